// Kernel skeletons shared by every storage form (instantiated in llb_f64.cu and
// llb_lowp.cu).  One thread owns one node; a block is 32 consecutive rows of 8
// consecutive columns, so a warp reads and writes 32 contiguous entries of each
// population plane.
//
// The resident state is the post-collision populations f*.  One step t computes,
// for every fluid, inlet and outlet node x:
//   1. pull  S_t(x,k):  f*_{t-1}(x - c_k, k)   if the source node is fluid or open
//                       f*_{t-1}(x, opp(k))    if it is a wall or wet obstacle
//                                              (half-way bounce-back)
//                       initial value w_k      if it is dead (its slot holds w_k)
//                                              or outside the lattice
//      -- the reference's push stream + bounce-back (Lattice.hpp:393-403) seen
//         from the receiving node: every population slot has exactly one writer;
//   2. the inlet/outlet closure with the boundary values of step t-1
//      (Lattice.hpp:409-410, run at the end of the reference's iteration t-1);
//   3. moments of fluid nodes, boundary values of step t for open nodes
//      (update_nodes + update_macro, Lattice.hpp:351-357);
//   4. equilibrium and collision (Lattice.hpp:363-382), store f*_t.
#pragma once

#include "llb_model.cuh"

namespace llb {

constexpr int BX = 32, BY = MAX_BLOCK_Y;  // one warp = 32 rows of one column

// warp_plain: every lane of the warp that pulls has a PLAIN node (a warp vote
// taken by the caller while the warp is converged; false is always correct).
// Such warps read straight from the sources; the others take one branch-free
// path on every lane, where a bounce-back source is only another address
// (plain lanes skip the bounce-bit load).
// b_pre: the node's bounce byte when the caller has it already (NO_BB: load it).
// I: the type of the slot arithmetic -- long long in general; int where every
// offset of the nine planes fits in 32 bits (a batch's lattices), which saves
// the 64-bit multiply-adds of the 18 accesses of a node.
constexpr unsigned NO_BB = 0x100u;
template <class M, class I = long long>
__device__ __forceinline__ void pull(const Geometry& g, const typename M::T* __restrict__ fin, int i, int j,
                                     I node, uint8_t m, bool warp_plain, typename M::R* f,
                                     unsigned b_pre = NO_BB) {
    const I P = static_cast<I>(g.plane), ld = static_cast<I>(g.ld);
    f[0] = M::load(fin + node);
    if (warp_plain) {
#pragma unroll
        for (int k = 1; k < 9; ++k) f[k] = M::load(fin + (k * P + node - (DJ(k) * ld + DI(k))));
    } else if (i > 0 && j > 0 && i < g.rows - 1 && j < g.cols - 1) {
        const unsigned b = (m & MASK_PLAIN) ? 0u : (b_pre != NO_BB ? b_pre : ld_keep(g.bb + node, l2_keep_policy()));
#pragma unroll
        for (int k = 1; k < 9; ++k) {
            const I a = ((b >> (k - 1)) & 1u) ? opp(k) * P + node : k * P + node - (DJ(k) * ld + DI(k));
            f[k] = M::load(fin + a);
        }
    } else {
        // open nodes on the lattice edge: sources outside keep their initial value
#pragma unroll
        for (int k = 1; k < 9; ++k) {
            const int si = i - DI(k), sj = j - DJ(k);
            typename M::R v = M::keep(k);
            if (si >= 0 && sj >= 0 && si < g.rows && sj < g.cols) {
                const I src = static_cast<I>(sj) * ld + si;
                // a bounce-back source reflects this node's own population; fluid,
                // open and dead sources are read where they are
                v = mask_class(g.mask[src]) == CLS_BB ? M::load(fin + (opp(k) * P + node))
                                                      : M::load(fin + (k * P + src));
            }
            f[k] = v;
        }
    }
}

// Closure + choice of (rho, u) for an open node at step t (t >= 1), or for the
// initial step (t == 0: no closure, pressure nodes start at rest).
template <class M>
__device__ __forceinline__ void open_node(const OpenTable& ot, int q, uint8_t m, long long t, typename M::R* f,
                                          double& rho, double& ux, double& uy) {
    const int side = mask_side(m), bc = mask_bc(m);
    const double2 cur = ot.vals[static_cast<long long>(t % ot.cap) * ot.n_open + q];
    if (bc == BC_ZH_PRES) {
        rho = cur.x;
        if (t == 0) {
            ux = 0.0;
            uy = 0.0;
        } else {
            const double2 prev = ot.vals[static_cast<long long>((t - 1) % ot.cap) * ot.n_open + q];
            M::closure_pressure(f, side, prev.x, prev.y, ux, uy);
        }
    } else {
        if (bc == BC_ZH_VEL && t > 0) {
            const double2 prev = ot.vals[static_cast<long long>((t - 1) % ot.cap) * ot.n_open + q];
            M::closure_velocity(f, side, prev.x, prev.y);
        }
        rho = 1.0;  // open nodes collide with global_rho == 1 (never written for them)
        ux = cur.x;
        uy = cur.y;
    }
}

__device__ __forceinline__ long long current_step(const StepSync& ss) {
    return (ss.tbase ? *ss.tbase : 0LL) + ss.t_off;
}

// Non-finite densities raise bit 0 of the flag word (one atomic per warp that
// saw one).  No block-wide barrier: warps of a block finish independently.
__device__ __forceinline__ void flag_numerics(const StepSync& ss, bool bad) {
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(ss.flags, 1u);
}

// Stores of a warp cover whole 32-byte sectors when every lane of a sector
// writes: lanes of inactive nodes that share a sector with an active node
// store the initial values too (dead slots must keep them; wall and obstacle
// slots are never read), so L2 need not merge a partial sector with DRAM
// contents.  Lanes whose whole sector is inactive skip.
template <class M>
__device__ __forceinline__ bool sector_has_active(bool active) {
    constexpr int lanes_per_sector = 32 / sizeof(typename M::T);
    const unsigned ballot = __ballot_sync(0xffffffffu, active);
    const int lane = threadIdx.x & 31;
    const unsigned group = ((1u << lanes_per_sector) - 1u) << (lane & ~(lanes_per_sector - 1));
    return (ballot & group) != 0u;
}

// Partially saturated obstacles (PSBounceBackPolicy<2>, PSBounceBackPolicy.hpp:177-293).
// The reference, after streaming, rewrites for every wet obstacle x and every
// direction k whose neighbour x_f = x + c_k is fluid or open the population
// x_f receives from x:
//   pop(x_f, k) = p - (1 - b)(p - e_opp) t + b ((pop(x_f, k) - e_k) - (p - w_k rho_x)),
//   p = f*(x_f, opp k) (streamed into x), e from x_f's rho and u of the step,
//   rho_x = 1 (global_rho of an obstacle is never updated), t = 1 / tau_ps.
// Every term is known to x_f at the end of its own step, so x_f computes the
// value and writes it into the obstacle's (otherwise unused) slot (x, k);
// next step's pull reads it there as from any source.  The equilibria are the
// policy's own expressions, evaluated in its order.
__device__ __forceinline__ double ps_equilibrium(int k, double rho, double ux, double uy) {
    constexpr double one18 = (1.0 / 18.0);
    constexpr double one36 = (1.0 / 36.0);
    const double u2 = ux * ux + uy * uy;
    switch (k) {
    case 1: return one18 * rho * (2 + 6 * ux + 9 * ux * ux - 3 * u2);
    case 3: return one18 * rho * (2 - 6 * ux + 9 * ux * ux - 3 * u2);
    case 2: return one18 * rho * (2 + 6 * uy + 9 * uy * uy - 3 * u2);
    case 4: return one18 * rho * (2 - 6 * uy + 9 * uy * uy - 3 * u2);
    case 5: return one36 * rho * (1 + 3 * (ux + uy) + 9 * ux * uy + 3 * u2);
    case 7: return one36 * rho * (1 - 3 * (ux + uy) + 9 * ux * uy + 3 * u2);
    case 6: return one36 * rho * (1 - 3 * (ux - uy) - 9 * ux * uy + 3 * u2);
    default: return one36 * rho * (1 + 3 * (ux - uy) - 9 * ux * uy + 3 * u2);
    }
}

// s: the node's populations before collision, f: after; bits: ps bits of the node.
template <typename T>
__device__ __forceinline__ void ps_push(const Geometry& g, T* __restrict__ fout, long long node, unsigned bits,
                                        const double* s, const double* f, double rho, double ux, double uy, double t) {
    constexpr double one18 = (1.0 / 18.0);
    constexpr double one36 = (1.0 / 36.0);
#pragma unroll
    for (int k = 1; k < 9; ++k) {
        if (!((bits >> (k - 1)) & 1u)) continue;
        const long long x = node - (DJ(k) * g.ld + DI(k));  // the obstacle
        const double b = g.psb[x];
        const double p = f[opp(k)];
        const double ek = ps_equilibrium(k, rho, ux, uy);
        const double eo = ps_equilibrium(opp(k), rho, ux, uy);
        const double wr = k <= 4 ? 2 * one18 * 1.0 : one36 * 1.0;
        fout[k * g.plane + x] = p - (1.0 - b) * (p - eo) * t + b * ((s[k] - ek) - (p - wr));
    }
}

// One node of a step (steps 1-4 above).  Every lane of the warp calls it
// (warp votes inside).  inside: (i, j) is a node of the lattice, m its mask;
// write_sector: the node's 32-byte sector holds an active node, so an
// inactive node of it stores the initial values; padding: (i, j) is a padding
// row of a column (rows <= i < ld), stored like a dead node; b_pre: the
// node's bounce byte if already loaded (NO_BB otherwise).
// INIT == true: step 0 from the initial equilibrium (Lattice.hpp:326-328).
template <class M, int COLL, bool MACRO, bool INIT, bool PS>
__device__ __forceinline__ void step_node(const Geometry& g, const OpenTable& ot, const Collision& c,
                                          const typename M::T* __restrict__ fin, typename M::T* __restrict__ fout,
                                          const MacroOut& mo, const StepSync& ss, int i, int j, long long node,
                                          bool inside, uint8_t m, bool write_sector, bool padding,
                                          unsigned b_pre = NO_BB) {
    bool bad = false;
    const uint8_t cls = mask_class(m);
    const bool warp_plain = __all_sync(0xffffffffu, !(inside && class_active(cls)) || (m & MASK_PLAIN));
    if (inside) {
        if (class_active(cls)) {
            typename M::R f[9];
            if (INIT) {
#pragma unroll
                for (int k = 0; k < 9; ++k) f[k] = M::keep(k);
            } else {
                pull<M>(g, fin, i, j, node, m, warp_plain, f, b_pre);
            }
            // moments stay in the model's arithmetic type up to the collision
            typename M::R rr, xr, yr;
            if (cls == CLS_OPEN) {
                const long long t = INIT ? 0 : current_step(ss);
                double rho, ux, uy;
                open_node<M>(ot, g.open_idx[node], m, t, f, rho, ux, uy);
                rr = M::from_f64(rho);
                xr = static_cast<typename M::R>(ux);
                yr = static_cast<typename M::R>(uy);
            } else {
                M::moments(f, rr, xr, yr);
                bad = !M::finite(rr);
            }
            if (MACRO) {
                const long long d = static_cast<long long>(j) * g.rows + i;
                const long long N = static_cast<long long>(g.rows) * g.cols;
                mo.rho[d] = M::rho_f64(rr);
                mo.u[d] = xr;
                mo.u[d + N] = yr;
            }
            [[maybe_unused]] typename M::R s_ps[9];
            [[maybe_unused]] unsigned psbits = 0;
            if constexpr (PS) {
                psbits = g.ps[node];
#pragma unroll
                for (int k = 0; k < 9; ++k) s_ps[k] = f[k];
            }
            M::template collide<COLL>(f, rr, xr, yr, c);
#pragma unroll
            for (int k = 0; k < 9; ++k) M::store(fout + k * g.plane + node, f[k]);
            if constexpr (PS) {
                if (psbits) ps_push(g, fout, node, psbits, s_ps, f, rr, xr, yr, c.ps_t);
            }
        } else {
            // a partially saturated obstacle's slots hold what its neighbours write
            if (write_sector && !(PS && cls == CLS_BB)) {
#pragma unroll
                for (int k = 0; k < 9; ++k) M::store(fout + k * g.plane + node, M::keep(k));
            }
            if (MACRO) {
                const long long d = static_cast<long long>(j) * g.rows + i;
                const long long N = static_cast<long long>(g.rows) * g.cols;
                mo.rho[d] = 1.0;  // global_rho / global_u keep their initial values off active nodes
                mo.u[d] = 0.0;
                mo.u[d + N] = 0.0;
            }
        }
    } else if (write_sector && padding) {
        // padding rows (dead) of a column that shares a sector with active nodes
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(fout + k * g.plane + node, M::keep(k));
    }
    flag_numerics(ss, bad);
}

// Programmatic dependent launch: a step kernel launched with programmatic
// stream serialization may start while the previous kernel on the stream
// drains.  It reads the lattice's own tables first (they do not change
// between steps), then waits (griddepcontrol.wait returns once the previous
// grid has completed and its writes are visible) before it touches the
// populations, and lets the next step's launch begin as soon as every block
// is past that point.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_wait_then_release() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Block: 32 rows (one warp per column) x blockDim.y columns, blockDim.y <= BY.
template <class M, int COLL, bool MACRO, bool INIT, bool PS = false>
__global__ void __launch_bounds__(BX* BY) k_step(Geometry g, OpenTable ot, Collision c,
                                                 const typename M::T* __restrict__ fin,
                                                 typename M::T* __restrict__ fout, MacroOut mo, StepSync ss) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const bool inside = i < g.rows && j < g.cols;
    const long long node = static_cast<long long>(j) * g.ld + i;
    const uint8_t m = inside ? ld_keep(g.mask + node, l2_keep_policy()) : CLS_DEAD;
    const bool write_sector = sector_has_active<M>(class_active(mask_class(m)));
    pdl_wait_then_release();
    step_node<M, COLL, MACRO, INIT, PS>(g, ot, c, fin, fout, mo, ss, i, j, node, inside, m, write_sector,
                                        j < g.cols && i < g.ld);
}

// Plain steps over the active-sector list: one thread per node of every
// 32-byte sector of a population plane that holds an active node (the
// sectors' ids in g.sectors; the listed nodes' mask and bounce bytes in
// g.smask / g.sbb, so a thread's first loads are independent of each
// other).  Sectors of obstacle interiors and dead regions are neither read
// nor written, and every lane of a warp has a node to update or to complete
// its sector, which the one-thread-per-node grid cannot give on porous
// geometry (there a third of its lanes idle).  Same per-node arithmetic as
// k_step.
constexpr int LIST_BLOCK = 256;
template <class M, int COLL>
__global__ void __launch_bounds__(LIST_BLOCK, 5) k_step_list(Geometry g, OpenTable ot, Collision c,
                                                          const typename M::T* __restrict__ fin,
                                                          typename M::T* __restrict__ fout, MacroOut mo,
                                                          StepSync ss) {
    constexpr int SN = LIST_BYTES / sizeof(typename M::T);  // nodes per listed block
    const long long t = static_cast<long long>(blockIdx.x) * LIST_BLOCK + threadIdx.x;
    const long long e = t / SN;
    const bool valid = e < g.n_sectors;
    long long node = 0;
    int i = 0, j = 0;
    uint8_t m = CLS_DEAD;
    unsigned b = 0;
    if (valid) {
        m = g.smask[t];
        b = g.sbb[t];
        node = static_cast<long long>(g.sectors[e]) * SN + (t & (SN - 1));
        // node < 2^31 for every lattice that has a list
        const unsigned un = static_cast<unsigned>(node), uj = un / static_cast<unsigned>(g.ld);
        j = static_cast<int>(uj);
        i = static_cast<int>(un - uj * static_cast<unsigned>(g.ld));
    }
    // padding rows of a listed sector carry a dead mask: like a dead node of
    // the lattice, they store the initial values
    step_node<M, COLL, false, false, false>(g, ot, c, fin, fout, mo, ss, i, j, node, valid, m, valid, valid, b);
}

// Every slot of a population buffer set to the node-independent initial value
// of its direction (dead nodes keep it for ever; other slots are overwritten).
template <class M>
__global__ void k_fill_keep(typename M::T* __restrict__ f, long long plane) {
    const long long n = 9 * plane;
    for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < n;
         x += static_cast<long long>(gridDim.x) * blockDim.x)
        M::store(f + x, M::keep(static_cast<int>(x / plane)));
}

// populations S_t = stream + bounce-back + closures of the resident state,
// written as a dense (R, C, 9) FP64 tensor (0 off active nodes).
template <class M>
__global__ void __launch_bounds__(BX* BY) k_finalize(Geometry g, OpenTable ot, const typename M::T* __restrict__ fin,
                                                     double* __restrict__ out, long long t) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= g.rows || j >= g.cols) return;
    const long long node = static_cast<long long>(j) * g.ld + i;
    const long long d = static_cast<long long>(j) * g.rows + i;
    const long long N = static_cast<long long>(g.rows) * g.cols;
    const uint8_t m = g.mask[node];
    const uint8_t cls = mask_class(m);
    if (!class_active(cls)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) out[d + k * N] = 0.0;
        return;
    }
    typename M::R f[9];
    pull<M>(g, fin, i, j, node, m, false, f);
    if (cls == CLS_OPEN && t > 0) {
        const int q = g.open_idx[node];
        const double2 prev = ot.vals[static_cast<long long>((t - 1) % ot.cap) * ot.n_open + q];
        if (mask_bc(m) == BC_ZH_VEL) M::closure_velocity(f, mask_side(m), prev.x, prev.y);
        else if (mask_bc(m) == BC_ZH_PRES) {
            double ux, uy;
            M::closure_pressure(f, mask_side(m), prev.x, prev.y, ux, uy);
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) out[d + k * N] = M::to_f64(f[k], k);
}

// after_collision_populations as a dense (R, C, 9) FP64 tensor.
template <class M>
__global__ void __launch_bounds__(BX* BY) k_export(Geometry g, const typename M::T* __restrict__ fin,
                                                   double* __restrict__ out) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= g.rows || j >= g.cols) return;
    const long long node = static_cast<long long>(j) * g.ld + i;
    const long long d = static_cast<long long>(j) * g.rows + i;
    const long long N = static_cast<long long>(g.rows) * g.cols;
    const bool act = class_active(mask_class(g.mask[node]));
#pragma unroll
    for (int k = 0; k < 9; ++k) out[d + k * N] = act ? M::to_f64(M::load(fin + k * g.plane + node), k) : 0.0;
}

// ---------------------------------------------------------------------------
// compensated FP64 reductions (Neumaier), deterministic order
// ---------------------------------------------------------------------------
struct Neu {
    double s, c;
};
__device__ __forceinline__ Neu neu_add(Neu a, double x) {
    const double t = a.s + x;
    if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
    else a.c += (x - t) + a.s;
    a.s = t;
    return a;
}
__device__ __forceinline__ Neu neu_merge(Neu a, Neu b) {
    Neu r = neu_add(a, b.s);
    r.c += b.c;
    return r;
}

// Block-wide reduction of NV compensated sums; thread 0 of the block writes
// partials[blockIdx][v] = (s, c).  Fixed shuffle and warp order.
template <int NV>
__device__ __forceinline__ void block_reduce_store(Neu (&acc)[NV], double2* partials) {
    __shared__ Neu sh[32][NV];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        for (int off = 16; off > 0; off >>= 1) {
            Neu o;
            o.s = __shfl_down_sync(0xffffffffu, acc[v].s, off);
            o.c = __shfl_down_sync(0xffffffffu, acc[v].c, off);
            if (lane + off < 32) acc[v] = neu_merge(acc[v], o);
        }
        if (lane == 0) sh[warp][v] = acc[v];
    }
    __syncthreads();
    if (tid == 0) {
        for (int v = 0; v < NV; ++v) {
            Neu r = sh[0][v];
            for (int w = 1; w < nwarps; ++w) r = neu_merge(r, sh[w][v]);
            partials[static_cast<long long>(blockIdx.x) * NV + v] = make_double2(r.s, r.c);
        }
    }
}

// final pass: one block folds the per-block partials in index order
template <int NV>
__global__ void k_reduce_partials(const double2* __restrict__ partials, int nblocks, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    for (int v = 0; v < NV; ++v) {
        Neu r{0.0, 0.0};
        for (int b = 0; b < nblocks; ++b) {
            const double2 p = partials[static_cast<long long>(b) * NV + v];
            r = neu_merge(r, Neu{p.x, p.y});
        }
        out[v] = r.s + r.c;
    }
}

// mass and momentum of the resident post-collision state over active nodes
template <class M>
__global__ void __launch_bounds__(256) k_mass_momentum(Geometry g, const typename M::T* __restrict__ fin,
                                                       double2* partials) {
    Neu acc[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    const long long N = static_cast<long long>(g.rows) * g.cols;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < N; x += stride) {
        const int j = static_cast<int>(x / g.rows), i = static_cast<int>(x - static_cast<long long>(j) * g.rows);
        const long long node = static_cast<long long>(j) * g.ld + i;
        if (!class_active(mask_class(g.mask[node]))) continue;
        double f[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) f[k] = M::to_f64(M::load(fin + k * g.plane + node), k);
        const double m = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
        const double mx = (f[1] + f[5] + f[8]) - (f[3] + f[6] + f[7]);
        const double my = (f[2] + f[5] + f[6]) - (f[4] + f[7] + f[8]);
        acc[0] = neu_add(acc[0], m);
        acc[1] = neu_add(acc[1], mx);
        acc[2] = neu_add(acc[2], my);
    }
    block_reduce_store<3>(acc, partials);
}

// FlowAnalyzer<2>::compute_flow_properties (FlowAnalyzer.hpp:394-427): the value
// of bit k is the neighbour x + c_k's population in direction opp(k).
template <class M>
__device__ __forceinline__ double force_input(const Geometry& g, const typename M::T* __restrict__ fin, long long i,
                                              long long j, int k) {
    const long long ni = i + DI(k), nj = j + DJ(k);
    if (ni < 0 || nj < 0 || ni >= g.rows || nj >= g.cols) return 0.0;
    const int b = opp(k);
    return M::to_f64(M::load(fin + b * g.plane + nj * g.ld + ni), b);
}

template <class M>
__global__ void __launch_bounds__(256) k_flow_forces(Geometry g, const typename M::T* __restrict__ fin,
                                                     const int64_t* __restrict__ pts, const uint16_t* __restrict__ dirs,
                                                     long long n, double2* partials) {
    Neu acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
    constexpr double SQRT2 = 1.4142135623730951;  // sqrt(2) rounded to double
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
        const long long i = pts[2 * q], j = pts[2 * q + 1];
        const unsigned b = dirs[q];
        double local_lift = 0., local_drag = 0.;
        if (b & (1u << 1)) local_drag -= force_input<M>(g, fin, i, j, 1);
        if (b & (1u << 2)) local_lift -= force_input<M>(g, fin, i, j, 2);
        if (b & (1u << 3)) local_drag += force_input<M>(g, fin, i, j, 3);
        if (b & (1u << 4)) local_lift += force_input<M>(g, fin, i, j, 4);
        if (b & (1u << 5)) {
            const double v = force_input<M>(g, fin, i, j, 5);
            local_drag -= (v) * SQRT2 / 2.0;
            local_lift -= (v) * SQRT2 / 2.0;
        }
        if (b & (1u << 6)) {
            const double v = force_input<M>(g, fin, i, j, 6);
            local_drag += (v) * SQRT2 / 2.0;
            local_lift -= (v) * SQRT2 / 2.0;
        }
        if (b & (1u << 7)) {
            const double v = force_input<M>(g, fin, i, j, 7);
            local_drag += (v) * SQRT2 / 2.0;
            local_lift += (v) * SQRT2 / 2.0;
        }
        if (b & (1u << 8)) {
            const double v = force_input<M>(g, fin, i, j, 8);
            local_drag -= (v) * SQRT2 / 2.0;
            local_lift += (v) * SQRT2 / 2.0;
        }
        acc[0] = neu_add(acc[0], local_lift);
        acc[1] = neu_add(acc[1], local_drag);
    }
    block_reduce_store<2>(acc, partials);
}

template <class M>
__global__ void k_gather_forces(Geometry g, const typename M::T* __restrict__ fin, const int64_t* __restrict__ pts,
                                const uint16_t* __restrict__ dirs, long long n, double* __restrict__ out) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const long long i = pts[2 * q], j = pts[2 * q + 1];
    const unsigned b = dirs[q];
#pragma unroll
    for (int k = 1; k < 9; ++k) out[q * 8 + (k - 1)] = (b & (1u << k)) ? force_input<M>(g, fin, i, j, k) : 0.0;
}

}  // namespace llb

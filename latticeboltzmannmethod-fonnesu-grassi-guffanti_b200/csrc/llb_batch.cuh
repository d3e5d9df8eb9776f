// Batched step: many independent lattices (uneven sizes, BGK or TRT, own tau)
// advanced by one persistent launch.
//
// Every lattice is described by a BatchLattice in device memory; the work list
// holds one item per (lattice, block of slots) for lattices on compacted
// planes (llb_compact.cuh: only active nodes, every lane busy) and per
// (lattice, tile of 32 rows x blockDim.y columns) for lattices on dense
// planes.  A persistent grid walks the items with a grid-stride loop, so
// lattices of any size share the launch and the load balances at item
// granularity.  A lattice
// joins the batch at batch step s0 with its step index t0 and current buffer
// cur0; at batch step s it is at step t0 + (s - s0) and reads buffer
// cur0 ^ ((s - s0) & 1), so lattices that joined at different times coexist and
// no per-step bookkeeping is written.
//
// With steps > 1 one launch advances all lattices several steps, separated by a
// grid barrier; the host launches it cooperatively (all blocks co-resident).
// The barrier's spin is bounded: on timeout it raises the batch error flag and
// the kernel returns.
#pragma once

#include "llb_compact.cuh"

namespace llb {

struct BatchLattice {
    Geometry g;
    OpenTable ot;
    Collision c;
    void* f[2];     // the planes the batch steps: dense, or compacted when `compact`
    long long t0;   // lattice step index at batch step s0
    long long s0;
    long long t_end;  // the lattice stops before step index t_end (later batch steps leave it as it is)
    int cur0;       // buffer holding the lattice's state at batch step s0
    int nti;        // row tiles: ceil(rows / 32)
    int compact;    // 1: compacted planes (cg), items are blocks of slots
    unsigned* flags;
    CompactGeo cg;
};

constexpr long long BARRIER_LIMIT = 1LL << 22;
constexpr unsigned BATCH_FLAG_TIMEOUT = 1u;

// Generation barrier across the grid (blocks must be co-resident); a block
// gives up after `limit` polls.  A block that gave up has counted itself, so
// the host clears [count, generation] before the next launch (the batch's
// error path).
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks, long long limit) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        volatile unsigned* vgen = gen;
        const unsigned g0 = *vgen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(count, 1u) == nblocks - 1) {
            *count = 0u;
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            long long it = 0;
            while (*vgen == g0) {
                if (++it > limit) { ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

// Work-list item flag, bit 30 of the item's lattice index: every node of the
// dense tile is a fluid node whose eight sources are fluid or open (PLAIN; such
// a node is never on the lattice edge).  The tile then pulls straight from its
// sources without waiting for its mask bytes: the population loads leave
// right after the lattice descriptor, one memory round trip earlier.  Set on
// the host from the lattice's per-column flags of 32-row segments (built with
// its mask).
constexpr int ITEM_PLAIN = 1 << 30;
__host__ __device__ __forceinline__ int item_lattice(int x) { return x & (ITEM_PLAIN - 1); }

// One tile of one lattice: `tile` packs its row-tile index (low 16 bits) and
// column-tile index (high 16 bits), computed on the host; plain_tile: the
// item's ITEM_PLAIN flag.
template <class M>
__device__ __forceinline__ void batch_tile(const BatchLattice* __restrict__ Lp, int tile, long long s,
                                           bool plain_tile) {
    using T = typename M::T;
    const long long d = s - Lp->s0;
    // both buffers are read with the step fields, so the population addresses
    // wait for one descriptor round trip, not two
    const void* const fa = Lp->f[0];
    const void* const fb = Lp->f[1];
    const int cur = Lp->cur0 ^ static_cast<int>(d & 1);
    const long long t = Lp->t0 + d;
    if (t >= Lp->t_end) return;  // block-uniform: the lattice has finished
    const T* __restrict__ fin = static_cast<const T*>(cur ? fb : fa);
    T* __restrict__ fout = static_cast<T*>(const_cast<void*>(cur ? fa : fb));
    const Geometry& g = Lp->g;  // read where used (L1), not copied into registers
    unsigned* const flags = Lp->flags;
    const int i = (tile & 0xffff) * BX + threadIdx.x;
    const int j = (static_cast<unsigned>(tile) >> 16) * blockDim.y + threadIdx.y;
    // 32-bit slot arithmetic: a batch admits only lattices whose nine planes
    // hold fewer than 2^31 slots
    const int P = static_cast<int>(g.plane);
    const int ld = g.ld;
    const int node = j * ld + i;
    if (plain_tile) {
        // every lane holds a PLAIN fluid node: the pull of a plain warp, the
        // moments and the collision, as below
        typename M::R f[9];
        f[0] = M::load(fin + node);
#pragma unroll
        for (int k = 1; k < 9; ++k) f[k] = M::load(fin + (k * P + node - (DJ(k) * ld + DI(k))));
        typename M::R rr, xr, yr;
        M::moments(f, rr, xr, yr);
        const bool bad = !M::finite(rr);
        if (Lp->c.model == 0) M::template collide<0>(f, rr, xr, yr, Lp->c);
        else M::template collide<1>(f, rr, xr, yr, Lp->c);
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(fout + (k * P + node), f[k]);
        if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 1u);
        return;
    }
    const bool inside = i < g.rows && j < g.cols;
    const uint8_t m = inside ? g.mask[node] : CLS_DEAD;
    const uint8_t cls = mask_class(m);
    const bool write_sector = sector_has_active<M>(class_active(cls));
    const bool warp_plain = __all_sync(0xffffffffu, !(inside && class_active(cls)) || (m & MASK_PLAIN));
    bool bad = false;
    if (inside && class_active(cls)) {
        typename M::R f[9];
        pull<M, int>(g, fin, i, j, node, m, warp_plain, f);
        typename M::R rr, xr, yr;
        if (cls == CLS_OPEN) {
            double rho, ux, uy;
            open_node<M>(Lp->ot, g.open_idx[node], m, t, f, rho, ux, uy);
            rr = M::from_f64(rho);
            xr = static_cast<typename M::R>(ux);
            yr = static_cast<typename M::R>(uy);
        } else {
            M::moments(f, rr, xr, yr);
            bad = !M::finite(rr);
        }
        if (Lp->c.model == 0) M::template collide<0>(f, rr, xr, yr, Lp->c);
        else M::template collide<1>(f, rr, xr, yr, Lp->c);
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(fout + (k * P + node), f[k]);
    } else if (write_sector && j < g.cols && i < g.ld) {
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(fout + (k * P + node), M::keep(k));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 1u);
}

// One item of a compacted lattice: (threads of the block) consecutive slots.
template <class M>
__device__ __forceinline__ void batch_slots(const BatchLattice* __restrict__ Lp, int item, long long s) {
    using T = typename M::T;
    const long long d = s - Lp->s0;
    const void* const fa = Lp->f[0];  // read with the step fields (see batch_tile)
    const void* const fb = Lp->f[1];
    const long long t = Lp->t0 + d;
    if (t >= Lp->t_end) return;  // block-uniform: the lattice has finished
    const int cur = Lp->cur0 ^ static_cast<int>(d & 1);
    const T* __restrict__ fin = static_cast<const T*>(cur ? fb : fa);
    T* __restrict__ fout = static_cast<T*>(const_cast<void*>(cur ? fa : fb));
    const int nthr = blockDim.x * blockDim.y;
    const long long slot = static_cast<long long>(item) * nthr + threadIdx.y * blockDim.x + threadIdx.x;
    // the descriptor's fields are read where they are used (L1-resident), not
    // copied into registers
    const bool bad =
        compact_slot<M, -1, int>(Lp->g, Lp->cg, Lp->ot, Lp->c, fin, fout, [t] { return t; }, static_cast<int>(slot));
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(Lp->flags, 1u);
}

// Resident blocks per SM of the one-step batch kernels (256-thread budget):
// 8 for the shifted forms (32 registers, full occupancy, some words spilled:
// the 256 problems of config 4 ran 67.9k MLUPS against 64.7k at 6 blocks and
// 40 registers, and 61.7k at 5 blocks and 48 registers), 4 for FP64 (64
// registers, no spills).
template <class M>
__host__ __device__ constexpr int batch_min_blocks() { return sizeof(typename M::T) == 8 ? 4 : 8; }

// One batch step, one block per item: the dense tiles (items[0, n)) ...
template <class M>
__global__ void __launch_bounds__(BX* BY, batch_min_blocks<M>()) k_batch_tiles(const BatchLattice* __restrict__ lats,
                                                       const int2* __restrict__ items, const long long* sbase,
                                                       long long soff) {
    const int2 it = items[blockIdx.x];
    batch_tile<M>(lats + item_lattice(it.x), it.y, *sbase + soff, (it.x & ITEM_PLAIN) != 0);
}

// ... and the compacted slot blocks, in a launch of their own (each kernel
// gets the registers its own path needs).
template <class M>
__global__ void __launch_bounds__(BX* BY, batch_min_blocks<M>()) k_batch_slots(const BatchLattice* __restrict__ lats,
                                                       const int2* __restrict__ items, const long long* sbase,
                                                       long long soff) {
    const int2 it = items[blockIdx.x];
    batch_slots<M>(lats + it.x, it.y, *sbase + soff);
}

// One cooperative launch: `steps` batch steps starting at batch step
// (*sbase + soff) over every item, a grid barrier between steps.
template <class M>
__global__ void __launch_bounds__(BX* BY, 5) k_batch_step(const BatchLattice* __restrict__ lats,
                                                       const int2* __restrict__ items, int n_items,
                                                       const long long* sbase, long long soff, int steps,
                                                       unsigned* bar, unsigned* err, long long bar_limit) {
    const long long s0 = *sbase + soff;
    for (int st = 0; st < steps; ++st) {
        const long long s = s0 + st;
        // the next item's entry is loaded while this one is computed
        int2 it = blockIdx.x < n_items ? items[blockIdx.x] : make_int2(0, 0);
        for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
            const int nxt = item + gridDim.x;
            const int2 it_next = nxt < n_items ? items[nxt] : it;
            const BatchLattice* Lp = lats + item_lattice(it.x);
            if (Lp->compact) batch_slots<M>(Lp, it.y, s);
            else batch_tile<M>(Lp, it.y, s, (it.x & ITEM_PLAIN) != 0);
            it = it_next;
        }
        if (st + 1 < steps && !grid_barrier(bar, bar + 1, gridDim.x, bar_limit)) {
            if (threadIdx.x == 0 && threadIdx.y == 0) atomicOr(err, BATCH_FLAG_TIMEOUT);
            return;
        }
    }
}

// rho and u of the current populations S_t of one lattice (pull, closure,
// moments or prescribed values), dense (R, C) and (R, C, 2).
template <class M>
__global__ void __launch_bounds__(BX* BY) k_macro_now(Geometry g, OpenTable ot, const typename M::T* __restrict__ fin,
                                                     long long t, double* __restrict__ rho_out,
                                                     double* __restrict__ u_out) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= g.rows || j >= g.cols) return;
    const long long node = static_cast<long long>(j) * g.ld + i;
    const long long dd = static_cast<long long>(j) * g.rows + i;
    const long long N = static_cast<long long>(g.rows) * g.cols;
    const uint8_t m = g.mask[node];
    const uint8_t cls = mask_class(m);
    double rho = 1.0, ux = 0.0, uy = 0.0;
    if (class_active(cls)) {
        typename M::R f[9];
        pull<M>(g, fin, i, j, node, m, false, f);
        if (cls == CLS_OPEN) {
            open_node<M>(ot, g.open_idx[node], m, t, f, rho, ux, uy);
        } else {
            typename M::R r, x, y;
            M::moments(f, r, x, y);
            rho = M::rho_f64(r);
            ux = x;
            uy = y;
        }
    }
    rho_out[dd] = rho;
    u_out[dd] = ux;
    u_out[dd + N] = uy;
}

}  // namespace llb

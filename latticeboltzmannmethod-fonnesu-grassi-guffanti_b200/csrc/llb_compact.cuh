// Plain steps over column-compacted storage (pipeline PIPE_COMPACT; layout in
// llb_internal.cuh, CompactGeo).  Only the fluid and open nodes have slots, so
// a step moves the bytes of active nodes and nothing else: on obstacle-rich
// lattices the dense layouts also pull obstacle interiors through DRAM (the
// 64-byte bursts at the ends of every active run of a column), which the
// compacted planes do not have.
//
// One thread owns one slot.  Its first loads (the node's info and neighbour
// offsets) depend on nothing, so the pull is one memory round trip behind the
// launch, as in the one-thread-per-node dense kernel, and every lane of a
// warp has a node (no lanes idle over obstacles).  The pull reads the same
// sources as k_step and the arithmetic is the same: the bits are identical.
#pragma once

#include "llb_kernels.cuh"

namespace llb {

constexpr int COMPACT_BLOCK = 256;  // threads per block (the copies: 8 chunks of 32 slots)

// Position of the n-th set bit (n from 0) of m; m has more than n set bits.
__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
    int pos = 0, c;
    c = __popc(m & 0xffffu);
    if (n >= c) { n -= c; m >>= 16; pos += 16; }
    c = __popc(m & 0xffu);
    if (n >= c) { n -= c; m >>= 8; pos += 8; }
    c = __popc(m & 0xfu);
    if (n >= c) { n -= c; m >>= 4; pos += 4; }
    c = __popc(m & 0x3u);
    if (n >= c) { n -= c; m >>= 2; pos += 2; }
    c = static_cast<int>(m & 1u);
    if (n >= c) pos += 1;
    return pos;
}

__device__ __forceinline__ unsigned below(int r) { return (1u << r) - 1u; }  // r in [0, 31]

// Rows of the 32 slots of chunk w: row of this lane's slot (-1 past the
// column's active nodes), the first slot of the chunk and the column.
// Warp-uniform control flow: every lane loads the same segment entries.
struct ChunkPos {
    int j, row, t, tend;
};
__device__ __forceinline__ ChunkPos chunk_rows(const CompactGeo& cg, long long w, int lane) {
    const int2 ch = cg.chunk[w];
    ChunkPos p;
    p.j = ch.x;
    const int2* sc = cg.seg + static_cast<long long>(ch.x) * cg.nseg;
    int s = ch.y >> 5;
    const int2 e = sc[s];
    const unsigned lowr = below(ch.y & 31);
    p.t = e.y + __popc(static_cast<unsigned>(e.x) & lowr) + lane;
    p.tend = cg.col[ch.x + 1];
    unsigned m = static_cast<unsigned>(e.x) & ~lowr;
    p.row = -1;
    int base = 0;
    for (;;) {
        const int cnt = __popc(m);
        if (p.row < 0 && lane < base + cnt) p.row = (s << 5) + nth_set_bit(m, lane - base);
        base += cnt;
        if (base >= 32 || ++s >= cg.nseg) break;
        m = static_cast<unsigned>(sc[s].x);
    }
    return p;
}

// Slot of row i in column j (or of the next active row below it) and whether
// row i of column j is active.
__device__ __forceinline__ int col_slot(const CompactGeo& cg, int j, int i, int& act) {
    const int2 e = cg.seg[static_cast<long long>(j) * cg.nseg + (i >> 5)];
    const unsigned x = static_cast<unsigned>(e.x);
    act = static_cast<int>((x >> (i & 31)) & 1u);
    return e.y + __popc(x & below(i & 31));
}

// Pull of a node that needs every source tested: an open node (it may lie on
// the lattice edge) or a fluid node with a dead source.  dn: its dense index.
template <class M>
__device__ __forceinline__ void pull_compact_general(const Geometry& g, const CompactGeo& cg,
                                                     const typename M::T* __restrict__ fin, long long t,
                                                     unsigned dn, typename M::R* f) {
    const long long P = cg.cplane;
    const int j = static_cast<int>(dn / static_cast<unsigned>(g.ld));
    const int i = static_cast<int>(dn - static_cast<unsigned>(j) * static_cast<unsigned>(g.ld));
    f[0] = M::load(fin + t);
#pragma unroll
    for (int k = 1; k < 9; ++k) {
        const int si = i - DI(k), sj = j - DJ(k);
        typename M::R v = M::keep(k);
        if (si >= 0 && sj >= 0 && si < g.rows && sj < g.cols) {
            int act;
            const long long c = col_slot(cg, sj, si, act);
            if (act) v = M::load(fin + k * P + c);
            else if (mask_class(g.mask[static_cast<long long>(sj) * g.ld + si]) == CLS_BB)
                v = M::load(fin + opp(k) * P + t);
        }
        f[k] = v;
    }
}

// One slot of a step (steps 1-4 of llb_kernels.cuh) over the compacted planes:
// pull, closure, moments, collision, store.  Padding slots store the initial
// values, so every 32-byte sector of a column's run is written whole.  Every
// lane of the warp calls it (warp vote inside).  Returns whether a non-finite
// density was seen.  COLL: 0 BGK, 1 TRT, -1 the lattice's own (c.model; a
// batch holds both).
//
// One slot per thread: a variant that gave each thread 2 (FP32) or 4 (FP16)
// slots with all their loads issued first ran slower on B200 in every form
// (porous 4096^2: FP16 103.7k -> 77.7k, FP32 98.3k -> 93.1k MLUPS).
// tstep: callable returning the step index, evaluated for open nodes only (a
// step index read from device memory stays off every other lane's path and
// out of its registers).
// I: the type of the slot arithmetic (long long, or int where the nine planes
// hold fewer than 2^31 slots).
template <class M, int COLL, class I, class TStep>
__device__ __forceinline__ bool compact_slot(const Geometry& g, const CompactGeo& cg, const OpenTable& ot,
                                             const Collision& c, const typename M::T* __restrict__ fin,
                                             typename M::T* __restrict__ fout, TStep tstep, I t) {
    const bool in = t < cg.n_slots;
    unsigned info = 0, nb = 0;
    if (in) {
        info = cg.info[t];
        nb = cg.nb[t];
    }
    const uint8_t m = static_cast<uint8_t>(info & 0xffu);
    const uint8_t cls = mask_class(m);
    const bool node = class_active(cls);
    const bool general = cls == CLS_OPEN || (node && (m & COMPACT_DEAD_SRC));
    const bool warp_plain = __all_sync(0xffffffffu, !node || ((m & MASK_PLAIN) && !general));
    const I P = static_cast<I>(cg.cplane);
    bool bad = false;
    if (node) {
        typename M::R f[9];
        if (!general) {
            // fluid node: both neighbouring columns exist; a source that is not
            // a wall or obstacle is active
            const I cL = t - static_cast<I>(nb & 0xffffu);
            const I cR = t + static_cast<I>(nb >> 16);
            const unsigned bb = (m & MASK_PLAIN) ? 0u : (info >> 8);
            const I aL = ((bb >> 0) & 1u) ? 0 : 1;  // row i of column j - 1 active (direction 1's source)
            const I aR = ((bb >> 2) & 1u) ? 0 : 1;  // row i of column j + 1 active (direction 3's source)
            I src[9];
            src[1] = cL;       // (i, j-1)
            src[2] = t + 1;    // (i+1, j)
            src[3] = cR;       // (i, j+1)
            src[4] = t - 1;    // (i-1, j)
            src[5] = cL + aL;  // (i+1, j-1)
            src[6] = cR + aR;  // (i+1, j+1)
            src[7] = cR - 1;   // (i-1, j+1)
            src[8] = cL - 1;   // (i-1, j-1)
            f[0] = M::load(fin + t);
            if (warp_plain) {
#pragma unroll
                for (int k = 1; k < 9; ++k) f[k] = M::load(fin + (k * P + src[k]));
            } else {
#pragma unroll
                for (int k = 1; k < 9; ++k) {
                    const I a = ((bb >> (k - 1)) & 1u) ? opp(k) * P + t : k * P + src[k];
                    f[k] = M::load(fin + a);
                }
            }
        } else {
            pull_compact_general<M>(g, cg, fin, t, nb, f);
        }
        typename M::R rr, xr, yr;
        if (cls == CLS_OPEN) {
            double rho, ux, uy;
            open_node<M>(ot, g.open_idx[nb], m, tstep(), f, rho, ux, uy);
            rr = M::from_f64(rho);
            xr = static_cast<typename M::R>(ux);
            yr = static_cast<typename M::R>(uy);
        } else {
            M::moments(f, rr, xr, yr);
            bad = !M::finite(rr);
        }
        if (COLL == 0 || (COLL < 0 && c.model == 0)) M::template collide<0>(f, rr, xr, yr, c);
        else M::template collide<1>(f, rr, xr, yr, c);
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(fout + (k * P + t), f[k]);
    } else if (in) {
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(fout + (k * P + t), M::keep(k));
    }
    return bad;
}

// Resident blocks per SM of the plain compacted step: 5 for FP64 (48
// registers, no spills); 8 for the shifted forms (32 registers, full
// occupancy, a few words spilled: on porous 4096^2 FP16 ran 118k MLUPS
// against 104k at 6 blocks and 40 registers, FP32 101.5k against 98.7k).
template <class M>
__host__ __device__ constexpr int compact_min_blocks() { return sizeof(typename M::T) == 8 ? 5 : 8; }

// One plain step over the compacted planes: one thread per slot.  I: int when
// the nine planes hold fewer than 2^31 slots (32-bit slot arithmetic), else
// long long.
template <class M, int COLL, class I>
__global__ void __launch_bounds__(COMPACT_BLOCK, compact_min_blocks<M>()) k_step_compact(
    Geometry g, CompactGeo cg, OpenTable ot, Collision c, const typename M::T* __restrict__ fin,
    typename M::T* __restrict__ fout, StepSync ss) {
    const I t = static_cast<I>(blockIdx.x) * COMPACT_BLOCK + static_cast<I>(threadIdx.x);
    const bool bad = compact_slot<M, COLL, I>(g, cg, ot, c, fin, fout, [&] { return current_step(ss); }, t);
    flag_numerics(ss, bad);
}

// Copies between the dense planes and the compacted ones (to_compact: dense ->
// compact).  Padding slots get the initial values.
template <class M, bool TO_COMPACT>
__global__ void __launch_bounds__(COMPACT_BLOCK) k_compact_copy(Geometry g, CompactGeo cg,
                                                                typename M::T* __restrict__ dense,
                                                                typename M::T* __restrict__ comp) {
    const int lane = threadIdx.x & 31;
    const long long w = (static_cast<long long>(blockIdx.x) * COMPACT_BLOCK + threadIdx.x) >> 5;
    if (w >= cg.n_chunks) return;
    const ChunkPos p = chunk_rows(cg, w, lane);
    if (p.row >= 0) {
        const long long dn = static_cast<long long>(p.j) * g.ld + p.row;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (TO_COMPACT) comp[k * cg.cplane + p.t] = dense[k * g.plane + dn];
            else dense[k * g.plane + dn] = comp[k * cg.cplane + p.t];
        }
    } else if (TO_COMPACT && p.t < p.tend) {
#pragma unroll
        for (int k = 0; k < 9; ++k) M::store(comp + k * cg.cplane + p.t, M::keep(k));
    }
}

}  // namespace llb

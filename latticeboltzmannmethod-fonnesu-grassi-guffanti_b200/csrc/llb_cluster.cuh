// Small lattices resident in the distributed shared memory of one
// thread-block cluster (pipeline PIPE_CLUSTER).
//
// Config 1 (129 x 129, 16 641 nodes) is launch-bound: with one launch per
// step a step costs about 3 us of launch, ramp-up and drain for well under a
// microsecond of work.  Here one cluster of up to 16 blocks runs a chunk of
// steps in one launch.  Block r of the cluster owns a slab of columns
// [c0, c1) and keeps, in its own shared memory, both population buffers of
// its slab plus one halo column on each side, the slab's mask, bounce bytes
// and open-node indices.  A step reads only this block's shared memory; a
// block writes the populations that leave its slab (directions 1, 5, 8 from
// its last column, 3, 6, 7 from its first) straight into the neighbouring
// block's halo column (distributed shared memory), and one cluster barrier
// (arrive.release / wait.acquire) ends the step.  The state goes to global
// memory once per launch.  The pull follows pull() in llb_kernels.cuh source
// for source and the per-node arithmetic is the storage model's, so results
// are bit-identical to the other kernels.  No software spin: the barrier is
// the cluster's own and every thread reaches it the same number of times.
#pragma once

#include <cooperative_groups.h>

#include "llb_kernels.cuh"

namespace llb {

constexpr int CLUSTER_THREADS = 1024;  // 32 rows x 32 warps per block
constexpr int CLUSTER_MAX_CTAS = 16;   // non-portable cluster size (8 is the portable one)

// Shared-memory layout of one block: L = wmax + 2 local columns (halo, slab,
// halo) of R rows.  pop[b][k][l][i] for buffers b = 0, 1; mask of all L
// columns; bounce bytes, open indices and the list of active nodes of the
// slab.
struct ClusterSmem {
    int R, L;
    __host__ __device__ long long pop_elems() const { return 9LL * L * R; }
    __host__ __device__ long long slab() const { return static_cast<long long>(L - 2) * R; }
    // byte offset of the open indices (after the populations, masks and bounce bytes)
    template <class T>
    __host__ __device__ long long oid_offset() const {
        const long long tab = static_cast<long long>(L) * R + slab();
        return 2 * pop_elems() * static_cast<long long>(sizeof(T)) + ((tab + 15) / 16) * 16;
    }
    template <class T>
    __host__ __device__ long long bytes() const { return oid_offset<T>() + 2 * slab() * 4; }
};

// Slab of block r of nc: columns [c0, c1).
__host__ __device__ inline void cluster_slab(int C, int nc, int r, int& c0, int& c1) {
    c0 = static_cast<int>((static_cast<long long>(r) * C) / nc);
    c1 = static_cast<int>((static_cast<long long>(r + 1) * C) / nc);
}

template <class M, int COLL>
__global__ void __launch_bounds__(CLUSTER_THREADS, 1)
    k_step_cluster(Geometry g, OpenTable ot, Collision c, typename M::T* f0, typename M::T* f1, int cur,
                   long long t0, int steps, unsigned* flags, int wmax) {
    using T = typename M::T;
    using Rt = typename M::R;
    namespace cg = cooperative_groups;
    extern __shared__ __align__(128) unsigned char cl_smem[];
    cg::cluster_group cl = cg::this_cluster();
    const int r = static_cast<int>(cl.block_rank());
    const int nc = static_cast<int>(cl.num_blocks());
    const int R = g.rows, C = g.cols;
    int c0, c1;
    cluster_slab(C, nc, r, c0, c1);
    const int W = c1 - c0;
    const ClusterSmem lay{R, wmax + 2};
    const long long PE = lay.pop_elems();  // elements of one buffer
    const int P = lay.L * R;               // elements of one direction plane
    T* pop = reinterpret_cast<T*>(cl_smem);
    uint8_t* msk = reinterpret_cast<uint8_t*>(pop + 2 * PE);  // L x R
    uint8_t* bbs = msk + static_cast<long long>(lay.L) * R;   // (L - 2) x R, slab only
    int32_t* oid = reinterpret_cast<int32_t*>(cl_smem + lay.oid_offset<T>());  // slab
    uint32_t* lst = reinterpret_cast<uint32_t*>(oid + lay.slab());              // active nodes: l << 16 | i
    __shared__ int wsum[32];
    __shared__ int wtot;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nthr = blockDim.x * blockDim.y;
    const T* g0 = cur ? f1 : f0;  // the state at step t0 - 1 (buffer 0 here)
    const T* g1 = cur ? f0 : f1;

    // Load the slab and its halo columns: both buffers (inactive nodes hold
    // the initial values in both), masks of all local columns, bounce bytes
    // and open indices of the slab.  A column outside the lattice is never read.
    for (long long e = tid; e < static_cast<long long>(lay.L) * R; e += nthr) {
        const int l = static_cast<int>(e / R), i = static_cast<int>(e - static_cast<long long>(l) * R);
        const int j = c0 - 1 + l;
        if (j < 0 || j >= C || l > W + 1) continue;
        const long long node = static_cast<long long>(j) * g.ld + i;
        const uint8_t m = g.mask[node];
        msk[e] = m;
        if (l >= 1 && l <= W) {
            bbs[e - R] = (m & MASK_PLAIN) ? 0u : g.bb[node];
            oid[e - R] = mask_class(m) == CLS_OPEN ? g.open_idx[node] : -1;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            pop[k * P + e] = g0[k * g.plane + node];
            pop[PE + k * P + e] = g1[k * g.plane + node];
        }
    }
    // neighbours write into this block's halo columns from the first step on
    cl.sync();

    // the neighbours' shared memory (same layout; their slab widths differ by at most one)
    T* left = r > 0 ? cl.map_shared_rank(pop, r - 1) : nullptr;
    T* right = r + 1 < nc ? cl.map_shared_rank(pop, r + 1) : nullptr;
    int lc0, lc1;
    cluster_slab(C, nc, r > 0 ? r - 1 : 0, lc0, lc1);
    const int left_halo = lc1 - lc0 + 1;  // local column of the left neighbour's right halo

    const int n_loc = W * R;
    const int warp = tid >> 5, lane = tid & 31, nwarps = nthr >> 5;
    // The slab's active nodes, column by column (a block-wide compaction):
    // walls and obstacles take no thread, so a slab of up to 1024 active
    // nodes is one node per thread.
    int n_act = 0;
    for (int base = 0; base < n_loc; base += nthr) {
        const int n = base + tid;
        bool a = false;
        unsigned ent = 0;
        if (n < n_loc) {
            const int l = n / R + 1, i = n - (l - 1) * R;
            a = class_active(mask_class(msk[l * R + i]));
            ent = (static_cast<unsigned>(l) << 16) | static_cast<unsigned>(i);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, a);
        if (lane == 0) wsum[warp] = __popc(bal);
        __syncthreads();
        if (warp == 0) {  // exclusive prefix sum of the warps' counts
            const int v = lane < nwarps ? wsum[lane] : 0;
            int x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane < nwarps) wsum[lane] = x - v;
            if (lane == 31) wtot = x;
        }
        __syncthreads();
        if (a) lst[n_act + wsum[warp] + __popc(bal & ((1u << lane) - 1u))] = ent;
        n_act += wtot;
        __syncthreads();  // wsum and wtot are rewritten by the next round
    }

    for (int s = 0; s < steps; ++s) {
        const T* in = pop + (s & 1) * PE;
        T* out = pop + ((s & 1) ^ 1) * PE;
        const long long t = t0 + s;
        for (int base = warp * 32; base < n_act; base += nthr) {
            const int q = base + lane;
            const bool here = q < n_act;
            const unsigned ent = here ? lst[q] : (1u << 16);
            const int l = static_cast<int>(ent >> 16);  // local column
            const int i = static_cast<int>(ent & 0xffffu);
            const int j = c0 + l - 1;                   // global column
            const int e = l * R + i;              // local index
            const uint8_t m = here ? msk[e] : CLS_DEAD;
            const uint8_t cls = mask_class(m);
            const bool act = here && class_active(cls);
            const bool warp_plain = __all_sync(0xffffffffu, !act || (m & MASK_PLAIN));
            bool bad = false;
            if (act) {
                Rt f[9];
                f[0] = M::load(in + e);
                if (warp_plain) {
#pragma unroll
                    for (int k = 1; k < 9; ++k) f[k] = M::load(in + (k * P + e - (DJ(k) * R + DI(k))));
                } else if (i > 0 && j > 0 && i < R - 1 && j < C - 1) {
                    const unsigned b = bbs[e - R];
#pragma unroll
                    for (int k = 1; k < 9; ++k) {
                        const int a = ((b >> (k - 1)) & 1u) ? opp(k) * P + e : k * P + e - (DJ(k) * R + DI(k));
                        f[k] = M::load(in + a);
                    }
                } else {
#pragma unroll
                    for (int k = 1; k < 9; ++k) {
                        const int si = i - DI(k), sj = j - DJ(k);
                        Rt v = M::keep(k);
                        if (si >= 0 && sj >= 0 && si < R && sj < C) {
                            const int se = (l - DJ(k)) * R + si;
                            v = mask_class(msk[se]) == CLS_BB ? M::load(in + (opp(k) * P + e))
                                                              : M::load(in + (k * P + se));
                        }
                        f[k] = v;
                    }
                }
                Rt rr, xr, yr;
                if (cls == CLS_OPEN) {
                    double rho, ux, uy;
                    open_node<M>(ot, oid[e - R], m, t, f, rho, ux, uy);
                    rr = M::from_f64(rho);
                    xr = static_cast<Rt>(ux);
                    yr = static_cast<Rt>(uy);
                } else {
                    M::moments(f, rr, xr, yr);
                    bad = !M::finite(rr);
                }
                M::template collide<COLL>(f, rr, xr, yr, c);
#pragma unroll
                for (int k = 0; k < 9; ++k) M::store(out + (k * P + e), f[k]);
                // populations that leave the slab, into the neighbours' halo columns
                const long long ob = ((s & 1) ^ 1) * PE;
                if (l == W && right) {
                    M::store(right + ob + 1 * P + i, f[1]);
                    M::store(right + ob + 5 * P + i, f[5]);
                    M::store(right + ob + 8 * P + i, f[8]);
                }
                if (l == 1 && left) {
                    const int le = left_halo * R + i;
                    M::store(left + ob + 3 * P + le, f[3]);
                    M::store(left + ob + 6 * P + le, f[6]);
                    M::store(left + ob + 7 * P + le, f[7]);
                }
            }
            if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flags, 1u);
        }
        cl.sync();
    }

    // the state after the last step, back to global memory (the slab only)
    const T* fin_s = pop + (steps & 1) * PE;
    T* dst = ((cur ^ steps) & 1) ? f1 : f0;
    for (int n = tid; n < n_loc; n += nthr) {
        const int l = n / R + 1, i = n - (l - 1) * R;
        const long long node = static_cast<long long>(c0 + l - 1) * g.ld + i;
        const int e = l * R + i;
#pragma unroll
        for (int k = 0; k < 9; ++k) dst[k * g.plane + node] = fin_s[k * P + e];
    }
}

}  // namespace llb

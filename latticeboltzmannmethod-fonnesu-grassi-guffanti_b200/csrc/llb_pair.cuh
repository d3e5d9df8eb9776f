// Two time steps per pass (temporal blocking through shared memory).
//
// A plain step reads 9 populations and writes 9 per active node, so at the
// copy bandwidth the step rate is fixed by the bytes per node.  This kernel
// advances two steps per pass over HBM: for each tile of TI rows x TJ columns
// the producer warp brings f*_{t-1} of the tile plus a two-node halo (all 9
// planes, unshifted) and the node mask plus a three-node halo into a shared
// memory stage with cp.async.bulk.tensor (each CTA loads its own boxes).  The consumer
// warps then
//   A. compute step t for the tile plus a one-node halo, (TI+2) x (TJ+2)
//      nodes, into a shared-memory buffer `mid` (inactive nodes store their
//      initial values there, as dead slots hold them in HBM);
//   B. compute step t+1 for the tile's own nodes from `mid` and store f*_{t+1}
//      to HBM.
// f*_t never reaches HBM, so a pair of steps moves the bytes of one.  The
// halo nodes of step A are computed again by the neighbouring tiles: (TI+2)
// (TJ+2) / (TI TJ) of the step-A work.  Every node update is the per-node
// arithmetic of k_step and k_step_tma in the same order, and `mid` holds the
// storage type T, so results are bit-identical to two single steps.
//
// Box origins: populations at (i0 - HA, j0 - 2), HA = max(2, 16 / sizeof(T))
// so that the TMA x coordinate stays 16-byte aligned (i0 is a multiple of 32),
// BI rows (a multiple of 16 / sizeof(T), so the inner box extent is a multiple
// of 16 bytes) and TJ + 4 columns; mask at (i0 - 16, j0 - 3), TI + 32 rows and
// TJ + 6 columns.  Coordinates outside the tensors read zeros: a zero mask is
// a dead node.
//
// Waits: every mbarrier wait is bounded.  The consumer warps agree on a
// timeout through a shared flag read after a named barrier that every consumer
// warp reaches (each wait before it is bounded), so no warp is left at a
// barrier; on timeout the kernel sets FLAG_TIMEOUT and the producer waits
// (bounded) for the copies it issued before returning.
#pragma once

#include "llb_tma.cuh"

namespace llb {

// CPS: CTAs per SM (the persistent grid is CPS x the SM count).  Two CTAs
// with one stage each let one CTA compute while the other waits for its tile
// or at a phase barrier.
template <typename T, int TI_, int TJ_, int S_, int W_, int CPS_ = 1>
struct PairCfg {
    static constexpr bool PAIR = true;
    static constexpr int CPS = CPS_;
    static constexpr int TI = TI_, TJ = TJ_, S = S_, W = W_;
    static constexpr int A = 16 / static_cast<int>(sizeof(T));     // elements per 16 bytes
    static constexpr int HA = A >= 2 ? A : 2;                       // box rows above the tile
    static constexpr int BI = (HA + TI + 2 + A - 1) / A * A;        // box rows, down to i0 + TI + 1
    static constexpr int BJ = TJ + 4;                               // box columns, j0 - 2 .. j0 + TJ + 1
    static constexpr int BIM = TI + 32;                             // mask rows from i0 - 16
    static constexpr int BJM = TJ + 6;                              // mask columns from j0 - 3
    static constexpr int RI = TI + 2, RJ = TJ + 2;                  // step-A region from (i0 - 1, j0 - 1)
    static constexpr int PLANE_BYTES = round128(BI * BJ * static_cast<int>(sizeof(T)));
    static constexpr int MASK_BYTES = round128(BIM * BJM);
    static constexpr int STAGE_BYTES = 9 * PLANE_BYTES + MASK_BYTES;
    static constexpr unsigned TX_BYTES = 9u * BI * BJ * sizeof(T) + static_cast<unsigned>(BIM * BJM);
    static constexpr int MID_PLANE = RI * RJ;  // elements per plane of mid
    static constexpr int MID_BYTES = round128(9 * MID_PLANE * static_cast<int>(sizeof(T)));
    static constexpr int SMEM_BYTES = S * STAGE_BYTES + MID_BYTES + 2 * S * 8 + 16;
    static constexpr int THREADS = 32 * (W + 1);
    static_assert(TI % 32 == 0 && BI <= 256 && BJ <= 256 && BIM <= 256 && BJM <= 256, "TMA box limits");
    static_assert(SMEM_BYTES <= 232448 && CPS * (SMEM_BYTES + 1024) <= 233472, "shared memory per SM");
};

__device__ __forceinline__ void consumer_barrier(int threads) {
    asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

template <class M, int COLL, class CFG>
__global__ void __launch_bounds__(CFG::THREADS, CFG::CPS)
    k_step_pair(const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap mmap,
                const __grid_constant__ CUtensorMap, Geometry g,
                OpenTable ot, Collision c, const typename M::T* __restrict__ fin, typename M::T* __restrict__ fout,
                StepSync ss) {
    using T = typename M::T;
    using R = typename M::R;
    constexpr int TI = CFG::TI, TJ = CFG::TJ, S = CFG::S, W = CFG::W;
    constexpr int BI = CFG::BI, BIM = CFG::BIM, RI = CFG::RI, HA = CFG::HA, MP = CFG::MID_PLANE;
    extern __shared__ __align__(128) unsigned char smem[];
    T* mid = reinterpret_cast<T*>(smem + S * CFG::STAGE_BYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * CFG::STAGE_BYTES + CFG::MID_BYTES);
    uint64_t* empty = full + S;
    int* abort_flag = reinterpret_cast<int*>(empty + S);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nti = (g.rows + TI - 1) / TI;
    const long long ntiles = static_cast<long long>(nti) * ((g.cols + TJ - 1) / TJ);

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == 0) {
        // ---------------- producer ----------------
        if (lane != 0) return;
        long long n = 0;
        for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++n) {
            const int s = static_cast<int>(n % S);
            const unsigned round = static_cast<unsigned>(n / S);
            if (n >= S && !mbar_wait(&empty[s], (round - 1) & 1u, ss.wait_limit)) {
                atomicOr(ss.flags, FLAG_TIMEOUT);
                break;
            }
            const int i0 = static_cast<int>(tile % nti) * TI, j0 = static_cast<int>(tile / nti) * TJ;
            unsigned char* st = smem + s * CFG::STAGE_BYTES;
            mbar_expect_tx(&full[s], CFG::TX_BYTES);
#pragma unroll
            for (int k = 0; k < 9; ++k) tma_load_3d(st + k * CFG::PLANE_BYTES, &pmap, i0 - HA, j0 - 2, k, &full[s]);
            tma_load_2d(st + 9 * CFG::PLANE_BYTES, &mmap, i0 - 16, j0 - 3, &full[s]);
        }
        // Do not leave with copies in flight: wait for the last fill of every stage.
        const long long issued = n;
        for (int s = 0; s < S && s < issued; ++s) {
            const long long last = issued - 1 - ((issued - 1 - s) % S);
            if (!mbar_wait(&full[s], static_cast<unsigned>(last / S) & 1u)) atomicOr(ss.flags, FLAG_TIMEOUT);
        }
        return;
    }

    // ---------------- consumers ----------------
    const int cw = warp - 1, ct = threadIdx.x - 32;
    const long long t0 = current_step(ss);
    long long n = 0;
    bool bad = false;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++n) {
        const int s = static_cast<int>(n % S);
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&full[s], static_cast<unsigned>(n / S) & 1u, ss.wait_limit));
        if (!ok && lane == 0) *abort_flag = 1;
        consumer_barrier(32 * W);
        if (*abort_flag) {
            if (lane == 0 && !ok) atomicOr(ss.flags, FLAG_TIMEOUT);
            break;
        }
        const int i0 = static_cast<int>(tile % nti) * TI, j0 = static_cast<int>(tile / nti) * TJ;
        const unsigned char* st = smem + s * CFG::STAGE_BYTES;
        const uint8_t* sm = st + 9 * CFG::PLANE_BYTES;
        auto box = [&](int k) { return reinterpret_cast<const T*>(st + k * CFG::PLANE_BYTES); };
        // mask of lattice node (i0 + li, j0 + cj)
        auto mask_at = [&](int li, int cj) { return sm[(cj + 3) * BIM + li + 16]; };

        // ---- A: step t on the tile and a one-node halo, into mid ----
        for (int idx = ct; idx < CFG::RI * CFG::RJ; idx += 32 * W) {
            const int li = idx % RI - 1, cj = idx / RI - 1;
            const int i = i0 + li, j = j0 + cj;
            const uint8_t m = mask_at(li, cj);  // 0 outside the lattice and on padding rows
            const uint8_t cls = mask_class(m);
            T* dst = mid + (cj + 1) * RI + (li + 1);
            if (class_active(cls)) {
                R f[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    // source (li - DI, cj - DJ) of plane k, or this node's own value of
                    // plane opp(k) when the source is a wall or wet obstacle
                    const bool bbk = k > 0 && !(m & MASK_PLAIN) &&
                                     mask_class(mask_at(li - DI(k), cj - DJ(k))) == CLS_BB;
                    const T* p = bbk ? box(opp(k)) + (cj + 2) * BI + li + HA
                                     : box(k) + (cj - DJ(k) + 2) * BI + (li - DI(k)) + HA;
                    f[k] = M::load(p);
                }
                R rr, xr, yr;
                if (cls == CLS_OPEN) {
#pragma unroll
                    for (int k = 1; k < 9; ++k) {
                        const int si = i - DI(k), sj = j - DJ(k);
                        if (si < 0 || sj < 0 || si >= g.rows || sj >= g.cols) f[k] = M::keep(k);
                    }
                    double rho, ux, uy;
                    open_node<M>(ot, g.open_idx[static_cast<long long>(j) * g.ld + i], m, t0, f, rho, ux, uy);
                    rr = M::from_f64(rho);
                    xr = static_cast<R>(ux);
                    yr = static_cast<R>(uy);
                } else {
                    M::moments(f, rr, xr, yr);
                    bad |= !M::finite(rr);
                }
                M::template collide<COLL>(f, rr, xr, yr, c);
#pragma unroll
                for (int k = 0; k < 9; ++k) M::store(dst + k * MP, f[k]);
            } else {
#pragma unroll
                for (int k = 0; k < 9; ++k) M::store(dst + k * MP, M::keep(k));
            }
        }
        consumer_barrier(32 * W);

        // ---- B: step t + 1 on the tile, from mid, to HBM ----
        for (int task = cw; task < (TI / 32) * TJ; task += W) {
            const int li = (task % (TI / 32)) * 32 + lane;
            const int cj = task / (TI / 32);
            const int i = i0 + li, j = j0 + cj;
            const bool inside = i < g.rows && j < g.cols;
            const uint8_t m = mask_at(li, cj);
            const uint8_t cls = mask_class(m);
            const bool write_sector = sector_has_active<M>(class_active(cls));
            const long long node = static_cast<long long>(j) * g.ld + i;
            if (inside && class_active(cls)) {
                R f[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    const bool bbk = k > 0 && !(m & MASK_PLAIN) &&
                                     mask_class(mask_at(li - DI(k), cj - DJ(k))) == CLS_BB;
                    const T* p = bbk ? mid + opp(k) * MP + (cj + 1) * RI + li + 1
                                     : mid + k * MP + (cj - DJ(k) + 1) * RI + (li - DI(k)) + 1;
                    f[k] = M::load(p);
                }
                R rr, xr, yr;
                if (cls == CLS_OPEN) {
#pragma unroll
                    for (int k = 1; k < 9; ++k) {
                        const int si = i - DI(k), sj = j - DJ(k);
                        if (si < 0 || sj < 0 || si >= g.rows || sj >= g.cols) f[k] = M::keep(k);
                    }
                    double rho, ux, uy;
                    open_node<M>(ot, g.open_idx[node], m, t0 + 1, f, rho, ux, uy);
                    rr = M::from_f64(rho);
                    xr = static_cast<R>(ux);
                    yr = static_cast<R>(uy);
                } else {
                    M::moments(f, rr, xr, yr);
                    bad |= !M::finite(rr);
                }
                M::template collide<COLL>(f, rr, xr, yr, c);
#pragma unroll
                for (int k = 0; k < 9; ++k) M::store(fout + k * g.plane + node, f[k]);
            } else if (write_sector && j < g.cols && i < g.ld) {
#pragma unroll
                for (int k = 0; k < 9; ++k) M::store(fout + k * g.plane + node, M::keep(k));
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        consumer_barrier(32 * W);  // mid is rewritten by the next tile's step A
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(ss.flags, 1u);
}

}  // namespace llb

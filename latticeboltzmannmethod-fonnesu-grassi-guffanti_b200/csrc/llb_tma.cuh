// TMA-pipelined step kernel.
//
// The lattice is cut into tiles of TI rows x TJ columns.  Persistent CTAs walk
// the tiles; in each CTA one producer warp streams, for every tile, the 9
// population boxes the tile pulls from (plane k shifted by -c_k) and the tile's
// node-mask with a one-node halo into a ring of S shared-memory stages with
// cp.async.bulk.tensor (each CTA loads its own boxes), completion tracked by mbarriers.
// W consumer warps compute the tile's nodes from shared memory and store the
// new post-collision populations straight to HBM.  The bytes in flight live in
// shared memory instead of registers, so HBM stays busy with few warps.
//
// TMA needs the innermost start coordinate x aligned to 16 bytes.  A plane that
// pulls from row i-1 therefore loads from x = i0 - A (A = 16 / sizeof(T)) and a
// plane that pulls from row i+1 from x = i0; every box is TI + A rows tall and
// the consumer offsets its row index.  Column shifts need no alignment; each
// box is TJ + 1 columns wide, reaching one column toward the tile's own nodes,
// so it holds both the values the tile pulls from plane k and the tile's own
// values of plane k (which a bounce-back source reflects).  A bounce-back is
// then only a different shared-memory address.  Coordinates outside the tensor
// read zeros (a zero mask byte is a dead node).
//
// Every wait is bounded: on timeout the kernel sets bit 1 of the flag word,
// the producer waits (bounded) for the copies it issued, and the CTA returns.
#pragma once

#include <cuda.h>

#include "llb_kernels.cuh"

namespace llb {

constexpr long long WAIT_LIMIT = DEFAULT_WAIT_LIMIT;  // try_wait polls before the drain gives up
constexpr unsigned FLAG_TIMEOUT = 2u;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity to complete, at most `limit`
// polls; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long limit = WAIT_LIMIT) {
    for (long long it = 0; it < limit; ++it)
        if (mbar_test(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

constexpr int round128(int b) { return (b + 127) / 128 * 128; }

// Compile-time layout of one pipeline configuration.
// BBX: the producer also brings the tile's bounce bytes (one byte per node,
// bit k-1 set when direction k's source is a wall or wet obstacle), so a
// non-PLAIN node tests one byte instead of its eight neighbours' masks.
template <typename T, int TI_, int TJ_, int S_, int W_, bool BBX_ = false>
struct TmaCfg {
    static constexpr bool PAIR = false;
    static constexpr bool BBX = BBX_;
    static constexpr int CPS = 1;  // CTAs per SM
    static constexpr int TI = TI_, TJ = TJ_, S = S_, W = W_;
    static constexpr int A = 16 / static_cast<int>(sizeof(T));  // rows per 16 bytes
    static constexpr int BI = TI + A;                           // rows of a population box
    static constexpr int BJ = TJ + 1;                           // columns of a population box
    static constexpr int BIM = TI + 32;                         // rows of the mask box (x0 = i0 - 16)
    static constexpr int BJM = TJ + 2;                          // columns of the mask box (y0 = j0 - 1)
    static constexpr int PLANE_BYTES = round128(BI * BJ * static_cast<int>(sizeof(T)));
    static constexpr int MASK_BYTES = round128(BIM * BJM);
    static constexpr int BB_BYTES = BBX ? round128(TI * TJ) : 0;  // bounce-byte box (x0 = i0, y0 = j0)
    static constexpr int STAGE_BYTES = 9 * PLANE_BYTES + MASK_BYTES + BB_BYTES;
    static constexpr unsigned TX_BYTES =
        9u * BI * BJ * sizeof(T) + static_cast<unsigned>(BIM * BJM) + (BBX ? static_cast<unsigned>(TI * TJ) : 0u);
    static constexpr int SMEM_BYTES = S * STAGE_BYTES + 2 * S * 8;
    static constexpr int THREADS = 32 * (W + 1);
    static_assert(TI % 32 == 0 && BI <= 256 && BIM <= 256 && BJM <= 256, "TMA box limits");
};

// Box of plane k: origin x0 = i0 - A if DI(k) = +1 else i0, y0 = j0 - 1 if
// DJ(k) = +1 else j0.  Element index, inside it, of the value node (li, cj) of
// the tile pulls (source x - c_k) and of the node's own value.
template <class CFG>
__device__ __forceinline__ constexpr int pulled_index(int k, int li, int cj) {
    return (cj + (DJ(k) == -1 ? 1 : 0)) * CFG::BI + li + (DI(k) == 1 ? CFG::A - 1 : (DI(k) == -1 ? 1 : 0));
}
template <class CFG>
__device__ __forceinline__ constexpr int own_index(int k, int li, int cj) {
    return (cj + (DJ(k) == 1 ? 1 : 0)) * CFG::BI + li + (DI(k) == 1 ? CFG::A : 0);
}

template <class M, int COLL, class CFG>
__global__ void __launch_bounds__(CFG::THREADS, 1)
    k_step_tma(const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap mmap,
               const __grid_constant__ CUtensorMap bmap, Geometry g,
               OpenTable ot, Collision c, const typename M::T* __restrict__ fin, typename M::T* __restrict__ fout,
               StepSync ss) {
    using T = typename M::T;
    using R = typename M::R;
    constexpr int TI = CFG::TI, TJ = CFG::TJ, S = CFG::S, W = CFG::W, BIM = CFG::BIM;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * CFG::STAGE_BYTES);
    uint64_t* empty = full + S;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nti = (g.rows + TI - 1) / TI;
    const long long ntiles = static_cast<long long>(nti) * ((g.cols + TJ - 1) / TJ);

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == 0) {
        // ---------------- producer ----------------
        if (lane != 0) return;
        long long n = 0;
        bool ok = true;
        for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++n) {
            const int s = static_cast<int>(n % S);
            const unsigned round = static_cast<unsigned>(n / S);
            if (n >= S && !mbar_wait(&empty[s], (round - 1) & 1u, ss.wait_limit)) {
                atomicOr(ss.flags, FLAG_TIMEOUT);
                ok = false;
                break;
            }
            const int i0 = static_cast<int>(tile % nti) * TI, j0 = static_cast<int>(tile / nti) * TJ;
            unsigned char* st = smem + s * CFG::STAGE_BYTES;
            mbar_expect_tx(&full[s], CFG::TX_BYTES);
#pragma unroll
            for (int k = 0; k < 9; ++k)
                tma_load_3d(st + k * CFG::PLANE_BYTES, &pmap, DI(k) == 1 ? i0 - CFG::A : i0, DJ(k) == 1 ? j0 - 1 : j0,
                            k, &full[s]);
            tma_load_2d(st + 9 * CFG::PLANE_BYTES, &mmap, i0 - 16, j0 - 1, &full[s]);
            if constexpr (CFG::BBX) tma_load_2d(st + 9 * CFG::PLANE_BYTES + CFG::MASK_BYTES, &bmap, i0, j0, &full[s]);
        }
        // Do not leave with copies in flight: wait for the last fill of every stage.
        const long long issued = n;
        for (int s = 0; s < S && s < issued; ++s) {
            const long long last = issued - 1 - ((issued - 1 - s) % S);  // last n that used stage s
            if (!mbar_wait(&full[s], static_cast<unsigned>(last / S) & 1u)) atomicOr(ss.flags, FLAG_TIMEOUT);
        }
        (void)ok;
        return;
    }

    // ---------------- consumers ----------------
    const int cw = warp - 1;
    long long n = 0;
    bool bad = false;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++n) {
        const int s = static_cast<int>(n % S);
        // warp-uniform outcome: the warp's later ballots need every lane
        if (!__all_sync(0xffffffffu, mbar_wait(&full[s], static_cast<unsigned>(n / S) & 1u, ss.wait_limit))) {
            if (lane == 0) atomicOr(ss.flags, FLAG_TIMEOUT);
            break;
        }
        const int i0 = static_cast<int>(tile % nti) * TI, j0 = static_cast<int>(tile / nti) * TJ;
        const unsigned char* st = smem + s * CFG::STAGE_BYTES;
        const uint8_t* sm = st + 9 * CFG::PLANE_BYTES;
        for (int task = cw; task < (TI / 32) * TJ; task += W) {
            const int li = (task % (TI / 32)) * 32 + lane;
            const int cj = task / (TI / 32);
            const int i = i0 + li, j = j0 + cj;
            const bool inside = i < g.rows && j < g.cols;
            const uint8_t m = sm[(cj + 1) * BIM + li + 16];  // 0 outside the lattice
            const uint8_t cls = mask_class(m);
            const bool write_sector = sector_has_active<M>(class_active(cls));
            const long long node = static_cast<long long>(j) * g.ld + i;
            if (inside && class_active(cls)) {
                R f[9];
                auto plane = [&](int k) { return reinterpret_cast<const T*>(st + k * CFG::PLANE_BYTES); };
                if (m & MASK_PLAIN) {
#pragma unroll
                    for (int k = 0; k < 9; ++k) f[k] = M::load(plane(k) + pulled_index<CFG>(k, li, cj));
                } else {
                    f[0] = M::load(plane(0) + pulled_index<CFG>(0, li, cj));
                    [[maybe_unused]] unsigned bbits = 0;
                    if constexpr (CFG::BBX) bbits = (st + 9 * CFG::PLANE_BYTES + CFG::MASK_BYTES)[cj * TI + li];
#pragma unroll
                    for (int k = 1; k < 9; ++k) {
                        // bounce-back source: this node's own value of direction opp(k)
                        bool bb;
                        if constexpr (CFG::BBX) bb = (bbits >> (k - 1)) & 1u;
                        else bb = mask_class(sm[(cj + 1 - DJ(k)) * BIM + li + 16 - DI(k)]) == CLS_BB;
                        const T* p = bb ? plane(opp(k)) + own_index<CFG>(opp(k), li, cj)
                                        : plane(k) + pulled_index<CFG>(k, li, cj);
                        f[k] = M::load(p);
                    }
                }
                R rr, xr, yr;
                if (cls == CLS_OPEN) {
                    // sources outside the lattice (the boxes read zeros there) keep w_k
#pragma unroll
                    for (int k = 1; k < 9; ++k) {
                        const int si = i - DI(k), sj = j - DJ(k);
                        if (si < 0 || sj < 0 || si >= g.rows || sj >= g.cols) f[k] = M::keep(k);
                    }
                    double rho, ux, uy;
                    open_node<M>(ot, g.open_idx[node], m, current_step(ss), f, rho, ux, uy);
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
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(ss.flags, 1u);
}

}  // namespace llb

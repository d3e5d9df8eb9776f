// Launch wrappers for one storage model M (included by llb_f64.cu and llb_lowp.cu).
#pragma once

#include "llb_kernels.cuh"
#include "llb_launch.h"
#include "llb_tma.cuh"
#include "llb_pair.cuh"
#include "llb_batch.cuh"
#include "llb_compact.cuh"
#include "llb_cluster.cuh"

namespace llb {

// Launch of kernel k with programmatic stream serialization (the kernel waits
// for the previous one itself: pdl_wait_then_release).
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

template <class M>
cudaError_t do_step(const LaunchCtx& x, const void* fin, void* fout, bool init, bool macro) {
    using T = typename M::T;
    const int by = x.block_y >= 1 && x.block_y <= BY ? x.block_y : BY;
    const dim3 block(BX, by), grid = node_grid(x.g, BX, by);
    const T* in = static_cast<const T*>(fin);
    T* out = static_cast<T*>(fout);
    // the one-thread-per-node steps overlap their launch with the previous
    // step's drain (small lattices are launch-bound)
#define LLB_STEP(COLL, MAC, INI) \
    return launch_pdl(k_step<M, COLL, MAC, INI>, grid, block, x.stream, x.g, x.ot, x.c, in, out, x.mo, x.ss)
#define LLB_STEP_PS(COLL, MAC, INI) \
    return launch_pdl(k_step<M, COLL, MAC, INI, true>, grid, block, x.stream, x.g, x.ot, x.c, in, out, x.mo, x.ss)
    if constexpr (std::is_same_v<M, ModelF64>) {
        if (x.g.ps) {  // partially saturated obstacles
            if (x.c.model == 0) {
                if (init) { if (macro) LLB_STEP_PS(0, true, true); else LLB_STEP_PS(0, false, true); }
                else { if (macro) LLB_STEP_PS(0, true, false); else LLB_STEP_PS(0, false, false); }
            } else {
                if (init) { if (macro) LLB_STEP_PS(1, true, true); else LLB_STEP_PS(1, false, true); }
                else { if (macro) LLB_STEP_PS(1, true, false); else LLB_STEP_PS(1, false, false); }
            }
            return cudaGetLastError();
        }
    }
#undef LLB_STEP_PS
    if (!init && !macro && x.g.sectors && x.g.n_sectors > 0) {  // plain step over the active-sector list
        const long long threads = static_cast<long long>(x.g.n_sectors) * (LIST_BYTES / static_cast<int>(sizeof(T)));
        const unsigned blocks = static_cast<unsigned>((threads + LIST_BLOCK - 1) / LIST_BLOCK);
        if (x.c.model == 0) k_step_list<M, 0><<<blocks, LIST_BLOCK, 0, x.stream>>>(x.g, x.ot, x.c, in, out, x.mo, x.ss);
        else k_step_list<M, 1><<<blocks, LIST_BLOCK, 0, x.stream>>>(x.g, x.ot, x.c, in, out, x.mo, x.ss);
        return cudaGetLastError();
    }
    if (x.c.model == 0) {
        if (init) { if (macro) LLB_STEP(0, true, true); else LLB_STEP(0, false, true); }
        else { if (macro) LLB_STEP(0, true, false); else LLB_STEP(0, false, false); }
    } else {
        if (init) { if (macro) LLB_STEP(1, true, true); else LLB_STEP(1, false, true); }
        else { if (macro) LLB_STEP(1, true, false); else LLB_STEP(1, false, false); }
    }
#undef LLB_STEP
    return cudaGetLastError();
}

template <class M>
cudaError_t do_step_compact(const LaunchCtx& x, const CompactGeo& cg, const void* fin, void* fout) {
    using T = typename M::T;
    if (cg.n_slots <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((cg.n_slots + COMPACT_BLOCK - 1) / COMPACT_BLOCK);
    const T* in = static_cast<const T*>(fin);
    T* out = static_cast<T*>(fout);
#define LLB_COMPACT(COLL, I) \
    k_step_compact<M, COLL, I><<<blocks, COMPACT_BLOCK, 0, x.stream>>>(x.g, cg, x.ot, x.c, in, out, x.ss)
    if (cg.cplane * 9 < (1LL << 31)) {
        if (x.c.model == 0) LLB_COMPACT(0, int);
        else LLB_COMPACT(1, int);
    } else {
        if (x.c.model == 0) LLB_COMPACT(0, long long);
        else LLB_COMPACT(1, long long);
    }
#undef LLB_COMPACT
    return cudaGetLastError();
}

// Cluster plan of a lattice (llb_cluster.cuh): 16 blocks (8 where a
// non-portable cluster of 16 cannot be placed), slabs of at most wmax
// columns, the shared memory a block needs.  False when the slab and its
// halos do not fit one block's shared memory or no cluster can be placed.
template <class M>
bool do_cluster_plan(int R, int C, int device, ClusterPlan* plan) {
    using T = typename M::T;
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    if (R >= (1 << 16)) return false;  // the active-node list packs rows in 16 bits
    for (int nc : {CLUSTER_MAX_CTAS, 8}) {
        if (C < nc) continue;
        const int wmax = (C + nc - 1) / nc;
        const long long bytes = ClusterSmem{R, wmax + 2}.bytes<T>();
        if (bytes > optin) continue;
        bool ok = true;
        for (auto k : {k_step_cluster<M, 0>, k_step_cluster<M, 1>}) {
            // the most the device allows next to the kernel's static shared
            // memory, so launches of every lattice's plan are valid
            cudaFuncAttributes fa{};
            if (cudaFuncGetAttributes(&fa, k) != cudaSuccess ||
                bytes + static_cast<long long>(fa.sharedSizeBytes) > optin ||
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     optin - static_cast<int>(fa.sharedSizeBytes)) != cudaSuccess ||
                (nc > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
                ok = false;
                break;
            }
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(nc);
            cfg.blockDim = dim3(BX, CLUSTER_THREADS / BX);
            cfg.dynamicSmemBytes = static_cast<size_t>(bytes);
            cudaLaunchAttribute at;
            at.id = cudaLaunchAttributeClusterDimension;
            at.val.clusterDim.x = nc;
            at.val.clusterDim.y = 1;
            at.val.clusterDim.z = 1;
            cfg.attrs = &at;
            cfg.numAttrs = 1;
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess || n < 1) {
                ok = false;
                break;
            }
        }
        (void)cudaGetLastError();  // a refused size is a plan that does not exist, not an error
        if (ok) {
            plan->nc = nc;
            plan->wmax = wmax;
            plan->smem = bytes;
            return true;
        }
    }
    return false;
}

// `steps` plain steps in one launch of one cluster.
template <class M>
cudaError_t do_step_cluster(const LaunchCtx& x, const ClusterPlan& p, void* f0, void* f1, int cur, long long t0,
                            int steps) {
    using T = typename M::T;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.nc);
    cfg.blockDim = dim3(BX, CLUSTER_THREADS / BX);
    cfg.dynamicSmemBytes = static_cast<size_t>(p.smem);
    cfg.stream = x.stream;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = p.nc;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    T* a = static_cast<T*>(f0);
    T* b = static_cast<T*>(f1);
    if (x.c.model == 0)
        return cudaLaunchKernelEx(&cfg, k_step_cluster<M, 0>, x.g, x.ot, x.c, a, b, cur, t0, steps, x.ss.flags, p.wmax);
    return cudaLaunchKernelEx(&cfg, k_step_cluster<M, 1>, x.g, x.ot, x.c, a, b, cur, t0, steps, x.ss.flags, p.wmax);
}

template <class M>
cudaError_t do_compact_copy(const LaunchCtx& x, const CompactGeo& cg, void* dense, void* comp, bool to_compact) {
    using T = typename M::T;
    if (cg.n_chunks <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((static_cast<long long>(cg.n_chunks) * 32 + COMPACT_BLOCK - 1) / COMPACT_BLOCK);
    T* d = static_cast<T*>(dense);
    T* c = static_cast<T*>(comp);
    if (to_compact) k_compact_copy<M, true><<<blocks, COMPACT_BLOCK, 0, x.stream>>>(x.g, cg, d, c);
    else k_compact_copy<M, false><<<blocks, COMPACT_BLOCK, 0, x.stream>>>(x.g, cg, d, c);
    return cudaGetLastError();
}

template <class M>
cudaError_t do_fill_keep(const LaunchCtx& x, void* buf) {
    k_fill_keep<M><<<1024, 256, 0, x.stream>>>(static_cast<typename M::T*>(buf), x.g.plane);
    return cudaGetLastError();
}

template <class M>
cudaError_t do_finalize(const LaunchCtx& x, const void* fin, double* out, long long t) {
    k_finalize<M><<<node_grid(x.g, BX, BY), dim3(BX, BY), 0, x.stream>>>(
        x.g, x.ot, static_cast<const typename M::T*>(fin), out, t);
    return cudaGetLastError();
}

template <class M>
cudaError_t do_export(const LaunchCtx& x, const void* fin, double* out) {
    k_export<M><<<node_grid(x.g, BX, BY), dim3(BX, BY), 0, x.stream>>>(x.g, static_cast<const typename M::T*>(fin), out);
    return cudaGetLastError();
}

template <class M>
cudaError_t do_mass(const LaunchCtx& x, const void* fin, double2* partials, int nblocks, double* out3) {
    k_mass_momentum<M><<<nblocks, 256, 0, x.stream>>>(x.g, static_cast<const typename M::T*>(fin), partials);
    k_reduce_partials<3><<<1, 32, 0, x.stream>>>(partials, nblocks, out3);
    return cudaGetLastError();
}

template <class M>
cudaError_t do_forces(const LaunchCtx& x, const void* fin, const int64_t* pts, const uint16_t* dirs, long long n,
                      double2* partials, int nblocks, double* out2) {
    k_flow_forces<M><<<nblocks, 256, 0, x.stream>>>(x.g, static_cast<const typename M::T*>(fin), pts, dirs, n, partials);
    k_reduce_partials<2><<<1, 32, 0, x.stream>>>(partials, nblocks, out2);
    return cudaGetLastError();
}

template <class M>
cudaError_t do_gather(const LaunchCtx& x, const void* fin, const int64_t* pts, const uint16_t* dirs, long long n,
                      double* out) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    k_gather_forces<M><<<blocks, 256, 0, x.stream>>>(x.g, static_cast<const typename M::T*>(fin), pts, dirs, n, out);
    return cudaGetLastError();
}

// ---- TMA-pipelined step -------------------------------------------------------
template <class M, class CFG>
void fill_plan(int cfg, TmaPlan* p) {
    p->cfg = cfg;
    p->pair = CFG::PAIR;
    p->ctas_per_sm = CFG::CPS;
    if constexpr (!CFG::PAIR) p->bbx = CFG::BBX;
    p->TI = CFG::TI;
    p->TJ = CFG::TJ;
    p->S = CFG::S;
    p->W = CFG::W;
    p->BI = CFG::BI;
    p->BJ = CFG::BJ;
    p->BIM = CFG::BIM;
    p->BJM = CFG::BJM;
    p->smem = CFG::SMEM_BYTES;
    p->threads = CFG::THREADS;
}

template <class M, class CFG>
cudaError_t do_step_tma(const LaunchCtx& x, const CUtensorMap* pmap, const CUtensorMap* mmap,
                        const CUtensorMap* bmap, const void* fin, void* fout, int grid) {
    using T = typename M::T;
    auto k0 = k_step_tma<M, 0, CFG>;
    auto k1 = k_step_tma<M, 1, CFG>;
    auto kern = x.c.model == 0 ? k0 : k1;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CFG::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    kern<<<grid, CFG::THREADS, CFG::SMEM_BYTES, x.stream>>>(*pmap, *mmap, *bmap, x.g, x.ot, x.c,
                                                             static_cast<const T*>(fin), static_cast<T*>(fout), x.ss);
    return cudaGetLastError();
}

template <class M, class CFG>
cudaError_t do_step_pair(const LaunchCtx& x, const CUtensorMap* pmap, const CUtensorMap* mmap,
                         const CUtensorMap* bmap, const void* fin, void* fout, int grid) {
    using T = typename M::T;
    auto k0 = k_step_pair<M, 0, CFG>;
    auto k1 = k_step_pair<M, 1, CFG>;
    auto kern = x.c.model == 0 ? k0 : k1;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CFG::SMEM_BYTES);
    // CFG::CPS CTAs of this kernel share an SM's shared memory
    if (e == cudaSuccess && CFG::CPS > 1)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    kern<<<grid, CFG::THREADS, CFG::SMEM_BYTES, x.stream>>>(*pmap, *mmap, *bmap, x.g, x.ot, x.c,
                                                             static_cast<const T*>(fin), static_cast<T*>(fout), x.ss);
    return cudaGetLastError();
}

// ---- batched step ----------------------------------------------------------------
template <class M>
cudaError_t do_batch_step(const BatchLaunch& b) {
    const dim3 block(BX, b.block_y);
    auto kern = k_batch_step<M>;
    if (!b.cooperative) {
        // one step: a block per item, dense tiles and compacted slot blocks in
        // launches of their own
        if (b.n_dense > 0) k_batch_tiles<M><<<b.n_dense, block, 0, b.stream>>>(b.lats, b.items, b.sbase, b.soff);
        if (b.n_items > b.n_dense)
            k_batch_slots<M><<<b.n_items - b.n_dense, block, 0, b.stream>>>(b.lats, b.items + b.n_dense, b.sbase,
                                                                            b.soff);
        return cudaGetLastError();
    }
    const BatchLattice* lats = b.lats;
    const int2* items = b.items;
    int n_items = b.n_items;
    const long long* sbase = b.sbase;
    long long soff = b.soff;
    int steps = b.steps;
    unsigned* bar = b.bar;
    unsigned* err = b.err;
    long long bar_limit = b.bar_limit;
    void* args[] = {&lats, &items, &n_items, &sbase, &soff, &steps, &bar, &err, &bar_limit};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kern), dim3(b.grid), block, args, 0, b.stream);
}

template <class M>
int do_batch_max_grid(int block_y, int sm_count) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_step<M>, BX * block_y, 0) != cudaSuccess)
        return 0;
    return per_sm * sm_count;
}

template <class M>
cudaError_t do_macro_now(const LaunchCtx& x, const void* fin, long long t, double* rho, double* u) {
    k_macro_now<M><<<node_grid(x.g, BX, BY), dim3(BX, BY), 0, x.stream>>>(
        x.g, x.ot, static_cast<const typename M::T*>(fin), t, rho, u);
    return cudaGetLastError();
}

}  // namespace llb

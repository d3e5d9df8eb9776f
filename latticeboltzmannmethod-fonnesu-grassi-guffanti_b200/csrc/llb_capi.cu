// C ABI of libllalbm_cuda.so (declared in include/llalbm_cuda.h).
//
// A handle owns one lattice on one device: its CUDA stream, the node mask, the
// resident populations (two buffers, ping-pong), the open-boundary value ring,
// output buffers and a device step counter.  Multi-step calls are replayed from
// CUDA graphs of GRAPH_STEPS kernels (one graph per buffer parity).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/llalbm_cuda.h"
#include "llb_handle.h"
#include "llb_launch.h"

using namespace llb;

namespace {

constexpr int GRAPH_STEPS = 32;  // even: a replay returns the state to the same buffer
thread_local std::string g_last_error;

}  // namespace


namespace {

int fail(llb_handle h, int code, const std::string& msg) {
    g_last_error = msg;
    if (h) h->err = msg;
    return code;
}

int cuda_fail(llb_handle h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(h, e == cudaErrorMemoryAllocation ? LLB_E_NOMEM : LLB_E_CUDA, m);
}

#define LLB_CUDA(h, call)                                   \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

// Device memory of lattices comes from a stream-ordered pool per device that
// the library owns.  A lattice's buffers are allocated and freed in the order
// of its stream (cudaMallocFromPoolAsync / cudaFreeAsync), so retiring a
// lattice never synchronises the device -- cudaFree can, and a solve server
// retiring lattices would stall every other lattice's kernels -- and the pool
// keeps freed memory for the next lattice rather than returning it to the
// driver at each synchronisation.
constexpr int MAX_POOL_DEVICES = 64;
cudaMemPool_t lattice_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[MAX_POOL_DEVICES] = {};
    if (device < 0 || device >= MAX_POOL_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = pool;
    }
    return pools[device];
}

template <typename T>
int dev_alloc(llb_handle h, T** p, size_t bytes) {
    cudaMemPool_t pool = lattice_pool(h->device);
    if (!pool) return fail(h, LLB_E_CUDA, "device memory pool unavailable");
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMallocFromPoolAsync");
    h->bytes += static_cast<int64_t>(bytes);
    return LLB_OK;
}

// Returns a buffer to the pool in the order of the handle's stream.
void dev_free(llb_handle h, void* p) {
    if (p) cudaFreeAsync(p, h->stream);
}

int select_device(llb_handle h) {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
    return LLB_OK;
}

LaunchCtx make_ctx(llb_handle h) {
    LaunchCtx x{};
    x.g.rows = static_cast<int>(h->R);
    x.g.cols = static_cast<int>(h->C);
    x.g.ld = h->ld;
    x.g.plane = h->plane;
    x.g.mask = h->d_mask;
    x.g.bb = h->d_bb;
    x.g.ps = h->d_ps;
    x.g.psb = h->d_psb;
    x.g.open_idx = h->d_open_idx;
    x.g.sectors = h->tma_cfg == PIPE_LIST ? h->d_sectors : nullptr;
    x.g.smask = h->d_smask;
    x.g.sbb = h->d_sbb;
    x.g.n_sectors = h->n_sectors;
    x.ot.vals = h->d_open;
    x.ot.n_open = h->n_open;
    x.ot.cap = h->cap;
    x.c = h->coll;
    x.mo.rho = h->d_rho;
    x.mo.u = h->d_u;
    x.ss.tbase = nullptr;
    x.ss.t_off = h->step;
    x.ss.flags = h->d_flags;
    x.ss.wait_limit = h->wait_limit;
    x.stream = h->stream;
    x.block_y = h->block_y;
    return x;
}

void release(llb_handle h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& g : h->graph)
        if (g) cudaGraphExecDestroy(g);
    void* bufs[] = {h->f[0], h->f[1], h->d_mask, h->d_bb, h->d_ps, h->d_psb, h->d_sectors, h->d_smask, h->d_sbb, h->d_open_idx, h->d_open, h->d_rho, h->d_u, h->d_dense,
                    h->d_step, h->d_flags, h->d_partials, h->d_red, h->d_fpts, h->d_fdirs, h->d_gather,
                    h->cf[0], h->cf[1], h->d_cnb, h->d_cseg, h->d_cchunk, h->d_ccol, h->d_cinfo};
    for (void* b : bufs) dev_free(h, b);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : h->flag_ev)
        if (e) cudaEventDestroy(e);
    if (h->h_flags) cudaFreeHost(h->h_flags);
    if (h->stream && h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
}

// ---------------------------------------------------------------------------
// node mask
// ---------------------------------------------------------------------------
constexpr uint8_t UNSET = 0xff;

int build_mask(const llb_desc* d, int ld, std::vector<uint8_t>& mask, std::vector<uint8_t>& bb,
               std::vector<uint8_t>& ps, std::vector<double>& psb, std::vector<int32_t>& open_idx,
               int64_t& n_nonplain, std::string& why) {
    const int64_t R = d->rows, C = d->cols;
    const bool partial = d->obstacle_bc == LLB_OBSTACLE_PARTIAL;
    // provisional codes in a grid with a one-node border of UNSET, so that
    // neighbour lookups need no bounds checks: 1 fluid, 2 wall/obstacle,
    // 3 inlet, 4 outlet, 5 partially saturated obstacle
    const int64_t P = R + 2;
    std::vector<uint8_t> cls(static_cast<size_t>(P * (C + 2)), UNSET);
    auto cell = [&](int64_t i, int64_t j) -> uint8_t& { return cls[static_cast<size_t>((i + 1) + P * (j + 1))]; };
    auto mark = [&](const int64_t* ij, int64_t n, uint8_t c, const char* name) -> bool {
        if (n > 0 && !ij) { why = std::string(name) + " list is NULL"; return false; }
        for (int64_t q = 0; q < n; ++q) {
            const int64_t i = ij[2 * q], j = ij[2 * q + 1];
            if (i < 0 || j < 0 || i >= R || j >= C) { why = std::string(name) + " node out of range"; return false; }
            uint8_t& s = cell(i, j);
            if (s != UNSET) { why = std::string(name) + " node also listed as another node kind"; return false; }
            s = c;
        }
        return true;
    };
    if (!mark(d->fluid_ij, d->n_fluid, 1, "fluid") || !mark(d->wall_ij, d->n_wall, 2, "wall") ||
        !mark(d->inlet_ij, d->n_inlet, 3, "inlet") || !mark(d->outlet_ij, d->n_outlet, 4, "outlet") ||
        !mark(d->obstacle_ij, d->n_obstacle, partial ? 5 : 2, "obstacle"))
        return LLB_E_GEOMETRY;
    auto active = [](uint8_t c) { return c == 1 || c == 3 || c == 4; };
    // offset in the bordered grid of the source x - c_k of direction k
    int64_t src_off[9];
    for (int k = 0; k < 9; ++k) src_off[k] = -(DI(k) + P * DJ(k));
    // The reference streams fluid nodes without bounds checks; a fluid node on
    // the lattice edge would write outside its tensors.
    for (int64_t q = 0; q < d->n_fluid; ++q) {
        const int64_t i = d->fluid_ij[2 * q], j = d->fluid_ij[2 * q + 1];
        if (i == 0 || j == 0 || i == R - 1 || j == C - 1) {
            why = "fluid node on the lattice edge (the reference streams it out of bounds)";
            return LLB_E_GEOMETRY;
        }
    }
    // obstacle direction bits must be the reference's rule (bit k iff x + c_k active)
    if (d->obstacle_dirs) {
        for (int64_t q = 0; q < d->n_obstacle; ++q) {
            const int64_t i = d->obstacle_ij[2 * q], j = d->obstacle_ij[2 * q + 1];
            const uint8_t* x = &cell(i, j);
            uint16_t b = 0;
            for (int k = 1; k < 9; ++k)
                if (active(x[-src_off[k]])) b |= static_cast<uint16_t>(1u << k);
            if (b != (d->obstacle_dirs[q] & 0x1feu)) {
                why = "obstacle direction bits differ from the neighbour rule of identify_obstacle_propagation";
                return LLB_E_UNSUPPORTED;
            }
        }
    }
    n_nonplain = 0;
    mask.assign(static_cast<size_t>(ld) * C, 0);
    bb.assign(static_cast<size_t>(ld) * C, 0);
    open_idx.assign(static_cast<size_t>(ld) * C, -1);
    if (partial) {
        ps.assign(static_cast<size_t>(ld) * C, 0);
        psb.assign(static_cast<size_t>(ld) * C, 1.0);
        for (int64_t q = 0; q < d->n_obstacle; ++q) {
            const double b = d->obstacle_b ? d->obstacle_b[q] : 1.0;
            if (!(b >= 0.0 && b <= 1.0)) { why = "obstacle b outside [0, 1]"; return LLB_E_INVALID; }
            psb[static_cast<size_t>(d->obstacle_ij[2 * q + 1] * ld + d->obstacle_ij[2 * q])] = b;
        }
    }
    auto side_code = [](int32_t bt) { return (bt >= 1 && bt <= 4) ? bt : SIDE_NONE; };
    static constexpr uint8_t kClass[6] = {CLS_DEAD, CLS_FLUID, CLS_BB, CLS_OPEN, CLS_OPEN, CLS_BB};
    for (int64_t j = 0; j < C; ++j) {
        const uint8_t* col = &cell(0, j);
        uint8_t* mcol = mask.data() + static_cast<size_t>(j * ld);
        uint8_t* bcol = bb.data() + static_cast<size_t>(j * ld);
        for (int64_t i = 0; i < R; ++i) {
            const uint8_t c = col[i];
            if (c == UNSET) continue;  // dead: mask and bounce bits stay 0
            uint8_t m = kClass[c];
            if (active(c)) {
                const uint8_t* x = col + i;
                bool plain = true;
                uint8_t b = 0, p = 0;
                for (int k = 1; k < 9; ++k) {
                    const uint8_t sk = x[src_off[k]];
                    plain &= active(sk);
                    b |= static_cast<uint8_t>((sk == 2) << (k - 1));
                    p |= static_cast<uint8_t>((sk == 5) << (k - 1));
                }
                if (plain) m |= MASK_PLAIN;
                else ++n_nonplain;
                bcol[i] = b;
                if (partial) ps[static_cast<size_t>(j * ld + i)] = p;
            }
            mcol[i] = m;
        }
    }
    auto set_open = [&](const int64_t* ij, const int32_t* side, int64_t n, int bc, int base) {
        for (int64_t q = 0; q < n; ++q) {
            const int64_t i = ij[2 * q], j = ij[2 * q + 1];
            const size_t x = static_cast<size_t>(j * ld + i);
            const int s = side ? side_code(side[q]) : SIDE_NONE;
            mask[x] = static_cast<uint8_t>((mask[x] & 7u) | (s << SIDE_SHIFT) | (bc << BC_SHIFT));
            open_idx[x] = static_cast<int32_t>(base + q);
        }
    };
    set_open(d->inlet_ij, d->inlet_side, d->n_inlet, d->inlet_bc, 0);
    set_open(d->outlet_ij, d->outlet_side, d->n_outlet, d->outlet_bc, static_cast<int>(d->n_inlet));
    return LLB_OK;
}

int ensure_partials(llb_handle h, int nblocks) {
    if (h->partial_blocks >= nblocks) return LLB_OK;
    if (h->d_partials) { dev_free(h, h->d_partials); h->d_partials = nullptr; }
    int rc = dev_alloc(h, &h->d_partials, sizeof(double2) * 3 * static_cast<size_t>(nblocks));
    if (rc) return rc;
    h->partial_blocks = nblocks;
    return LLB_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    // looked up once; lattices may be created from several threads
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return nullptr;
    }();
    return fn;
}

// Tensor maps of the two population buffers, (ld, C, 9) elements with boxes
// of BI x BJ x 1, and of the mask, (ld, C) bytes with boxes of BIM x BJM.
int build_maps(llb_handle h) {
    if (h->maps_ready) return LLB_OK;
    if (!tma_plan(h->storage, h->tma_cfg, &h->plan)) return fail(h, LLB_E_INVALID, "unknown pipeline configuration");
    auto enc = tensor_map_encoder();
    if (!enc) return fail(h, LLB_E_CUDA, "cuTensorMapEncodeTiled unavailable");
    const CUtensorMapDataType dt = h->storage == LLB_STORE_F64   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                   : h->storage == LLB_STORE_F32S ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(h->ld), static_cast<cuuint64_t>(h->C), 9};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(h->ld) * h->elem, static_cast<cuuint64_t>(h->plane) * h->elem};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(h->plan.BI), static_cast<cuuint32_t>(h->plan.BJ), 1};
    const cuuint32_t es[3] = {1, 1, 1};
    for (int b = 0; b < 2; ++b) {
        CUresult r = enc(&h->pmap[b], dt, 3, h->f[b], dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(h, LLB_E_CUDA, "cuTensorMapEncodeTiled (populations) failed");
    }
    const cuuint64_t mdims[2] = {static_cast<cuuint64_t>(h->ld), static_cast<cuuint64_t>(h->C)};
    const cuuint64_t mstrides[1] = {static_cast<cuuint64_t>(h->ld)};
    const cuuint32_t mbox[2] = {static_cast<cuuint32_t>(h->plan.BIM), static_cast<cuuint32_t>(h->plan.BJM)};
    CUresult r = enc(&h->mmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, h->d_mask, mdims, mstrides, mbox, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(h, LLB_E_CUDA, "cuTensorMapEncodeTiled (mask) failed");
    // bounce bytes, (ld, C) bytes with boxes of TI x TJ (a copy of the mask map
    // when the configuration does not load them: the kernel never reads it)
    h->bmap = h->mmap;
    if (h->plan.bbx) {
        const cuuint32_t bbox[2] = {static_cast<cuuint32_t>(h->plan.TI), static_cast<cuuint32_t>(h->plan.TJ)};
        r = enc(&h->bmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, h->d_bb, mdims, mstrides, bbox, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(h, LLB_E_CUDA, "cuTensorMapEncodeTiled (bounce bytes) failed");
    }
    h->maps_ready = true;
    return LLB_OK;
}

// Steps one plain-step launch advances: 2 for the two-step configurations.
int steps_per_launch(llb_handle h) {
    TmaPlan p;
    return h->tma_cfg >= 0 && tma_plan(h->storage, h->tma_cfg, &p) && p.pair ? 2 : 1;
}

// ---------------------------------------------------------------------------
// column-compacted storage (pipeline PIPE_COMPACT)
// ---------------------------------------------------------------------------
CompactGeo compact_geo(llb_handle h) {
    CompactGeo cg{};
    cg.info = h->d_cinfo;
    cg.nb = h->d_cnb;
    cg.seg = h->d_cseg;
    cg.chunk = h->d_cchunk;
    cg.col = h->d_ccol;
    cg.nseg = h->cnseg;
    cg.n_chunks = h->c_chunks;
    cg.n_slots = h->c_slots;
    cg.cplane = h->cplane;
    return cg;
}

// The state's copy in the dense planes, after steps on the compacted ones.
int state_to_dense(llb_handle h) {
    if (h->where != RES_COMPACT) return LLB_OK;
    cudaError_t e = launch_compact_copy(h->storage, make_ctx(h), compact_geo(h), h->f[h->cur], h->cf[h->cur], false);
    if (e != cudaSuccess) return cuda_fail(h, e, "compacted-to-dense copy");
    h->where = RES_BOTH;
    return LLB_OK;
}

// The state's copy in the compacted planes, before compacted steps.
int state_to_compact(llb_handle h) {
    if (h->where != RES_DENSE) return LLB_OK;
    cudaError_t e = launch_compact_copy(h->storage, make_ctx(h), compact_geo(h), h->f[h->cur], h->cf[h->cur], true);
    if (e != cudaSuccess) return cuda_fail(h, e, "dense-to-compacted copy");
    h->where = RES_BOTH;
    return LLB_OK;
}

void release_compact(llb_handle h) {
    for (void* p : {h->cf[0], h->cf[1], static_cast<void*>(h->d_cnb), static_cast<void*>(h->d_cseg),
                    static_cast<void*>(h->d_cchunk), static_cast<void*>(h->d_ccol), static_cast<void*>(h->d_cinfo)})
        dev_free(h, p);
    h->cf[0] = h->cf[1] = nullptr;
    h->d_cnb = nullptr;
    h->d_cseg = nullptr;
    h->d_cchunk = nullptr;
    h->d_ccol = nullptr;
    h->d_cinfo = nullptr;
    h->bytes -= h->compact_bytes;
    h->compact_bytes = 0;
    h->c_chunks = 0;
    h->cplane = 0;
    h->c_slots = 0;
}

// Compacted planes and their tables from the node mask and bounce bytes
// (dense (j * ld + i) layout).  Slots are taken column by column, rows in
// order; each column's run is padded to a whole 32-byte sector.
int build_compact_from(llb_handle h, const std::vector<uint8_t>& mask, const std::vector<uint8_t>& bb) {
    if (h->d_cseg) return LLB_OK;
    if (h->d_ps) return fail(h, LLB_E_UNSUPPORTED, "partially saturated obstacles run on the one-thread-per-node kernel");
    const int64_t R = h->R, C = h->C, ld = h->ld;
    const int64_t nseg = (R + 31) / 32;
    const int64_t pad = 32 / static_cast<int64_t>(h->elem);
    std::vector<int2> seg(static_cast<size_t>(C * nseg));
    std::vector<int32_t> col(static_cast<size_t>(C + 1));
    std::vector<uint16_t> info;
    info.reserve(static_cast<size_t>(h->n_active + C * pad));
    std::vector<int2> chunks;
    int64_t t = 0;
    for (int64_t j = 0; j < C; ++j) {
        if (t + R + pad >= (int64_t{1} << 31))
            return fail(h, LLB_E_UNSUPPORTED, "compacted planes need fewer than 2^31 slots");
        col[static_cast<size_t>(j)] = static_cast<int32_t>(t);
        int64_t in_col = 0;
        for (int64_t s = 0; s < nseg; ++s) {
            uint32_t m = 0;
            const int64_t t_seg = t;
            for (int64_t r = 0; r < 32 && 32 * s + r < R; ++r) {
                const int64_t i = 32 * s + r;
                const uint8_t mk = mask[static_cast<size_t>(j * ld + i)];
                if (!class_active(mask_class(mk))) continue;
                m |= 1u << r;
                uint8_t mb = mk;
                if (mask_class(mk) == CLS_FLUID && !(mk & MASK_PLAIN)) {
                    // fluid nodes never lie on the lattice edge: every source is in range
                    for (int k = 1; k < 9; ++k) {
                        const int64_t si = i - DI(k), sj = j - DJ(k);
                        if (mask_class(mask[static_cast<size_t>(sj * ld + si)]) == CLS_DEAD) mb |= COMPACT_DEAD_SRC;
                    }
                }
                info.push_back(static_cast<uint16_t>(mb | (bb[static_cast<size_t>(j * ld + i)] << 8)));
                if (in_col % 32 == 0) chunks.push_back(make_int2(static_cast<int>(j), static_cast<int>(i)));
                ++in_col;
                ++t;
            }
            seg[static_cast<size_t>(j * nseg + s)] = make_int2(static_cast<int>(m), static_cast<int>(t_seg));
        }
        while (t % pad) {
            info.push_back(0);
            ++t;
        }
    }
    col[static_cast<size_t>(C)] = static_cast<int32_t>(t);
    if (chunks.empty()) return fail(h, LLB_E_UNSUPPORTED, "no active node");
    if (static_cast<uint64_t>(ld) * static_cast<uint64_t>(C) > 0xffffffffull)
        return fail(h, LLB_E_UNSUPPORTED, "compacted planes need fewer than 2^32 dense slots per plane");
    // neighbour offsets of every slot (dense index for nodes whose pull tests each source)
    auto slot_at = [&](int64_t j, int64_t i) -> int64_t {
        const int2 e = seg[static_cast<size_t>(j * nseg + (i >> 5))];
        const uint32_t below_i = (i & 31) ? (static_cast<uint32_t>(e.x) & ((1u << (i & 31)) - 1u)) : 0u;
        return e.y + __builtin_popcount(below_i);
    };
    std::vector<uint32_t> nb(info.size(), 0);
    for (int64_t j = 0; j < C; ++j) {
        int64_t q = col[static_cast<size_t>(j)];
        for (int64_t i = 0; i < R; ++i) {
            const uint8_t mk = mask[static_cast<size_t>(j * ld + i)];
            if (!class_active(mask_class(mk))) continue;
            const uint8_t mb = static_cast<uint8_t>(info[static_cast<size_t>(q)] & 0xffu);
            if (mask_class(mk) == CLS_OPEN || (mb & COMPACT_DEAD_SRC)) {
                nb[static_cast<size_t>(q)] = static_cast<uint32_t>(j * ld + i);
            } else {
                const int64_t dl = q - slot_at(j - 1, i), dr = slot_at(j + 1, i) - q;
                if (dl < 0 || dl > 0xffff || dr < 0 || dr > 0xffff)
                    return fail(h, LLB_E_UNSUPPORTED, "compacted planes: neighbour columns more than 65535 slots apart");
                nb[static_cast<size_t>(q)] = static_cast<uint32_t>(dl) | (static_cast<uint32_t>(dr) << 16);
            }
            ++q;
        }
    }
    const int64_t align = 256 / static_cast<int64_t>(h->elem);
    const long long cplane = static_cast<long long>((t + align - 1) / align * align);
    const int64_t before = h->bytes;
    void* cf0 = nullptr;
    void* cf1 = nullptr;
    int2 *d_seg = nullptr, *d_chunk = nullptr;
    int32_t* d_col = nullptr;
    uint16_t* d_info = nullptr;
    uint32_t* d_nb = nullptr;
    const size_t pbytes = static_cast<size_t>(cplane) * 9 * h->elem;
    int rc = dev_alloc(h, &cf0, pbytes);
    if (!rc) rc = dev_alloc(h, &cf1, pbytes);
    if (!rc) rc = dev_alloc(h, &d_seg, seg.size() * sizeof(int2));
    if (!rc) rc = dev_alloc(h, &d_chunk, chunks.size() * sizeof(int2));
    if (!rc) rc = dev_alloc(h, &d_col, col.size() * sizeof(int32_t));
    if (!rc) rc = dev_alloc(h, &d_info, info.size() * sizeof(uint16_t));
    if (!rc) rc = dev_alloc(h, &d_nb, nb.size() * sizeof(uint32_t));
    cudaError_t e = cudaSuccess;
    if (!rc) e = cudaMemcpyAsync(d_seg, seg.data(), seg.size() * sizeof(int2), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpyAsync(d_chunk, chunks.data(), chunks.size() * sizeof(int2), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpyAsync(d_col, col.data(), col.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpyAsync(d_info, info.data(), info.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpyAsync(d_nb, nb.data(), nb.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(h, e, "compacted-plane tables upload");
    if (rc) {
        for (void* p : {cf0, cf1, static_cast<void*>(d_seg), static_cast<void*>(d_chunk), static_cast<void*>(d_col),
                        static_cast<void*>(d_info), static_cast<void*>(d_nb)})
            dev_free(h, p);
        h->bytes = before;
        return rc;
    }
    h->cf[0] = cf0;
    h->cf[1] = cf1;
    h->d_cseg = d_seg;
    h->d_cchunk = d_chunk;
    h->d_ccol = d_col;
    h->d_cinfo = d_info;
    h->d_cnb = d_nb;
    h->c_slots = static_cast<long long>(t);
    h->cnseg = static_cast<int>(nseg);
    h->c_chunks = static_cast<int>(chunks.size());
    h->cplane = cplane;
    h->compact_bytes = h->bytes - before;
    return LLB_OK;
}

// As above, with the mask and bounce bytes read back from the device.
int build_compact(llb_handle h) {
    if (h->d_cseg) return LLB_OK;
    const size_t n = static_cast<size_t>(h->ld) * h->C;
    std::vector<uint8_t> mask(n), bb(n);
    LLB_CUDA(h, cudaMemcpyAsync(mask.data(), h->d_mask, n, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaMemcpyAsync(bb.data(), h->d_bb, n, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return build_compact_from(h, mask, bb);
}

// Whether the lattice fits one thread-block cluster (looked up once).
bool cluster_ok(llb_handle h) {
    if (h->cl_state == 0)
        h->cl_state = (!h->d_ps && cluster_plan(h->storage, static_cast<int>(h->R), static_cast<int>(h->C), h->device,
                                                &h->cl_plan))
                          ? 1
                          : -1;
    return h->cl_state > 0;
}

// One step kernel (two steps for a two-step configuration unless `single`).
// Inside a graph capture the step index is relative (graph_offset >= 0, base
// read from d_step); otherwise it is absolute.
int launch_one(llb_handle h, bool macro, long long graph_offset = -1, bool single = false) {
    LaunchCtx x = make_ctx(h);
    if (graph_offset >= 0) {
        x.ss.tbase = h->d_step;
        x.ss.t_off = graph_offset;
    }
    if (!macro && h->tma_cfg == PIPE_COMPACT) {
        cudaError_t e = launch_step_compact(h->storage, x, compact_geo(h), h->cf[h->cur], h->cf[h->cur ^ 1]);
        if (e != cudaSuccess) return cuda_fail(h, e, "compacted step kernel launch");
        h->cur ^= 1;
        ++h->step;
        return LLB_OK;
    }
    if (!macro && h->tma_cfg >= 0) {
        int rc = build_maps(h);
        if (rc) return rc;
        if (!(h->plan.pair && single)) {
            const long long ntiles =
                ((h->R + h->plan.TI - 1) / h->plan.TI) * ((h->C + h->plan.TJ - 1) / h->plan.TJ);
            const int grid = static_cast<int>(std::min<long long>(ntiles, static_cast<long long>(h->sm_count) * h->plan.ctas_per_sm));
            cudaError_t e = launch_step_tma(h->storage, h->plan, x, &h->pmap[h->cur], &h->mmap, &h->bmap,
                                            h->f[h->cur], h->f[h->cur ^ 1], grid);
            if (e != cudaSuccess) return cuda_fail(h, e, "pipelined step kernel launch");
            h->cur ^= 1;
            h->step += h->plan.pair ? 2 : 1;
            return LLB_OK;
        }
        // a lone step of a two-step configuration: the one-thread-per-node kernel
    }
    cudaError_t e = launch_step(h->storage, x, h->f[h->cur], h->f[h->cur ^ 1], false, macro);
    if (e != cudaSuccess) return cuda_fail(h, e, "step kernel launch");
    h->cur ^= 1;
    ++h->step;
    return LLB_OK;
}

int graph_for(llb_handle h, cudaGraphExec_t* out) {
    if (h->graph[h->cur]) { *out = h->graph[h->cur]; return LLB_OK; }
    const int cur0 = h->cur;
    const int64_t step0 = h->step;
    cudaGraph_t g = nullptr;
    LLB_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = LLB_OK;
    const int per = steps_per_launch(h);
    for (int s = 0; s < GRAPH_STEPS && rc == LLB_OK; s += per) rc = launch_one(h, false, s);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->cur = cur0;
    h->step = step0;
    if (rc != LLB_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&h->graph[cur0], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    *out = h->graph[cur0];
    return LLB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// dispatch to the storage-specific translation units
// ---------------------------------------------------------------------------
namespace llb {
cudaError_t launch_step(int s, const LaunchCtx& x, const void* fin, void* fout, bool init, bool macro) {
    return s == LLB_STORE_F64 ? launch_step_f64(x, fin, fout, init, macro) : launch_step_lowp(s, x, fin, fout, init, macro);
}
cudaError_t launch_batch_step(int s, const BatchLaunch& b) {
    return s == LLB_STORE_F64 ? launch_batch_step_f64(b) : launch_batch_step_lowp(s, b);
}
int batch_max_grid(int s, int block_y, int sm_count) {
    return s == LLB_STORE_F64 ? batch_max_grid_f64(block_y, sm_count) : batch_max_grid_lowp(s, block_y, sm_count);
}
cudaError_t launch_macro_now(int s, const LaunchCtx& x, const void* fin, long long t, double* rho, double* u) {
    return s == LLB_STORE_F64 ? launch_macro_now_f64(x, fin, t, rho, u) : launch_macro_now_lowp(s, x, fin, t, rho, u);
}
bool cluster_plan(int s, int R, int C, int device, ClusterPlan* plan) {
    return s == LLB_STORE_F64 ? cluster_plan_f64(R, C, device, plan) : cluster_plan_lowp(s, R, C, device, plan);
}
cudaError_t launch_step_cluster(int s, const LaunchCtx& x, const ClusterPlan& p, void* f0, void* f1, int cur,
                                long long t0, int steps) {
    return s == LLB_STORE_F64 ? launch_step_cluster_f64(x, p, f0, f1, cur, t0, steps)
                              : launch_step_cluster_lowp(s, x, p, f0, f1, cur, t0, steps);
}
cudaError_t launch_step_compact(int s, const LaunchCtx& x, const CompactGeo& cg, const void* fin, void* fout) {
    return s == LLB_STORE_F64 ? launch_step_compact_f64(x, cg, fin, fout) : launch_step_compact_lowp(s, x, cg, fin, fout);
}
cudaError_t launch_compact_copy(int s, const LaunchCtx& x, const CompactGeo& cg, void* dense, void* comp, bool to_compact) {
    return s == LLB_STORE_F64 ? launch_compact_copy_f64(x, cg, dense, comp, to_compact)
                              : launch_compact_copy_lowp(s, x, cg, dense, comp, to_compact);
}
cudaError_t launch_fill_keep(int s, const LaunchCtx& x, void* buf) {
    return s == LLB_STORE_F64 ? launch_fill_keep_f64(x, buf) : launch_fill_keep_lowp(s, x, buf);
}
cudaError_t launch_finalize(int s, const LaunchCtx& x, const void* fin, double* out, long long t) {
    return s == LLB_STORE_F64 ? launch_finalize_f64(x, fin, out, t) : launch_finalize_lowp(s, x, fin, out, t);
}
cudaError_t launch_export(int s, const LaunchCtx& x, const void* fin, double* out) {
    return s == LLB_STORE_F64 ? launch_export_f64(x, fin, out) : launch_export_lowp(s, x, fin, out);
}
cudaError_t launch_mass_momentum(int s, const LaunchCtx& x, const void* fin, double2* p, int nb, double* out3) {
    return s == LLB_STORE_F64 ? launch_mass_momentum_f64(x, fin, p, nb, out3) : launch_mass_momentum_lowp(s, x, fin, p, nb, out3);
}
cudaError_t launch_flow_forces(int s, const LaunchCtx& x, const void* fin, const int64_t* pts, const uint16_t* dirs,
                               long long n, double2* p, int nb, double* out2) {
    return s == LLB_STORE_F64 ? launch_flow_forces_f64(x, fin, pts, dirs, n, p, nb, out2)
                              : launch_flow_forces_lowp(s, x, fin, pts, dirs, n, p, nb, out2);
}
bool tma_plan(int s, int cfg, TmaPlan* out) {
    return s == LLB_STORE_F64 ? tma_plan_f64(cfg, out) : tma_plan_lowp(s, cfg, out);
}
cudaError_t launch_step_tma(int s, const TmaPlan& p, const LaunchCtx& x, const CUtensorMap* pm, const CUtensorMap* mm,
                            const CUtensorMap* bm, const void* fin, void* fout, int grid) {
    return s == LLB_STORE_F64 ? launch_step_tma_f64(p, x, pm, mm, bm, fin, fout, grid)
                              : launch_step_tma_lowp(s, p, x, pm, mm, bm, fin, fout, grid);
}
cudaError_t launch_gather_forces(int s, const LaunchCtx& x, const void* fin, const int64_t* pts, const uint16_t* dirs,
                                 long long n, double* out) {
    return s == LLB_STORE_F64 ? launch_gather_forces_f64(x, fin, pts, dirs, n, out)
                              : launch_gather_forces_lowp(s, x, fin, pts, dirs, n, out);
}
}  // namespace llb

// Hooks for llb_noalloc.cu: the launch context of a handle's resident state
// (with its device made current) and its error reporting.
namespace llb {
int handle_force_context(llb_handle h, LaunchCtx* ctx, const void** fin, double** d_out, int* storage,
                         int* device, int64_t* rows, int64_t* cols) {
    if (!h->initialized) return fail(h, LLB_E_STATE, "lattice not initialised");
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    *ctx = make_ctx(h);
    *fin = h->f[h->cur];
    *d_out = h->d_red;
    *storage = h->storage;
    *device = h->device;
    *rows = h->R;
    *cols = h->C;
    return LLB_OK;
}
int handle_fail(llb_handle h, int code, const char* msg) { return fail(h, code, msg); }
LaunchCtx handle_ctx(llb_handle h) { return make_ctx(h); }
int handle_dense_state(llb_handle h) { return state_to_dense(h); }
int handle_prepare_compact(llb_handle h) {
    int rc = select_device(h);
    if (rc) return rc;
    if (h->d_ps) return LLB_E_UNSUPPORTED;
    rc = build_compact(h);
    if (rc != LLB_OK) h->err.clear();
    return rc;
}
int handle_batch_layout(llb_handle h, bool compact) {
    int rc = select_device(h);
    if (rc) return rc;
    return compact ? state_to_compact(h) : state_to_dense(h);
}
void handle_batch_stepped(llb_handle h, bool compact) { h->where = compact ? RES_COMPACT : RES_DENSE; }
CompactGeo handle_compact_geo(llb_handle h) { return compact_geo(h); }
int handle_leave_compact(llb_handle h) {
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    h->where = RES_DENSE;
    if (h->tma_cfg != PIPE_COMPACT) return LLB_OK;
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    for (auto& g : h->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    h->tma_cfg = default_dense_pipeline(*h);
    h->maps_ready = false;
    release_compact(h);
    return LLB_OK;
}
}  // namespace llb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int llb_abi_version(void) { return LLB_ABI_VERSION; }

const char* llb_last_error(llb_handle h) { return h ? h->err.c_str() : g_last_error.c_str(); }

int llb_create(const llb_desc* d, llb_handle* out) {
    if (!d || !out) return fail(nullptr, LLB_E_INVALID, "null descriptor or output");
    *out = nullptr;
    if (d->rows < 3 || d->cols < 3 || d->rows > (1 << 30) || d->cols > (1 << 30) || d->rows * d->cols > (1LL << 36))
        return fail(nullptr, LLB_E_INVALID, "lattice dimensions out of range");
    if (d->n_fluid < 0 || d->n_wall < 0 || d->n_inlet < 0 || d->n_outlet < 0 || d->n_obstacle < 0)
        return fail(nullptr, LLB_E_INVALID, "negative node count");
    if (d->collision != LLB_BGK && d->collision != LLB_TRT) return fail(nullptr, LLB_E_INVALID, "bad collision");
    if (d->storage < LLB_STORE_F64 || d->storage > LLB_STORE_F16S) return fail(nullptr, LLB_E_INVALID, "bad storage");
    if (d->pattern != LLB_PATTERN_AB && d->pattern != LLB_PATTERN_AA) return fail(nullptr, LLB_E_INVALID, "bad pattern");
    if (d->pattern == LLB_PATTERN_AA) return fail(nullptr, LLB_E_UNSUPPORTED, "A-A pattern not available in this build");
    for (int bc : {d->inlet_bc, d->outlet_bc})
        if (bc < LLB_BC_ZH_VELOCITY || bc > LLB_BC_ZH_PRESSURE) return fail(nullptr, LLB_E_INVALID, "bad boundary policy");
    if (d->collision == LLB_BGK && !(d->tau > 0.0)) return fail(nullptr, LLB_E_INVALID, "tau must be > 0");
    if (d->collision == LLB_TRT && !(d->tau_even > 0.0 && d->tau_odd > 0.0))
        return fail(nullptr, LLB_E_INVALID, "tau_even and tau_odd must be > 0");
    if (d->obstacle_bc != LLB_OBSTACLE_BOUNCE_BACK && d->obstacle_bc != LLB_OBSTACLE_PARTIAL)
        return fail(nullptr, LLB_E_INVALID, "bad obstacle policy");
    if (d->obstacle_bc == LLB_OBSTACLE_PARTIAL) {
        if (!(d->ps_tau > 0.0)) return fail(nullptr, LLB_E_INVALID, "ps_tau must be > 0");
        if (d->storage != LLB_STORE_F64)
            return fail(nullptr, LLB_E_UNSUPPORTED, "partially saturated obstacles need FP64 storage");
    }
    const int64_t n_open = d->n_inlet + d->n_outlet;
    if (n_open > (1LL << 30)) return fail(nullptr, LLB_E_INVALID, "too many open nodes");
    const int cap = d->open_table_rows <= 0 ? 1 : d->open_table_rows;

    llb_handle h = new (std::nothrow) llb_lattice();
    if (!h) return fail(nullptr, LLB_E_NOMEM, "host allocation failed");
    h->device = d->device;
    h->storage = d->storage;
    h->pattern = d->pattern;
    h->R = d->rows;
    h->C = d->cols;
    h->elem = d->storage == LLB_STORE_F64 ? 8 : (d->storage == LLB_STORE_F32S ? 4 : 2);
    const int align = static_cast<int>(256 / h->elem);  // every column starts 256-byte aligned
    h->ld = static_cast<int>((d->rows + align - 1) / align * align);
    h->plane = static_cast<long long>(h->ld) * d->cols;
    h->n_open = static_cast<int>(n_open);
    h->cap = cap;
    if (d->collision == LLB_BGK) {
        h->coll.model = 0;
        h->coll.t = 1.0 / d->tau;  // BGKCollision.hpp:142-143
        h->coll.omt = 1.0 - h->coll.t;
    } else {
        h->coll.model = 1;
        h->coll.ie = 1.0 / d->tau_even;  // TRTCollision.hpp:155-188
        h->coll.he = 0.5 * (1.0 / d->tau_even);
        h->coll.ho = 0.5 * (1.0 / d->tau_odd);
    }
    h->coll.tf = static_cast<float>(h->coll.t);
    h->coll.omtf = static_cast<float>(h->coll.omt);
    h->coll.ief = static_cast<float>(h->coll.ie);
    h->coll.hef = static_cast<float>(h->coll.he);
    h->coll.hof = static_cast<float>(h->coll.ho);
    if (d->obstacle_bc == LLB_OBSTACLE_PARTIAL) h->coll.ps_t = 1.0 / d->ps_tau;  // PSBounceBackPolicy.hpp:200

    std::vector<uint8_t> mask, bb, ps;
    std::vector<double> psb;
    std::vector<int32_t> open_idx;
    std::string why;
    int rc = build_mask(d, h->ld, mask, bb, ps, psb, open_idx, h->n_nonplain, why);
    if (rc != LLB_OK) { delete h; return fail(nullptr, rc, why); }
    h->n_active = d->n_fluid + d->n_inlet + d->n_outlet;
    {
        constexpr int64_t SEG = 32;  // rows of a warp of the batch's dense tiles
        const int64_t nti = (h->R + SEG - 1) / SEG;
        h->plain_seg.assign(static_cast<size_t>(nti * h->C), 0);
        for (int64_t j = 0; j < h->C; ++j)
            for (int64_t ti = 0; ti < nti; ++ti) {
                bool ok = (ti + 1) * SEG <= h->R;
                for (int64_t i = ti * SEG; ok && i < (ti + 1) * SEG; ++i) {
                    const uint8_t m = mask[static_cast<size_t>(j * h->ld + i)];
                    ok = mask_class(m) == CLS_FLUID && (m & MASK_PLAIN);
                }
                h->plain_seg[static_cast<size_t>(j * nti + ti)] = ok ? 1 : 0;
            }
    }
    h->tma_cfg = default_pipeline(*h);
    if (!ps.empty()) h->tma_cfg = -1;  // partially saturated obstacles: one thread per node only
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { delete h; return fail(nullptr, LLB_E_NODEVICE, "no CUDA device"); }
    if (d->device < 0 || d->device >= ndev) { delete h; return fail(nullptr, LLB_E_NODEVICE, "device ordinal out of range"); }

    auto bail = [&](int code) { std::string m = h->err; release(h); return fail(nullptr, code, m); };
    if ((rc = select_device(h))) return bail(rc);
    if (h->tma_cfg == PIPE_GRID && ps.empty() && cluster_default_size(*h) && cluster_ok(h))
        h->tma_cfg = PIPE_CLUSTER;
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaStreamCreate"));
    e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
    if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaDeviceGetAttribute"));
    const size_t pop_bytes = static_cast<size_t>(h->plane) * 9 * h->elem;
    const size_t N = static_cast<size_t>(h->R * h->C);
    if ((rc = dev_alloc(h, &h->f[0], pop_bytes)) || (rc = dev_alloc(h, &h->f[1], pop_bytes)) ||
        (rc = dev_alloc(h, &h->d_mask, mask.size())) || (rc = dev_alloc(h, &h->d_bb, bb.size())) ||
        (rc = dev_alloc(h, &h->d_open_idx, open_idx.size() * sizeof(int32_t))) ||
        (rc = dev_alloc(h, &h->d_open, sizeof(double2) * static_cast<size_t>(std::max<int64_t>(n_open, 1)) * cap)) ||
        (rc = dev_alloc(h, &h->d_rho, sizeof(double) * N)) || (rc = dev_alloc(h, &h->d_u, sizeof(double) * 2 * N)) ||
        (rc = dev_alloc(h, &h->d_step, sizeof(long long))) || (rc = dev_alloc(h, &h->d_flags, sizeof(unsigned))) || (rc = dev_alloc(h, &h->d_red, sizeof(double) * 4)))
        return bail(rc);
    if (!ps.empty() && ((rc = dev_alloc(h, &h->d_ps, ps.size())) || (rc = dev_alloc(h, &h->d_psb, psb.size() * sizeof(double)))))
        return bail(rc);
    e = cudaMemcpyAsync(h->d_mask, mask.data(), mask.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && h->d_ps)
        e = cudaMemcpyAsync(h->d_ps, ps.data(), ps.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && h->d_psb)
        e = cudaMemcpyAsync(h->d_psb, psb.data(), psb.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_bb, bb.data(), bb.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->d_open_idx, open_idx.data(), open_idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(h->d_open, 0, sizeof(double2) * static_cast<size_t>(std::max<int64_t>(n_open, 1)) * cap, h->stream);
    // every slot starts at its direction's initial value: dead nodes keep it
    if (e == cudaSuccess) e = launch_fill_keep(h->storage, make_ctx(h), h->f[0]);
    if (e == cudaSuccess) e = launch_fill_keep(h->storage, make_ctx(h), h->f[1]);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return bail(cuda_fail(h, e, "lattice upload"));
    if (h->tma_cfg == PIPE_COMPACT && build_compact_from(h, mask, bb) != LLB_OK) {
        // the dense kernels serve every lattice: fall back to their default
        h->tma_cfg = default_dense_pipeline(*h);
        h->err.clear();
    }
    *out = h;
    return LLB_OK;
}

int llb_destroy(llb_handle h) {
    if (!h) return fail(nullptr, LLB_E_INVALID, "null handle");
    release(h);
    return LLB_OK;
}

int llb_set_open_values(llb_handle h, int64_t t_first, int32_t count, const double* values) {
    if (!h || t_first < 0 || count < 0) return fail(h, LLB_E_INVALID, "bad arguments");
    if (h->n_open == 0 || count == 0) return LLB_OK;
    if (!values) return fail(h, LLB_E_INVALID, "null values");
    if (count > h->cap) return fail(h, LLB_E_INVALID, "more rows than the open-value ring holds");
    int rc = select_device(h);
    if (rc) return rc;
    const size_t row = sizeof(double2) * static_cast<size_t>(h->n_open);
    int32_t r = 0;
    while (r < count) {
        const int64_t slot = (t_first + r) % h->cap;
        const int32_t run = static_cast<int32_t>(std::min<int64_t>(count - r, h->cap - slot));
        LLB_CUDA(h, cudaMemcpyAsync(reinterpret_cast<char*>(h->d_open) + slot * row,
                                    reinterpret_cast<const char*>(values) + static_cast<size_t>(r) * row, row * run,
                                    cudaMemcpyHostToDevice, h->stream));
        r += run;
    }
    return LLB_OK;
}

int llb_init(llb_handle h, uint32_t flags) {
    if (!h) return fail(nullptr, LLB_E_INVALID, "null handle");
    int rc = select_device(h);
    if (rc) return rc;
    h->cur = 0;
    h->step = 0;
    LaunchCtx x = make_ctx(h);
    const bool macro = (flags & LLB_STEP_MACRO) != 0;
    cudaError_t e = launch_step(h->storage, x, nullptr, h->f[0], true, macro);
    if (e != cudaSuccess) return cuda_fail(h, e, "init kernel launch");
    h->step = 1;
    h->initialized = true;
    h->macro_valid = macro;
    h->where = RES_DENSE;
    return LLB_OK;
}

int llb_step(llb_handle h, int32_t nsteps, uint32_t flags) {
    if (!h || nsteps < 0) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "llb_step before llb_init");
    if (nsteps == 0) return LLB_OK;
    int rc = select_device(h);
    if (rc) return rc;
    const bool macro = (flags & LLB_STEP_MACRO) != 0;
    int32_t plain = macro ? nsteps - 1 : nsteps;
    const bool compact = h->tma_cfg == PIPE_COMPACT;
    if (plain > 0 && (rc = compact ? state_to_compact(h) : state_to_dense(h))) return rc;
    if (plain > 0) h->where = compact ? RES_COMPACT : RES_DENSE;  // where the steps below leave it
    if (plain >= GRAPH_STEPS && h->tma_cfg != PIPE_CLUSTER) {
        cudaGraphExec_t g = nullptr;
        if ((rc = graph_for(h, &g))) return rc;
        while (plain >= GRAPH_STEPS) {
            // the replay's step base; a pageable source is staged at call time
            LLB_CUDA(h, cudaMemcpyAsync(h->d_step, &h->step, sizeof(long long), cudaMemcpyHostToDevice, h->stream));
            LLB_CUDA(h, cudaGraphLaunch(g, h->stream));
            h->step += GRAPH_STEPS;
            plain -= GRAPH_STEPS;
        }
    }
    if (h->tma_cfg == PIPE_CLUSTER) {
        // chunks of steps, each one launch of the cluster
        while (plain > 0) {
            const int n = std::min<int32_t>(plain, CLUSTER_CHUNK);
            cudaError_t e =
                launch_step_cluster(h->storage, make_ctx(h), h->cl_plan, h->f[0], h->f[1], h->cur, h->step, n);
            if (e != cudaSuccess) return cuda_fail(h, e, "cluster step kernel launch");
            h->cur ^= n & 1;
            h->step += n;
            plain -= n;
        }
    }
    const int per = steps_per_launch(h);
    for (; plain >= per; plain -= per)
        if ((rc = launch_one(h, false))) return rc;
    if (plain > 0 && (rc = launch_one(h, false, -1, true))) return rc;
    if (macro) {
        // output steps write rho and u from the dense kernel
        if ((rc = state_to_dense(h))) return rc;
        if ((rc = launch_one(h, true))) return rc;
        h->where = RES_DENSE;
        h->macro_valid = true;
    }
    return LLB_OK;
}

int llb_get_step(llb_handle h, int64_t* step) {
    if (!h || !step) return fail(h, LLB_E_INVALID, "bad arguments");
    *step = h->step;
    return LLB_OK;
}

int llb_get_macro(llb_handle h, double* rho, double* u) {
    if (!h) return fail(nullptr, LLB_E_INVALID, "null handle");
    if (!h->macro_valid) return fail(h, LLB_E_STATE, "no step has written rho/u yet");
    int rc = select_device(h);
    if (rc) return rc;
    const size_t N = static_cast<size_t>(h->R * h->C);
    if (rho) LLB_CUDA(h, cudaMemcpyAsync(rho, h->d_rho, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    if (u) LLB_CUDA(h, cudaMemcpyAsync(u, h->d_u, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

int llb_compute_macro(llb_handle h, double* rho, double* u) {
    if (!h || (!rho && !u)) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "lattice not initialised");
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    LaunchCtx x = make_ctx(h);
    cudaError_t e = launch_macro_now(h->storage, x, h->f[h->cur], h->step, h->d_rho, h->d_u);
    if (e != cudaSuccess) return cuda_fail(h, e, "macro kernel launch");
    const size_t N = static_cast<size_t>(h->R * h->C);
    if (rho) LLB_CUDA(h, cudaMemcpyAsync(rho, h->d_rho, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    if (u) LLB_CUDA(h, cudaMemcpyAsync(u, h->d_u, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

static int dense_out(llb_handle h, double* host, bool finalize) {
    if (!h || !host) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "lattice not initialised");
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    const size_t bytes = sizeof(double) * 9 * static_cast<size_t>(h->R * h->C);
    if (!h->d_dense && (rc = dev_alloc(h, &h->d_dense, bytes))) return rc;
    LaunchCtx x = make_ctx(h);
    cudaError_t e = finalize ? launch_finalize(h->storage, x, h->f[h->cur], h->d_dense, h->step)
                             : launch_export(h->storage, x, h->f[h->cur], h->d_dense);
    if (e != cudaSuccess) return cuda_fail(h, e, "export kernel launch");
    LLB_CUDA(h, cudaMemcpyAsync(host, h->d_dense, bytes, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

int llb_get_populations(llb_handle h, double* populations) { return dense_out(h, populations, true); }
int llb_get_post_collision(llb_handle h, double* populations) { return dense_out(h, populations, false); }

int llb_set_force_points(llb_handle h, const int64_t* ij, const uint16_t* dirs, int64_t n) {
    if (!h || n < 0 || (n > 0 && (!ij || !dirs))) return fail(h, LLB_E_INVALID, "bad arguments");
    for (int64_t q = 0; q < n; ++q)
        if (ij[2 * q] < 0 || ij[2 * q + 1] < 0 || ij[2 * q] >= h->R || ij[2 * q + 1] >= h->C)
            return fail(h, LLB_E_INVALID, "force point out of range");
    int rc = select_device(h);
    if (rc) return rc;
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    for (void* p : {static_cast<void*>(h->d_fpts), static_cast<void*>(h->d_fdirs), static_cast<void*>(h->d_gather)})
        dev_free(h, p);
    h->d_fpts = nullptr;
    h->d_fdirs = nullptr;
    h->d_gather = nullptr;
    h->n_fpts = n;
    if (n == 0) return LLB_OK;
    if ((rc = dev_alloc(h, &h->d_fpts, sizeof(int64_t) * 2 * n)) || (rc = dev_alloc(h, &h->d_fdirs, sizeof(uint16_t) * n)) ||
        (rc = dev_alloc(h, &h->d_gather, sizeof(double) * 8 * n)))
        return rc;
    LLB_CUDA(h, cudaMemcpyAsync(h->d_fpts, ij, sizeof(int64_t) * 2 * n, cudaMemcpyHostToDevice, h->stream));
    LLB_CUDA(h, cudaMemcpyAsync(h->d_fdirs, dirs, sizeof(uint16_t) * n, cudaMemcpyHostToDevice, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

int llb_flow_forces(llb_handle h, double lift_drag[2]) {
    if (!h || !lift_drag) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "lattice not initialised");
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    const int nb = force_blocks(h->n_fpts);
    if ((rc = ensure_partials(h, nb))) return rc;
    LaunchCtx x = make_ctx(h);
    cudaError_t e = launch_flow_forces(h->storage, x, h->f[h->cur], h->d_fpts, h->d_fdirs, h->n_fpts, h->d_partials, nb, h->d_red);
    if (e != cudaSuccess) return cuda_fail(h, e, "force kernel launch");
    LLB_CUDA(h, cudaMemcpyAsync(lift_drag, h->d_red, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

int llb_gather_force_inputs(llb_handle h, double* values) {
    if (!h || (h->n_fpts > 0 && !values)) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "lattice not initialised");
    if (h->n_fpts == 0) return LLB_OK;
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    LaunchCtx x = make_ctx(h);
    cudaError_t e = launch_gather_forces(h->storage, x, h->f[h->cur], h->d_fpts, h->d_fdirs, h->n_fpts, h->d_gather);
    if (e != cudaSuccess) return cuda_fail(h, e, "gather kernel launch");
    LLB_CUDA(h, cudaMemcpyAsync(values, h->d_gather, sizeof(double) * 8 * h->n_fpts, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

int llb_mass_momentum(llb_handle h, double out[3]) {
    if (!h || !out) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "lattice not initialised");
    int rc = select_device(h);
    if (rc) return rc;
    if ((rc = state_to_dense(h))) return rc;
    const int64_t N = h->R * h->C;
    const int nb = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(148 * 8, (N + 255) / 256)));
    if ((rc = ensure_partials(h, nb))) return rc;
    LaunchCtx x = make_ctx(h);
    cudaError_t e = launch_mass_momentum(h->storage, x, h->f[h->cur], h->d_partials, nb, h->d_red);
    if (e != cudaSuccess) return cuda_fail(h, e, "reduction kernel launch");
    LLB_CUDA(h, cudaMemcpyAsync(out, h->d_red, sizeof(double) * 3, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

int llb_synchronize(llb_handle h) {
    if (!h) return fail(nullptr, LLB_E_INVALID, "null handle");
    int rc = select_device(h);
    if (rc) return rc;
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return LLB_OK;
}

// The flag word's meaning, shared by the whole and the split checks.
static int numerics_status(llb_handle h, unsigned flags) {
    if (flags & 2u) return fail(h, LLB_E_TIMEOUT, "a pipelined step kernel gave up waiting for its copies");
    if (flags & 1u) return fail(h, LLB_E_NUMERIC, "non-finite density detected");
    return LLB_OK;
}

int llb_check_numerics(llb_handle h) {
    if (!h) return fail(nullptr, LLB_E_INVALID, "null handle");
    int rc = select_device(h);
    if (rc) return rc;
    unsigned flags = 0;
    LLB_CUDA(h, cudaMemcpyAsync(&flags, h->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned), h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    return numerics_status(h, flags);
}

int llb_check_numerics_begin(llb_handle h, int32_t slot) {
    if (!h || slot < 0 || slot >= 8) return fail(h, LLB_E_INVALID, "bad arguments");
    int rc = select_device(h);
    if (rc) return rc;
    if (!h->h_flags) LLB_CUDA(h, cudaHostAlloc(reinterpret_cast<void**>(&h->h_flags), 8 * sizeof(unsigned), cudaHostAllocDefault));
    if (!h->flag_ev[slot]) LLB_CUDA(h, cudaEventCreateWithFlags(&h->flag_ev[slot], cudaEventDisableTiming));
    LLB_CUDA(h, cudaMemcpyAsync(&h->h_flags[slot], h->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned), h->stream));
    LLB_CUDA(h, cudaEventRecord(h->flag_ev[slot], h->stream));
    return LLB_OK;
}

int llb_check_numerics_end(llb_handle h, int32_t slot) {
    if (!h || slot < 0 || slot >= 8) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->flag_ev[slot]) return fail(h, LLB_E_STATE, "no llb_check_numerics_begin on this slot");
    int rc = select_device(h);
    if (rc) return rc;
    LLB_CUDA(h, cudaEventSynchronize(h->flag_ev[slot]));
    return numerics_status(h, h->h_flags[slot]);
}

int llb_event_record(llb_handle h, int32_t slot) {
    if (!h || slot < 0 || slot >= 8) return fail(h, LLB_E_INVALID, "bad arguments");
    int rc = select_device(h);
    if (rc) return rc;
    if (!h->ev[slot]) LLB_CUDA(h, cudaEventCreate(&h->ev[slot]));
    LLB_CUDA(h, cudaEventRecord(h->ev[slot], h->stream));
    return LLB_OK;
}

int llb_event_elapsed_ms(llb_handle h, int32_t a, int32_t b, float* ms) {
    if (!h || !ms || a < 0 || a >= 8 || b < 0 || b >= 8 || !h->ev[a] || !h->ev[b])
        return fail(h, LLB_E_INVALID, "bad arguments");
    int rc = select_device(h);
    if (rc) return rc;
    LLB_CUDA(h, cudaEventSynchronize(h->ev[b]));
    LLB_CUDA(h, cudaEventElapsedTime(ms, h->ev[a], h->ev[b]));
    return LLB_OK;
}

// The active-sector list of a lattice (built on first use): every 32-byte
// sector of a population plane holding an active node, ordered by tiles of
// 32 rows x 8 columns (the one-thread grid's block) and column by column
// inside a tile, with the mask and bounce bytes of the listed nodes.
static int build_sector_list(llb_handle h) {
    if (h->d_sectors) return LLB_OK;
    if (h->d_ps) return fail(h, LLB_E_UNSUPPORTED, "partially saturated obstacles run on the one-thread-per-node kernel");
    if (static_cast<int64_t>(h->ld) * h->C >= (1LL << 31))
        return fail(h, LLB_E_UNSUPPORTED, "no active-sector list for 2^31 or more slots per plane");
    const size_t n = static_cast<size_t>(h->ld) * h->C;
    std::vector<uint8_t> mask(n), bb(n);
    LLB_CUDA(h, cudaMemcpyAsync(mask.data(), h->d_mask, n, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaMemcpyAsync(bb.data(), h->d_bb, n, cudaMemcpyDeviceToHost, h->stream));
    LLB_CUDA(h, cudaStreamSynchronize(h->stream));
    const int64_t SN = LIST_BYTES / static_cast<int64_t>(h->elem), ld = h->ld;
    std::vector<int32_t> sectors;
    for (int64_t j0 = 0; j0 < h->C; j0 += 8)
        for (int64_t i0 = 0; i0 < ld; i0 += 32)
            for (int64_t j = j0; j < std::min<int64_t>(j0 + 8, h->C); ++j)
                for (int64_t base = j * ld + i0; base < j * ld + std::min<int64_t>(i0 + 32, ld); base += SN) {
                    bool any = false;
                    for (int64_t q = 0; q < SN; ++q) any |= class_active(mask_class(mask[static_cast<size_t>(base + q)]));
                    if (any) sectors.push_back(static_cast<int32_t>(base / SN));
                }
    if (sectors.empty()) return fail(h, LLB_E_UNSUPPORTED, "no active node");
    std::vector<uint8_t> smask(sectors.size() * SN), sbb(sectors.size() * SN);
    for (size_t e = 0; e < sectors.size(); ++e)
        for (int64_t q = 0; q < SN; ++q) {
            const size_t node = static_cast<size_t>(sectors[e]) * SN + q;
            smask[e * SN + q] = mask[node];
            sbb[e * SN + q] = bb[node];
        }
    // the handle takes the three buffers only when all of them are filled
    int32_t* d_sec = nullptr;
    uint8_t *d_sm = nullptr, *d_sb = nullptr;
    int rc = dev_alloc(h, &d_sec, sectors.size() * sizeof(int32_t));
    if (!rc) rc = dev_alloc(h, &d_sm, smask.size());
    if (!rc) rc = dev_alloc(h, &d_sb, sbb.size());
    cudaError_t e = cudaSuccess;
    if (!rc) e = cudaMemcpyAsync(d_sec, sectors.data(), sectors.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess) e = cudaMemcpyAsync(d_sm, smask.data(), smask.size(), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess) e = cudaMemcpyAsync(d_sb, sbb.data(), sbb.size(), cudaMemcpyHostToDevice, h->stream);
    if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(h, e, "active-sector list upload");
    if (rc) {
        const size_t sizes[3] = {sectors.size() * sizeof(int32_t), smask.size(), sbb.size()};
        void* bufs[3] = {d_sec, d_sm, d_sb};
        for (int q = 0; q < 3; ++q)
            if (bufs[q]) {
                dev_free(h, bufs[q]);
                h->bytes -= static_cast<int64_t>(sizes[q]);
            }
        return rc;
    }
    h->d_sectors = d_sec;
    h->d_smask = d_sm;
    h->d_sbb = d_sb;
    h->n_sectors = static_cast<int>(sectors.size());
    return LLB_OK;
}

int llb_set_pipeline(llb_handle h, int32_t config) {
    if (!h || config < PIPE_CLUSTER || config >= TMA_CONFIGS)
        return fail(h, LLB_E_INVALID, "config must be -4, -3, -2, -1 or in [0, 7)");
    if (config != PIPE_GRID && h->d_ps)
        return fail(h, LLB_E_UNSUPPORTED, "partially saturated obstacles run on the one-thread-per-node kernel");
    if (config == PIPE_COMPACT && !h->own_stream)
        return fail(h, LLB_E_STATE, "a lattice in a batch is stepped by the batch's kernels");
    if (config == PIPE_CLUSTER) {
        int rc = select_device(h);
        if (rc) return rc;
        if (!cluster_ok(h))
            return fail(h, LLB_E_UNSUPPORTED, "the lattice's column slabs do not fit the shared memory of one cluster");
    }
    if (config != h->tma_cfg) {
        int rc = select_device(h);
        if (rc) return rc;
        if (config == PIPE_LIST && (rc = build_sector_list(h))) return rc;
        if (config == PIPE_COMPACT && (rc = build_compact(h))) return rc;
        if (h->tma_cfg == PIPE_COMPACT && (rc = state_to_dense(h))) return rc;
        LLB_CUDA(h, cudaStreamSynchronize(h->stream));
        for (auto& g : h->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        h->tma_cfg = config;
        h->maps_ready = false;
    }
    return LLB_OK;
}

int llb_get_pipeline(llb_handle h, int32_t* config) {
    if (!h || !config) return fail(h, LLB_E_INVALID, "bad arguments");
    *config = h->tma_cfg;
    return LLB_OK;
}

// Device buffers of the active-sector list, released when the tuner does not
// keep the list kernel.
static void release_sector_list(llb_handle h) {
    const int64_t SN = LIST_BYTES / static_cast<int64_t>(h->elem);
    if (h->d_sectors) {
        dev_free(h, h->d_sectors);
        dev_free(h, h->d_smask);
        dev_free(h, h->d_sbb);
        h->bytes -= static_cast<int64_t>(h->n_sectors) * (static_cast<int64_t>(sizeof(int32_t)) + 2 * SN);
    }
    h->d_sectors = nullptr;
    h->d_smask = nullptr;
    h->d_sbb = nullptr;
    h->n_sectors = 0;
}

int llb_tune_pipeline(llb_handle h, int32_t trial_steps, int32_t* best, float* ms_per_step) {
    if (!h || trial_steps < 2 || trial_steps > (1 << 20)) return fail(h, LLB_E_INVALID, "bad arguments");
    if (!h->initialized) return fail(h, LLB_E_STATE, "llb_tune_pipeline before llb_init");
    int rc = select_device(h);
    if (rc) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    LLB_CUDA(h, cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(h, ce, "cudaEventCreate");
    }
    const int original = h->tma_cfg;
    int chosen = original;
    float chosen_ms = -1.0f;
    static constexpr int kCandidates[] = {PIPE_GRID, PIPE_LIST, PIPE_COMPACT, PIPE_CLUSTER, 0, 1, 2, 3, 4, 5, 6};
    for (int cfg : kCandidates) {
        if (llb_set_pipeline(h, cfg) != LLB_OK) continue;  // not available for this lattice
        // warm-up (tensor maps, graphs), then the timed steps
        if ((rc = llb_step(h, trial_steps, 0))) break;
        cudaError_t te = cudaEventRecord(e0, h->stream);
        if (te != cudaSuccess) {
            rc = cuda_fail(h, te, "cudaEventRecord");
            break;
        }
        if ((rc = llb_step(h, trial_steps, 0))) break;
        float ms = 0.0f;
        te = cudaEventRecord(e1, h->stream);
        if (te == cudaSuccess) te = cudaEventSynchronize(e1);
        if (te == cudaSuccess) te = cudaEventElapsedTime(&ms, e0, e1);
        if (te != cudaSuccess) {
            rc = cuda_fail(h, te, "timing a pipeline configuration");
            break;
        }
        if (chosen_ms < 0.0f || ms < chosen_ms) {
            chosen_ms = ms;
            chosen = cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = llb_set_pipeline(h, chosen))) return rc;
    if (chosen != PIPE_LIST) release_sector_list(h);
    if (chosen != PIPE_COMPACT) release_compact(h);
    if (best) *best = chosen;
    if (ms_per_step) *ms_per_step = chosen_ms < 0.0f ? 0.0f : chosen_ms / static_cast<float>(trial_steps);
    return LLB_OK;
}

int llb_set_wait_limit(llb_handle h, int64_t polls) {
    if (!h || polls < -1) return fail(h, LLB_E_INVALID, "polls must be >= 0, or -1 for the default");
    const long long lim = polls < 0 ? DEFAULT_WAIT_LIMIT : static_cast<long long>(polls);
    if (lim != h->wait_limit) {
        int rc = select_device(h);
        if (rc) return rc;
        LLB_CUDA(h, cudaStreamSynchronize(h->stream));
        for (auto& g : h->graph)  // the limit is a kernel argument captured in the graphs
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        h->wait_limit = lim;
    }
    return LLB_OK;
}

int llb_set_launch_shape(llb_handle h, int32_t block_y) {
    if (!h || block_y < 1 || block_y > MAX_BLOCK_Y) return fail(h, LLB_E_INVALID, "block_y must be in [1, 8]");
    if (block_y != h->block_y) {
        int rc = select_device(h);
        if (rc) return rc;
        LLB_CUDA(h, cudaStreamSynchronize(h->stream));
        for (auto& g : h->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        h->block_y = block_y;
    }
    return LLB_OK;
}

int llb_device_bytes(llb_handle h, int64_t* bytes) {
    if (!h || !bytes) return fail(h, LLB_E_INVALID, "bad arguments");
    *bytes = h->bytes;
    return LLB_OK;
}

}  // extern "C"

// Batches of lattices (C ABI llb_batch_*): independent D2Q9 problems of uneven
// sizes, collision models and relaxation times advanced together, one
// persistent launch per step (or per several steps, cooperatively), replayed
// from CUDA graphs.  Lattices can join and leave between calls: a solve server
// admits requests into a running batch as memory frees up.
//
// Every lattice of a batch is an ordinary llb_handle (created by llb_create,
// stepped to step 0 by llb_init) whose stream is the batch's stream, so its
// results are read with the single-lattice calls (llb_get_populations,
// llb_compute_macro, llb_flow_forces, ...).
#include <cuda_runtime.h>

#include <algorithm>
#include <limits>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/llalbm_cuda.h"
#include "llb_batch.cuh"
#include "llb_handle.h"
#include "llb_launch.h"

using namespace llb;

namespace {
constexpr int BATCH_GRAPH_STEPS = 32;  // even: a replay keeps every lattice's buffer parity
static_assert(BX == 32, "a handle's plain_seg flags segments of 32 rows, one dense tile's rows");
}  // namespace

struct llb_batch {
    int device = 0;
    int storage = LLB_STORE_F32S;
    cudaStream_t stream = nullptr;
    int sm_count = 148;
    std::vector<llb_handle> slot;        // nullptr: free slot
    std::vector<BatchLattice> desc;      // per slot
    std::vector<int> order;              // active slots in descriptor order
    BatchLattice* d_desc = nullptr;
    int desc_cap = 0;
    int2* d_items = nullptr;
    int items_cap = 0;
    int n_items = 0;
    int n_dense = 0;                     // items[0, n_dense): dense tiles; the rest compacted slot blocks
    long long step = 0;                  // batch step counter
    long long* d_sbase = nullptr;
    unsigned* d_bar = nullptr;           // [count, generation]
    unsigned* d_err = nullptr;
    long long bar_limit = BARRIER_LIMIT;  // polls of the grid barrier before a block gives up
    int layout = LLB_LAYOUT_AUTO;         // which lattices the batch steps on compacted planes
    int block_y = 4;
    int spl = 1;                         // steps per launch
    bool dirty = true;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // by parity of the batch step
    cudaEvent_t ev[8] = {};
    std::string err;
};

namespace {

int bfail(llb_batch_handle b, int code, const std::string& m) {
    if (b) b->err = m;
    return code;
}

#define LLB_BCUDA(b, call)                                                               \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return bfail(b, e_ == cudaErrorMemoryAllocation ? LLB_E_NOMEM : LLB_E_CUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));            \
    } while (0)

void drop_graph(llb_batch_handle b) {
    for (auto& g : b->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// Batch steps a lattice has taken since it was anchored: the batch's, up to
// its stop step.
long long steps_taken(llb_batch_handle b, const BatchLattice& d) {
    return std::max(0LL, std::min(b->step - d.s0, d.t_end - d.t0));
}

// Per-lattice step, buffer and state residence implied by the batch counter.
void sync_handle(llb_batch_handle b, int s) {
    llb_handle h = b->slot[s];
    const BatchLattice& d = b->desc[s];
    const long long delta = steps_taken(b, d);
    h->step = d.t0 + delta;
    h->cur = d.cur0 ^ static_cast<int>(delta & 1);
    if (delta > 0) handle_batch_stepped(h, d.compact != 0);
}

// A lattice stepped through its own handle since the last batch call is
// re-anchored at its current step and buffer, its state brought back into
// the layout the batch steps.
int reanchor_if_moved(llb_batch_handle b, int s) {
    llb_handle h = b->slot[s];
    BatchLattice& d = b->desc[s];
    const long long delta = steps_taken(b, d);
    if (h->step != d.t0 + delta || h->cur != (d.cur0 ^ static_cast<int>(delta & 1))) {
        d.t0 = h->step;
        d.s0 = b->step;
        d.cur0 = h->cur;
        b->dirty = true;
        if (handle_batch_layout(h, d.compact != 0) != LLB_OK) return bfail(b, LLB_E_CUDA, llb_last_error(h));
    }
    return LLB_OK;
}

// Slots of one work-list item of a compacted lattice: one per thread of a block.
int64_t slots_per_item(const llb_batch_handle b) { return static_cast<int64_t>(BX) * b->block_y; }

// Whether the batch steps this lattice on its compacted planes (building them
// if needed; a lattice without them runs on the dense ones).
bool want_compact(llb_batch_handle b, llb_handle h) {
    if (b->layout == LLB_LAYOUT_DENSE) return false;
    if (b->layout == LLB_LAYOUT_AUTO && !obstacle_rich(*h)) return false;
    return handle_prepare_compact(h) == LLB_OK;
}

// Descriptor fields that follow the lattice's layout and position.
void anchor(llb_batch_handle b, int s, bool compact) {
    llb_handle h = b->slot[s];
    BatchLattice& d = b->desc[s];
    d.compact = compact ? 1 : 0;
    d.f[0] = compact ? h->cf[0] : h->f[0];
    d.f[1] = compact ? h->cf[1] : h->f[1];
    d.cg = compact ? handle_compact_geo(h) : CompactGeo{};
    d.t0 = h->step;
    d.s0 = b->step;
    d.cur0 = h->cur;
    b->dirty = true;
}

int rebuild(llb_batch_handle b) {
    if (!b->dirty) return LLB_OK;
    drop_graph(b);
    b->order.clear();
    std::vector<BatchLattice> dev;
    std::vector<int2> items, slot_items;
    for (int s = 0; s < static_cast<int>(b->slot.size()); ++s) {
        if (!b->slot[s]) continue;
        const int idx = static_cast<int>(dev.size());
        b->order.push_back(s);
        dev.push_back(b->desc[s]);
        // every lattice, large or small, is items of the one work list: one
        // persistent launch advances the whole batch
        const BatchLattice& d = b->desc[s];
        if (d.compact) {
            const int64_t n = (d.cg.n_slots + slots_per_item(b) - 1) / slots_per_item(b);
            for (int64_t t = 0; t < n; ++t) slot_items.push_back(make_int2(idx, static_cast<int>(t)));
        } else {
            // tiles in column-major order, (row tile, column tile) packed in 16
            // bits each; ITEM_PLAIN on tiles whose every node is a PLAIN fluid node
            const int by = b->block_y, cols = d.g.cols, ntj = (cols + by - 1) / by;
            const std::vector<uint8_t>& seg = b->slot[s]->plain_seg;
            const bool have = seg.size() == static_cast<size_t>(d.nti) * static_cast<size_t>(cols);
            for (int tj = 0; tj < ntj; ++tj)
                for (int ti = 0; ti < d.nti; ++ti) {
                    bool plain = have;
                    for (int y = 0; plain && y < by; ++y) {
                        const int c = tj * by + y;
                        plain = c < cols && seg[static_cast<size_t>(c) * d.nti + ti] != 0;
                    }
                    items.push_back(make_int2(idx | (plain ? ITEM_PLAIN : 0), ti | (tj << 16)));
                }
        }
    }
    const int n_dense = static_cast<int>(items.size());
    items.insert(items.end(), slot_items.begin(), slot_items.end());
    LLB_BCUDA(b, cudaStreamSynchronize(b->stream));
    if (static_cast<int>(dev.size()) > b->desc_cap) {
        if (b->d_desc) cudaFree(b->d_desc);
        b->desc_cap = std::max<int>(static_cast<int>(dev.size()), 2 * b->desc_cap);
        LLB_BCUDA(b, cudaMalloc(&b->d_desc, sizeof(BatchLattice) * b->desc_cap));
    }
    if (static_cast<int>(items.size()) > b->items_cap) {
        if (b->d_items) cudaFree(b->d_items);
        b->items_cap = std::max<int>(static_cast<int>(items.size()), 2 * b->items_cap);
        LLB_BCUDA(b, cudaMalloc(&b->d_items, sizeof(int2) * b->items_cap));
    }
    if (!dev.empty())
        LLB_BCUDA(b, cudaMemcpyAsync(b->d_desc, dev.data(), sizeof(BatchLattice) * dev.size(), cudaMemcpyHostToDevice,
                                     b->stream));
    if (!items.empty())
        LLB_BCUDA(b, cudaMemcpyAsync(b->d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice,
                                     b->stream));
    LLB_BCUDA(b, cudaStreamSynchronize(b->stream));
    b->n_items = static_cast<int>(items.size());
    b->n_dense = n_dense;
    b->dirty = false;
    return LLB_OK;
}

BatchLaunch launch_desc(llb_batch_handle b, long long soff, int steps) {
    BatchLaunch L{};
    L.lats = b->d_desc;
    L.items = b->d_items;
    L.n_items = b->n_items;
    L.n_dense = b->n_dense;
    L.sbase = b->d_sbase;
    L.soff = soff;
    L.steps = steps;
    L.bar = b->d_bar;
    L.err = b->d_err;
    L.bar_limit = b->bar_limit;
    L.block_y = b->block_y;
    L.stream = b->stream;
    L.cooperative = steps > 1;
    const int maxg = batch_max_grid(b->storage, b->block_y, b->sm_count);
    L.grid = std::max(1, std::min(b->n_items, maxg > 0 ? maxg : b->sm_count));
    return L;
}

int set_base(llb_batch_handle b) {
    LLB_BCUDA(b, cudaMemcpyAsync(b->d_sbase, &b->step, sizeof(long long), cudaMemcpyHostToDevice, b->stream));
    return LLB_OK;
}

// Every lattice one step: one launch of the work-list kernel.
int launch_one_step(llb_batch_handle b, long long soff) {
    if (b->n_items > 0) {
        cudaError_t e = launch_batch_step(b->storage, launch_desc(b, soff, 1));
        if (e != cudaSuccess) return bfail(b, LLB_E_CUDA, std::string("batched kernel: ") + cudaGetErrorString(e));
    }
    return LLB_OK;
}

int launch_steps(llb_batch_handle b, int32_t nsteps) {
    int rc;
    if (b->n_items == 0) {
        b->step += nsteps;
        return LLB_OK;
    }
    if (b->spl > 1) {
        // cooperative launches of spl steps each
        while (nsteps > 0) {
            const int k = std::min<int>(nsteps, b->spl);
            if ((rc = set_base(b))) return rc;
            cudaError_t e = launch_batch_step(b->storage, launch_desc(b, 0, k));
            if (e != cudaSuccess) return bfail(b, LLB_E_CUDA, std::string("batched kernel: ") + cudaGetErrorString(e));
            b->step += k;
            nsteps -= k;
        }
        return LLB_OK;
    }
    if (nsteps >= BATCH_GRAPH_STEPS) {
        cudaGraphExec_t& gx = b->graph[b->step & 1];
        if (!gx) {
            cudaGraph_t g = nullptr;
            LLB_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int lr = LLB_OK;
            for (int s = 0; s < BATCH_GRAPH_STEPS && lr == LLB_OK; ++s) lr = launch_one_step(b, s);
            cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
            if (lr != LLB_OK || ee != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return lr != LLB_OK ? lr : bfail(b, LLB_E_CUDA, "capture of the batched step graph failed");
            }
            cudaError_t ie = cudaGraphInstantiate(&gx, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return bfail(b, LLB_E_CUDA, "cudaGraphInstantiate (batch)");
        }
        while (nsteps >= BATCH_GRAPH_STEPS) {
            if ((rc = set_base(b))) return rc;
            LLB_BCUDA(b, cudaGraphLaunch(gx, b->stream));
            b->step += BATCH_GRAPH_STEPS;
            nsteps -= BATCH_GRAPH_STEPS;
        }
    }
    if (nsteps > 0) {
        if ((rc = set_base(b))) return rc;
        for (int s = 0; s < nsteps; ++s)
            if ((rc = launch_one_step(b, s))) return rc;
        b->step += nsteps;
    }
    return LLB_OK;
}

}  // namespace

extern "C" {

int llb_batch_create(int32_t device, int32_t storage, llb_batch_handle* out) {
    if (!out || storage < LLB_STORE_F64 || storage > LLB_STORE_F16S) return LLB_E_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return LLB_E_NODEVICE;
    llb_batch_handle b = new (std::nothrow) llb_batch();
    if (!b) return LLB_E_NOMEM;
    b->device = device;
    b->storage = storage;
    auto bail = [&](int rc) {
        llb_batch_destroy(b);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(LLB_E_CUDA);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(LLB_E_CUDA);
    cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&b->d_sbase, sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&b->d_bar, 2 * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&b->d_err, sizeof(unsigned)) != cudaSuccess)
        return bail(LLB_E_NOMEM);
    if (cudaMemsetAsync(b->d_bar, 0, 2 * sizeof(unsigned), b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_err, 0, sizeof(unsigned), b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return bail(LLB_E_CUDA);
    *out = b;
    return LLB_OK;
}

int llb_batch_destroy(llb_batch_handle b) {
    if (!b) return LLB_E_INVALID;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (llb_handle h : b->slot)
        if (h) llb_destroy(h);
    drop_graph(b);
    for (void* p : {static_cast<void*>(b->d_desc), static_cast<void*>(b->d_items), static_cast<void*>(b->d_sbase),
                    static_cast<void*>(b->d_bar), static_cast<void*>(b->d_err)})
        if (p) cudaFree(p);
    for (auto& e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return LLB_OK;
}

int llb_batch_add(llb_batch_handle b, const llb_desc* desc, const double* open_values, int32_t rows, int32_t* slot) {
    if (!b || !desc || !slot) return LLB_E_INVALID;
    if (desc->storage != b->storage || desc->pattern != LLB_PATTERN_AB || desc->device != b->device)
        return bfail(b, LLB_E_INVALID, "lattice storage, pattern or device differs from the batch");
    if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
    llb_handle h = nullptr;
    int rc = llb_create(desc, &h);
    if (rc != LLB_OK) return bfail(b, rc, llb_last_error(nullptr));
    if (open_values && rows > 0 && (rc = llb_set_open_values(h, 0, rows, open_values)) != LLB_OK) {
        llb_destroy(h);
        return bfail(b, rc, "boundary values rejected");
    }
    if ((rc = llb_batch_attach(b, h, slot)) != LLB_OK) llb_destroy(h);
    return rc;
}

int llb_batch_attach(llb_batch_handle b, llb_handle h, int32_t* slot) {
    if (!b || !h || !slot) return LLB_E_INVALID;
    if (h->storage != b->storage || h->pattern != LLB_PATTERN_AB || h->device != b->device)
        return bfail(b, LLB_E_INVALID, "lattice storage, pattern or device differs from the batch");
    if (!h->own_stream) return bfail(b, LLB_E_STATE, "lattice already belongs to a batch");
    if (h->d_ps) return bfail(b, LLB_E_UNSUPPORTED, "partially saturated obstacles run on the single-lattice path");
    // the batch's kernels index a lattice's nine planes with 32-bit offsets,
    // and a dense tile's row and column tile indices with 16 bits each
    if (10 * static_cast<int64_t>(h->plane) >= (int64_t{1} << 31) || (h->R + BX - 1) / BX >= (1 << 16) ||
        h->C >= (1 << 16))
        return bfail(b, LLB_E_UNSUPPORTED, "lattice too large for a batch (32-bit plane offsets, 16-bit tile indices)");
    if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
    // the batch steps the compacted planes (built here, on the lattice's own
    // stream, so a chunk running on the batch's stream is not waited for);
    // lattices without them run on the dense ones
    const bool compact = want_compact(b, h);
    if (!compact && handle_leave_compact(h) != LLB_OK) return bfail(b, LLB_E_CUDA, llb_last_error(h));
    // the lattice works on the batch's stream from now on
    LLB_BCUDA(b, cudaStreamSynchronize(h->stream));
    cudaStreamDestroy(h->stream);
    h->stream = b->stream;
    h->own_stream = false;
    // on failure the handle gets a stream of its own again so the caller can destroy it
    auto give_back = [&](int rc, const std::string& why) {
        cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        h->own_stream = true;
        return bfail(b, rc, why);
    };
    if (!h->initialized) {
        const int rc = llb_init(h, 0);
        if (rc != LLB_OK) return give_back(rc, "llb_init failed");
    }
    if (handle_batch_layout(h, compact) != LLB_OK) return give_back(LLB_E_CUDA, llb_last_error(h));
    BatchLattice d{};
    const LaunchCtx x = handle_ctx(h);
    d.g = x.g;
    d.ot = x.ot;
    d.c = x.c;
    d.compact = compact ? 1 : 0;
    d.f[0] = compact ? h->cf[0] : h->f[0];
    d.f[1] = compact ? h->cf[1] : h->f[1];
    if (compact) d.cg = handle_compact_geo(h);
    d.t_end = std::numeric_limits<long long>::max();
    d.t0 = h->step;
    d.s0 = b->step;
    d.cur0 = h->cur;
    d.nti = static_cast<int>((h->R + BX - 1) / BX);
    d.flags = h->d_flags;
    int s = 0;
    while (s < static_cast<int>(b->slot.size()) && b->slot[s]) ++s;
    if (s == static_cast<int>(b->slot.size())) {
        b->slot.push_back(nullptr);
        b->desc.push_back(BatchLattice{});
    }
    b->slot[s] = h;
    b->desc[s] = d;
    b->dirty = true;
    *slot = s;
    return LLB_OK;
}

int llb_batch_detach(llb_batch_handle b, int32_t slot, llb_handle* out) {
    if (!b || !out || slot < 0 || slot >= static_cast<int>(b->slot.size()) || !b->slot[slot]) return LLB_E_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
    sync_handle(b, slot);
    llb_handle h = b->slot[slot];
    // the handle's own stream starts after the batch work queued so far
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    LLB_BCUDA(b, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ev, b->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev, 0);
    if (ev) cudaEventDestroy(ev);
    if (e != cudaSuccess) {
        cudaStreamDestroy(st);
        return bfail(b, LLB_E_CUDA, std::string("detach: ") + cudaGetErrorString(e));
    }
    h->stream = st;
    h->own_stream = true;
    b->slot[slot] = nullptr;
    b->dirty = true;
    *out = h;
    return LLB_OK;
}

int llb_batch_remove(llb_batch_handle b, int32_t slot) {
    if (!b || slot < 0 || slot >= static_cast<int>(b->slot.size()) || !b->slot[slot]) return LLB_E_INVALID;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    llb_destroy(b->slot[slot]);
    b->slot[slot] = nullptr;
    b->dirty = true;
    return LLB_OK;
}

int llb_batch_step(llb_batch_handle b, int32_t nsteps) {
    if (!b || nsteps < 0) return LLB_E_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
    int rc = LLB_OK;
    for (int s = 0; s < static_cast<int>(b->slot.size()); ++s)
        if (b->slot[s] && (rc = reanchor_if_moved(b, s)) != LLB_OK) return rc;
    rc = rebuild(b);
    if (rc != LLB_OK) return rc;
    if ((rc = launch_steps(b, nsteps)) != LLB_OK) return rc;
    for (int s = 0; s < static_cast<int>(b->slot.size()); ++s)
        if (b->slot[s]) sync_handle(b, s);
    return LLB_OK;
}

int llb_batch_lattice(llb_batch_handle b, int32_t slot, llb_handle* out) {
    if (!b || !out || slot < 0 || slot >= static_cast<int>(b->slot.size()) || !b->slot[slot]) return LLB_E_INVALID;
    sync_handle(b, slot);
    *out = b->slot[slot];
    return LLB_OK;
}

int llb_batch_set_config(llb_batch_handle b, int32_t block_y, int32_t steps_per_launch) {
    if (!b || block_y < 1 || block_y > MAX_BLOCK_Y || steps_per_launch < 1 || steps_per_launch > 1024)
        return LLB_E_INVALID;
    if (block_y != b->block_y) b->dirty = true;
    b->block_y = block_y;
    b->spl = steps_per_launch;
    drop_graph(b);
    return LLB_OK;
}

int llb_batch_get_config(llb_batch_handle b, int32_t* block_y, int32_t* steps_per_launch) {
    if (!b || !block_y || !steps_per_launch) return LLB_E_INVALID;
    *block_y = b->block_y;
    *steps_per_launch = b->spl;
    return LLB_OK;
}

int llb_batch_tune(llb_batch_handle b, int32_t trial_steps, int32_t* block_y, int32_t* steps_per_launch,
                   float* ms_per_step) {
    if (!b || trial_steps < 1) return LLB_E_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
    static const int shapes[] = {1, 2, 4, 8};
    static const int spls[] = {1, 8};
    static const int layouts[] = {LLB_LAYOUT_AUTO, LLB_LAYOUT_COMPACT, LLB_LAYOUT_DENSE};
    float best = 1e30f;
    int best_by = b->block_y, best_spl = b->spl, best_layout = b->layout;
    for (int e = 0; e < 2; ++e)
        if (!b->ev[e]) LLB_BCUDA(b, cudaEventCreate(&b->ev[e]));
    for (int layout : layouts) {
      int rc = llb_batch_set_layout(b, layout);
      if (rc != LLB_OK) return rc;
      for (int by : shapes) {
        for (int spl : spls) {
            rc = llb_batch_set_config(b, by, spl);
            if (rc != LLB_OK) return rc;
            if ((rc = llb_batch_step(b, std::min(trial_steps, 8))) != LLB_OK) return rc;  // graph capture, warm-up
            LLB_BCUDA(b, cudaEventRecord(b->ev[0], b->stream));
            if ((rc = llb_batch_step(b, trial_steps)) != LLB_OK) return rc;
            LLB_BCUDA(b, cudaEventRecord(b->ev[1], b->stream));
            LLB_BCUDA(b, cudaEventSynchronize(b->ev[1]));
            float ms = 0.f;
            LLB_BCUDA(b, cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
            if (ms < best) {
                best = ms;
                best_by = by;
                best_spl = spl;
                best_layout = layout;
            }
        }
      }
    }
    int rc = llb_batch_set_layout(b, best_layout);
    if (rc == LLB_OK) rc = llb_batch_set_config(b, best_by, best_spl);
    if (rc != LLB_OK) return rc;
    if (block_y) *block_y = best_by;
    if (steps_per_launch) *steps_per_launch = best_spl;
    if (ms_per_step) *ms_per_step = best / static_cast<float>(trial_steps);
    return LLB_OK;
}

int llb_batch_get_step(llb_batch_handle b, int64_t* step) {
    if (!b || !step) return LLB_E_INVALID;
    *step = b->step;
    return LLB_OK;
}

int llb_batch_query(llb_batch_handle b, int32_t* done) {
    if (!b || !done) return LLB_E_INVALID;
    cudaSetDevice(b->device);
    const cudaError_t e = cudaStreamQuery(b->stream);
    if (e == cudaSuccess) {
        *done = 1;
        return LLB_OK;
    }
    if (e == cudaErrorNotReady) {
        *done = 0;
        return LLB_OK;
    }
    return bfail(b, LLB_E_CUDA, std::string("cudaStreamQuery: ") + cudaGetErrorString(e));
}

int llb_batch_synchronize(llb_batch_handle b) {
    if (!b) return LLB_E_INVALID;
    cudaSetDevice(b->device);
    LLB_BCUDA(b, cudaStreamSynchronize(b->stream));
    unsigned err = 0;
    LLB_BCUDA(b, cudaMemcpy(&err, b->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err) {
        // blocks that gave up had counted themselves at the barrier: clear
        // [count, generation] too, or the next launch's first barrier could
        // let blocks through before all of them arrive
        LLB_BCUDA(b, cudaMemset(b->d_bar, 0, 2 * sizeof(unsigned)));
        LLB_BCUDA(b, cudaMemset(b->d_err, 0, sizeof(unsigned)));
        return bfail(b, LLB_E_TIMEOUT, "batched kernel gave up a grid barrier");
    }
    return LLB_OK;
}

int llb_batch_set_layout(llb_batch_handle b, int32_t layout) {
    if (!b || layout < LLB_LAYOUT_AUTO || layout > LLB_LAYOUT_DENSE) return LLB_E_INVALID;
    if (layout == b->layout) return LLB_OK;
    if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
    b->layout = layout;
    // every attached lattice moves into the layout it now takes, at its current step
    for (int s = 0; s < static_cast<int>(b->slot.size()); ++s) {
        llb_handle h = b->slot[s];
        if (!h) continue;
        sync_handle(b, s);
        const bool compact = want_compact(b, h);
        if (handle_batch_layout(h, compact) != LLB_OK) return bfail(b, LLB_E_CUDA, llb_last_error(h));
        anchor(b, s, compact);
    }
    drop_graph(b);
    return LLB_OK;
}

int llb_batch_get_layout(llb_batch_handle b, int32_t* layout) {
    if (!b || !layout) return LLB_E_INVALID;
    *layout = b->layout;
    return LLB_OK;
}

int llb_batch_set_stop(llb_batch_handle b, int32_t slot, int64_t stop_step) {
    if (!b || slot < 0 || slot >= static_cast<int>(b->slot.size()) || !b->slot[slot] || stop_step < -1)
        return LLB_E_INVALID;
    BatchLattice& d = b->desc[slot];
    // re-anchor at the lattice's current position, then set the stop
    sync_handle(b, slot);
    llb_handle h = b->slot[slot];
    d.t0 = h->step;
    d.s0 = b->step;
    d.cur0 = h->cur;
    d.t_end = stop_step < 0 ? std::numeric_limits<long long>::max() : std::max<long long>(stop_step, h->step);
    b->dirty = true;
    return LLB_OK;
}

int llb_batch_set_wait_limit(llb_batch_handle b, int64_t polls) {
    if (!b || polls < -1) return LLB_E_INVALID;
    const long long lim = polls < 0 ? BARRIER_LIMIT : static_cast<long long>(polls);
    if (lim != b->bar_limit) {
        if (cudaSetDevice(b->device) != cudaSuccess) return LLB_E_CUDA;
        LLB_BCUDA(b, cudaStreamSynchronize(b->stream));
        drop_graph(b);  // the limit is a kernel argument captured in the graphs
        b->bar_limit = lim;
    }
    return LLB_OK;
}

int llb_batch_set_stream_priority(llb_batch_handle b, int32_t priority) {
    if (!b) return LLB_E_INVALID;
    for (llb_handle h : b->slot)
        if (h) return bfail(b, LLB_E_STATE, "stream priority can only change on an empty batch");
    cudaSetDevice(b->device);
    int lo = 0, hi = 0;
    LLB_BCUDA(b, cudaDeviceGetStreamPriorityRange(&lo, &hi));
    const int p = std::min(std::max(static_cast<int>(priority), hi), lo);  // hi is the greatest priority
    cudaStream_t st = nullptr;
    LLB_BCUDA(b, cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, p));
    LLB_BCUDA(b, cudaStreamSynchronize(b->stream));
    drop_graph(b);
    cudaStreamDestroy(b->stream);
    b->stream = st;
    return LLB_OK;
}

int llb_batch_event_record(llb_batch_handle b, int32_t slot) {
    if (!b || slot < 0 || slot >= 8) return LLB_E_INVALID;
    cudaSetDevice(b->device);
    if (!b->ev[slot]) LLB_BCUDA(b, cudaEventCreate(&b->ev[slot]));
    LLB_BCUDA(b, cudaEventRecord(b->ev[slot], b->stream));
    return LLB_OK;
}

int llb_batch_event_elapsed_ms(llb_batch_handle b, int32_t a, int32_t c, float* ms) {
    if (!b || !ms || a < 0 || a >= 8 || c < 0 || c >= 8 || !b->ev[a] || !b->ev[c]) return LLB_E_INVALID;
    LLB_BCUDA(b, cudaEventSynchronize(b->ev[c]));
    LLB_BCUDA(b, cudaEventElapsedTime(ms, b->ev[a], b->ev[c]));
    return LLB_OK;
}

int llb_batch_info(llb_batch_handle b, int64_t* lattices, int64_t* nodes, int64_t* device_bytes) {
    if (!b) return LLB_E_INVALID;
    int64_t n = 0, nn = 0, bytes = 0;
    for (llb_handle h : b->slot) {
        if (!h) continue;
        ++n;
        nn += h->R * h->C;
        bytes += h->bytes;
    }
    if (lattices) *lattices = n;
    if (nodes) *nodes = nn;
    if (device_bytes) *device_bytes = bytes;
    return LLB_OK;
}

const char* llb_batch_last_error(llb_batch_handle b) { return b ? b->err.c_str() : ""; }

}  // extern "C"

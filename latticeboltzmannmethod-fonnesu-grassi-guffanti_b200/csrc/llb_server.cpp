// Solve server (C ABI llb_server_*).  Requests -- one lattice, its boundary
// values and a step count -- arrive from any thread.  One worker thread keeps
// every admitted lattice resident on the device and advances them together.
//
// Batched mode (continuous batching): requests are admitted first come, first
// served while their device memory fits the budget.  The worker advances the
// running batch in chunks of at most max_chunk steps, never past the earliest
// completion.  Admission of newly arrived requests (mask build, allocation,
// upload, step 0) happens on the host while the previous chunk is still running
// on the device, and they join the batch at the next chunk boundary, so their
// work overlaps the work of the requests already running.  A finished request's
// result -- rho and u of the state after its last step -- is copied to host
// memory and its lattice is freed, which makes room for the queue.
//
// Sequential mode serves the same requests one at a time through the plain
// single-lattice path (the comparison for the batched mode).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/llalbm_cuda.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    llb_desc desc{};
    std::vector<int64_t> fluid, wall, inlet, outlet, obstacle;
    std::vector<int32_t> inlet_side, outlet_side;
    std::vector<uint16_t> dirs;
    std::vector<double> values;
    int32_t rows = 0;
    int64_t steps = 0;
    int64_t remaining = 0;      // batch steps still to run
    int32_t slot = -1;
    int state = LLB_REQ_QUEUED;
    int64_t bytes = 0;          // device bytes charged against the budget
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::vector<double> rho, u;
    std::string error;
};

// Device bytes a lattice of this description holds once created: two
// population buffers, the node mask, bounce bits and open-node index, the macroscopic
// outputs and the boundary-value ring (plus a small fixed allowance).
int64_t estimate_bytes(const llb_desc& d, int32_t rows) {
    const int64_t elem = d.storage == LLB_STORE_F64 ? 8 : d.storage == LLB_STORE_F32S ? 4 : 2;
    const int64_t align = 256 / elem;
    const int64_t n = (d.rows + align - 1) / align * align * d.cols;
    const int64_t nn = d.rows * d.cols;
    const int64_t open = std::max<int64_t>(d.n_inlet + d.n_outlet, 1);
    return 2 * 9 * elem * n + 6 * n + 24 * nn + 16 * open * std::max<int32_t>(rows, 1) + (1 << 16);
}

}  // namespace

struct llb_server {
    int device = 0;
    int storage = LLB_STORE_F32S;
    int mode = LLB_SERVE_BATCHED;
    int64_t budget = 0;
    int32_t max_chunk = 256;
    llb_batch_handle batch = nullptr;
    std::mutex mu;
    std::condition_variable cv_work;   // the worker: new requests or stop
    std::condition_variable cv_done;   // waiters: a request finished
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> all;
    std::vector<std::shared_ptr<Request>> running;   // touched by the worker only
    int64_t n_running = 0;
    int64_t next_id = 1;
    int64_t in_use = 0;
    bool stop = false;
    std::thread worker;
    int64_t node_steps = 0;
    int64_t completed = 0;
    int64_t failed = 0;
    int64_t chunks = 0;
    int64_t batch_steps = 0;
    std::string error;
};

namespace {

// Marks a request finished (rc == LLB_OK: reads its result through h first).
void finish(llb_server_handle s, const std::shared_ptr<Request>& r, llb_handle h, int rc, const char* what) {
    if (rc == LLB_OK) {
        const size_t N = static_cast<size_t>(r->desc.rows * r->desc.cols);
        r->rho.resize(N);
        r->u.resize(2 * N);
        rc = llb_compute_macro(h, r->rho.data(), r->u.data());
    }
    std::string msg;
    if (rc != LLB_OK) msg = std::string(what) + ": " + (h ? llb_last_error(h) : llb_last_error(nullptr));
    std::lock_guard<std::mutex> lk(s->mu);
    r->t_done = now_s();
    if (rc == LLB_OK) {
        r->state = LLB_REQ_DONE;
        s->node_steps += r->desc.rows * r->desc.cols * r->steps;
        s->completed += 1;
    } else {
        r->state = LLB_REQ_FAILED;
        r->error = msg;
        r->rho.clear();
        r->u.clear();
        s->failed += 1;
    }
    s->in_use -= r->bytes;
    s->cv_done.notify_all();
}

// One request through the plain single-lattice path: steps - 1 collisions
// (llb_init is the first), then rho and u of the state the last step reads.
void serve_plain(llb_server_handle s, const std::shared_ptr<Request>& r) {
    llb_handle h = nullptr;
    llb_desc d = r->desc;
    int rc = llb_create(&d, &h);
    if (rc == LLB_OK && r->rows > 0) rc = llb_set_open_values(h, 0, r->rows, r->values.data());
    if (rc == LLB_OK) rc = llb_init(h, 0);
    int64_t left = r->steps - 2;
    while (rc == LLB_OK && left > 0) {
        const int32_t n = static_cast<int32_t>(std::min<int64_t>(left, 1 << 20));
        rc = llb_step(h, n, 0);
        left -= n;
    }
    if (rc == LLB_OK) rc = llb_synchronize(h);
    finish(s, r, h, rc, "plain path");
    if (h) llb_destroy(h);
}

void sequential_loop(llb_server_handle s) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) return;  // stop requested and nothing left
            r = s->queue.front();
            s->queue.pop_front();
            r->state = LLB_REQ_RUNNING;
            r->t_admit = now_s();
            s->in_use += r->bytes;
            s->n_running = 1;
        }
        serve_plain(s, r);
        std::lock_guard<std::mutex> lk(s->mu);
        s->n_running = 0;
    }
}

// Admits queued requests while the budget allows (the queue head always when
// nothing runs); returns them in arrival order.
std::vector<std::shared_ptr<Request>> take_admissible(llb_server_handle s, bool block) {
    std::vector<std::shared_ptr<Request>> out;
    std::unique_lock<std::mutex> lk(s->mu);
    if (block) s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
    while (!s->queue.empty()) {
        auto& r = s->queue.front();
        if (s->in_use + r->bytes > s->budget && !(s->running.empty() && out.empty())) break;
        r->state = LLB_REQ_RUNNING;
        r->t_admit = now_s();
        s->in_use += r->bytes;
        out.push_back(r);
        s->queue.pop_front();
    }
    return out;
}

void batched_loop(llb_server_handle s) {
    bool inflight = false;   // a chunk was launched and not yet waited for
    for (;;) {
        const bool idle = s->running.empty() && !inflight;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (idle && s->stop && s->queue.empty()) return;
        }
        // 1. admissions (overlap the chunk in flight)
        for (auto& r : take_admissible(s, idle)) {
            llb_desc d = r->desc;
            int32_t slot = -1;
            const int rc = llb_batch_add(s->batch, &d, r->rows > 0 ? r->values.data() : nullptr, r->rows, &slot);
            if (rc != LLB_OK) {
                std::lock_guard<std::mutex> lk(s->mu);
                r->state = LLB_REQ_FAILED;
                r->error = std::string("admission failed: ") + llb_batch_last_error(s->batch);
                r->t_done = now_s();
                s->in_use -= r->bytes;
                s->failed += 1;
                s->cv_done.notify_all();
                continue;
            }
            llb_handle h = nullptr;
            int64_t actual = 0;
            if (llb_batch_lattice(s->batch, slot, &h) == LLB_OK && llb_device_bytes(h, &actual) == LLB_OK) {
                std::lock_guard<std::mutex> lk(s->mu);
                s->in_use += actual - r->bytes;
                r->bytes = actual;
            }
            r->slot = slot;
            r->remaining = r->steps - 2;  // llb_batch_add ran the first collision
            std::lock_guard<std::mutex> lk(s->mu);
            s->running.push_back(r);
            s->n_running = static_cast<int64_t>(s->running.size());
        }
        // 2. wait for the chunk in flight, retire what it finished
        int rc = LLB_OK;
        if (inflight) {
            rc = llb_batch_synchronize(s->batch);
            inflight = false;
        }
        std::vector<std::shared_ptr<Request>> keep;
        for (auto& r : s->running) {
            if (r->remaining > 0 && rc == LLB_OK) {
                keep.push_back(r);
                continue;
            }
            llb_handle h = nullptr;
            const int hr = rc == LLB_OK ? llb_batch_lattice(s->batch, r->slot, &h) : rc;
            finish(s, r, h, hr, "batched step");
            llb_batch_remove(s->batch, r->slot);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->running.swap(keep);
            s->n_running = static_cast<int64_t>(s->running.size());
        }
        if (s->running.empty()) continue;
        // 3. next chunk: up to the earliest completion
        int64_t chunk = s->max_chunk;
        for (auto& r : s->running) chunk = std::min(chunk, r->remaining);
        rc = llb_batch_step(s->batch, static_cast<int32_t>(chunk));
        for (auto& r : s->running) r->remaining -= chunk;
        if (rc != LLB_OK) {
            // every running request fails at the next retirement pass
            for (auto& r : s->running) r->remaining = 0;
            std::lock_guard<std::mutex> lk(s->mu);
            s->error = std::string("batched step failed: ") + llb_batch_last_error(s->batch);
        }
        inflight = true;
        std::lock_guard<std::mutex> lk(s->mu);
        s->chunks += 1;
        s->batch_steps += chunk;
    }
}

}  // namespace

extern "C" {

int llb_server_create(int32_t device, int32_t storage, int32_t mode, int64_t budget_bytes, int32_t max_chunk_steps,
                      llb_server_handle* out) {
    if (!out) return LLB_E_INVALID;
    *out = nullptr;
    if (budget_bytes <= 0 || max_chunk_steps < 1 || storage < LLB_STORE_F64 || storage > LLB_STORE_F16S ||
        (mode != LLB_SERVE_BATCHED && mode != LLB_SERVE_SEQUENTIAL))
        return LLB_E_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return LLB_E_NODEVICE;
    llb_server_handle s = new (std::nothrow) llb_server();
    if (!s) return LLB_E_NOMEM;
    s->device = device;
    s->storage = storage;
    s->mode = mode;
    s->budget = budget_bytes;
    s->max_chunk = max_chunk_steps;
    if (mode == LLB_SERVE_BATCHED) {
        const int rc = llb_batch_create(device, storage, &s->batch);
        if (rc != LLB_OK) {
            delete s;
            return rc;
        }
        llb_batch_set_config(s->batch, 8, 1);
    }
    try {
        s->worker = std::thread(mode == LLB_SERVE_BATCHED ? batched_loop : sequential_loop, s);
    } catch (...) {
        if (s->batch) llb_batch_destroy(s->batch);
        delete s;
        return LLB_E_NOMEM;
    }
    *out = s;
    return LLB_OK;
}

int llb_server_destroy(llb_server_handle s) {
    if (!s) return LLB_E_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (auto& r : s->queue) {
            r->state = LLB_REQ_FAILED;
            r->error = "server stopped before admission";
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->batch) llb_batch_destroy(s->batch);
    delete s;
    return LLB_OK;
}

int llb_server_submit(llb_server_handle s, const llb_desc* d, const double* open_values, int32_t rows, int64_t steps,
                      int64_t* request_id) {
    if (!s || !d || !request_id || steps < 2 || rows < 0 || (rows > 0 && !open_values) || d->rows <= 0 ||
        d->cols <= 0)
        return LLB_E_INVALID;
    auto r = std::make_shared<Request>();
    r->desc = *d;
    auto copy_ij = [](const int64_t* p, int64_t n, std::vector<int64_t>& v) {
        if (n > 0 && p) v.assign(p, p + 2 * n);
    };
    copy_ij(d->fluid_ij, d->n_fluid, r->fluid);
    copy_ij(d->wall_ij, d->n_wall, r->wall);
    copy_ij(d->inlet_ij, d->n_inlet, r->inlet);
    copy_ij(d->outlet_ij, d->n_outlet, r->outlet);
    copy_ij(d->obstacle_ij, d->n_obstacle, r->obstacle);
    if (d->n_inlet > 0 && d->inlet_side) r->inlet_side.assign(d->inlet_side, d->inlet_side + d->n_inlet);
    if (d->n_outlet > 0 && d->outlet_side) r->outlet_side.assign(d->outlet_side, d->outlet_side + d->n_outlet);
    if (d->n_obstacle > 0 && d->obstacle_dirs) r->dirs.assign(d->obstacle_dirs, d->obstacle_dirs + d->n_obstacle);
    r->desc.fluid_ij = r->fluid.empty() ? nullptr : r->fluid.data();
    r->desc.wall_ij = r->wall.empty() ? nullptr : r->wall.data();
    r->desc.inlet_ij = r->inlet.empty() ? nullptr : r->inlet.data();
    r->desc.outlet_ij = r->outlet.empty() ? nullptr : r->outlet.data();
    r->desc.obstacle_ij = r->obstacle.empty() ? nullptr : r->obstacle.data();
    r->desc.inlet_side = r->inlet_side.empty() ? nullptr : r->inlet_side.data();
    r->desc.outlet_side = r->outlet_side.empty() ? nullptr : r->outlet_side.data();
    r->desc.obstacle_dirs = r->dirs.empty() ? nullptr : r->dirs.data();
    const int64_t n_open = d->n_inlet + d->n_outlet;
    if (rows > 0) r->values.assign(open_values, open_values + static_cast<size_t>(rows) * n_open * 2);
    r->rows = rows;
    r->steps = steps;
    r->desc.open_table_rows = std::max<int32_t>(rows, 1);
    r->desc.storage = s->storage;
    r->desc.device = s->device;
    r->desc.pattern = LLB_PATTERN_AB;
    r->bytes = estimate_bytes(r->desc, rows);
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->bytes > s->budget) {
        s->error = "request needs more device memory than the whole budget";
        return LLB_E_NOMEM;
    }
    if (s->stop) return LLB_E_STATE;
    r->id = s->next_id++;
    r->t_submit = now_s();
    s->all[r->id] = r;
    s->queue.push_back(r);
    *request_id = r->id;
    s->cv_work.notify_all();
    return LLB_OK;
}

int llb_server_poll(llb_server_handle s, int64_t id, int32_t* state) {
    if (!s || !state) return LLB_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return LLB_E_INVALID;
    *state = it->second->state;
    return LLB_OK;
}

int llb_server_wait(llb_server_handle s, int64_t id, double timeout_s) {
    if (!s || timeout_s < 0) return LLB_E_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return LLB_E_INVALID;
    auto r = it->second;
    const bool ended = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        return r->state == LLB_REQ_DONE || r->state == LLB_REQ_FAILED;
    });
    if (!ended) return LLB_E_TIMEOUT;
    if (r->state == LLB_REQ_FAILED) {
        s->error = r->error;
        return LLB_E_CUDA;
    }
    return LLB_OK;
}

int llb_server_result(llb_server_handle s, int64_t id, double* rho, double* u, double times[3]) {
    if (!s) return LLB_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return LLB_E_INVALID;
    auto r = it->second;
    if (r->state == LLB_REQ_FAILED) {
        s->error = r->error;
        s->all.erase(it);
        return LLB_E_CUDA;
    }
    if (r->state != LLB_REQ_DONE) return LLB_E_STATE;
    if (rho) std::memcpy(rho, r->rho.data(), sizeof(double) * r->rho.size());
    if (u) std::memcpy(u, r->u.data(), sizeof(double) * r->u.size());
    if (times) {
        times[0] = r->t_submit;
        times[1] = r->t_admit;
        times[2] = r->t_done;
    }
    s->all.erase(it);
    return LLB_OK;
}

int llb_server_stats(llb_server_handle s, llb_server_counters* out) {
    if (!s || !out) return LLB_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->failed = s->failed;
    out->node_steps = s->node_steps;
    out->queued = static_cast<int64_t>(s->queue.size());
    out->running = s->n_running;
    out->bytes_in_use = s->in_use;
    out->chunks = s->chunks;
    out->batch_steps = s->batch_steps;
    out->clock_s = now_s();
    return LLB_OK;
}

const char* llb_server_last_error(llb_server_handle s) { return s ? s->error.c_str() : ""; }

}  // extern "C"

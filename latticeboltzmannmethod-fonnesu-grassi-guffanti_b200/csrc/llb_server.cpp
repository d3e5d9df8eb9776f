// Solve server (C ABI llb_server_*).  Requests -- one lattice, its boundary
// values and a step count -- arrive from any thread and are served by native
// threads that keep every admitted lattice resident on the device.
//
// Batched mode (continuous batching) runs three kinds of threads:
//  * preparer threads admit queued requests -- shortest work first (lattice
//    nodes x steps) by default, or first come, first served -- while their
//    device memory fits the budget and the resident lattice nodes stay under
//    a cap (enough nodes to keep HBM busy; more only stretches every
//    request's time on the device), and create each lattice (mask build,
//    compacted planes, allocation, upload) on a stream of its own, several at
//    a time;
//  * the worker moves prepared lattices into one of two lanes, each a batch on
//    its own stream (lattices of fewer than 2^20 nodes in the small lane), and
//    advances each lane chunk by chunk, max_chunk steps at a time: a lattice
//    carries its own stop step, so one that finishes inside a chunk stops
//    there on the device while the others run on.  The lanes run
//    concurrently and independently: a lane whose chunk is done is drained
//    and relaunched at once while the other runs on.  The small lane's stream
//    has the higher scheduling priority, so a small request keeps its own step
//    rate beside large lattices.  Prepared lattices join at their lane's next
//    chunk boundary, so their work overlaps the work already running;
//  * the reaper takes finished lattices out of the worker's way, copies their
//    result -- the rho and u the reference's Lattice holds after
//    perform_lbm(steps) -- to host memory and frees them, which returns their
//    bytes to the budget.
//
// Sequential mode serves the same requests one at a time through the plain
// single-lattice path (the comparison for the batched mode).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/llalbm_cuda.h"
#include "llb_handle.h"

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
    llb_handle h = nullptr;     // the lattice while it is prepared, running or retired
    int rc = LLB_OK;            // outcome of its steps
    bool counted_nodes = false;  // its nodes count against the resident-node cap
    std::vector<double> rho, u;
    std::string error;
};

// Device bytes a lattice of this description holds once created, at most:
// two population buffers, the node mask, bounce bits and open-node index, the
// macroscopic outputs and the boundary-value ring (plus a small fixed
// allowance), and -- unless the lattice cannot be obstacle-rich -- its
// compacted planes and their tables.  Admission reserves this bound, so the
// bytes in use never exceed the budget; the preparer then charges the bytes
// the lattice actually holds.
int64_t estimate_bytes(const llb_desc& d, int32_t rows) {
    const int64_t elem = d.storage == LLB_STORE_F64 ? 8 : d.storage == LLB_STORE_F32S ? 4 : 2;
    const int64_t align = 256 / elem;
    const int64_t n = (d.rows + align - 1) / align * align * d.cols;
    const int64_t nn = d.rows * d.cols;
    const int64_t open = std::max<int64_t>(d.n_inlet + d.n_outlet, 1);
    int64_t bytes = 2 * 9 * elem * n + 6 * n + 24 * nn + 16 * open * std::max<int32_t>(rows, 1) + (1 << 16);
    // a node that is not PLAIN has one of the non-active nodes (or a node
    // outside the lattice) among its eight neighbours, and each of those
    // neighbours at most eight such nodes
    const int64_t active = d.n_fluid + d.n_inlet + d.n_outlet;
    const int64_t nonplain_max = 8 * (nn - active + 2 * (d.rows + d.cols) + 4);
    if (static_cast<double>(nonplain_max) >= TMA_MIN_NONPLAIN * static_cast<double>(active)) {
        // slots: the active nodes, each column padded to a 32-byte sector
        const int64_t slots = active + d.cols * (32 / elem) + align;
        const int64_t nseg = (d.rows + 31) / 32;
        bytes += 2 * 9 * elem * slots + 6 * slots + 8 * d.cols * nseg + 8 * (slots / 32 + d.cols) + 4 * (d.cols + 1);
    }
    return bytes;
}

}  // namespace

struct llb_server {
    int device = 0;
    int storage = LLB_STORE_F32S;
    int mode = LLB_SERVE_BATCHED;
    int64_t budget = 0;
    int32_t max_chunk = 256;
    int64_t node_cap = LLB_SERVE_DEFAULT_NODE_CAP;  // resident lattice nodes, at most (batched mode)
    int order = LLB_ADMIT_SHORTEST_FIRST;
    int64_t resident_nodes = 0;
    llb_batch_handle batch[2] = {nullptr, nullptr};  // small lane, large lane
    std::mutex mu;
    std::condition_variable cv_prep;   // the preparer: queued requests, freed bytes, stop
    std::condition_variable cv_work;   // the worker: prepared lattices, stop
    std::condition_variable cv_reap;   // the reaper: finished lattices, worker done
    std::condition_variable cv_done;   // waiters: a request finished
    std::deque<std::shared_ptr<Request>> queue;   // submitted, not admitted
    std::deque<std::shared_ptr<Request>> ready;   // created on the device, waiting for a lane
    std::deque<std::shared_ptr<Request>> dying;   // out of their lane, waiting for the result copy
    std::map<int64_t, std::shared_ptr<Request>> all;
    std::vector<std::shared_ptr<Request>> running[2];  // per lane; touched by the worker only
    int64_t admitted = 0;              // admitted and not finished
    int64_t next_id = 1;
    int64_t in_use = 0;
    bool stop = false, preparer_done = false, worker_done = false;
    int preparers_live = 0;
    std::vector<std::thread> preparers;
    std::thread worker, reaper;
    int64_t node_steps = 0;
    int64_t completed = 0;
    int64_t failed = 0;
    int64_t chunks = 0;
    int64_t batch_steps = 0;
    double admit_s = 0, wait_s = 0, retire_s = 0;
    std::string error;
};

namespace {

// Marks a request finished and returns its bytes to the budget (its lattice
// is already destroyed).
void complete(llb_server_handle s, const std::shared_ptr<Request>& r, int rc, const std::string& msg) {
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
    s->admitted -= 1;
    if (r->counted_nodes) s->resident_nodes -= r->desc.rows * r->desc.cols;
    s->cv_done.notify_all();
    s->cv_prep.notify_all();
}

// Copies the result of a finished lattice (rc == LLB_OK) and destroys it.
void retire(llb_server_handle s, const std::shared_ptr<Request>& r, int rc, const char* what) {
    llb_handle h = r->h;
    if (rc == LLB_OK) {
        const size_t N = static_cast<size_t>(r->desc.rows * r->desc.cols);
        r->rho.resize(N);
        r->u.resize(2 * N);
        rc = llb_compute_macro(h, r->rho.data(), r->u.data());
    }
    std::string msg;
    if (rc != LLB_OK) msg = std::string(what) + ": " + (h ? llb_last_error(h) : llb_last_error(nullptr));
    if (h) llb_destroy(h);
    r->h = nullptr;
    complete(s, r, rc, msg);
}

// One request through the plain single-lattice path: steps - 1 collisions
// (llb_init is the first), then rho and u of the state the last step reads.
void serve_plain(llb_server_handle s, const std::shared_ptr<Request>& r) {
    llb_desc d = r->desc;
    int rc = llb_create(&d, &r->h);
    if (rc == LLB_OK && r->rows > 0) rc = llb_set_open_values(r->h, 0, r->rows, r->values.data());
    if (rc == LLB_OK) rc = llb_init(r->h, 0);
    int64_t left = r->steps - 2;
    while (rc == LLB_OK && left > 0) {
        const int32_t n = static_cast<int32_t>(std::min<int64_t>(left, 1 << 20));
        rc = llb_step(r->h, n, 0);
        left -= n;
    }
    if (rc == LLB_OK) rc = llb_synchronize(r->h);
    retire(s, r, rc, "plain path");
}

void sequential_loop(llb_server_handle s) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_prep.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) return;  // stop requested and nothing left
            r = s->queue.front();
            s->queue.pop_front();
            r->state = LLB_REQ_RUNNING;
            r->t_admit = now_s();
            s->in_use += r->bytes;
            s->admitted += 1;
        }
        serve_plain(s, r);
    }
}

constexpr int64_t LARGE_LANE_NODES = 1 << 20;

int lane_of(const Request& r) { return r.desc.rows * r.desc.cols >= LARGE_LANE_NODES ? 1 : 0; }

// The queued request admitted next (shortest work first, or the oldest), if
// it fits the budget and the resident-node cap; queue.end() otherwise.  A
// request is always admitted when nothing else runs.  Called with s->mu held.
std::deque<std::shared_ptr<Request>>::iterator next_admission(llb_server_handle s) {
    auto pick = s->queue.begin();
    if (pick == s->queue.end()) return pick;
    if (s->order == LLB_ADMIT_SHORTEST_FIRST) {
        auto work = [](const Request& r) { return r.desc.rows * r.desc.cols * r.steps; };
        for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
            if (work(**it) < work(**pick)) pick = it;
    }
    const Request& r = **pick;
    if (s->admitted == 0) return pick;
    if (s->in_use + r.bytes > s->budget) return s->queue.end();
    if (s->resident_nodes + r.desc.rows * r.desc.cols > s->node_cap) return s->queue.end();
    return pick;
}

void preparer_loop(llb_server_handle s) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_prep.wait(lk, [&] { return s->stop || next_admission(s) != s->queue.end(); });
            if (s->stop) {
                if (--s->preparers_live == 0) {
                    s->preparer_done = true;
                    s->cv_work.notify_all();
                }
                return;
            }
            auto it = next_admission(s);
            r = *it;
            s->queue.erase(it);
            r->state = LLB_REQ_RUNNING;
            r->t_admit = now_s();
            s->in_use += r->bytes;
            s->admitted += 1;
            s->resident_nodes += r->desc.rows * r->desc.cols;
            r->counted_nodes = true;
        }
        const double t0 = now_s();
        llb_desc d = r->desc;
        int rc = llb_create(&d, &r->h);
        if (rc == LLB_OK && r->rows > 0) rc = llb_set_open_values(r->h, 0, r->rows, r->values.data());
        // the compacted planes of an obstacle-rich lattice (the lanes step
        // those on compacted planes, the others on dense ones), built here
        // rather than on the worker's path
        if (rc == LLB_OK && obstacle_rich(*r->h)) llb_set_pipeline(r->h, -3);
        if (rc == LLB_OK) rc = llb_synchronize(r->h);
        int64_t actual = 0;
        if (rc == LLB_OK) rc = llb_device_bytes(r->h, &actual);
        if (rc != LLB_OK) {
            retire(s, r, rc, "admission failed");
            continue;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use += actual - r->bytes;
        r->bytes = actual;
        s->admit_s += now_s() - t0;
        s->ready.push_back(r);
        s->cv_work.notify_all();
    }
}

void reaper_loop(llb_server_handle s) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_reap.wait(lk, [&] { return !s->dying.empty() || s->worker_done; });
            if (s->dying.empty()) return;
            r = s->dying.front();
            s->dying.pop_front();
        }
        const double t0 = now_s();
        retire(s, r, r->rc, "batched step");
        std::lock_guard<std::mutex> lk(s->mu);
        s->retire_s += now_s() - t0;
    }
}

// Waits for a lane's chunk, measures it, hands what it finished to the reaper.
void drain_lane(llb_server_handle s, int ln) {
    llb_batch_handle b = s->batch[ln];
    const double t0 = now_s();
    const int rc = llb_batch_synchronize(b);
    std::vector<std::shared_ptr<Request>> keep;
    for (auto& r : s->running[ln]) {
        if (r->remaining > 0 && rc == LLB_OK) {
            keep.push_back(r);
            continue;
        }
        llb_handle h = nullptr;
        const int dr = llb_batch_detach(b, r->slot, &h);
        if (dr == LLB_OK) {
            r->h = h;
            r->rc = rc;
        } else {
            llb_batch_remove(b, r->slot);
            r->h = nullptr;
            r->rc = dr;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->dying.push_back(r);
        s->cv_reap.notify_all();
    }
    s->running[ln].swap(keep);
    std::lock_guard<std::mutex> lk(s->mu);
    s->wait_s += now_s() - t0;
}

// Next chunk of a lane: max_chunk steps, or fewer when every running lattice
// finishes sooner; a lattice that finishes inside the chunk stops at its own
// stop step on the device.
void launch_lane(llb_server_handle s, int ln) {
    llb_batch_handle b = s->batch[ln];
    int64_t n = 0;
    for (auto& r : s->running[ln]) n = std::max(n, r->remaining);
    n = std::min<int64_t>(n, s->max_chunk);
    const int rc = llb_batch_step(b, static_cast<int32_t>(n));
    for (auto& r : s->running[ln]) r->remaining -= std::min(n, r->remaining);
    std::lock_guard<std::mutex> lk(s->mu);
    if (rc != LLB_OK) {
        // every running request of the lane fails at its next drain
        for (auto& r : s->running[ln]) r->remaining = 0;
        s->error = std::string("batched step failed: ") + llb_batch_last_error(b);
    }
    s->chunks += 1;
    s->batch_steps += n;
}

// The lanes are independent: whichever lane's chunk has finished is drained
// and relaunched at once, while the other lane keeps running.
void batched_loop(llb_server_handle s) {
    bool inflight[2] = {false, false};  // a chunk was launched on the lane and not yet drained
    for (;;) {
        const bool idle = s->running[0].empty() && s->running[1].empty() && !inflight[0] && !inflight[1];
        std::deque<std::shared_ptr<Request>> joining;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (idle) s->cv_work.wait(lk, [&] { return !s->ready.empty() || s->preparer_done; });
            if (idle && s->ready.empty() && s->preparer_done) {
                s->worker_done = true;
                s->cv_reap.notify_all();
                return;
            }
            joining.swap(s->ready);
        }
        // 1. prepared lattices join their lane (step 0 queued on the lane's stream,
        //    behind a chunk in flight)
        for (auto& r : joining) {
            const int ln = lane_of(*r);
            int32_t slot = -1;
            const int rc = llb_batch_attach(s->batch[ln], r->h, &slot);
            if (rc != LLB_OK) {
                r->rc = rc;
                std::lock_guard<std::mutex> lk(s->mu);
                s->dying.push_back(r);
                s->cv_reap.notify_all();
                continue;
            }
            r->slot = slot;
            r->remaining = r->steps - 2;  // step 0 was the first collision
            // the lattice stops on the device after its last step, whatever the chunk
            llb_handle view = nullptr;
            int64_t t_now = 0;
            if (llb_batch_lattice(s->batch[ln], slot, &view) == LLB_OK && llb_get_step(view, &t_now) == LLB_OK)
                llb_batch_set_stop(s->batch[ln], slot, t_now + r->remaining);
            s->running[ln].push_back(r);
        }
        // 2. every lane whose chunk is done (or that has none): drain, relaunch
        bool progressed = !joining.empty();
        for (int ln = 0; ln < 2; ++ln) {
            if (inflight[ln]) {
                int32_t done = 0;
                if (llb_batch_query(s->batch[ln], &done) == LLB_OK && !done) continue;
                inflight[ln] = false;
                progressed = true;
            } else if (s->running[ln].empty()) {
                continue;
            }
            drain_lane(s, ln);
            if (s->running[ln].empty()) continue;
            launch_lane(s, ln);
            inflight[ln] = true;
            progressed = true;
        }
        if (!progressed) {
            // both lanes busy: doze until a prepared lattice arrives or a moment passes
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait_for(lk, std::chrono::microseconds(200), [&] { return !s->ready.empty(); });
        }
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
    auto drop = [&](int rc) {
        for (auto& c : s->batch)
            if (c) llb_batch_destroy(c);
        delete s;
        return rc;
    };
    if (mode == LLB_SERVE_BATCHED) {
        for (auto& b : s->batch) {
            const int rc = llb_batch_create(device, storage, &b);
            if (rc != LLB_OK) return drop(rc);
            // obstacle-rich lattices on compacted planes, the others on dense
            // planes (whose all-PLAIN tiles skip the mask), 32 x 2 threads per
            // block, one step per launch: on the config-4 problems dense tiles
            // ran 81.7k MLUPS against 69.0k on compacted planes (B200)
            llb_batch_set_layout(b, LLB_LAYOUT_AUTO);
            llb_batch_set_config(b, 2, 1);
        }
        // the small lane's blocks go first, so small requests keep their own
        // step rate beside large lattices
        llb_batch_set_stream_priority(s->batch[0], std::numeric_limits<int32_t>::min());
    }
    try {
        if (mode == LLB_SERVE_BATCHED) {
            s->reaper = std::thread(reaper_loop, s);
            s->worker = std::thread(batched_loop, s);
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            const int np = static_cast<int>(std::min(4u, std::max(1u, hw / 2)));
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->preparers_live = np;
            }
            for (int i = 0; i < np; ++i) s->preparers.emplace_back(preparer_loop, s);
        } else {
            s->worker = std::thread(sequential_loop, s);
        }
    } catch (...) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = s->preparer_done = s->worker_done = true;
        }
        s->cv_prep.notify_all();
        s->cv_work.notify_all();
        s->cv_reap.notify_all();
        for (auto& t : s->preparers)
            if (t.joinable()) t.join();
        for (std::thread* t : {&s->worker, &s->reaper})
            if (t->joinable()) t->join();
        return drop(LLB_E_NOMEM);
    }
    *out = s;
    return LLB_OK;
}

int llb_server_set_admission(llb_server_handle s, int64_t max_resident_nodes, int32_t order) {
    if (!s || max_resident_nodes < 0 || (order != LLB_ADMIT_SHORTEST_FIRST && order != LLB_ADMIT_FIFO))
        return LLB_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    s->node_cap = max_resident_nodes == 0 ? LLB_SERVE_DEFAULT_NODE_CAP : max_resident_nodes;
    s->order = order;
    s->cv_prep.notify_all();
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
    s->cv_prep.notify_all();
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    // running requests finish: the preparer stops admitting, the worker drains
    // its lanes, the reaper retires the last lattices
    for (auto& t : s->preparers)
        if (t.joinable()) t.join();
    for (std::thread* t : {&s->worker, &s->reaper})
        if (t->joinable()) t->join();
    for (auto& b : s->batch)
        if (b) llb_batch_destroy(b);
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
    s->cv_prep.notify_all();
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
    out->running = s->admitted;
    out->bytes_in_use = s->in_use;
    out->chunks = s->chunks;
    out->batch_steps = s->batch_steps;
    out->clock_s = now_s();
    out->admit_s = s->admit_s;
    out->wait_s = s->wait_s;
    out->retire_s = s->retire_s;
    return LLB_OK;
}

const char* llb_server_last_error(llb_server_handle s) { return s ? s->error.c_str() : ""; }

}  // extern "C"

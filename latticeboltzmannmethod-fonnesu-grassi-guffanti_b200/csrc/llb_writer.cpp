// Output writer (C ABI llb_writer_*): the reference's velocity text files
// (util::writer::write_lattice_file<2>, utils/writers/LatticeWriter.hpp:60-92)
// written off the stepping thread.
//
// A save enqueues a device-to-host copy of u into a pinned slot on the
// lattice's own stream and records an event; the caller goes on enqueuing
// steps.  One writer thread takes the slots in order, waits for each copy's
// event, formats the rows on a few threads and writes the two files.  The
// reference writes each value with `ostream << double` (default flags,
// precision 6, i.e. printf "%.6g" in the C locale) followed by a space, and
// ends each lattice row with std::endl; put_g6 below produces those bytes.
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "llb_handle.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

namespace llb_out {

struct Slot {
    double* buf = nullptr;  // host memory, (R, C, 2) column-major
    size_t cap = 0;         // doubles
    bool pinned = false;    // page-locked (else malloc: host saves without a device)
    cudaEvent_t ev = nullptr;
    int ev_device = -1;
    bool from_device = false;
    int device = 0;
    int64_t R = 0, C = 0, index = 0;
    bool busy = false;
};

}  // namespace llb_out

using llb_out::Slot;

struct llb_writer {
    std::string dir;
    int nthreads = 1;
    std::vector<Slot> slots;
    std::deque<int> queue;  // slots waiting for the writer thread, in save order
    int writing = -1;       // slot the writer thread holds
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::thread io;
    std::string bg_err;  // first error of the background work, not yet returned
    int bg_rc = LLB_OK;
    std::string err;     // message of the last failed call
    int64_t files = 0;
    double wait_s = 0.0, write_s = 0.0;
    std::vector<std::string> bx, by;  // per formatting thread: rows of u_x, u_y
    std::vector<std::vector<double>> bt;  // per formatting thread: its band, row-major
};

namespace {

int wfail(llb_writer_handle w, int rc, const std::string& msg) {
    if (w) w->err = msg;
    return rc;
}

// printf "%.6g" of v (the reference's `ostream << double`).  The six
// significant digits come from the exact binary value: v = m 2^e, so
// m 10^k 2^e with k = 5 - X (X the decimal exponent) is split into its
// integer part q and remainder r with 128-bit integer arithmetic, and q is
// rounded to nearest, ties to even, as printf does.  Values outside the
// fast range (|v| >= 2^52 or X outside [-17, 5], zero, subnormal, inf, nan)
// go through std::to_chars, which the C++ standard specifies as that same
// printf conversion.
using u128 = unsigned __int128;

struct Pow10 {
    u128 p[23];
    double d[48];  // 10^(x - 24) as doubles, for the first guess of X
    Pow10() {
        p[0] = 1;
        for (int k = 1; k < 23; ++k) p[k] = p[k - 1] * 10u;
        for (int x = 0; x < 48; ++x) d[x] = std::pow(10.0, x - 24);
    }
};
const Pow10 kPow10;

char* put_g6_slow(double v, char* p, char* end) {
    return std::to_chars(p, end, v, std::chars_format::general, 6).ptr;
}

char* put_g6(double v, char* p, char* end) {
    uint64_t bits;
    std::memcpy(&bits, &v, sizeof(bits));
    const int be = static_cast<int>((bits >> 52) & 0x7ff);
    if (be == 0 || be == 0x7ff) return put_g6_slow(v, p, end);
    const uint64_t m = (bits & ((1ull << 52) - 1)) | (1ull << 52);
    const int s = 1075 - be;  // v = m 2^-s
    if (s <= 0 || s >= 128) return put_g6_slow(v, p, end);
    // floor(log10 |v|) is X0 or X0 + 1; a comparison picks one, and the
    // exact test below corrects the guess near a power of ten
    int X = static_cast<int>(std::floor((be - 1023) * 0.30102999566398120));
    if (X >= -24 && X < 23 && std::fabs(v) >= kPow10.d[X + 25]) ++X;
    uint64_t N = 0;
    for (int it = 0; it < 4 && !N; ++it) {
        const int k = 5 - X;
        if (k < 0 || k > 22) return put_g6_slow(v, p, end);
        const u128 prod = static_cast<u128>(m) * kPow10.p[k];
        u128 q = prod >> s;
        const u128 r = prod - (q << s);
        const u128 half = static_cast<u128>(1) << (s - 1);
        if (q >= 1000000u) { ++X; continue; }  // X was one too small
        if (q < 100000u) { --X; continue; }    // one too large
        if (r > half || (r == half && (q & 1u))) ++q;
        if (q == 1000000u) { q = 100000u; ++X; }  // rounded up to the next power of ten
        N = static_cast<uint64_t>(q);
    }
    if (!N) return put_g6_slow(v, p, end);
    char d[6];
    for (int i = 5; i >= 0; --i) { d[i] = static_cast<char>('0' + N % 10); N /= 10; }
    int nd = 6;
    while (nd > 1 && d[nd - 1] == '0') --nd;
    if (bits >> 63) *p++ = '-';
    if (X >= -4 && X < 6) {
        if (X >= 0) {
            for (int i = 0; i <= X; ++i) *p++ = d[i];
            if (nd > X + 1) {
                *p++ = '.';
                for (int i = X + 1; i < nd; ++i) *p++ = d[i];
            }
        } else {
            *p++ = '0';
            *p++ = '.';
            for (int i = 0; i < -X - 1; ++i) *p++ = '0';
            for (int i = 0; i < nd; ++i) *p++ = d[i];
        }
    } else {
        *p++ = d[0];
        if (nd > 1) {
            *p++ = '.';
            for (int i = 1; i < nd; ++i) *p++ = d[i];
        }
        *p++ = 'e';
        *p++ = X < 0 ? '-' : '+';
        const int ax = X < 0 ? -X : X;  // 5..17 here
        *p++ = static_cast<char>('0' + ax / 10);
        *p++ = static_cast<char>('0' + ax % 10);
    }
    return p;
}

// Rows [i0, i1) of both component files: value, space; newline after each
// row.  u is column-major (a row's values lie R apart), so the band is first
// transposed tile by tile into t (row-major) and then formatted in order.
void format_rows(const double* u, int64_t R, int64_t C, int64_t i0, int64_t i1, std::string& sx, std::string& sy,
                 std::vector<double>& t) {
    constexpr int64_t TILE = 32;
    const int64_t N = R * C, B = i1 - i0;
    t.resize(static_cast<size_t>(2 * B * C));
    for (int d = 0; d < 2; ++d)
        for (int64_t jb = 0; jb < C; jb += TILE)
            for (int64_t ib = i0; ib < i1; ib += TILE) {
                const int64_t je = std::min(C, jb + TILE), ie = std::min(i1, ib + TILE);
                for (int64_t j = jb; j < je; ++j) {
                    const double* src = u + d * N + j * R;
                    double* dst = t.data() + d * B * C + j;
                    for (int64_t i = ib; i < ie; ++i) dst[(i - i0) * C] = src[i];
                }
            }
    for (int d = 0; d < 2; ++d) {
        std::string& s = d == 0 ? sx : sy;
        s.resize(static_cast<size_t>(B * (C * 14 + 1)));  // at most 13 characters and a space per value
        char* p = s.data();
        const double* row = t.data() + d * B * C;
        for (int64_t i = 0; i < B; ++i, row += C) {
            for (int64_t j = 0; j < C; ++j) {
                p = put_g6(row[j], p, p + 32);
                *p++ = ' ';
            }
            *p++ = '\n';
        }
        s.resize(static_cast<size_t>(p - s.data()));
    }
}

// Formats and writes one slot's two files; returns an error message or "".
// Formats band t of T; false if its buffers could not be allocated.
bool format_band(llb_writer* w, const Slot& s, int t, int T) noexcept {
    try {
        format_rows(s.buf, s.R, s.C, s.R * t / T, s.R * (t + 1) / T, w->bx[t], w->by[t], w->bt[t]);
        return true;
    } catch (...) {
        return false;
    }
}

std::string write_slot(llb_writer* w, const Slot& s) {
    const int64_t R = s.R;
    const int T = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(w->nthreads, R)));
    try {
        if (static_cast<int>(w->bx.size()) < T) {
            w->bx.resize(T);
            w->by.resize(T);
            w->bt.resize(T);
        }
    } catch (...) {
        return "host allocation of the formatting buffers failed";
    }
    // bands 1..T-1 on helper threads (a band whose thread cannot start runs here)
    std::vector<char> ok(static_cast<size_t>(T), 0);
    std::vector<std::thread> pool;
    std::vector<int> inline_bands;
    for (int t = 1; t < T; ++t) {
        try {
            pool.emplace_back([w, &s, &ok, t, T] { ok[static_cast<size_t>(t)] = format_band(w, s, t, T); });
        } catch (...) {
            inline_bands.push_back(t);
        }
    }
    ok[0] = format_band(w, s, 0, T);
    for (int t : inline_bands) ok[static_cast<size_t>(t)] = format_band(w, s, t, T);
    for (auto& th : pool) th.join();
    for (int t = 0; t < T; ++t)
        if (!ok[static_cast<size_t>(t)]) return "host allocation of the formatting buffers failed";
    for (int d = 0; d < 2; ++d) {
        const std::string path = w->dir + "/output-" + std::to_string(s.index) + (d == 0 ? "u_x.txt" : "u_y.txt");
        std::FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return "cannot open " + path + ": " + std::strerror(errno);
        bool ok = true;
        for (int t = 0; t < T && ok; ++t) {
            const std::string& b = d == 0 ? w->bx[t] : w->by[t];
            ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
        }
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) return "short write to " + path;
    }
    return "";
}

void io_loop(llb_writer* w) {
    std::unique_lock<std::mutex> lk(w->mu);
    for (;;) {
        w->cv_work.wait(lk, [&] { return w->stop || !w->queue.empty(); });
        if (w->queue.empty()) return;  // stop requested and nothing left
        const int k = w->queue.front();
        w->queue.pop_front();
        w->writing = k;
        Slot& s = w->slots[k];
        lk.unlock();
        std::string msg;
        int rc = LLB_OK;
        const double t0 = now_s();
        if (s.from_device) {
            cudaError_t e = cudaSetDevice(s.device);
            if (e == cudaSuccess) e = cudaEventSynchronize(s.ev);
            if (e != cudaSuccess) {
                msg = std::string("copy of u: ") + cudaGetErrorString(e);
                rc = LLB_E_CUDA;
            }
        }
        const double t1 = now_s();
        if (rc == LLB_OK) {
            msg = write_slot(w, s);
            if (!msg.empty()) rc = LLB_E_INVALID;
        }
        const double t2 = now_s();
        lk.lock();
        w->wait_s += t1 - t0;
        w->write_s += t2 - t1;
        if (rc == LLB_OK) ++w->files;
        else if (w->bg_rc == LLB_OK) {
            w->bg_rc = rc;
            w->bg_err = msg;
        }
        s.busy = false;
        w->writing = -1;
        w->cv_done.notify_all();
    }
}

// Takes the background error, if any, for the caller to return.
int take_bg(llb_writer* w) {
    if (w->bg_rc == LLB_OK) return LLB_OK;
    const int rc = w->bg_rc;
    w->err = w->bg_err;
    w->bg_rc = LLB_OK;
    w->bg_err.clear();
    return rc;
}

void release_buf(Slot& s) {
    if (s.buf) {
        if (s.pinned) cudaFreeHost(s.buf);
        else std::free(s.buf);
    }
    s.buf = nullptr;
    s.cap = 0;
    s.pinned = false;
}

// A free slot with room for n doubles, or -1 with w->err set.  Device saves
// need page-locked memory for the copy to be asynchronous; host saves take
// ordinary memory when no device is present.
int acquire(llb_writer* w, std::unique_lock<std::mutex>& lk, size_t n, bool device, int& rc) {
    int k = -1;
    w->cv_done.wait(lk, [&] {
        for (size_t i = 0; i < w->slots.size(); ++i)
            if (!w->slots[i].busy) { k = static_cast<int>(i); return true; }
        return false;
    });
    Slot& s = w->slots[k];
    if (s.cap < n || (device && !s.pinned)) {
        release_buf(s);
        if (cudaHostAlloc(reinterpret_cast<void**>(&s.buf), n * sizeof(double), cudaHostAllocPortable) == cudaSuccess) {
            s.pinned = true;
        } else {
            cudaGetLastError();
            s.buf = device ? nullptr : static_cast<double*>(std::malloc(n * sizeof(double)));
            if (!s.buf) {
                rc = wfail(w, LLB_E_NOMEM, "host allocation of the output slot failed");
                return -1;
            }
        }
        s.cap = n;
    }
    return k;
}

}  // namespace

extern "C" {

int llb_writer_create(const char* dir, int32_t slots, int32_t threads, llb_writer_handle* out) {
    if (!dir || !out || slots < 0 || slots > 64 || threads < 0 || threads > 256) return LLB_E_INVALID;
    *out = nullptr;
    llb_writer* w = new (std::nothrow) llb_writer;
    if (!w) return LLB_E_NOMEM;
    w->dir = dir;
    w->slots.resize(slots ? slots : 3);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    w->nthreads = threads ? threads : static_cast<int>(std::min(16u, hw));
    try {
        w->io = std::thread(io_loop, w);
    } catch (...) {
        delete w;
        return LLB_E_NOMEM;
    }
    *out = w;
    return LLB_OK;
}

int llb_writer_save_u(llb_writer_handle w, llb_handle h, int64_t index) {
    if (!w || !h || index < 0) return wfail(w, LLB_E_INVALID, "bad arguments");
    if (!h->macro_valid) return wfail(w, LLB_E_STATE, "no step has written u yet");
    std::unique_lock<std::mutex> lk(w->mu);
    int rc = take_bg(w);
    if (rc) return rc;
    const size_t n = static_cast<size_t>(h->R * h->C) * 2;
    const int k = acquire(w, lk, n, true, rc);
    if (k < 0) return rc;
    Slot& s = w->slots[k];
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess && s.ev_device != h->device) {
        if (s.ev) cudaEventDestroy(s.ev);
        s.ev = nullptr;
        s.ev_device = -1;
        e = cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming);
        if (e == cudaSuccess) s.ev_device = h->device;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.buf, h->d_u, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(s.ev, h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return wfail(w, LLB_E_CUDA, std::string("enqueueing the copy of u: ") + cudaGetErrorString(e));
    }
    s.from_device = true;
    s.device = h->device;
    s.R = h->R;
    s.C = h->C;
    s.index = index;
    s.busy = true;
    w->queue.push_back(k);
    w->cv_work.notify_one();
    return LLB_OK;
}

int llb_writer_save_host(llb_writer_handle w, const double* u, int64_t rows, int64_t cols, int64_t index) {
    if (!w || !u || rows < 1 || cols < 1 || rows > (1 << 30) || cols > (1 << 30) || rows * cols > (1LL << 36) ||
        index < 0)
        return wfail(w, LLB_E_INVALID, "bad arguments");
    std::unique_lock<std::mutex> lk(w->mu);
    int rc = take_bg(w);
    if (rc) return rc;
    const size_t n = static_cast<size_t>(rows * cols) * 2;
    const int k = acquire(w, lk, n, false, rc);
    if (k < 0) return rc;
    Slot& s = w->slots[k];
    std::memcpy(s.buf, u, n * sizeof(double));
    s.from_device = false;
    s.R = rows;
    s.C = cols;
    s.index = index;
    s.busy = true;
    w->queue.push_back(k);
    w->cv_work.notify_one();
    return LLB_OK;
}

int llb_writer_flush(llb_writer_handle w) {
    if (!w) return LLB_E_INVALID;
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv_done.wait(lk, [&] {
        return std::none_of(w->slots.begin(), w->slots.end(), [](const Slot& s) { return s.busy; });
    });
    return take_bg(w);
}

int llb_writer_stats(llb_writer_handle w, int64_t* files, double* wait_s, double* write_s) {
    if (!w) return LLB_E_INVALID;
    std::lock_guard<std::mutex> lk(w->mu);
    if (files) *files = w->files;
    if (wait_s) *wait_s = w->wait_s;
    if (write_s) *write_s = w->write_s;
    return LLB_OK;
}

int llb_writer_destroy(llb_writer_handle w) {
    if (!w) return LLB_OK;
    const int rc = llb_writer_flush(w);
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->stop = true;
    }
    w->cv_work.notify_all();
    if (w->io.joinable()) w->io.join();
    for (Slot& s : w->slots) {
        release_buf(s);
        if (s.ev) {
            cudaSetDevice(s.ev_device);
            cudaEventDestroy(s.ev);
        }
    }
    delete w;
    return rc;
}

const char* llb_writer_last_error(llb_writer_handle w) { return w ? w->err.c_str() : "null writer"; }

}  // extern "C"

// bpc_server.cu -- request server: encode and decode requests of mixed size,
// admitted against a device-memory budget and overlapped on the GPU.
//
// Memory.  The budget is reserved once, at creation, as one device arena; every
// request's output (the slot stream of an encode, the coefficients of a decode)
// is carved out of it first-fit and returned to it by bpc_server_release.  No
// cudaMalloc or cudaFree runs while requests are served, so an allocation never
// synchronises the device under other requests' kernels.  Inputs and LUTs are
// the caller's device buffers and stay resident there.
//
// Scheduling.  Requests are admitted strictly in arrival order (no request can
// starve behind smaller ones) whenever one of the `max_in_flight` streams is
// free and the head request's output fits in the arena.  Each admitted request
// is one launch of the plain coder (work-ordered for requests of more than two
// warp waves, its scratch allocated with the output) on its own stream,
// followed by a 4-byte copy of its status word and an event; launches on different streams run
// concurrently, so the CTAs of a newly admitted request fill the SMs that an
// earlier request's tail leaves idle.  Each slot has one stream per priority
// class (up to three hardware priority levels) and a request runs in the class
// of its size (up to 2^22 coefficients; up to 2^24; larger): the block
// scheduler then dispatches a small request's CTAs ahead of the not-yet-started
// CTAs of a large one, so small requests are not stuck behind large ones
// (running CTAs are never preempted).  The device feeds streams through a
// limited number of hardware queues (CUDA_DEVICE_MAX_CONNECTIONS, 8 unless the
// process sets it before CUDA initialises); streams that share a queue run in
// order, so a process serving small requests beside large ones should set it
// to 32 (8 slots x 3 classes = 24 streams).  A worker thread admits
// requests and polls the events; the latency of a request is measured on the
// host clock from its submission to the moment the worker sees its event
// complete.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bpc_paco.h"
#include "bpc_arena.h"
#include "bpc_kernels.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Lut {
    const int *d;
    int n, passes, levels;
};

struct Request {
    long long ticket;
    int dir;
    const int *in;
    int X, Y, lut, cb;
    size_t bytes;        // output, plus the work-order scratch when sched_off > 0
    size_t sched_off;    // byte offset of that scratch in the allocation (0: none)
    Clock::time_point t0;
};

struct Slot {
    std::vector<cudaStream_t> st_by_prio;  // [0] = highest priority
    cudaStream_t st = nullptr;             // stream of the current request
    cudaEvent_t ev = nullptr;
    int *d_status = nullptr;
    int *h_status = nullptr;
    bool busy = false;
    Request r{};
    size_t off = 0;
};

struct Done {
    long long ticket;
    int *out;
    double us;
    int status;
};

struct Server {
    std::mutex mu;
    std::condition_variable cv;       // worker: new request, release, stop
    std::condition_variable cv_done;  // pollers: new completion
    std::thread worker;
    bool stop = false;
    int device = 0;
    unsigned char *base = nullptr;
    size_t budget = 0;
    bpc::Arena arena;
    std::vector<Lut> luts;
    std::deque<Request> queue;
    std::vector<Slot> slots;
    std::deque<Done> done;
    std::unordered_map<const int *, std::pair<size_t, size_t>> owned;  // output -> (offset, bytes)
    int *d_status = nullptr;
    int *h_status = nullptr;
    long long next_ticket = 0, completed = 0;
    int in_flight = 0;
};

constexpr size_t kAlign = 256;

constexpr int kMaxClasses = 3;

// priority class of a request: 0 (highest) up to 2^22 coefficients, 1 up to
// 2^24, 2 above
int priority_level(int X, int Y, int nprio) {
    const unsigned long long n = (unsigned long long)X * (unsigned long long)Y;
    int lg = 0;
    while ((2ULL << lg) <= n) ++lg;  // floor(log2(n))
    const int p = (lg - 21) / 2;
    return p < 0 ? 0 : (p >= nprio ? nprio - 1 : p);
}

double micros(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::micro>(b - a).count();
}

// enqueue one admitted request on its slot's stream (lock held)
void launch(Server *s, Slot &sl) {
    const Request &r = sl.r;
    const Lut &L = s->luts[r.lut];
    int *out = reinterpret_cast<int *>(s->base + sl.off);
    sl.st = sl.st_by_prio[priority_level(r.X, r.Y, (int)sl.st_by_prio.size())];
    int rc = cudaMemsetAsync(sl.d_status, 0, sizeof(int), sl.st) == cudaSuccess ? BPC_OK : BPC_ERR_CUDA;
    int *sched = r.sched_off ? reinterpret_cast<int *>(s->base + sl.off + r.sched_off) : nullptr;
    // several requests share the SMs at once: the forms with the fewest
    // instructions, not the latency forms of a launch alone on the GPU
    if (!rc)
        rc = bpc::code_device(r.dir == BPC_CODE, r.in, out, r.X, r.Y, L.d, L.n, L.passes, L.levels, r.cb, sl.d_status,
                              nullptr, 0, sl.st, 0, -1, sched, false);
    if (!rc && cudaMemcpyAsync(sl.h_status, sl.d_status, sizeof(int), cudaMemcpyDeviceToHost, sl.st) != cudaSuccess)
        rc = BPC_ERR_CUDA;
    if (!rc && cudaEventRecord(sl.ev, sl.st) != cudaSuccess) rc = BPC_ERR_CUDA;
    if (rc) {  // nothing useful was queued: report the failure, give the memory back
        s->arena.release(sl.off, r.bytes);
        s->done.push_back({r.ticket, nullptr, micros(r.t0, Clock::now()), rc});
        s->cv_done.notify_all();
        return;
    }
    sl.busy = true;
    s->in_flight++;
}

void work(Server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        for (Slot &sl : s->slots) {  // completions
            if (!sl.busy) continue;
            const cudaError_t e = cudaEventQuery(sl.ev);
            if (e == cudaErrorNotReady) continue;
            const Clock::time_point t = Clock::now();
            const int st = e == cudaSuccess ? *sl.h_status : BPC_ERR_CUDA;
            int *out = reinterpret_cast<int *>(s->base + sl.off);
            s->owned[out] = {sl.off, sl.r.bytes};
            s->done.push_back({sl.r.ticket, out, micros(sl.r.t0, t), st});
            sl.busy = false;
            s->in_flight--;
            s->completed++;
            progressed = true;
        }
        if (progressed) s->cv_done.notify_all();
        while (!s->stop && !s->queue.empty()) {  // admission, strictly first come first served
            Slot *free_slot = nullptr;
            for (Slot &sl : s->slots)
                if (!sl.busy) {
                    free_slot = &sl;
                    break;
                }
            if (!free_slot) break;
            size_t off = 0;
            if (!s->arena.alloc(s->queue.front().bytes, &off)) break;
            free_slot->r = s->queue.front();
            free_slot->off = off;
            s->queue.pop_front();
            launch(s, *free_slot);
            progressed = true;
        }
        if (s->stop && s->in_flight == 0) break;
        if (s->in_flight == 0) {
            // nothing on the GPU: sleep until a submission, a release or stop
            s->cv.wait(lk);
        } else if (!progressed) {
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        }
    }
}

Server *as_server(void *p) { return static_cast<Server *>(p); }

}  // namespace

extern "C" int bpc_server_create(long long budget_bytes, int max_in_flight, void **srv) {
    if (!srv || budget_bytes <= 0 || max_in_flight < 1 || max_in_flight > 64) return BPC_ERR_ARG;
    *srv = nullptr;
    Server *s = new Server();
    cudaGetDevice(&s->device);
    s->budget = (size_t)budget_bytes / kAlign * kAlign;
    cudaError_t e = cudaMalloc(&s->base, s->budget);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "bpc: server arena of %lld bytes: %s\n", budget_bytes, cudaGetErrorString(e));
        cudaGetLastError();
        delete s;
        return BPC_ERR_NOMEM;
    }
    s->arena.init(s->budget);
    s->slots.resize(max_in_flight);
    int least = 0, greatest = 0;
    bool ok = cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess &&
              cudaMalloc(&s->d_status, sizeof(int) * max_in_flight) == cudaSuccess &&
              cudaHostAlloc(&s->h_status, sizeof(int) * max_in_flight, cudaHostAllocDefault) == cudaSuccess;
    int nprio = ok ? least - greatest + 1 : 1;
    nprio = nprio < 1 ? 1 : (nprio > kMaxClasses ? kMaxClasses : nprio);
    for (int k = 0; ok && k < max_in_flight; ++k) {
        Slot &sl = s->slots[k];
        sl.d_status = s->d_status + k;
        sl.h_status = s->h_status + k;
        for (int q = 0; ok && q < nprio; ++q) {
            cudaStream_t st = nullptr;
            ok = cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, greatest + q) == cudaSuccess;
            if (ok) sl.st_by_prio.push_back(st);
        }
        ok = ok && cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        std::fprintf(stderr, "bpc: server set-up failed\n");
        for (Slot &sl : s->slots) {
            if (sl.ev) cudaEventDestroy(sl.ev);
            for (cudaStream_t st : sl.st_by_prio) cudaStreamDestroy(st);
        }
        cudaFree(s->d_status);
        cudaFreeHost(s->h_status);
        cudaFree(s->base);
        delete s;
        return BPC_ERR_CUDA;
    }
    s->worker = std::thread(work, s);
    *srv = s;
    return BPC_OK;
}

extern "C" int bpc_server_register_lut(void *srv, const int *d_lut, int lut_n, int passes, int levels, int *lut_id) {
    Server *s = as_server(srv);
    if (!s || !d_lut || lut_n <= 0 || !lut_id || (passes != 2 && passes != 3) || levels < 1 || levels > 16)
        return BPC_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    s->luts.push_back({d_lut, lut_n, passes, levels});
    *lut_id = (int)s->luts.size() - 1;
    return BPC_OK;
}

extern "C" long long bpc_server_submit(void *srv, int direction, const int *d_in, int X, int Y, int lut_id,
                                       int cb_size) {
    Server *s = as_server(srv);
    if (!s || !d_in || (direction != BPC_CODE && direction != BPC_DECODE) || (cb_size != 64 && cb_size != 32) ||
        X <= 0 || Y <= 0 || X % cb_size || Y % cb_size ||
        !bpc::aligned_to(d_in, direction == BPC_CODE ? bpc::kEncInAlign : bpc::kDecInAlign))
        return BPC_ERR_ARG;
    size_t bytes = ((size_t)X * (size_t)Y * sizeof(int) + kAlign - 1) / kAlign * kAlign;
    size_t sched_off = 0;
    const int ncb = (X / cb_size) * (Y / cb_size);
    // decided for the server's device, as the worker thread (which has that
    // device current) decides again when it launches the request
    if (bpc::order_pays(direction == BPC_CODE, ncb, cb_size, s->device)) {  // large request: work-ordered coding
        sched_off = bytes;
        bytes += ((size_t)bpc::sched_ints(ncb, cb_size) * sizeof(int) + kAlign - 1) / kAlign * kAlign;
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (lut_id < 0 || lut_id >= (int)s->luts.size() || s->stop) return BPC_ERR_ARG;
    if (bytes > s->budget) return BPC_ERR_TOO_LARGE;  // could never be admitted
    const long long t = s->next_ticket++;
    s->queue.push_back({t, direction, d_in, X, Y, lut_id, cb_size, bytes, sched_off, Clock::now()});
    s->cv.notify_one();
    return t;
}

extern "C" int bpc_server_cancel(void *srv, long long ticket) {
    Server *s = as_server(srv);
    if (!s) return BPC_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
        if (it->ticket != ticket) continue;
        s->done.push_back({ticket, nullptr, micros(it->t0, Clock::now()), BPC_ERR_CANCELLED});
        s->queue.erase(it);
        s->cv.notify_one();  // the next request may now be at the head
        s->cv_done.notify_all();
        return BPC_OK;
    }
    return BPC_ERR_ARG;  // unknown, already on the GPU, or finished
}

extern "C" int bpc_server_poll(void *srv, int max, int wait_us, long long *tickets, int **outputs,
                               double *latency_us, int *status, int *n) {
    Server *s = as_server(srv);
    if (!s || max < 0 || !n) return BPC_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_us > 0)
        s->cv_done.wait_for(lk, std::chrono::microseconds(wait_us), [s] { return !s->done.empty(); });
    int k = 0;
    for (; k < max && !s->done.empty(); ++k) {
        const Done &d = s->done.front();
        if (tickets) tickets[k] = d.ticket;
        if (outputs) outputs[k] = d.out;
        if (latency_us) latency_us[k] = d.us;
        if (status) status[k] = d.status;
        s->done.pop_front();
    }
    *n = k;
    return BPC_OK;
}

extern "C" int bpc_server_release(void *srv, const int *output) {
    Server *s = as_server(srv);
    if (!s || !output) return BPC_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->owned.find(output);
    if (it == s->owned.end()) return BPC_ERR_ARG;
    s->arena.release(it->second.first, it->second.second);
    s->owned.erase(it);
    s->cv.notify_one();
    return BPC_OK;
}

extern "C" int bpc_server_state(void *srv, long long *queued, long long *in_flight, long long *bytes_used,
                                long long *completed) {
    Server *s = as_server(srv);
    if (!s) return BPC_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    if (queued) *queued = (long long)s->queue.size();
    if (in_flight) *in_flight = s->in_flight;
    if (bytes_used) *bytes_used = (long long)s->arena.used();
    if (completed) *completed = s->completed;
    return BPC_OK;
}

extern "C" int bpc_server_destroy(void *srv) {
    Server *s = as_server(srv);
    if (!s) return BPC_ERR_ARG;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;  // queued requests are dropped; in-flight ones finish
        s->cv.notify_all();
    }
    s->worker.join();
    for (Slot &sl : s->slots) {
        cudaEventDestroy(sl.ev);
        for (cudaStream_t st : sl.st_by_prio) cudaStreamDestroy(st);
    }
    cudaFree(s->d_status);
    cudaFreeHost(s->h_status);
    cudaFree(s->base);
    delete s;
    return BPC_OK;
}

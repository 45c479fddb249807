// oza_server.cpp -- request loop for streams of independent FP64 GEMMs with
// continuous batching:
//
//  * submit() queues a request (device pointers, slice count) and returns an id;
//  * one scheduler thread admits queued requests in arrival order while their
//    workspaces fit in a device arena of the configured budget and a stream
//    slot is free, and launches everything it admitted as one grouped batch
//    (the grouped kernels of oza_kernels.cu) on that slot's stream -- a batch
//    of one request runs the single-GEMM launch sequence instead.  Scheme I
//    requests (chosen where Scheme II's 20 moduli cannot reach an accuracy
//    target) always run as a batch of one;
//  * up to max_inflight batches run at once on separate streams, so requests
//    that arrive while a batch is on the GPU are admitted as soon as a slot and
//    memory free up, and their work overlaps on the device;
//  * completion is detected from each batch's event; the workspaces go back to
//    the arena and wait() returns per-request timestamps.
//
// Workspaces and the CRT constant tables stay resident: the arena is one
// allocation made at creation, the tables are uploaded once per device.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "oza_capi.h"
#include "oza_internal.h"
#include "oza_kernels.h"

namespace {

oza_status_t sfail(oza_status_t st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    oza::set_last_error(buf);
    return st;
}

constexpr size_t kAlign = 1024;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator over [0, size) with coalescing of free ranges.
class Arena {
public:
    void reset(size_t size) {
        size_ = size;
        used_ = peak_ = 0;
        free_.clear();
        if (size) free_[0] = size;
    }
    bool alloc(size_t n, size_t* off) {
        n = align_up(n ? n : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            *off = it->first;
            const size_t rest = it->second - n;
            const size_t next = it->first + n;
            free_.erase(it);
            if (rest) free_[next] = rest;
            used_ += n;
            if (used_ > peak_) peak_ = used_;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t n) {
        n = align_up(n ? n : 1);
        used_ -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

private:
    size_t size_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

struct Request {
    uint64_t id = 0;
    size_t M = 0, N = 0, K = 0;
    const double* A = nullptr;
    const double* B = nullptr;
    double* C = nullptr;
    int S = 0;
    int scheme = OZA_SCHEME2;
    size_t ws_bytes = 0, ws_off = 0;
    oza_request_stats_t stats{};
    bool done = false;
};

// Per-request workspace: shiftA, shiftB, A planes, B^T planes, and the GEMM's
// output planes: CRT coefficient bytes (Scheme II) or INT32 groups (Scheme I).
struct WsLayout {
    size_t Mp, Np, Kp, off[5], bytes;
    WsLayout(size_t M, size_t N, size_t K, int S, int scheme = OZA_SCHEME2) {
        Mp = oza::round_up(M, oza::kTileM);
        Np = oza::round_up(N, oza::kTileN);
        Kp = oza::round_up(K, oza::kTileK);
        const size_t s = (size_t)S;
        // Scheme I: one INT32 plane per accumulation unit (groups split at large K)
        const size_t out = scheme == OZA_SCHEME1
                               ? (size_t)oza::make_pairs(scheme, S, K).num_groups * Mp * Np * sizeof(int32_t)
                               : s * Mp * Np;
        const size_t sz[5] = {M * 4, N * 4, s * Mp * Kp, s * Np * Kp, out};
        size_t o = 0;
        for (int i = 0; i < 5; ++i) {
            off[i] = o;
            o = align_up(o + sz[i]);
        }
        bytes = o;
    }
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<Request*> reqs;
    oza::GroupPlan* plan = nullptr;
    size_t blk_off = 0, blk_bytes = 0;   // colmax + error word
    size_t tab_off = 0, tab_bytes = 0;   // device tables
    uint8_t* pinned = nullptr;           // staging: error word readback, then the table image
    size_t pinned_cap = 0;
    bool launch_failed = false;
};

}  // namespace

struct oza_server {
    oza_executor* ex = nullptr;
    oza_server_config_t cfg{};
    uint8_t* arena_base = nullptr;
    Arena arena;                                      // scheduler thread only
    std::vector<Slot> slots;                          // scheduler thread only
    std::mutex mu;                                    // guards everything below
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    bool kick = false;                                // new work or a finished batch
    bool failed = false;
    std::string fail_msg;
    oza_server_stats_t st{};
    std::chrono::steady_clock::time_point t0;
    std::thread worker;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void run();
    bool poll();
    bool launch();
    // Runs on the CUDA callback thread: no CUDA calls.
    static void CUDART_CB batch_done(void* p) {
        auto* s = static_cast<oza_server*>(p);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->kick = true;
        }
        s->cv_work.notify_one();
    }
};

bool oza_server::poll() {
    bool progressed = false;
    for (Slot& sl : slots) {
        if (!sl.busy) continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady) continue;
        const double t = now();
        int code = 0;
        if (q == cudaSuccess) std::memcpy(&code, sl.pinned, sizeof(int));
        else cudaGetLastError();
        const int status =
            (q != cudaSuccess || sl.launch_failed) ? OZA_CUDA_ERROR : (code ? OZA_TIMEOUT : OZA_OK);
        for (Request* r : sl.reqs) arena.release(r->ws_off, r->ws_bytes);
        arena.release(sl.blk_off, sl.blk_bytes);
        if (sl.tab_bytes) arena.release(sl.tab_off, sl.tab_bytes);
        sl.tab_bytes = 0;
        oza::group_plan_destroy(sl.plan);
        sl.plan = nullptr;
        sl.busy = false;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (Request* r : sl.reqs) {
                r->stats.done_s = t;
                r->stats.status = status;
                r->done = true;
            }
            st.completed += sl.reqs.size();
            st.arena_used = arena.used();
            if (status != OZA_OK) {
                failed = true;
                if (q != cudaSuccess) fail_msg = cudaGetErrorString(q);
                else if (status == OZA_TIMEOUT) fail_msg = "a device-side wait expired";
            }
        }
        sl.reqs.clear();
        cv_done.notify_all();
        progressed = true;
    }
    return progressed;
}

bool oza_server::launch() {
    Slot* sl = nullptr;
    for (Slot& s : slots)
        if (!s.busy) {
            sl = &s;
            break;
        }
    if (!sl) return false;
    std::vector<Request*> batch;
    {
        std::lock_guard<std::mutex> lk(mu);
        // Arrival order; stop at the first request that does not fit now.  A
        // Scheme I request runs alone: it ends a batch and starts its own.
        while (!queue.empty() && (int)batch.size() < cfg.max_batch) {
            Request* r = queue.front();
            if (r->scheme == OZA_SCHEME1 && !batch.empty()) break;
            if (!arena.alloc(r->ws_bytes, &r->ws_off)) break;
            queue.pop_front();
            batch.push_back(r);
            if (r->scheme == OZA_SCHEME1) break;
        }
    }
    if (batch.empty()) return false;
    auto requeue = [&](const char* why) {
        for (Request* r : batch) arena.release(r->ws_off, r->ws_bytes);
        std::lock_guard<std::mutex> lk(mu);
        for (auto it = batch.rbegin(); it != batch.rend(); ++it) queue.push_front(*it);
        (void)why;
    };
    size_t ncol = 0;
    for (Request* r : batch) ncol += r->N;
    sl->blk_bytes = align_up(ncol * 8) + kAlign;
    if (!arena.alloc(sl->blk_bytes, &sl->blk_off)) {
        requeue("no memory for the batch block");
        return false;
    }
    unsigned long long* colmax = reinterpret_cast<unsigned long long*>(arena_base + sl->blk_off);
    int* err = reinterpret_cast<int*>(arena_base + sl->blk_off + align_up(ncol * 8));
    std::vector<oza::GroupProblem> probs(batch.size());
    size_t cofs = 0;
    for (size_t i = 0; i < batch.size(); ++i) {
        const Request* r = batch[i];
        const WsLayout L(r->M, r->N, r->K, r->S, r->scheme);
        uint8_t* w = arena_base + r->ws_off;
        oza::GroupProblem& p = probs[i];
        p.A = r->A;
        p.B = r->B;
        p.C = r->C;
        p.M = r->M;
        p.N = r->N;
        p.K = r->K;
        p.Mp = L.Mp;
        p.Np = L.Np;
        p.Kp = L.Kp;
        p.S = r->S;
        p.k_param = r->scheme == OZA_SCHEME2 ? oza_scheme2_k_param(r->S, r->K) : 0;
        p.shiftA = reinterpret_cast<int32_t*>(w + L.off[0]);
        p.shiftB = reinterpret_cast<int32_t*>(w + L.off[1]);
        p.a_planes = reinterpret_cast<int8_t*>(w + L.off[2]);
        p.b_planes = reinterpret_cast<int8_t*>(w + L.off[3]);
        p.coef = w + L.off[4];
        p.colmax = colmax + cofs;
        cofs += r->N;
    }
    // A batch of one runs the single-GEMM launch sequence (no device tables);
    // larger batches run the grouped kernels.
    const bool single = batch.size() == 1;
    oza::GroupPlan* plan = nullptr;
    cudaError_t e = cudaSuccess;
    sl->tab_bytes = 0;
    if (!single) {
        e = oza::group_plan_build(probs.data(), (int)probs.size(), err, &plan);
        if (e != cudaSuccess) {
            arena.release(sl->blk_off, sl->blk_bytes);
            requeue("plan");
            std::lock_guard<std::mutex> lk(mu);
            failed = true;
            fail_msg = std::string("batch plan: ") + cudaGetErrorString(e);
            return false;
        }
        sl->tab_bytes = oza::group_plan_table_bytes(plan);
        if (!arena.alloc(sl->tab_bytes, &sl->tab_off)) {
            oza::group_plan_destroy(plan);
            arena.release(sl->blk_off, sl->blk_bytes);
            sl->tab_bytes = 0;
            requeue("no memory for the batch tables");
            return false;
        }
    }
    const size_t need = kAlign + sl->tab_bytes;
    if (sl->pinned_cap < need) {
        if (sl->pinned) cudaFreeHost(sl->pinned);
        sl->pinned = nullptr;
        sl->pinned_cap = 0;
        const size_t cap = need > (4u << 20) ? need * 2 : (4u << 20);
        if (cudaHostAlloc(reinterpret_cast<void**>(&sl->pinned), cap, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            oza::group_plan_destroy(plan);
            if (sl->tab_bytes) arena.release(sl->tab_off, sl->tab_bytes);
            sl->tab_bytes = 0;
            arena.release(sl->blk_off, sl->blk_bytes);
            requeue("pinned staging");
            std::lock_guard<std::mutex> lk(mu);
            failed = true;
            fail_msg = "pinned staging allocation failed";
            return false;
        }
        sl->pinned_cap = cap;
    }
    const double t = now();
    if (single) {
        // The single-GEMM launch sequence of oza_gemm (the steps in order).
        const oza::GroupProblem& p = probs[0];
        const int scheme = batch[0]->scheme;
        const int beta = scheme == OZA_SCHEME1 ? oza_scheme1_beta(p.K) : 0;
        oza::GemmPlan g;
        g.a_planes = p.a_planes;
        g.b_planes = p.b_planes;
        g.planes = p.S;
        g.Mp = p.Mp;
        g.Np = p.Np;
        g.Kp = p.Kp;
        g.M = p.M;
        g.N = p.N;
        g.pairs = oza::make_pairs(scheme, p.S, p.K);
        g.err = err;
        g.sms = ex->sms;
        g.ctc = scheme == OZA_SCHEME1 ? reinterpret_cast<int32_t*>(p.coef) : nullptr;
        g.coef = scheme == OZA_SCHEME2 ? p.coef : nullptr;
        e = cudaMemsetAsync(err, 0, sizeof(int), sl->st);
        if (e == cudaSuccess) e = oza::launch_stats_rows(p.A, p.M, p.K, p.k_param, p.shiftA, ex->sms, sl->st);
        if (e == cudaSuccess) e = oza::launch_stats_cols(p.B, p.K, p.N, p.colmax, ex->sms, sl->st);
        if (e == cudaSuccess)
            e = oza::launch_slice_rows(scheme, p.A, p.M, p.K, p.shiftA, p.S, beta, p.k_param, p.a_planes, p.Mp, p.Kp,
                                       ex->sms, sl->st, 0, err);
        if (e == cudaSuccess)
            e = oza::launch_slice_cols(scheme, p.B, p.K, p.N, p.colmax, p.k_param, p.S, beta, p.shiftB, p.b_planes,
                                       p.Np, p.Kp, sl->st, err);
        if (e == cudaSuccess) e = oza::launch_gemm_i8(g, sl->st);
        if (e == cudaSuccess && scheme == OZA_SCHEME2)
            e = oza::launch_crt_coef(p.coef, p.Mp, p.Np, p.M, p.N, p.S, p.shiftA, p.shiftB, p.C, ex->sms, sl->st);
        if (e == cudaSuccess && scheme == OZA_SCHEME1)
            e = oza::launch_reconstruct1(g.ctc, p.Mp, p.Np, p.M, p.N, p.S, beta, p.shiftA, p.shiftB, p.C, ex->sms,
                                         sl->st, &g.pairs);
    } else {
        std::memcpy(sl->pinned + kAlign, oza::group_plan_image(plan), sl->tab_bytes);
        void* tab = arena_base + sl->tab_off;
        oza::group_plan_bind(plan, tab);
        e = cudaMemcpyAsync(tab, sl->pinned + kAlign, sl->tab_bytes, cudaMemcpyHostToDevice, sl->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), sl->st);
        if (e == cudaSuccess) e = oza::group_plan_launch(plan, colmax, ncol, ex->sms, sl->st, nullptr);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl->pinned, err, sizeof(int), cudaMemcpyDeviceToHost, sl->st);
    if (e == cudaSuccess) e = cudaEventRecord(sl->done, sl->st);
    // Wake the scheduler as soon as the batch is done (after the event, so the
    // scheduler then finds it complete).
    if (e == cudaSuccess) e = cudaLaunchHostFunc(sl->st, &oza_server::batch_done, this);
    sl->plan = plan;
    sl->reqs = batch;
    sl->busy = true;
    sl->launch_failed = e != cudaSuccess;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Request* r : batch) {
            r->stats.admit_s = t;
            r->stats.batch_size = (int)batch.size();
        }
        st.batches += 1;
        st.admitted += batch.size();
        if ((int)batch.size() > st.max_batch_seen) st.max_batch_seen = (int)batch.size();
        st.arena_used = arena.used();
        st.arena_peak = arena.peak();
        if (e != cudaSuccess) {
            failed = true;
            fail_msg = std::string("batch launch: ") + cudaGetErrorString(e);
        }
    }
    if (e != cudaSuccess) {
        // Nothing usable was queued after the failure; complete the batch
        // through the event path with an error status.
        cudaGetLastError();
        cudaEventRecord(sl->done, sl->st);
    }
    return true;
}

void oza_server::run() {
    cudaSetDevice(ex->device);
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(mu);
            kick = false;
        }
        bool progressed = poll();
        while (launch()) progressed = true;
        bool idle = true;
        for (const Slot& s : slots) idle = idle && !s.busy;
        std::unique_lock<std::mutex> lk(mu);
        if (stop && queue.empty() && idle) break;
        if (progressed) continue;
        // Submissions and finished batches kick the loop; the timeout is only
        // a safety net.
        cv_work.wait_for(lk, std::chrono::milliseconds(idle ? 100 : 2), [this] { return kick || stop; });
    }
}

extern "C" {

oza_status_t oza_server_create(oza_exec_t ex, const oza_server_config_t* cfg, oza_server_t* out) {
    if (!out) return sfail(OZA_INVALID_ARG, "oza_server_create: null output handle");
    *out = nullptr;
    if (!ex || !cfg) return sfail(OZA_INVALID_ARG, "oza_server_create: null argument");
    if (cfg->workspace_budget < (1u << 20) || cfg->max_inflight < 1 || cfg->max_inflight > 16 || cfg->max_batch < 1)
        return sfail(OZA_INVALID_ARG, "oza_server_create: budget >= 1 MiB, 1 <= max_inflight <= 16, max_batch >= 1");
    oza::DeviceGuard dg(ex->device);
    if (!dg.ok) return sfail(OZA_CUDA_ERROR, "CUDA: Failed to set device %d", ex->device);
    cudaError_t e = oza::upload_tables();
    if (e != cudaSuccess) return sfail(OZA_CUDA_ERROR, "CUDA: constant tables: %s", cudaGetErrorString(e));
    auto* s = new (std::nothrow) oza_server();
    if (!s) return sfail(OZA_OOM, "oza_server_create: host allocation failed");
    s->ex = ex;
    s->cfg = *cfg;
    e = cudaMalloc(reinterpret_cast<void**>(&s->arena_base), cfg->workspace_budget);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return sfail(OZA_OOM, "oza_server_create: workspace arena of %zu bytes: %s", cfg->workspace_budget,
                     cudaGetErrorString(e));
    }
    s->arena.reset(cfg->workspace_budget);
    s->slots.resize(cfg->max_inflight);
    for (Slot& sl : s->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        for (Slot& sl : s->slots) {
            if (sl.st) cudaStreamDestroy(sl.st);
            if (sl.done) cudaEventDestroy(sl.done);
        }
        cudaFree(s->arena_base);
        delete s;
        return sfail(OZA_CUDA_ERROR, "oza_server_create: streams: %s", cudaGetErrorString(e));
    }
    s->st.workspace_budget = cfg->workspace_budget;
    s->t0 = std::chrono::steady_clock::now();
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return OZA_OK;
}

size_t oza_server_request_bytes(int scheme, size_t M, size_t N, size_t K, int slices) {
    if (scheme != OZA_SCHEME1 && scheme != OZA_SCHEME2) return 0;
    if (M == 0 || N == 0 || K == 0 || slices < 1 || slices > 20) return 0;
    // beyond Scheme II's INT32-exact bound
    if (scheme == OZA_SCHEME2 && (double)K * 125.0 * 125.0 >= 2147483648.0) return 0;
    return WsLayout(M, N, K, slices, scheme).bytes;
}

oza_status_t oza_server_submit(oza_server_t s, int scheme, size_t M, size_t N, size_t K, const double* A,
                               const double* B, double* C, int slices, uint64_t* id) {
    // Sizes first (the same limits as oza_ws_create), then the handles.
    if (M == 0 || N == 0 || K == 0 || M > (1u << 30) || N > (1u << 30) || K > (1u << 30))
        return sfail(OZA_INVALID_ARG, "oza_server_submit: dimensions must be in [1, 2^30]");
    if (slices < 1 || slices > 20) return sfail(OZA_INVALID_ARG, "oza_server_submit: slices must be in [1, 20]");
    {
        const oza_status_t chk = oza::check_problem("oza_server_submit", scheme, M, N, K, slices);
        if (chk != OZA_OK) return chk;
    }
    if (!s || !id) return sfail(OZA_INVALID_ARG, "oza_server_submit: null argument");
    if (!A || !B || !C) return sfail(OZA_INVALID_ARG, "oza_server_submit: null matrix pointer");
    const size_t bytes = WsLayout(M, N, K, slices, scheme).bytes;
    // The batch block (column maxima, error word) and the batch's device
    // tables (work units: 16 bytes per S x 128 x 256 tile) come from the arena too.
    const size_t batch_extra = align_up(N * 8) + 2 * kAlign + bytes / 1024 + (1u << 20);
    if (bytes + batch_extra > s->cfg.workspace_budget)
        return sfail(OZA_OOM, "oza_server_submit: a %zu x %zu x %zu request needs %zu workspace bytes, over the "
                              "budget of %zu", M, N, K, bytes, s->cfg.workspace_budget);
    auto* r = new (std::nothrow) Request();
    if (!r) return sfail(OZA_OOM, "oza_server_submit: host allocation failed");
    r->M = M;
    r->N = N;
    r->K = K;
    r->A = A;
    r->B = B;
    r->C = C;
    r->S = slices;
    r->scheme = scheme;
    r->ws_bytes = bytes;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return sfail(OZA_INVALID_ARG, "oza_server_submit: server is shutting down");
        }
        r->id = s->next_id++;
        s->kick = true;
        r->stats.submit_s = s->now();
        r->stats.slices = slices;
        r->stats.workspace_bytes = bytes;
        s->queue.push_back(r);
        s->reqs[r->id] = r;
        s->st.submitted += 1;
        *id = r->id;
    }
    s->cv_work.notify_one();
    return OZA_OK;
}

oza_status_t oza_server_wait(oza_server_t s, uint64_t id, double timeout_s, oza_request_stats_t* stats) {
    if (!s) return sfail(OZA_INVALID_ARG, "oza_server_wait: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return sfail(OZA_INVALID_ARG, "oza_server_wait: unknown request %llu", (unsigned long long)id);
    Request* r = it->second;
    const auto pred = [r] { return r->done; };
    if (timeout_s < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return sfail(OZA_TIMEOUT, "oza_server_wait: request %llu not complete after %.3f s", (unsigned long long)id,
                     timeout_s);
    if (stats) *stats = r->stats;
    const int status = r->stats.status;
    s->reqs.erase(it);
    delete r;
    if (status != OZA_OK)
        return sfail((oza_status_t)status, "oza_server_wait: request %llu failed: %s", (unsigned long long)id,
                     s->fail_msg.c_str());
    return OZA_OK;
}

oza_status_t oza_server_get_stats(oza_server_t s, oza_server_stats_t* out) {
    if (!s || !out) return sfail(OZA_INVALID_ARG, "oza_server_get_stats: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->queued = s->queue.size();
    return OZA_OK;
}

oza_status_t oza_server_destroy(oza_server_t s) {
    if (!s) return OZA_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->kick = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    oza::DeviceGuard dg(s->ex->device);
    for (Slot& sl : s->slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        oza::group_plan_destroy(sl.plan);
        if (sl.pinned) cudaFreeHost(sl.pinned);
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    for (auto& kv : s->reqs) delete kv.second;
    cudaFree(s->arena_base);
    delete s;
    return OZA_OK;
}

}  // extern "C"

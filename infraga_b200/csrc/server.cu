// Request server: continuous batching of ray-fan and eigenray requests on one
// GPU (C ABI in include/infraga_gpu.h, iga_server_*).
//
// The reference has no serving layer (its CLI runs one job per process); this
// is the runtime around the fan and eigen kernels:
//   - atmospheres stay resident (the caller's iga_atmo_t handles);
//   - a scheduler thread admits queued requests whenever a slot (a CUDA stream
//     with its own buffers) is free and the request's device memory fits the
//     HBM budget; later, smaller requests may pass a queued request that does
//     not fit yet, so memory freed by a finishing request is used at once;
//   - admitted fan requests run asynchronously on their slot's stream
//     (H2D of the angles, the fan kernel, D2H of the results, then a host
//     callback that wakes the scheduler), so requests that arrive while others
//     are on the GPU overlap with them;
//   - eigenray requests run on worker threads, each with its own stream (the
//     search is host-driven round by round);
//   - fan kernels of large requests are capped at a fraction of the resident
//     CTA slots, and small requests use high-priority streams, so a short
//     request is not queued behind a long persistent kernel.
// Each request's results depend only on the request (per-ray determinism of
// the kernels), so a result is the same alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/infraga_gpu.h"
#include "handle.h"

using namespace iga_internal;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    long long id = 0;
    int kind = 0;   // 0 fan, 1 eigen
    iga_atmo_s* atmo = nullptr;
    iga_fan_params fp{};
    iga_eig_params ep{};
    std::vector<double> th, ph;
    std::vector<iga_eig_pair> pairs;
    size_t need = 0;   // device bytes
    // results
    std::vector<double> rows;
    std::vector<int> index;
    std::vector<long long> ray_steps;
    std::vector<int> ray_status;
    long long total_steps = 0;
    int status = IGA_OK;
    bool done = false;
    double t_submit = 0.0, t_start = 0.0, t_done = 0.0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    bool high = false;             // high-priority stream (small requests)
    Request* req = nullptr;
    void* d_mem = nullptr;
    size_t d_bytes = 0;
    void* h_pin = nullptr;
    size_t h_bytes = 0;
    std::atomic<int> finished{0};
    struct iga_server_s* server = nullptr;
};

// byte layout of one fan request on the device / in pinned memory
struct FanLayout {
    size_t ws, th, ph, arr, n, st, steps, total;
    static size_t al(size_t x) { return (x + 255) & ~size_t(255); }
    FanLayout(int n_rays, int bounces) {
        const size_t nr = (size_t)n_rays, nb = (size_t)bounces + 1;
        ws = 0;
        th = ws + al(256);
        ph = th + al(nr * sizeof(double));
        arr = ph + al(nr * sizeof(double));
        n = arr + al(nr * nb * IGA_ARRIVAL_COLS * sizeof(double));
        st = n + al(nr * sizeof(int));
        steps = st + al(nr * sizeof(int));
        total = steps + al(nr * sizeof(long long));
    }
};

}  // namespace

struct iga_server_s {
    iga_server_config cfg{};
    int n_sm = 0, fan_cap_ctas = 0;
    std::mutex mu;
    std::condition_variable cv_work;   // scheduler
    std::condition_variable cv_done;   // waiters
    std::condition_variable cv_eig;    // eigen workers
    std::deque<Request*> pending;
    std::deque<Request*> eig_queue;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    std::vector<std::unique_ptr<Slot>> slots;
    size_t bytes_in_use = 0;
    long long next_id = 1;
    bool stop = false;
    int eig_running = 0;
    std::thread sched;
    std::vector<std::thread> eig_threads;
    std::vector<cudaStream_t> eig_streams;
    // statistics
    std::vector<double> lat_fan, lat_eig;
    long long steps_done = 0, rays_done = 0, eig_rows = 0, n_done = 0;
    double t_first_submit = -1.0, t_last_done = 0.0;
};

namespace {

void CUDART_CB on_slot_done(void* p) {
    // Runs on a CUDA callback thread: no CUDA calls and no blocking on the
    // server mutex (the scheduler may hold it across CUDA calls); a wake-up
    // that races the scheduler's wait is caught by its 2 ms timed wait.
    Slot* s = static_cast<Slot*>(p);
    s->finished.store(1, std::memory_order_release);
    s->server->cv_work.notify_all();
}

void finish_request(iga_server_s* S, Request* r) {
    r->t_done = now_s();
    r->done = true;
    S->bytes_in_use -= r->need;
    S->n_done++;
    S->t_last_done = std::max(S->t_last_done, r->t_done);
    if (r->status == IGA_OK) {
        S->steps_done += r->total_steps;
        if (r->kind == 0) { S->rays_done += (long long)r->th.size(); S->lat_fan.push_back(r->t_done - r->t_submit); }
        else { S->eig_rows += (long long)r->index.size(); S->lat_eig.push_back(r->t_done - r->t_submit); }
    }
    S->cv_done.notify_all();
}

// Copy a finished slot's pinned results into its request (scheduler thread, lock held).
void collect(iga_server_s* S, Slot& s) {
    Request* r = s.req;
    const int n = (int)r->th.size(), nb = r->fp.bounces + 1;
    FanLayout L(n, r->fp.bounces);
    const char* h = static_cast<const char*>(s.h_pin);
    const int* n_arr = reinterpret_cast<const int*>(h + L.n);
    const int* stat = reinterpret_cast<const int*>(h + L.st);
    const long long* steps = reinterpret_cast<const long long*>(h + L.steps);
    const double* arr = reinterpret_cast<const double*>(h + L.arr);
    r->ray_steps.assign(steps, steps + n);
    r->ray_status.assign(stat, stat + n);
    r->total_steps = 0;
    size_t tot = 0;
    for (int i = 0; i < n; i++) { r->total_steps += steps[i]; tot += (size_t)n_arr[i]; }
    r->rows.resize(tot * IGA_ARRIVAL_COLS);
    r->index.resize(tot);
    size_t w = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n_arr[i]; j++, w++) {
            memcpy(&r->rows[w * IGA_ARRIVAL_COLS], arr + ((size_t)i * nb + j) * IGA_ARRIVAL_COLS,
                   IGA_ARRIVAL_COLS * sizeof(double));
            r->index[w] = i;
        }
    s.req = nullptr;
    s.finished.store(0);
    finish_request(S, r);
}

// Launch a fan request on a free slot (scheduler thread, lock held).
int launch_fan(iga_server_s* S, Slot& s, Request* r) {
    const int n = (int)r->th.size();
    FanLayout L(n, r->fp.bounces);
    if (s.d_bytes < L.total) {
        if (s.d_mem) cudaFreeAsync(s.d_mem, s.stream);
        s.d_mem = nullptr; s.d_bytes = 0;
        IGA_CUDA(cudaMallocAsync(&s.d_mem, L.total, s.stream), "server: cudaMallocAsync");
        s.d_bytes = L.total;
    }
    if (s.h_bytes < L.total) {
        if (s.h_pin) cudaFreeHost(s.h_pin);
        s.h_pin = nullptr; s.h_bytes = 0;
        IGA_CUDA(cudaMallocHost(&s.h_pin, L.total), "server: cudaMallocHost");
        s.h_bytes = L.total;
    }
    char* d = static_cast<char*>(s.d_mem);
    char* h = static_cast<char*>(s.h_pin);
    memcpy(h + L.th, r->th.data(), n * sizeof(double));
    memcpy(h + L.ph, r->ph.data(), n * sizeof(double));
    IGA_CUDA(cudaMemcpyAsync(d + L.th, h + L.th, L.arr - L.th, cudaMemcpyHostToDevice, s.stream), "server: H2D");
    const int big = n > S->cfg.small_rays;
    int rc = fan_device(r->atmo, &r->fp, reinterpret_cast<double*>(d + L.th), reinterpret_cast<double*>(d + L.ph), n,
                        reinterpret_cast<double*>(d + L.arr), reinterpret_cast<int*>(d + L.n),
                        reinterpret_cast<long long*>(d + L.steps), reinterpret_cast<int*>(d + L.st), nullptr,
                        d + L.ws, s.stream, big ? S->fan_cap_ctas : 0);
    if (rc) return rc;
    IGA_CUDA(cudaMemcpyAsync(h + L.arr, d + L.arr, L.total - L.arr, cudaMemcpyDeviceToHost, s.stream), "server: D2H");
    s.req = r;
    s.finished.store(0);
    IGA_CUDA(cudaLaunchHostFunc(s.stream, on_slot_done, &s), "server: cudaLaunchHostFunc");
    return IGA_OK;
}

void scheduler(iga_server_s* S) {
    cudaSetDevice(S->cfg.device);
    std::unique_lock<std::mutex> lk(S->mu);
    while (true) {
        // finished fan slots
        for (auto& sp : S->slots) {
            Slot& s = *sp;
            if (s.req && s.finished.load(std::memory_order_acquire)) collect(S, s);
        }
        if (S->stop) {
            bool busy = S->eig_running > 0;
            for (auto& sp : S->slots) busy |= sp->req != nullptr;
            if (!busy) break;
        }
        // admission
        for (auto it = S->pending.begin(); it != S->pending.end();) {
            Request* r = *it;
            if (S->bytes_in_use + r->need > S->cfg.hbm_budget && S->bytes_in_use > 0) { ++it; continue; }
            if (r->kind == 1) {
                if (S->eig_running + (int)S->eig_queue.size() >= S->cfg.eig_workers) { ++it; continue; }
                S->bytes_in_use += r->need;
                r->t_start = now_s();
                S->eig_queue.push_back(r);
                S->cv_eig.notify_one();
                it = S->pending.erase(it);
                continue;
            }
            // fan: a free slot of the right priority class, else any free slot
            const bool small = (int)r->th.size() <= S->cfg.small_rays;
            Slot* free_slot = nullptr;
            for (auto& sp : S->slots)
                if (!sp->req && sp->high == small) { free_slot = sp.get(); break; }
            if (!free_slot)
                for (auto& sp : S->slots)
                    if (!sp->req) { free_slot = sp.get(); break; }
            if (!free_slot) { ++it; continue; }
            S->bytes_in_use += r->need;
            r->t_start = now_s();
            int rc = launch_fan(S, *free_slot, r);
            it = S->pending.erase(it);
            if (rc) {
                r->status = rc;
                free_slot->req = nullptr;
                finish_request(S, r);
            }
        }
        S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
    }
}

void eig_worker(iga_server_s* S, cudaStream_t st) {
    cudaSetDevice(S->cfg.device);
    std::unique_lock<std::mutex> lk(S->mu);
    while (true) {
        S->cv_eig.wait(lk, [&] { return S->stop || !S->eig_queue.empty(); });
        if (S->eig_queue.empty()) {
            if (S->stop) break;
            continue;
        }
        Request* r = S->eig_queue.front();
        S->eig_queue.pop_front();
        S->eig_running++;
        lk.unlock();
        std::vector<double> rows;
        std::vector<int> idx;
        long long steps = 0;
        int rc = eig_search(r->atmo, &r->ep, r->pairs.data(), (int)r->pairs.size(), st, rows, idx, steps);
        lk.lock();
        S->eig_running--;
        r->status = rc;
        r->rows = std::move(rows);
        r->index = std::move(idx);
        r->total_steps = steps;
        finish_request(S, r);
        S->cv_work.notify_all();
    }
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

int iga_server_config_default(iga_server_config* c) {
    if (!c) return IGA_E_INVALID;
    memset(c, 0, sizeof(*c));
    c->device = 0;
    c->hbm_budget = (size_t)8 << 30;
    c->max_inflight = 8;
    c->eig_workers = 2;
    c->small_rays = 4096;
    c->big_fan_sm_frac = 0.75;
    return IGA_OK;
}

int iga_server_create(const iga_server_config* cfg, iga_server_t* out) {
    if (!cfg || !out || cfg->max_inflight < 1 || cfg->eig_workers < 0 || cfg->hbm_budget == 0 ||
        !(cfg->big_fan_sm_frac > 0.0 && cfg->big_fan_sm_frac <= 1.0))
        return IGA_E_INVALID;
    *out = nullptr;
    auto* S = new (std::nothrow) iga_server_s();
    if (!S) return IGA_E_NOMEM;
    S->cfg = *cfg;
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) { delete S; return cuda_fail(e, "server: cudaSetDevice"); }
    cudaDeviceGetAttribute(&S->n_sm, cudaDevAttrMultiProcessorCount, cfg->device);
    // a large fan kernel gets at most this many CTAs (resident capacity is a few per SM)
    S->fan_cap_ctas = std::max(1, (int)(S->n_sm * 3 * cfg->big_fan_sm_frac));
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    for (int i = 0; i < cfg->max_inflight; i++) {
        auto s = std::make_unique<Slot>();
        s->server = S;
        s->high = (i % 2) == 1;
        e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, s->high ? hi : lo);
        if (e != cudaSuccess) { iga_server_destroy(S); return cuda_fail(e, "server: cudaStreamCreate"); }
        S->slots.push_back(std::move(s));
    }
    for (int i = 0; i < cfg->eig_workers; i++) {
        cudaStream_t st;
        e = cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi);
        if (e != cudaSuccess) { iga_server_destroy(S); return cuda_fail(e, "server: cudaStreamCreate"); }
        S->eig_streams.push_back(st);
    }
    S->sched = std::thread(scheduler, S);
    for (auto st : S->eig_streams) S->eig_threads.emplace_back(eig_worker, S, st);
    *out = S;
    return IGA_OK;
}

int iga_server_submit_fan(iga_server_t S, iga_atmo_t atmo, const iga_fan_params* p, const double* theta_deg,
                          const double* phi_deg, int n_rays, long long* id) {
    if (!S || !atmo || !p || !id || n_rays < 0 || (n_rays > 0 && (!theta_deg || !phi_deg))) return IGA_E_INVALID;
    int rc = validate(p, n_rays);
    if (rc) return rc;
    if (atmo->device != S->cfg.device) return IGA_E_INVALID;
    auto r = std::make_unique<Request>();
    r->kind = 0;
    r->atmo = atmo;
    r->fp = *p;
    r->th.assign(theta_deg, theta_deg + n_rays);
    r->ph.assign(phi_deg, phi_deg + n_rays);
    r->need = FanLayout(n_rays, p->bounces).total;
    if (r->need > S->cfg.hbm_budget) return IGA_E_NOMEM;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return IGA_E_INVALID;
    r->id = S->next_id++;
    r->t_submit = now_s();
    if (S->t_first_submit < 0) S->t_first_submit = r->t_submit;
    *id = r->id;
    if (n_rays == 0) { r->done = true; r->t_done = r->t_submit; S->reqs.emplace(r->id, std::move(r)); return IGA_OK; }
    S->pending.push_back(r.get());
    S->reqs.emplace(r->id, std::move(r));
    S->cv_work.notify_all();
    return IGA_OK;
}

int iga_server_submit_eig(iga_server_t S, iga_atmo_t atmo, const iga_eig_params* p, const iga_eig_pair* pairs,
                          int n_pairs, long long* id) {
    if (!S || !atmo || !p || !id || n_pairs < 0 || (n_pairs > 0 && !pairs)) return IGA_E_INVALID;
    if (S->cfg.eig_workers < 1) return IGA_E_UNSUPPORTED;
    if (atmo->device != S->cfg.device) return IGA_E_INVALID;
    auto r = std::make_unique<Request>();
    r->kind = 1;
    r->atmo = atmo;
    r->ep = *p;
    r->pairs.assign(pairs, pairs + n_pairs);
    // worst-case trace buffers of one round (eig3d.cu: requests + results, two launches)
    const size_t searches = (size_t)n_pairs * (size_t)(p->bnc_max - p->bnc_min + 1);
    r->need = 2 * std::max<size_t>(searches * 128, 1024) * 256;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return IGA_E_INVALID;
    r->id = S->next_id++;
    r->t_submit = now_s();
    if (S->t_first_submit < 0) S->t_first_submit = r->t_submit;
    *id = r->id;
    S->pending.push_back(r.get());
    S->reqs.emplace(r->id, std::move(r));
    S->cv_work.notify_all();
    return IGA_OK;
}

int iga_server_wait(iga_server_t S, long long id, double timeout_s, int* done) {
    if (!S || !done) return IGA_E_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return IGA_E_INVALID;
    Request* r = it->second.get();
    if (!r->done && timeout_s != 0.0) {
        auto pred = [&] { return r->done; };
        if (timeout_s < 0.0) S->cv_done.wait(lk, pred);
        else S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
    }
    *done = r->done ? 1 : 0;
    return IGA_OK;
}

int iga_server_fetch(iga_server_t S, long long id, double* rows, int cap, int* n_out, int* index,
                     long long* total_steps, double* latency_s) {
    if (!S || !n_out || (cap > 0 && !rows)) return IGA_E_INVALID;
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->reqs.find(id);
        if (it == S->reqs.end() || !it->second->done) return IGA_E_INVALID;
        const int n = (int)it->second->index.size();
        *n_out = n;
        if (it->second->status != IGA_OK) {
            const int st = it->second->status;
            S->reqs.erase(it);
            return st;
        }
        if (n > cap) return IGA_E_TRUNCATED;   // kept: call again with more room
        r = std::move(it->second);
        S->reqs.erase(it);
    }
    const int n = (int)r->index.size();
    if (n > 0) memcpy(rows, r->rows.data(), (size_t)n * IGA_ARRIVAL_COLS * sizeof(double));
    if (index && n > 0) memcpy(index, r->index.data(), (size_t)n * sizeof(int));
    if (total_steps) *total_steps = r->total_steps;
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    return IGA_OK;
}

int iga_server_get_stats(iga_server_t S, iga_server_stats* st) {
    if (!S || !st) return IGA_E_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    memset(st, 0, sizeof(*st));
    st->completed = S->n_done;
    st->pending = (long long)S->pending.size();
    st->fan_p50_s = percentile(S->lat_fan, 0.50);
    st->fan_p99_s = percentile(S->lat_fan, 0.99);
    st->eig_p50_s = percentile(S->lat_eig, 0.50);
    st->eig_p99_s = percentile(S->lat_eig, 0.99);
    std::vector<double> all(S->lat_fan);
    all.insert(all.end(), S->lat_eig.begin(), S->lat_eig.end());
    st->p50_s = percentile(all, 0.50);
    st->p99_s = percentile(all, 0.99);
    st->ray_steps = S->steps_done;
    st->rays = S->rays_done;
    st->eigenrays = S->eig_rows;
    st->wall_s = S->t_first_submit < 0 ? 0.0 : S->t_last_done - S->t_first_submit;
    st->bytes_in_use = S->bytes_in_use;
    return IGA_OK;
}

int iga_server_destroy(iga_server_t S) {
    if (!S) return IGA_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->pending.clear();
        S->cv_work.notify_all();
        S->cv_eig.notify_all();
    }
    if (S->sched.joinable()) S->sched.join();
    for (auto& t : S->eig_threads) if (t.joinable()) t.join();
    for (auto& sp : S->slots) {
        if (sp->stream) cudaStreamSynchronize(sp->stream);
        if (sp->d_mem) cudaFreeAsync(sp->d_mem, sp->stream);
        if (sp->stream) { cudaStreamSynchronize(sp->stream); cudaStreamDestroy(sp->stream); }
        if (sp->h_pin) cudaFreeHost(sp->h_pin);
    }
    for (auto st : S->eig_streams) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
    delete S;
    return IGA_OK;
}

}  // extern "C"

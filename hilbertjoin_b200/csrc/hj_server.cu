// hj_server.cu -- the join-serving loop (no reference counterpart).
//
// Point sets are uploaded once and stay resident on the device. Joins are
// submitted from any host thread into a queue and return a request id at once.
// A pool of `max_inflight` worker threads, each with its own device context and
// CUDA stream, takes requests in arrival order as soon as (a) a worker is free
// and (b) the request fits the memory budget; its kernels then run
// concurrently with the other admitted requests' kernels on the same device
// (continuous batching across streams). A request larger than the whole budget
// is rejected with HJ_ERR_BUSY. Every request's count is computed by the same
// pipeline as a standalone call, so a result does not depend on what else is
// in flight.
//
// Memory: each worker's engine context keeps its device buffers between
// requests (reused, grow-only). The budget is charged with what every worker
// really holds, measured after each request, and with the estimate of each
// running request where that is larger (engine_join_bytes_estimate). A worker
// that holds more than its share of the budget (budget / max_inflight) when
// it finishes frees its buffers, and every idle worker frees them when no
// queued request fits. So the device memory of the server's requests
// stays within the budget, up to what a request takes beyond its estimate
// while it runs. When the head of the queue does not fit, a free worker may
// take a later request that does (backfill), unless the head has waited
// longer than kHeadWaitMs.
//
// With batch_max > 1 (tensor-core forms) a free worker takes the queue's head
// and then further queued requests of the same dtype while they fit in the
// budget, up to batch_max, and runs them as one batch (hj_batch_count_device:
// every request's sort and index, then ONE persistent launch over all their
// work items). A request's count is the same either way; a batch that cannot
// run (e.g. d > 256) falls back to one call per request.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/hj.h"
#include "hj_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct DevSet {
    void *ptr = nullptr;
    uint64_t n = 0;
    uint32_t d = 0;
    int dtype_bytes = 8;
    int users = 0;        // queued or running requests referencing the set
    bool released = false;
};

struct Request {
    uint64_t id = 0;
    uint64_t a = 0, b = 0;
    double eps = 0;
    uint64_t mem = 0;
    Clock::time_point t_submit, t_start, t_end;
    bool done = false;
    hj_result res{};
};

}  // namespace

struct hj_server {
    hj_server_opts opts{};
    int device = 0;
    int centring = HJ_CENTRING_GLOBAL;  // of the requests' tensor-core joins (hj_server_opts.block_centring)
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::map<uint64_t, Request> reqs;
    std::map<uint64_t, DevSet> sets;
    uint64_t next_id = 1, next_set = 1;
    std::vector<uint64_t> held;     // per worker: bytes its context holds (measured)
    std::vector<uint64_t> charged;  // per worker: max(held, estimate of its running requests)
    bool stop = false;
    std::vector<std::thread> workers;
};

constexpr double kHeadWaitMs = 1000.0;

static uint64_t request_bytes(const hj_server *s, const DevSet &a, const DevSet &b, bool self) {
    return hj::engine_join_bytes_estimate(a.n, self ? a.n : b.n, a.d, a.dtype_bytes, s->opts.form, self,
                                          s->centring != HJ_CENTRING_GLOBAL);
}

static uint64_t charged_by_others(const hj_server *s, int w) {
    uint64_t t = 0;
    for (size_t v = 0; v < s->charged.size(); ++v)
        if ((int)v != w) t += s->charged[v];
    return t;
}

// Fills a finished request's result and releases its memory and sets (lock held).
static void finish_request(hj_server *s, uint64_t id, int status, uint64_t count, int form_used,
                           uint64_t candidate_pairs, uint64_t band_pairs) {
    Request &r = s->reqs[id];
    r.t_end = Clock::now();
    r.done = true;
    r.res.count = count;
    r.res.status = status;
    r.res.form_used = status == HJ_OK ? form_used : -1;
    r.res.queue_ms = std::chrono::duration<double, std::milli>(r.t_start - r.t_submit).count();
    r.res.run_ms = std::chrono::duration<double, std::milli>(r.t_end - r.t_start).count();
    r.res.latency_ms = std::chrono::duration<double, std::milli>(r.t_end - r.t_submit).count();
    r.res.candidate_pairs = status == HJ_OK ? candidate_pairs : 0;
    r.res.band_pairs = status == HJ_OK ? band_pairs : 0;
    for (uint64_t sid : {r.a, r.b}) {
        auto it = s->sets.find(sid);
        if (it != s->sets.end()) {
            if (--it->second.users == 0 && it->second.released) {
                cudaFree(it->second.ptr);
                s->sets.erase(it);
            }
        }
        if (r.a == r.b) break;
    }
}

static bool tc_form(int f) {
    return f == HJ_FORM_TC_FP16 || f == HJ_FORM_TC_TF32 || f == HJ_FORM_TC_BF16X3 || f == HJ_FORM_AUTO;
}

static void worker_main(hj_server *s, int w) {
    cudaSetDevice(s->device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    const int batch_max = tc_form(s->opts.form) && s->opts.batch_max > 1 ? s->opts.batch_max : 1;
    const uint64_t budget = s->opts.memory_budget_bytes;
    const uint64_t share = budget / (uint64_t)std::max(1, s->opts.max_inflight);
    for (;;) {
        std::vector<uint64_t> ids;
        std::vector<Request> rqs;
        std::vector<DevSet> sa, sb;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            size_t pick = 0;
            for (;;) {
                if (s->stop) {
                    lk.unlock();
                    hj::engine_ctx_trim(s->device, stream);
                    if (stream) cudaStreamDestroy(stream);
                    return;
                }
                if (!s->queue.empty()) {
                    const uint64_t others = charged_by_others(s, w);
                    auto fits = [&](const Request &r) { return others + std::max(s->held[w], r.mem) <= budget; };
                    const Request &head = s->reqs[s->queue.front()];
                    const double head_wait =
                        std::chrono::duration<double, std::milli>(Clock::now() - head.t_submit).count();
                    bool found = false;
                    for (size_t q = 0; q < s->queue.size(); ++q) {
                        if (q > 0 && head_wait > kHeadWaitMs) break;  // no backfill past a starving head
                        if (fits(s->reqs[s->queue[q]])) {
                            pick = q;
                            found = true;
                            break;
                        }
                    }
                    if (found) break;
                    if (s->held[w] > 0) {
                        // nothing fits: an idle worker frees its buffers (every idle
                        // worker does so when woken), then all check again
                        lk.unlock();
                        hj::engine_ctx_trim(s->device, stream);
                        lk.lock();
                        s->held[w] = s->charged[w] = 0;
                        s->cv_work.notify_all();
                        continue;
                    }
                }
                s->cv_work.wait(lk);
            }
            // the picked request, then (batching) followers of the same dtype that fit
            int dtype = 0;
            uint64_t est = 0;
            while (pick < s->queue.size() && (int)ids.size() < batch_max) {
                Request &r = s->reqs[s->queue[pick]];
                const DevSet &a = s->sets[r.a];
                if (!ids.empty() && (a.dtype_bytes != dtype ||
                                     charged_by_others(s, w) + std::max(s->held[w], est + r.mem) > budget)) {
                    ++pick;
                    continue;
                }
                dtype = a.dtype_bytes;
                est += r.mem;
                ids.push_back(r.id);
                s->queue.erase(s->queue.begin() + (long)pick);
                r.t_start = Clock::now();
                rqs.push_back(r);
                sa.push_back(a);
                sb.push_back(s->sets[r.b]);
            }
            s->charged[w] = std::max(s->held[w], est);
            s->cv_work.notify_all();
        }
        hj_opts o;
        hj_opts_init(&o);
        o.form = s->opts.form;
        o.tc_centring = s->centring;
        o.device = s->device;
        o.stream = stream;
        const size_t k = ids.size();
        std::vector<int> status(k, HJ_OK);
        std::vector<uint64_t> count(k, 0), cand(k, 0), band(k, 0);
        std::vector<int> form_used(k, s->opts.form);
        bool batched = false;
        if (k > 1) {
            std::vector<hj_batch_job> jobs(k);
            for (size_t i = 0; i < k; ++i) {
                std::memset(&jobs[i], 0, sizeof(jobs[i]));
                jobs[i].a = sa[i].ptr;
                jobs[i].na = sa[i].n;
                jobs[i].d = sa[i].d;
                jobs[i].eps = rqs[i].eps;
                if (rqs[i].a != rqs[i].b) {
                    jobs[i].b = sb[i].ptr;
                    jobs[i].nb = sb[i].n;
                }
            }
            hj_batch *b = nullptr;
            if (hj_batch_create(jobs.data(), (uint32_t)k, sa[0].dtype_bytes, &o, &b) == HJ_OK) {
                hj_stats st;
                if (hj_batch_counts(b, count.data(), &st) == HJ_OK) {
                    batched = true;
                    hj::batch_job_candidates(b, cand.data());
                    for (size_t i = 0; i < k; ++i) form_used[i] = st.form_used;
                }
                hj_batch_destroy(b);
            }
        }
        if (!batched) {
            for (size_t i = 0; i < k; ++i) {
                hj_stats st;
                if (rqs[i].a == rqs[i].b)
                    status[i] = hj_self_join_count_device(sa[i].ptr, sa[i].dtype_bytes, sa[i].n, sa[i].d, rqs[i].eps,
                                                          &o, &count[i], &st);
                else
                    status[i] = hj_join_count_device(sa[i].ptr, sa[i].n, sb[i].ptr, sb[i].n, sa[i].dtype_bytes,
                                                     sa[i].d, rqs[i].eps, &o, &count[i], &st);
                if (status[i] == HJ_OK) {
                    form_used[i] = st.form_used;
                    cand[i] = st.candidate_pairs;
                    band[i] = st.band_pairs;
                }
            }
        }
        // what the context holds now; above this worker's share it is freed
        uint64_t held = hj::engine_ctx_bytes(s->device);
        if (held > share) {
            hj::engine_ctx_trim(s->device, stream);
            held = 0;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->held[w] = s->charged[w] = held;
            for (size_t i = 0; i < k; ++i) finish_request(s, ids[i], status[i], count[i], form_used[i], cand[i], band[i]);
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

extern "C" {

void hj_server_opts_init(hj_server_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->memory_budget_bytes = 40ull << 30;
    o->max_inflight = 8;
    o->device = -1;
    o->form = HJ_FORM_PLAIN_FP64;
}

int hj_server_create(const hj_server_opts *opts, hj_server **out) {
    if (!out) return HJ_ERR_INVALID_ARG;
    hj_server_opts o;
    hj_server_opts_init(&o);
    if (opts) o = *opts;
    if (o.memory_budget_bytes == 0) o.memory_budget_bytes = 40ull << 30;
    if (o.max_inflight <= 0) o.max_inflight = 8;
    int dev = o.device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return HJ_ERR_NO_DEVICE;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || dev >= ndev) {
        cudaGetLastError();
        return HJ_ERR_NO_DEVICE;
    }
    hj_server *s = new hj_server();
    s->opts = o;
    s->device = dev;
    s->centring = o.block_centring ? HJ_CENTRING_AUTO : HJ_CENTRING_GLOBAL;
    s->held.assign(o.max_inflight, 0);
    s->charged.assign(o.max_inflight, 0);
    for (int i = 0; i < o.max_inflight; ++i) s->workers.emplace_back(worker_main, s, i);
    *out = s;
    return HJ_OK;
}

int hj_server_destroy(hj_server *s) {
    if (!s) return HJ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    cudaSetDevice(s->device);
    for (auto &kv : s->sets) cudaFree(kv.second.ptr);
    delete s;
    return HJ_OK;
}

int hj_set_upload(hj_server *s, const void *pts, int dtype_bytes, uint64_t n, uint32_t d, uint64_t *set_id) {
    if (!s || !set_id || (n && !pts) || (dtype_bytes != 4 && dtype_bytes != 8) || d == 0) return HJ_ERR_INVALID_ARG;
    cudaSetDevice(s->device);
    void *p = nullptr;
    size_t bytes = n * d * (size_t)dtype_bytes;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        return HJ_ERR_OOM;
    }
    if (bytes && cudaMemcpy(p, pts, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return HJ_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    uint64_t id = s->next_set++;
    DevSet ds;
    ds.ptr = p;
    ds.n = n;
    ds.d = d;
    ds.dtype_bytes = dtype_bytes;
    s->sets[id] = ds;
    *set_id = id;
    return HJ_OK;
}

int hj_set_release(hj_server *s, uint64_t set_id) {
    if (!s) return HJ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->sets.find(set_id);
    if (it == s->sets.end() || it->second.released) return HJ_ERR_NOT_FOUND;
    if (it->second.users == 0) {
        cudaSetDevice(s->device);
        cudaFree(it->second.ptr);
        s->sets.erase(it);
    } else {
        it->second.released = true;  // freed when its last request finishes
    }
    return HJ_OK;
}

int hj_submit(hj_server *s, uint64_t set_a, uint64_t set_b, double eps, uint64_t *request_id) {
    if (!s || !request_id) return HJ_ERR_INVALID_ARG;
    if (set_b == 0) set_b = set_a;
    std::lock_guard<std::mutex> lk(s->mu);
    auto ia = s->sets.find(set_a), ib = s->sets.find(set_b);
    if (ia == s->sets.end() || ib == s->sets.end() || ia->second.released || ib->second.released)
        return HJ_ERR_NOT_FOUND;
    if (ia->second.d != ib->second.d || ia->second.dtype_bytes != ib->second.dtype_bytes)
        return HJ_ERR_INVALID_ARG;
    Request r;
    r.id = s->next_id++;
    r.a = set_a;
    r.b = set_b;
    r.eps = eps;
    r.mem = request_bytes(s, ia->second, ib->second, set_a == set_b);
    r.t_submit = Clock::now();
    if (r.mem > s->opts.memory_budget_bytes) return HJ_ERR_BUSY;
    ia->second.users++;
    if (set_b != set_a) ib->second.users++;
    s->reqs[r.id] = r;
    s->queue.push_back(r.id);
    *request_id = r.id;
    s->cv_work.notify_one();
    return HJ_OK;
}

int hj_poll(hj_server *s, uint64_t request_id, int *done, hj_result *result) {
    if (!s || !done) return HJ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return HJ_ERR_NOT_FOUND;
    *done = it->second.done ? 1 : 0;
    if (it->second.done) {
        if (result) *result = it->second.res;
        s->reqs.erase(it);
    }
    return HJ_OK;
}

int hj_wait(hj_server *s, uint64_t request_id, double timeout_ms, hj_result *result) {
    if (!s) return HJ_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] {
        auto it = s->reqs.find(request_id);
        return it == s->reqs.end() || it->second.done;
    };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred))
        return HJ_ERR_TIMEOUT;
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return HJ_ERR_NOT_FOUND;
    if (result) *result = it->second.res;
    s->reqs.erase(it);
    return HJ_OK;
}

}  // extern "C"

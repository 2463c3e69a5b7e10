// Serving loop: continuous batching of snapshot imaging requests.
//
// The reference images one snapshot per process invocation (SVDIntegratedImager.cu:1773-1854). A
// server keeps `num_slots` imaging engines resident (each with its own CUDA stream, grids, cuFFT
// plans and tile bins) and a worker thread per slot. Requests queue in arrival order; a request is
// admitted when a slot is free and its device-memory estimate fits in the HBM budget next to what
// the other slots hold. A slot's engine keeps its buffers (they only grow), so a slot is charged
// the largest estimate it has served (its resident buffers) and, while it runs a request, the
// larger of that and the request's estimate: the charges of all slots never exceed the budget, so
// the engines' resident buffers stay inside it too. Admitted requests run concurrently, so their kernels overlap on the
// GPU, and a new request starts the moment a slot frees up. Each request records its queueing,
// running and total latency (host wall clock, submit to completion).
#include "svdi_internal.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace svdi {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
    uint64_t ticket = 0;
    svdi_host_ms ms{};
    size_t N = 0;
    float cell = 0.0f;
    float* out = nullptr;
    size_t est_bytes = 0;
    int status = SVDI_OK;
    std::string error;
    int slot = -1;
    bool done = false;
    Clock::time_point t_submit, t_start, t_end;
};

}  // namespace
}  // namespace svdi

struct svdi_server {
    svdi_options opt{};
    int num_slots = 0;
    size_t budget = 0;
    size_t in_use = 0;                // sum of the slots' charges
    std::vector<size_t> resident;     // per slot: the largest estimate it has served
    int fault_every = 0;
    uint64_t next_ticket = 1;
    uint64_t admitted = 0;
    std::vector<svdi_engine*> engines;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<svdi::Request>> queue;
    std::map<uint64_t, std::shared_ptr<svdi::Request>> requests;
    bool stop = false;
};

namespace svdi {
namespace {

// Device bytes one request needs in a slot: raw inputs, collapsed visibilities, binned records,
// one moment plane per Chebyshev term (the estimate assumes `planes` planes) and the image.
size_t request_bytes(const svdi_host_ms& ms, size_t N, double sigma, int planes) {
    const size_t n = ms.num_samples;
    const size_t G = (size_t)std::ceil(sigma * (double)N) + 8;
    return n * (26 + 8 + 20) + ms.num_rows * 36 + (size_t)planes * G * G * 8 + N * N * 4 + (64u << 20);
}

void worker_loop(svdi_server* s, int slot) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stop && s->queue.empty()) return;
                // continuous batching: take the oldest queued request that fits the HBM budget
                // (this slot's charge grows from its resident buffers to the request's estimate)
                const size_t res = s->resident[slot];
                auto it = s->queue.begin();
                for (; it != s->queue.end(); ++it)
                    if (s->in_use - res + std::max(res, (*it)->est_bytes) <= s->budget) break;
                if (it != s->queue.end()) {
                    r = *it;
                    s->queue.erase(it);
                    s->in_use += std::max(res, r->est_bytes) - res;
                    s->resident[slot] = std::max(res, r->est_bytes);
                    ++s->admitted;
                    break;
                }
                if (!s->queue.empty() && res > 0) {
                    // nothing queued fits next to the other slots' buffers: give this idle slot's
                    // buffers back (a fresh engine) so that the queue cannot stall on resident memory
                    lk.unlock();
                    svdi_engine* fresh = nullptr;
                    const bool ok = svdi_engine_create(&s->opt, &fresh) == SVDI_OK;
                    if (ok) {
                        svdi_engine_destroy(s->engines[slot]);
                        s->engines[slot] = fresh;
                    }
                    lk.lock();
                    if (ok) {
                        s->in_use -= res;
                        s->resident[slot] = 0;
                        s->cv_work.notify_all();
                        continue;
                    }
                }
                s->cv_work.wait(lk);
            }
        }
        r->slot = slot;
        r->t_start = Clock::now();
        int st = SVDI_OK;
        std::string err;
        if (s->fault_every > 0 && (r->ticket % (uint64_t)s->fault_every) == 0) {
            // host-side fault injection (tests): the request fails before any device work
            st = SVDI_ERR_INTERNAL;
            err = "injected host fault";
        } else {
            st = svdi_engine_image_host(s->engines[slot], &r->ms, r->N, r->cell, r->out);
            if (st != SVDI_OK) err = svdi_last_error();
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->status = st;
            r->error = err;
            r->t_end = Clock::now();
            r->done = true;  // the slot stays charged its resident buffers
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace
}  // namespace svdi

using namespace svdi;

extern "C" {

int svdi_server_create(const svdi_options* opt, int num_slots, size_t hbm_budget_bytes, int fault_every,
                       svdi_server** out) {
    if (!out || num_slots < 1 || num_slots > 64) {
        set_error("num_slots must be in 1..64");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    std::unique_ptr<svdi_server> s(new svdi_server());
    if (opt) s->opt = *opt;
    else svdi_default_options(&s->opt);
    s->num_slots = num_slots;
    s->fault_every = fault_every;
    SVDI_CUDA(cudaSetDevice(s->opt.device));
    if (hbm_budget_bytes == 0) {
        size_t free_b = 0, total_b = 0;
        SVDI_CUDA(cudaMemGetInfo(&free_b, &total_b));
        hbm_budget_bytes = free_b / 10 * 8;  // 80 % of the free HBM
    }
    s->budget = hbm_budget_bytes;
    s->resident.assign((size_t)num_slots, 0);
    for (int i = 0; i < num_slots; ++i) {
        svdi_engine* e = nullptr;
        const int st = svdi_engine_create(&s->opt, &e);
        if (st != SVDI_OK) {
            for (auto* x : s->engines) svdi_engine_destroy(x);
            return st;
        }
        s->engines.push_back(e);
    }
    svdi_server* raw = s.get();
    for (int i = 0; i < num_slots; ++i) s->workers.emplace_back(worker_loop, raw, i);
    *out = s.release();
    return SVDI_OK;
}

int svdi_server_submit(svdi_server* s, const svdi_host_ms* ms, size_t N, float cell, float* out_image,
                       uint64_t* ticket) {
    if (!s || !ms || !out_image || !ticket) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (ms->num_samples == 0 || ms->num_rows == 0 || ms->num_channels == 0) {
        set_error("Measurement set is empty");
        return SVDI_ERR_EMPTY_INPUT;
    }
    if (ms->num_samples != ms->num_rows * ms->num_channels) {
        set_error("num_samples must equal num_rows * num_channels");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (N == 0 || N > 65536 || !(cell > 0.0f)) {
        set_error("Image_Size must be in 1..65536 and Cell_Size greater than zero");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_shared<Request>();
    r->ms = *ms;
    r->N = N;
    r->cell = cell;
    r->out = out_image;
    r->est_bytes = request_bytes(*ms, N, s->opt.sigma, s->opt.k_rule == SVDI_KRULE_BUCKET ? 8 : 2);
    if (r->est_bytes > s->budget) {
        set_error("request needs ~" + std::to_string(r->est_bytes >> 20) + " MiB of device memory, more than the "
                  "server's HBM budget of " + std::to_string(s->budget >> 20) + " MiB");
        return SVDI_ERR_OUT_OF_MEMORY;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            set_error("server is shutting down");
            return SVDI_ERR_INVALID_ARGUMENT;
        }
        r->ticket = s->next_ticket++;
        r->t_submit = Clock::now();
        s->requests[r->ticket] = r;
        s->queue.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return SVDI_OK;
}

int svdi_server_wait(svdi_server* s, uint64_t ticket, double timeout_s, svdi_request_info* info) {
    if (!s) {
        set_error("null server");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->requests.find(ticket);
        if (it == s->requests.end()) {
            set_error("unknown ticket");
            return SVDI_ERR_INVALID_ARGUMENT;
        }
        r = it->second;
        auto pred = [&] { return r->done; };
        if (timeout_s > 0) {
            if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
                set_error("timed out waiting for the request");
                return SVDI_ERR_INTERNAL;
            }
        } else {
            s->cv_done.wait(lk, pred);
        }
        s->requests.erase(ticket);
    }
    if (info) {
        info->status = r->status;
        info->slot = r->slot;
        info->num_samples = r->ms.num_samples;
        info->queue_ms = ms_between(r->t_submit, r->t_start);
        info->run_ms = ms_between(r->t_start, r->t_end);
        info->latency_ms = ms_between(r->t_submit, r->t_end);
    }
    if (r->status != SVDI_OK) set_error(r->error);
    return r->status;
}

int svdi_server_poll(svdi_server* s, uint64_t ticket, int* done) {
    if (!s || !done) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) {
        set_error("unknown ticket");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    *done = it->second->done ? 1 : 0;
    return SVDI_OK;
}

int svdi_server_stats(svdi_server* s, size_t* queued, size_t* hbm_in_use, size_t* hbm_budget, uint64_t* admitted) {
    if (!s) {
        set_error("null server");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = s->queue.size();
    if (hbm_in_use) *hbm_in_use = s->in_use;
    if (hbm_budget) *hbm_budget = s->budget;
    if (admitted) *admitted = s->admitted;
    return SVDI_OK;
}

int svdi_create(const svdi_options* opt, svdi_server** out) {
    return svdi_server_create(opt, SVDI_DEFAULT_SLOTS, 0, 0, out);
}

int svdi_submit(svdi_server* s, const svdi_host_ms* ms, size_t image_size, float cell_size, float* dirty_image,
                uint64_t* ticket) {
    return svdi_server_submit(s, ms, image_size, cell_size, dirty_image, ticket);
}

int svdi_poll(svdi_server* s, uint64_t ticket, int* done) { return svdi_server_poll(s, ticket, done); }

int svdi_wait(svdi_server* s, uint64_t ticket, double timeout_s, svdi_request_info* info) {
    return svdi_server_wait(s, ticket, timeout_s, info);
}

void svdi_destroy(svdi_server* s) { svdi_server_destroy(s); }

void svdi_server_destroy(svdi_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto* e : s->engines) svdi_engine_destroy(e);
    delete s;
}

}  // extern "C"

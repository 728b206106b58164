// bph_serve.cu -- continuous batching of potential solves for resident clients.
//
// A client is one instance of a bph_batch: its -4 pi rho_hat and its last
// potential (the warm state) stay on the device between requests, so every
// request after a client's first warm-starts its ADI from the previous
// solution, as consecutive potential_solver calls do (potential_solver.F90:
// 80-94: tstep > 1 warm 5 steps, else cold 20).
//
// One worker thread drives the GPU.  Requests queue in arrival order; each
// time the GPU is free the worker takes the oldest pending request of every
// client that has one (at most max_batch), splits them into first requests
// (cold) and later ones (warm), and solves each group in one batched call
// (one pass over the Green tables, one ADI launch over all their slots).
// Requests that arrive while a batch runs join the next one.  Clients are
// admitted while device memory allows: the number of resident clients is
// fixed at creation from the memory cap and the free device memory, and
// opening a client beyond it is refused with BPH_ERR_NOMEM.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bph_internal.cuh"

struct bph_server {
    bph_ctx *c = nullptr;
    bph_batch *batch = nullptr;
    int capacity = 0;   // resident clients
    int max_batch = 0;  // requests per batched call
    bool device_arrays = false;  // rho/pot are device arrays (else host arrays)
    size_t bytes_per_client = 0;

    struct Request {
        int client = -1;
        const double *rho = nullptr;
        double *pot = nullptr;
        int status = 1;  // 1: pending, else the final status
        double t_submit = 0.0, t_done = 0.0;
    };

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<long long> queue;                 // pending request ids in arrival order
    std::unordered_map<long long, Request> reqs;  // pending and completed, until polled done
    std::vector<char> open, warm;                // per client
    std::vector<int> inflight;                   // requests queued or running per client
    long long next_id = 1;
    long long batches = 0, solves = 0;
    int conv_nsteps = 0;  // converged mode: ADI steps per cycle (0: the drop-in solve)
    double conv_tol = 0.0;
    int conv_max_cycles = 0;
    bool conv_mixed = false;
    bool stop = false;
    std::thread worker;
};

namespace bph {
namespace {

constexpr int kPending = 1;

double now_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

void serve_loop(bph_server *s) {
    std::vector<long long> take;
    std::vector<char> take_warm;  // the client's state when the request was taken
    std::vector<int> group_inst;
    std::vector<const double *> group_rho;
    std::vector<double *> group_pot;
    std::vector<long long> group_ids;
    std::vector<int> group_status;
    for (;;) {
        take.clear();
        take_warm.clear();
        BatchConv conv;
        bool converged = false;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) return;  // stop requested and nothing left
            converged = s->conv_nsteps > 0;
            conv.nsteps = s->conv_nsteps;
            conv.tol = s->conv_tol;
            conv.max_cycles = s->conv_max_cycles;
            conv.mixed = s->conv_mixed;
            // oldest request of every client with one pending, in arrival order
            std::vector<char> seen((size_t)s->capacity, 0);
            for (auto it = s->queue.begin(); it != s->queue.end() && (int)take.size() < s->max_batch;) {
                const int cl = s->reqs[*it].client;
                if (!seen[(size_t)cl]) {
                    seen[(size_t)cl] = 1;
                    take.push_back(*it);
                    take_warm.push_back(s->warm[(size_t)cl]);
                    it = s->queue.erase(it);
                } else {
                    ++it;
                }
            }
        }
        // first requests of their clients run cold, the others warm
        for (int pass = 0; pass < 2; ++pass) {
            const bool warm_pass = (pass == 1);
            group_inst.clear();
            group_rho.clear();
            group_pot.clear();
            group_ids.clear();
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (size_t t = 0; t < take.size(); ++t) {
                    if ((take_warm[t] != 0) != warm_pass) continue;
                    const long long id = take[t];
                    const bph_server::Request &r = s->reqs[id];
                    group_inst.push_back(r.client);
                    group_rho.push_back(r.rho);
                    group_pot.push_back(r.pot);
                    group_ids.push_back(id);
                }
            }
            if (group_ids.empty()) continue;
            const int n = (int)group_ids.size();
            group_status.assign((size_t)n, BPH_OK);
            conv.cold = !warm_pass;
            int rc = batch_solve_core(s->batch, n, group_inst.data(), group_rho.data(), group_pot.data(), warm_pass,
                                      s->device_arrays, group_status.data(), converged ? &conv : nullptr);
            const double t = now_s();
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (int i = 0; i < n; ++i) {
                    bph_server::Request &r = s->reqs[group_ids[(size_t)i]];
                    r.status = rc ? rc : group_status[(size_t)i];
                    r.t_done = t;
                    // a client whose density was rejected keeps no usable state: its next request is cold
                    s->warm[(size_t)r.client] = (r.status == BPH_OK) ? 1 : 0;
                    --s->inflight[(size_t)r.client];
                }
                ++s->batches;
                s->solves += n;
            }
            s->cv_done.notify_all();
        }
    }
}

}  // namespace
}  // namespace bph

using namespace bph;

extern "C" {

int bph_server_create(bph_ctx_t *c, int max_clients, size_t mem_cap_bytes, int max_batch, int flags,
                      bph_server_t **out) {
    if (!out) {
        set_error("out-pointer is NULL");
        return BPH_ERR_INVALID;
    }
    *out = nullptr;
    if (!c || max_clients < 1 || max_clients > 4096 || max_batch < 0 || (flags & ~BPH_SERVER_DEVICE_ARRAYS)) {
        set_error("invalid context, client count (1..4096), batch size or flags");
        return BPH_ERR_INVALID;
    }
    const bool dev = (flags & BPH_SERVER_DEVICE_ARRAYS) != 0;
    if (!c->adi_seg && c->adi_smem) {
        set_error("serving needs the segmented or the grid-wide ADI kernels for this grid");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    cudaError_t e;
    // resident bytes of one client: slot array, -4 pi rho_hat, moments and
    // contraction output of its batch position, host-array staging (rho, pot)
    const size_t per = sizeof(double) * ((size_t)c->N * c->nplane + (size_t)c->N * c->np * (c->adi_seg ? 1 : 3) +
                                         2ull * c->g.mmax * c->np + 2ull * c->g.mmax * c->nb +
                                         (dev ? 0ull : 2ull * c->ntot));
    size_t free_b = 0, total_b = 0;
    e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
    const size_t margin = 256ull << 20;
    size_t budget = free_b > margin ? free_b - margin : 0;
    if (mem_cap_bytes && mem_cap_bytes < budget) budget = mem_cap_bytes;
    long long fit = (long long)(budget / per);
    if (!c->adi_seg && fit > 65535 / c->N) fit = 65535 / c->N;  // grid-wide ADI: capacity * numphi <= 65535
    const int cap = (int)(fit < max_clients ? fit : max_clients);
    if (cap < 1) {
        set_error("no client fits: %zu bytes per client, budget %zu", per, budget);
        return BPH_ERR_NOMEM;
    }
    bph_server *s = new bph_server();
    s->c = c;
    s->capacity = cap;
    s->max_batch = (max_batch == 0 || max_batch > cap) ? cap : max_batch;
    s->bytes_per_client = per;
    s->device_arrays = dev;
    s->open.assign((size_t)cap, 0);
    s->warm.assign((size_t)cap, 0);
    s->inflight.assign((size_t)cap, 0);
    int rc = bph_batch_create(c, cap, &s->batch);
    if (rc) {
        delete s;
        return rc;
    }
    s->worker = std::thread(serve_loop, s);
    *out = s;
    return BPH_OK;
}

int bph_server_set_converged(bph_server_t *s, int nsteps, double tol, int max_cycles, int mixed) {
    if (!s || nsteps < 0 || nsteps > 10000 || (nsteps > 0 && (max_cycles < 1 || !(tol >= 0.0)))) {
        set_error("invalid server or converged-mode arguments");
        return BPH_ERR_INVALID;
    }
    bph_ctx *c = s->c;
    if (nsteps > 0 && mixed && !c->adi_mixed_smem) {
        set_error("no mixed-precision ADI kernel is configured for this grid");
        return BPH_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (nsteps > 0) {
        // buffers first: a batch the worker takes after the mode changes finds them
        const int rc = batch_reserve_converged(s->batch, mixed != 0);
        if (rc) return rc;
    }
    s->conv_nsteps = nsteps;
    s->conv_tol = tol;
    s->conv_max_cycles = max_cycles;
    s->conv_mixed = mixed != 0;
    return BPH_OK;
}

int bph_server_capacity(const bph_server_t *s) { return s ? s->capacity : 0; }

int bph_server_open_client(bph_server_t *s, int *client) {
    if (!s || !client) {
        set_error("server or out-pointer is NULL");
        return BPH_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i = 0; i < s->capacity; ++i)
        if (!s->open[(size_t)i] && s->inflight[(size_t)i] == 0) {
            s->open[(size_t)i] = 1;
            s->warm[(size_t)i] = 0;
            *client = i;
            return BPH_OK;
        }
    set_error("all %d resident client slots are in use (device memory admission)", s->capacity);
    return BPH_ERR_NOMEM;
}

int bph_server_close_client(bph_server_t *s, int client) {
    if (!s) {
        set_error("server is NULL");
        return BPH_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (client < 0 || client >= s->capacity || !s->open[(size_t)client]) {
        set_error("client %d is not open", client);
        return BPH_ERR_INVALID;
    }
    // its queued requests still complete; the slot is reused once they have
    s->open[(size_t)client] = 0;
    return BPH_OK;
}

int bph_server_submit(bph_server_t *s, int client, const double *rho, double *pot, long long *request) {
    if (!s || !rho || !pot || !request) {
        set_error("server, arrays or out-pointer is NULL");
        return BPH_ERR_INVALID;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            set_error("server is shutting down");
            return BPH_ERR_STATE;
        }
        if (client < 0 || client >= s->capacity || !s->open[(size_t)client]) {
            set_error("client %d is not open", client);
            return BPH_ERR_INVALID;
        }
        const long long id = s->next_id++;
        bph_server::Request r;
        r.client = client;
        r.rho = rho;
        r.pot = pot;
        r.status = kPending;
        r.t_submit = now_s();
        s->reqs[id] = r;
        s->queue.push_back(id);
        ++s->inflight[(size_t)client];
        *request = id;
    }
    s->cv_work.notify_one();
    return BPH_OK;
}

int bph_server_poll(bph_server_t *s, long long request, double *latency_s) {
    if (!s) {
        set_error("server is NULL");
        return BPH_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) {
        set_error("unknown request %lld (never submitted, or already reported done)", request);
        return BPH_ERR_INVALID;
    }
    const int st = it->second.status;
    if (st == kPending) return BPH_PENDING;
    if (latency_s) *latency_s = it->second.t_done - it->second.t_submit;
    s->reqs.erase(it);
    if (st != BPH_OK) set_error("request %lld failed with status %d", request, st);
    return st;
}

int bph_server_wait(bph_server_t *s, long long request, double timeout_s, double *latency_s) {
    if (!s) {
        set_error("server is NULL");
        return BPH_ERR_INVALID;
    }
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto done = [&] {
            auto it = s->reqs.find(request);
            return it == s->reqs.end() || it->second.status != kPending;
        };
        if (timeout_s > 0.0) {
            if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
                set_error("request %lld still pending after %.3f s", request, timeout_s);
                return BPH_ERR_TIMEOUT;
            }
        } else {
            s->cv_done.wait(lk, done);
        }
    }
    return bph_server_poll(s, request, latency_s);
}

int bph_server_stats(const bph_server_t *s, long long *batches, long long *solves) {
    if (!s) {
        set_error("server is NULL");
        return BPH_ERR_INVALID;
    }
    bph_server *m = const_cast<bph_server *>(s);
    std::lock_guard<std::mutex> lk(m->mu);
    if (batches) *batches = m->batches;
    if (solves) *solves = m->solves;
    return BPH_OK;
}

int bph_server_destroy(bph_server_t *s) {
    if (!s) return BPH_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();  // queued requests finish first
    int rc = bph_batch_destroy(s->batch);
    delete s;
    return rc;
}

}  // extern "C"

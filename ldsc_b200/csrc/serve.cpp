// serve.cpp -- continuous batching of l2 and regression jobs over resident
// panels.  The server is a scheduler over the public C ABI: it owns n_slots
// engine contexts (each with its own stream, workspace and worker thread),
// admits queued jobs in arrival order as a slot and device memory free up,
// and lets admitted jobs run concurrently so their kernels overlap on the
// device.  It has no counterpart in the reference, which runs one
// computation per process (src/l2/mod.rs:439-575 fans chromosomes out over
// threads inside one run).
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ldsc_b200.h"
#include "regress.h"

namespace {

using Clock = std::chrono::steady_clock;

struct JobRec {
    uint64_t ticket = 0;
    ldsc_job job;
    uint64_t need = 0;  // device workspace bytes
    int state = 0;      // 0 queued, 1 running, 2 done
    int32_t pin = -1;   // slot that must run it (prewarm), or -1 for any
    ldsc_job_result res;
    Clock::time_point t_submit, t_start, t_end;
};

struct Slot {
    ldsc_ctx* ctx = nullptr;
    std::thread th;
    uint64_t cap = 0;        // workspace bytes this slot's context may hold
    bool busy = false;
    bool trim_req = false;   // give the workspace back (an older job needs the memory)
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

uint64_t regression_bytes(const ldsc_job& j) {
    if (j.kind == LDSC_JOB_H2P) {
        // block Grams, totals, solves, results, block starts, the summed LD score
        const ldsc_h2p_args& a = j.h2p;
        const uint64_t T = a.n_traits, n = a.n_snp, nb = a.n_blocks, K = a.n_annot;
        const uint64_t P = K + (a.fixed_intercept ? 0 : 1), Q = P + 1;
        const uint64_t C = (uint64_t)ldsc::part_trait_chunk((int)(T ? T : 1), (int)nb, (int)Q);  // traits per launch
        uint64_t b = 8 * C * (nb * Q * Q + Q * Q + (nb + 1) * P + 3 * nb) + 8 * T * (P * (1 + P + nb) + K + 7) +
                     4 * T * (2 * (nb + 1) + (n + 4095) / 4096) + 8 * n + 4096 + 256 * T;
        if (!a.device_pointers) b += 8 * T * n * (a.n_per_snp ? 2 : 1) + 8 * n * (K + 1);
        return b;
    }
    if (j.kind == LDSC_JOB_H2) {
        const ldsc_h2_args& a = j.h2;
        const uint64_t T = a.n_traits, n = a.n_snp, nb = a.n_blocks < n ? a.n_blocks : n;
        uint64_t b = T * (512 + 40 * nb) + 4096;
        if (!a.device_pointers) b += 8 * T * n * (a.n_per_snp ? 2 : 1) + 16 * n;
        return b;
    }
    const ldsc_rg_args& a = j.rg;
    const uint64_t P = a.n_pairs, n = a.n_snp, nb = a.n_blocks < n ? a.n_blocks : n;
    uint64_t b = 3 * P * (512 + 48 * nb) + P * 256 + 4096;
    if (!a.device_pointers) b += 16 * P * n + 16 * n;
    return b;
}

}  // namespace

struct ldsc_server {
    int device = 0;
    uint64_t budget = 0;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<JobRec*> pending;
    std::unordered_map<uint64_t, JobRec*> jobs;
    uint64_t next_ticket = 1, submitted = 0, completed = 0, running = 0;
    bool stop = false;

    uint64_t caps() const {
        uint64_t t = 0;
        for (const Slot& s : slots) t += s.cap;
        return t;
    }

    // First queued job that slot i can run now.  A job fits when the slot's
    // workspace already covers it, or when growing the slot keeps the sum of
    // all slots' workspaces within the budget.  When the oldest job fits in no
    // slot but would once idle slots give their workspace back, those slots
    // are asked to do so (later jobs may still pass it meanwhile).
    JobRec* pick(size_t i) {
        Slot& sl = slots[i];
        if (sl.trim_req) return nullptr;
        const uint64_t total = caps();
        for (size_t q = 0; q < pending.size(); q++) {
            JobRec* r = pending[q];
            if (r->pin >= 0 && r->pin != (int32_t)i) continue;
            if (r->need <= sl.cap || total - sl.cap + r->need <= budget) {
                if (r->need > sl.cap) sl.cap = r->need;
                pending.erase(pending.begin() + (long)q);
                return r;
            }
            if (q == 0) {
                uint64_t idle = 0;
                for (const Slot& o : slots)
                    if (!o.busy) idle += o.cap;
                if (total - idle + r->need <= budget) {
                    for (Slot& o : slots)
                        if (!o.busy && o.cap > 0) o.trim_req = true;
                    cv_work.notify_all();
                }
            }
        }
        return nullptr;
    }

    void run(size_t i, JobRec* r) {
        Slot& sl = slots[i];
        ldsc_job& j = r->job;
        ldsc_job_result& res = r->res;
        int rc = LDSC_E_INVALID;
        if (j.kind == LDSC_JOB_L2)
            rc = ldsc_l2_run(sl.ctx, j.panel, &j.l2, j.l2_out, j.maf_out, &res.perf);
        else if (j.kind == LDSC_JOB_H2)
            rc = ldsc_h2_batch(sl.ctx, &j.h2, j.h2_out);
        else if (j.kind == LDSC_JOB_RG)
            rc = ldsc_rg_batch(sl.ctx, &j.rg, j.rg_out);
        else if (j.kind == LDSC_JOB_H2P)
            rc = ldsc_h2_partitioned(sl.ctx, &j.h2p, j.h2p_out);
        res.status = rc;
        res.slot = (uint32_t)i;
        if (rc != LDSC_OK) ldsc_last_error(sl.ctx, res.error, sizeof res.error);
    }

    void worker(size_t i) {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            JobRec* r = nullptr;
            Slot& sl = slots[i];
            cv_work.wait(lk, [&] {
                if (stop) return true;
                r = pick(i);
                return r != nullptr || sl.trim_req;
            });
            if (sl.trim_req && !r) {
                lk.unlock();
                ldsc_ctx_trim(sl.ctx);
                lk.lock();
                sl.cap = 0;
                sl.trim_req = false;
                cv_work.notify_all();
                continue;
            }
            if (!r) return;  // stopping, nothing admissible
            sl.busy = true;
            running++;
            r->state = 1;
            r->t_start = Clock::now();
            lk.unlock();
            run(i, r);
            lk.lock();
            r->t_end = Clock::now();
            r->res.queue_ms = ms_between(r->t_submit, r->t_start);
            r->res.run_ms = ms_between(r->t_start, r->t_end);
            r->res.latency_ms = ms_between(r->t_submit, r->t_end);
            r->state = 2;
            sl.busy = false;
            running--;
            completed++;
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

int ldsc_server_create(int device, uint32_t n_slots, uint64_t device_budget, ldsc_server** out) {
    if (!out || n_slots == 0 || n_slots > 64) return LDSC_E_INVALID;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return LDSC_E_CUDA;
    }
    ldsc_server* srv = new ldsc_server();
    srv->device = device;
    if (device_budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete srv;
            return LDSC_E_CUDA;
        }
        const uint64_t headroom = 4ull << 30;
        device_budget = fr > headroom ? (uint64_t)(fr - headroom) : fr / 2;
    }
    srv->budget = device_budget;
    srv->slots.resize(n_slots);
    for (uint32_t i = 0; i < n_slots; i++) {
        int rc = ldsc_ctx_create(device, 0, &srv->slots[i].ctx);
        if (rc != LDSC_OK) {
            for (uint32_t k = 0; k < i; k++) ldsc_ctx_destroy(srv->slots[k].ctx);
            delete srv;
            return rc;
        }
    }
    for (uint32_t i = 0; i < n_slots; i++) srv->slots[i].th = std::thread([srv, i] { srv->worker(i); });
    *out = srv;
    return LDSC_OK;
}

static int submit_pinned(ldsc_server* srv, const ldsc_job* job, int32_t pin, uint64_t* ticket) {
    if (!srv || !job || !ticket) return LDSC_E_INVALID;
    if (job->kind != LDSC_JOB_L2 && job->kind != LDSC_JOB_H2 && job->kind != LDSC_JOB_RG &&
        job->kind != LDSC_JOB_H2P)
        return LDSC_E_INVALID;
    if (job->kind == LDSC_JOB_L2 && (!job->panel || (job->l2.n_snp && !job->l2_out))) return LDSC_E_INVALID;
    if (job->kind == LDSC_JOB_H2 && !job->h2_out) return LDSC_E_INVALID;
    if (job->kind == LDSC_JOB_RG && !job->rg_out) return LDSC_E_INVALID;
    if (job->kind == LDSC_JOB_H2P && !job->h2p_out) return LDSC_E_INVALID;
    JobRec* r = new JobRec();
    r->job = *job;
    std::memset(&r->res, 0, sizeof r->res);
    r->need = job->device_bytes;
    if (!r->need) {
        if (job->kind == LDSC_JOB_L2) {
            uint64_t n_indiv = 0, n_snp = 0;
            ldsc_panel_shape(job->panel, &n_indiv, &n_snp);
            if (ldsc_l2_workspace_bytes(&job->l2, n_indiv, &r->need) != LDSC_OK) {
                delete r;
                return LDSC_E_INVALID;
            }
        } else {
            r->need = regression_bytes(*job);
        }
    }
    std::lock_guard<std::mutex> g(srv->mu);
    if (srv->stop) {
        delete r;
        return LDSC_E_INVALID;
    }
    if (r->need > srv->budget) {
        delete r;
        return LDSC_E_NOMEM;
    }
    r->ticket = srv->next_ticket++;
    r->pin = pin;
    r->t_submit = Clock::now();
    srv->jobs[r->ticket] = r;
    srv->pending.push_back(r);
    srv->submitted++;
    *ticket = r->ticket;
    srv->cv_work.notify_all();
    return LDSC_OK;
}

int ldsc_server_submit(ldsc_server* srv, const ldsc_job* job, uint64_t* ticket) {
    return submit_pinned(srv, job, -1, ticket);
}

int ldsc_server_prewarm(ldsc_server* srv, const ldsc_job* job) {
    if (!srv || !job) return LDSC_E_INVALID;
    for (uint32_t i = 0; i < (uint32_t)srv->slots.size(); i++) {
        uint64_t t = 0;
        int rc = submit_pinned(srv, job, (int32_t)i, &t);
        if (rc == LDSC_OK) rc = ldsc_server_wait(srv, t, nullptr);
        if (rc != LDSC_OK) return rc;
    }
    return LDSC_OK;
}

int ldsc_server_wait(ldsc_server* srv, uint64_t ticket, ldsc_job_result* res) {
    if (!srv) return LDSC_E_INVALID;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) return LDSC_E_INVALID;
    JobRec* r = it->second;
    srv->cv_done.wait(lk, [&] { return r->state == 2; });
    if (res) *res = r->res;
    const int st = r->res.status;
    srv->jobs.erase(it);
    delete r;
    return st;
}

int ldsc_server_stats_get(ldsc_server* srv, ldsc_server_stats* st) {
    if (!srv || !st) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(srv->mu);
    std::memset(st, 0, sizeof *st);
    st->submitted = srv->submitted;
    st->completed = srv->completed;
    st->running = srv->running;
    st->queued = srv->pending.size();
    st->budget_bytes = srv->budget;
    st->reserved_bytes = srv->caps();
    for (const Slot& s : srv->slots) {
        st->graph_launches += ldsc_ctx_graph_launches(s.ctx);
        st->kernels += ldsc_ctx_kernel_count(s.ctx);
    }
    return LDSC_OK;
}

int ldsc_server_destroy(ldsc_server* srv) {
    if (!srv) return LDSC_OK;
    {
        std::lock_guard<std::mutex> g(srv->mu);
        srv->stop = true;
        // queued jobs never start; their waiters see the error
        for (JobRec* r : srv->pending) {
            r->res.status = LDSC_E_INVALID;
            std::snprintf(r->res.error, sizeof r->res.error, "server shut down before the job started");
            r->state = 2;
        }
        srv->pending.clear();
        srv->cv_work.notify_all();
        srv->cv_done.notify_all();
    }
    for (Slot& s : srv->slots)
        if (s.th.joinable()) s.th.join();
    for (Slot& s : srv->slots) ldsc_ctx_destroy(s.ctx);
    for (auto& kv : srv->jobs) delete kv.second;
    delete srv;
    return LDSC_OK;
}

}  // extern "C"

// vd_server.cu -- continuous-batching request loop over a batch (vd_server_* in
// vidyut_b200.h).  No counterpart in the reference, which runs one case per
// process.
//
// Requests (a discharge case: box, state, face fields, parameters, step count)
// are submitted from any host thread; the server copies their inputs into host
// memory it owns and queues them.  One worker thread owns a vd_batch on one GPU:
//   admit    queued requests, oldest first, each as soon as the batch's HBM arena
//            has room for it (a request that does not fit lets later, smaller
//            ones in -- backfill -- until it has waited 200 ms; from then on
//            admission is strictly in order, so the arena drains until it fits);
//   step     the resident cases together by one quantum of explicit steps (one
//            graph replay; cases with fewer steps left stop early);
//   retire   finished cases: their state comes back to host memory, their arena
//            region is freed and their waiters are woken.
// So requests that arrive while others run join the next quantum, and their work
// shares every launch with the cases already resident.  Latency is measured per
// request from submission to the moment its result is in host memory.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include "vd_host.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr double kHoldMs = 200.0;  // longest a request waits while smaller ones backfill

struct Request {
    int64_t id = 0;
    vd_box box{};
    vd_params prm{};
    int32_t periodic[3] = {0, 0, 0};
    int64_t nsteps = 0;
    std::vector<double> state;      // input, then the result
    std::vector<double> face[2][3]; // efield_ec, gradne_fc (empty when unused)
    uint64_t bytes = 0;             // arena bytes the case needs
    Clock::time_point t_submit, t_admit, t_done;
    int status = 1;                 // 1 queued, 2 resident, 0 done, < 0 failed
    int32_t case_id = -1;
    int64_t cells = 0;
};

int err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int err(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return vd_host::set_error(code, buf);
}

}  // namespace

struct vd_server {
    int dev = 0;
    int prec = VD_PREC_MIXED;
    int quantum = 25;
    vd_batch* batch = nullptr;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;            // submitted, not admitted
    std::map<int64_t, std::shared_ptr<Request>> all;       // every request not yet collected
    std::vector<std::shared_ptr<Request>> resident;        // worker thread only
    std::vector<double> latencies_ms;
    int64_t next_id = 1, submitted = 0, completed = 0, failed = 0, quanta = 0;
    int64_t cell_updates = 0, graph_builds = 0;
    uint64_t peak_bytes = 0;
    Clock::time_point t_first{}, t_last{};
    bool have_first = false;
    bool stop = false;
    int fatal = 0;
    std::thread worker;
};

namespace {

// worker: fail every resident and queued request with status code
void fail_all(vd_server* s, int code)
{
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto& r : s->resident) {
        r->status = code;
        r->t_done = Clock::now();
        s->failed++;
    }
    s->resident.clear();
    for (auto& r : s->queue) {
        r->status = code;
        r->t_done = Clock::now();
        s->failed++;
    }
    s->queue.clear();
    s->fatal = code;
    s->cv_done.notify_all();
}

void worker_main(vd_server* s)
{
    cudaSetDevice(s->dev);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        fail_all(s, VD_ERR_CUDA);
        return;
    }
    for (;;) {
        // admit
        std::vector<std::shared_ptr<Request>> cand;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty() || !s->resident.empty(); });
            if (s->stop) break;
            cand.assign(s->queue.begin(), s->queue.end());
        }
        std::vector<std::shared_ptr<Request>> admitted;
        for (auto& r : cand) {
            // a request that has waited kHoldMs without fitting stops the backfill,
            // so that the arena drains until it fits (no starvation of large cases)
            const double age_ms = std::chrono::duration<double, std::milli>(Clock::now() - r->t_submit).count();
            const double* ef[3] = {nullptr, nullptr, nullptr};
            const double* gn[3] = {nullptr, nullptr, nullptr};
            for (int d = 0; d < 3; d++) {
                if (!r->face[0][d].empty()) ef[d] = r->face[0][d].data();
                if (!r->face[1][d].empty()) gn[d] = r->face[1][d].data();
            }
            int32_t cid = -1;
            int rc = vd_batch_add_case(s->batch, &r->box, r->state.data(), ef, gn, &r->prm, r->periodic, r->nsteps,
                                       st, &cid);
            if (rc == VD_ERR_BUDGET) {
                if (age_ms > kHoldMs) break;
                continue;  // later, smaller requests may still fit
            }
            std::lock_guard<std::mutex> lk(s->mu);
            if (rc != VD_OK) {
                r->status = rc;
                r->t_done = Clock::now();
                s->failed++;
                s->cv_done.notify_all();
            } else {
                r->case_id = cid;
                r->status = 2;
                r->t_admit = Clock::now();
                admitted.push_back(r);
            }
            s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
        }
        s->resident.insert(s->resident.end(), admitted.begin(), admitted.end());
        if (s->resident.empty()) {
            // nothing fits although requests wait: only possible when a request was
            // accepted that exceeds an empty arena (submission rejects those)
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        vd_batch_stats bs;
        vd_batch_get_stats(s->batch, &bs);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->peak_bytes = std::max<uint64_t>(s->peak_bytes, bs.bytes_used);
        }
        // step one quantum
        int rc = vd_batch_step(s->batch, s->quantum, st);
        if (rc == VD_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = VD_ERR_CUDA;
        if (rc != VD_OK) {
            fail_all(s, rc);
            break;
        }
        vd_batch_get_stats(s->batch, &bs);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->quanta++;
            s->graph_builds = bs.graph_builds;
        }
        // cases that met a NaN or infinity fail (the reference aborts the run there)
        std::vector<int> bad;
        if ((rc = vd_host::batch_failed_cases(s->batch, &bad)) != VD_OK) {
            fail_all(s, rc);
            break;
        }
        // retire
        std::vector<std::shared_ptr<Request>> keep;
        for (auto& r : s->resident) {
            if (std::find(bad.begin(), bad.end(), r->case_id) != bad.end()) {
                vd_batch_remove_case(s->batch, r->case_id);
                std::lock_guard<std::mutex> lk(s->mu);
                r->t_done = Clock::now();
                r->status = VD_ERR_NONFINITE;
                s->failed++;
                for (int p = 0; p < 2; p++)
                    for (int d = 0; d < 3; d++) std::vector<double>().swap(r->face[p][d]);
                s->cv_done.notify_all();
                continue;
            }
            int64_t done = 0, left = 0;
            vd_batch_case_info(s->batch, r->case_id, &done, &left);
            if (left != 0) {
                keep.push_back(r);
                continue;
            }
            int rr = vd_batch_read_case(s->batch, r->case_id, r->state.data(), st);
            if (rr == VD_OK && cudaStreamSynchronize(st) != cudaSuccess) rr = VD_ERR_CUDA;
            vd_batch_remove_case(s->batch, r->case_id);
            std::lock_guard<std::mutex> lk(s->mu);
            r->t_done = Clock::now();
            if (rr == VD_OK) {
                r->status = 0;
                s->completed++;
                s->cell_updates += r->cells * r->nsteps;
                s->latencies_ms.push_back(
                    std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
                s->t_last = r->t_done;
            } else {
                r->status = rr;
                s->failed++;
            }
            for (int p = 0; p < 2; p++)
                for (int d = 0; d < 3; d++) std::vector<double>().swap(r->face[p][d]);
            s->cv_done.notify_all();
        }
        s->resident.swap(keep);
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
}

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double pos = q * (double)(v.size() - 1);
    size_t i = (size_t)pos;
    double f = pos - (double)i;
    if (i + 1 < v.size()) return v[i] * (1.0 - f) + v[i + 1] * f;
    return v[i];
}

}  // namespace

extern "C" {

int vd_server_create(vd_server** out, int precision, uint64_t hbm_budget_bytes, int max_cases, int quantum_steps)
{
    if (!out) return err(VD_ERR_ARG, "null output");
    *out = nullptr;
    if (quantum_steps < 1) return err(VD_ERR_ARG, "quantum_steps %d < 1", quantum_steps);
    vd_batch* b = nullptr;
    int rc = vd_batch_create(&b, precision, hbm_budget_bytes, max_cases);
    if (rc) return rc;
    vd_server* s = new vd_server;
    cudaGetDevice(&s->dev);
    s->prec = precision;
    s->quantum = quantum_steps;
    s->batch = b;
    s->budget = hbm_budget_bytes;
    s->worker = std::thread(worker_main, s);
    *out = s;
    return VD_OK;
}

int vd_server_destroy(vd_server* s)
{
    if (!s) return VD_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& kv : s->all)
            if (kv.second->status > 0) kv.second->status = VD_ERR_STATE;
    }
    s->cv_done.notify_all();
    int dev0 = 0;
    cudaGetDevice(&dev0);
    cudaSetDevice(s->dev);
    vd_batch_destroy(s->batch);
    cudaSetDevice(dev0);
    delete s;
    return VD_OK;
}

int vd_server_submit(vd_server* s, const vd_box* bx, const double* state, const double* const efield_ec[3],
                     const double* const gradne_fc[3], const vd_params* prm, const int32_t periodic[3],
                     int64_t nsteps, int64_t* request_id)
{
    if (!s || !bx || !state || !prm || !request_id) return err(VD_ERR_ARG, "null argument");
    if (nsteps < 1) return err(VD_ERR_ARG, "nsteps %lld < 1", (long long)nsteps);
    if (prm->precision != s->prec)
        return err(VD_ERR_ARG, "request precision %d differs from the server's %d", prm->precision, s->prec);
    const uint64_t need = vd_batch_case_bytes(bx, prm);
    if (need == 0) return VD_ERR_ARG;  // vd_batch_case_bytes left the reason in vd_last_error
    if (need > s->budget)
        return err(VD_ERR_BUDGET, "request needs %llu bytes of HBM; the server's budget is %llu",
                   (unsigned long long)need, (unsigned long long)s->budget);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->fatal) return err(s->fatal, "the server stopped after an error");
    }
    vd_host::MechInfo m;
    int rc = vd_host::mech_info(&m);
    if (rc) return rc;
    auto r = std::make_shared<Request>();
    r->box = *bx;
    r->prm = *prm;
    for (int d = 0; d < 3; d++) r->periodic[d] = periodic ? periodic[d] : 0;
    r->nsteps = nsteps;
    const int H = vd_host::stencil_halo(prm->hyp_order);
    int64_t gcells = 1, vcells = 1;
    for (int d = 0; d < 3; d++) {
        const int n = bx->hi[d] - bx->lo[d] + 1;
        gcells *= n + (d < bx->dim ? 2 * H : 0);
        vcells *= n;
    }
    r->cells = vcells;
    r->state.assign(state, state + gcells * VD_NVAR(m.ns));
    const bool ef = prm->elecenergy_solve && !prm->cs_technique;
    const bool gn = prm->elecenergy_solve && !prm->gradne_from_state;
    for (int d = 0; d < bx->dim; d++) {
        const int64_t fc = vcells / (bx->hi[d] - bx->lo[d] + 1) * (bx->hi[d] - bx->lo[d] + 2);
        if (ef) {
            if (!efield_ec || !efield_ec[d]) return err(VD_ERR_ARG, "efield_ec[%d] needed", d);
            r->face[0][d].assign(efield_ec[d], efield_ec[d] + fc);
        }
        if (gn) {
            if (!gradne_fc || !gradne_fc[d]) return err(VD_ERR_ARG, "gradne_fc[%d] needed", d);
            r->face[1][d].assign(gradne_fc[d], gradne_fc[d] + fc);
        }
    }
    r->bytes = need;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        r->t_submit = Clock::now();
        if (!s->have_first) {
            s->t_first = r->t_submit;
            s->have_first = true;
        }
        s->queue.push_back(r);
        s->all[r->id] = r;
        s->submitted++;
        *request_id = r->id;
    }
    s->cv_work.notify_one();
    return VD_OK;
}

int vd_server_wait(vd_server* s, int64_t request_id, double* state_out, double timeout_s, double* latency_ms)
{
    if (!s) return err(VD_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return err(VD_ERR_ARG, "no request %lld (unknown or already collected)",
                                       (long long)request_id);
    std::shared_ptr<Request> r = it->second;
    auto pred = [&] { return r->status <= 0; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, pred);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
        return err(VD_ERR_TIMEOUT, "request %lld not finished after %.3f s", (long long)request_id, timeout_s);
    }
    s->all.erase(request_id);
    if (r->status < 0) return err(r->status, "request %lld failed (status %d)", (long long)request_id, r->status);
    if (state_out) memcpy(state_out, r->state.data(), r->state.size() * sizeof(double));
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    return VD_OK;
}

int vd_server_get_stats(vd_server* s, vd_server_stats* out)
{
    if (!s || !out) return err(VD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->queued = (int64_t)s->queue.size();
    out->p50_ms = percentile(s->latencies_ms, 0.50);
    out->p99_ms = percentile(s->latencies_ms, 0.99);
    out->max_ms = s->latencies_ms.empty() ? 0.0 : *std::max_element(s->latencies_ms.begin(), s->latencies_ms.end());
    double span = s->have_first && s->completed ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
    out->span_s = span;
    out->solves_per_s = span > 0 ? (double)s->completed / span : 0.0;
    out->cell_updates_per_s = span > 0 ? (double)s->cell_updates / span : 0.0;
    out->bytes_budget = s->budget;
    out->peak_bytes_used = s->peak_bytes;
    out->quanta = s->quanta;
    out->graph_builds = s->graph_builds;
    return VD_OK;
}

}  // extern "C"

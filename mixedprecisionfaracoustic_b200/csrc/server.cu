// server.cu - serving loop: shot requests are admitted against an HBM budget,
// stay resident on the device and are advanced together (continuous
// batching): at every sync boundary (steps_per_sync steps) finished shots
// leave, their memory returns to the budget, and queued requests that now fit
// join the running batch.  Each request's arithmetic depends only on its own
// shot, so its traces are identical whether it runs alone or in a mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>

#include "batch.h"

using namespace bpk;

namespace {
using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    bp_config cfg{};
    std::vector<int> rx, ry, rz;
    std::vector<float> medium;          // 9 * cells, freed once resident
    size_t bytes = 0;
    int state = BP_REQ_QUEUED;
    bool cancel = false;
    Clock::time_point t_submit, t_done;
    std::vector<float> traces;          // [comp][rec][nt] when done
    std::string err;
    Shot* shot = nullptr;
};
}  // namespace

struct bp_server {
    int device = 0;
    size_t budget = 0;
    int sps = 100;
    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::deque<uint64_t> pending;
    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    size_t in_use = 0;
    bool stop = false;
    uint64_t next_id = 1;
    std::thread worker;
    // stats
    long long submitted = 0, admitted = 0, completed = 0, failed = 0, cancelled = 0;
    long long cell_updates = 0;
    double busy = 0;
    int max_resident = 0;
    std::vector<double> latencies;
    int worker_error = 0;
};

// One batch per (dim, order, precision, rounding) class; each class has its own stream
// so the classes' launches overlap on the device.
struct ClassBatch {
    BatchCore core;
    cudaStream_t st = nullptr;
    std::vector<Request*> running;       // parallel to core.shots
    bool changed = false;
};

static void server_loop(bp_server* s) {
    cudaSetDevice(s->device);
    std::map<int, std::unique_ptr<ClassBatch>> classes;
    auto klass = [](const bp_config& c) { return c.rounding * 1000 + c.dim * 100 + c.order * 10 + c.precision; };
    for (;;) {
        std::vector<Request*> admit;
        size_t nrun = 0;
        for (auto& kv : classes) nrun += kv.second->running.size();
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
            for (auto it = s->pending.begin(); it != s->pending.end();) {
                Request* r = s->reqs[*it].get();
                if (r->cancel) {
                    r->state = BP_REQ_CANCELLED;
                    r->t_done = Clock::now();
                    s->cancelled++;
                    it = s->pending.erase(it);
                    s->cv_done.notify_all();
                    continue;
                }
                if (s->in_use + r->bytes <= s->budget) {   // first fit in arrival order
                    s->in_use += r->bytes;
                    r->state = BP_REQ_RUNNING;
                    admit.push_back(r);
                    it = s->pending.erase(it);
                } else {
                    ++it;
                }
            }
            if (admit.empty() && nrun == 0) {
                s->cv.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
        }
        for (Request* r : admit) {
            const int key = klass(r->cfg);
            auto& cb = classes[key];
            if (!cb) {
                cb = std::make_unique<ClassBatch>();
                cudaStreamCreateWithFlags(&cb->st, cudaStreamNonBlocking);
                cb->core.init(s->device, cb->st);
                cb->core.dim = r->cfg.dim; cb->core.order = r->cfg.order; cb->core.prec = r->cfg.precision;
                cb->core.rounding = r->cfg.rounding;
                cb->core.steps_per_sync = s->sps;
            }
            const size_t n = r->medium.size() / 9;
            const float* p = r->medium.data();
            bp_medium m{p, p + n, p + 2 * n, p + 3 * n, p + 4 * n, p + 5 * n, p + 6 * n, p + 7 * n, p + 8 * n};
            auto sh = std::make_unique<Shot>();
            int rc = sh->create(&r->cfg, &m, cb->st);
            std::lock_guard<std::mutex> g(s->mu);
            if (rc) {
                sh->destroy();
                r->state = BP_REQ_FAILED;
                r->err = "shot creation failed";
                r->t_done = Clock::now();
                s->in_use -= r->bytes;
                s->failed++;
                s->cv_done.notify_all();
                continue;
            }
            r->medium.clear();
            r->medium.shrink_to_fit();
            r->shot = sh.get();
            cb->core.shots.push_back(std::move(sh));
            cb->running.push_back(r);
            cb->changed = true;
            s->admitted++;
        }
        nrun = 0;
        for (auto& kv : classes) nrun += kv.second->running.size();
        if (nrun == 0) continue;
        s->max_resident = std::max(s->max_resident, (int)nrun);
        const auto t0 = Clock::now();
        long long before = 0;
        bool err = false;
        for (auto& kv : classes) {
            ClassBatch& cb = *kv.second;
            before += cb.core.cell_updates;
            if (cb.running.empty()) continue;
            if (cb.changed) {
                if (cb.core.rebuild()) { err = true; break; }
                cb.changed = false;
            }
            if (cb.core.advance(s->sps)) { err = true; break; }
        }
        for (auto& kv : classes)
            if (cudaStreamSynchronize(kv.second->st) != cudaSuccess) err = true;
        const auto t1 = Clock::now();
        if (err) { s->worker_error = BP_ERR_CUDA; break; }
        long long after = 0;
        for (auto& kv : classes) after += kv.second->core.cell_updates;
        // retire finished or cancelled shots of every class
        for (auto& kv : classes) {
            ClassBatch& cb = *kv.second;
            std::vector<Request*> keep;
            std::vector<std::unique_ptr<Shot>> keep_shots;
            for (size_t i = 0; i < cb.running.size(); i++) {
                Request* r = cb.running[i];
                Shot* sh = cb.core.shots[i].get();
                bool cancel;
                {
                    std::lock_guard<std::mutex> g(s->mu);
                    cancel = r->cancel;
                }
                // a shot whose recorded values went non-finite is retired at
                // once as failed instead of running to its last step
                const int bad = sh->blowup_step(cb.st);
                if (sh->it_host < sh->cfg.nt && !cancel && !bad) {
                    keep.push_back(r);
                    keep_shots.push_back(std::move(cb.core.shots[i]));
                    continue;
                }
                std::vector<float> tr;
                if (!cancel && !bad) {
                    const size_t nt = sh->cfg.nt, nr = sh->cfg.nrec;
                    std::vector<float> u((size_t)BP_NTRACE * sh->nurec * nt);
                    if (!u.empty()) cudaMemcpy(u.data(), sh->desc.traces, u.size() * 4, cudaMemcpyDeviceToHost);
                    tr.resize((size_t)BP_NTRACE * nr * nt);
                    for (int c = 0; c < BP_NTRACE; c++)
                        for (size_t q = 0; q < nr; q++)
                            std::memcpy(tr.data() + ((size_t)c * nr + q) * nt,
                                        u.data() + ((size_t)c * sh->nurec + sh->urec_of[q]) * nt, nt * 4);
                }
                sh->destroy();
                cb.changed = true;
                std::lock_guard<std::mutex> g(s->mu);
                r->shot = nullptr;
                r->traces.swap(tr);
                r->t_done = Clock::now();
                r->state = cancel ? BP_REQ_CANCELLED : (bad ? BP_REQ_FAILED : BP_REQ_DONE);
                if (cancel) s->cancelled++;
                else if (bad) {
                    r->err = "non-finite value recorded at a receiver at step " + std::to_string(bad - 1);
                    s->failed++;
                } else {
                    s->completed++;
                    s->latencies.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
                }
                s->in_use -= r->bytes;
                s->cv_done.notify_all();
            }
            cb.core.shots.swap(keep_shots);
            cb.running.swap(keep);
        }
        {
            std::lock_guard<std::mutex> g(s->mu);
            s->busy += std::chrono::duration<double>(t1 - t0).count();
            s->cell_updates += after - before;
        }
    }
    // shutdown: drop resident shots and queued requests
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (auto& kv : classes)
            for (Request* r : kv.second->running) { r->state = BP_REQ_CANCELLED; r->shot = nullptr; }
        for (uint64_t id : s->pending) s->reqs[id]->state = BP_REQ_CANCELLED;
        s->pending.clear();
        s->cv_done.notify_all();
    }
    for (auto& kv : classes) {
        kv.second->core.release();
        cudaStreamDestroy(kv.second->st);
    }
}

extern "C" {

int bp_shot_bytes(const bp_config* cfg, size_t* bytes) {
    if (!bytes) { set_error("bad arguments"); return BP_ERR_ARG; }
    return Shot::plan_bytes(cfg, bytes);
}

int bp_server_create(int device, size_t hbm_budget, int steps_per_sync, bp_server** out) {
    if (!out || hbm_budget == 0 || steps_per_sync < 0) { set_error("bad arguments"); return BP_ERR_ARG; }
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        set_error("no such CUDA device");
        return BP_ERR_NO_DEVICE;
    }
    bp_server* s = new bp_server();
    s->device = device;
    s->budget = hbm_budget;
    s->sps = steps_per_sync > 0 ? steps_per_sync : 100;
    s->worker = std::thread(server_loop, s);
    *out = s;
    return BP_OK;
}

int bp_server_submit(bp_server* s, const bp_config* cfg, const bp_medium* medium, uint64_t* request_id) {
    if (!s || !cfg || !medium || !request_id) { set_error("bad arguments"); return BP_ERR_ARG; }
    size_t bytes = 0;
    int rc = Shot::plan_bytes(cfg, &bytes);
    if (rc) return rc;
    if (bytes > s->budget) { set_error("request needs more device memory than the budget"); return BP_ERR_BUDGET; }
    if (!medium->rho || !medium->rhof || !medium->M || !medium->C || !medium->H || !medium->H2mu || !medium->mu ||
        !medium->C1 || !medium->C2) {
        set_error("medium arrays missing");
        return BP_ERR_ARG;
    }
    auto r = std::make_unique<Request>();
    r->cfg = *cfg;
    r->rx.assign(cfg->rec_x, cfg->rec_x + cfg->nrec);
    r->rz.assign(cfg->rec_z, cfg->rec_z + cfg->nrec);
    if (cfg->dim == 3) r->ry.assign(cfg->rec_y, cfg->rec_y + cfg->nrec);
    else r->ry.assign(cfg->nrec, 0);
    r->cfg.rec_x = r->rx.data(); r->cfg.rec_y = r->ry.data(); r->cfg.rec_z = r->rz.data();
    r->cfg.nsnap = 0; r->cfg.snap_steps = nullptr; r->cfg.snap_masks = nullptr;
    const size_t n = (size_t)cfg->nx * (cfg->dim == 3 ? cfg->ny : 1) * cfg->nz;
    r->medium.resize(9 * n);
    const float* src[9] = {medium->rho, medium->rhof, medium->M, medium->C, medium->H, medium->H2mu, medium->mu,
                           medium->C1, medium->C2};
    for (int k = 0; k < 9; k++) std::memcpy(r->medium.data() + k * n, src[k], n * 4);
    r->bytes = bytes;
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) { set_error("server stopping"); return BP_ERR_STATE; }
    r->id = s->next_id++;
    *request_id = r->id;
    s->pending.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    s->submitted++;
    s->cv.notify_all();
    return BP_OK;
}

int bp_server_poll(bp_server* s, uint64_t id, int* state) {
    if (!s || !state) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request"); return BP_ERR_NOT_FOUND; }
    *state = it->second->state;
    return s->worker_error ? s->worker_error : BP_OK;
}

int bp_server_wait(bp_server* s, uint64_t id, double timeout_s) {
    if (!s) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request"); return BP_ERR_NOT_FOUND; }
    Request* r = it->second.get();
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    while (r->state == BP_REQ_QUEUED || r->state == BP_REQ_RUNNING) {
        if (s->worker_error) return s->worker_error;
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
            (r->state == BP_REQ_QUEUED || r->state == BP_REQ_RUNNING)) {
            set_error("request still running");
            return BP_ERR_TIMEOUT;
        }
    }
    return BP_OK;
}

int bp_server_cancel(bp_server* s, uint64_t id) {
    if (!s) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request"); return BP_ERR_NOT_FOUND; }
    it->second->cancel = true;
    s->cv.notify_all();
    return BP_OK;
}

int bp_server_get_traces(bp_server* s, uint64_t id, int comp, float* host, size_t n) {
    if (!s || !host || comp < 0 || comp >= BP_NTRACE) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request"); return BP_ERR_NOT_FOUND; }
    Request* r = it->second.get();
    if (r->state != BP_REQ_DONE) { set_error("request not finished"); return BP_ERR_STATE; }
    const size_t cs = (size_t)r->cfg.nrec * r->cfg.nt;
    if (n < cs) { set_error("host buffer too small"); return BP_ERR_ARG; }
    std::memcpy(host, r->traces.data() + comp * cs, cs * 4);
    return BP_OK;
}

int bp_server_release(bp_server* s, uint64_t id) {
    if (!s) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request"); return BP_ERR_NOT_FOUND; }
    int st = it->second->state;
    if (st == BP_REQ_QUEUED || st == BP_REQ_RUNNING) { set_error("request still active"); return BP_ERR_STATE; }
    s->reqs.erase(it);
    return BP_OK;
}

int bp_server_latency(bp_server* s, uint64_t id, double* seconds) {
    if (!s || !seconds) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request"); return BP_ERR_NOT_FOUND; }
    Request* r = it->second.get();
    if (r->state != BP_REQ_DONE) { set_error("request not finished"); return BP_ERR_STATE; }
    *seconds = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    return BP_OK;
}

int bp_server_get_stats(bp_server* s, bp_server_stats* st) {
    if (!s || !st) { set_error("bad arguments"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(s->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = s->submitted; st->admitted = s->admitted; st->completed = s->completed;
    st->failed = s->failed; st->cancelled = s->cancelled; st->cell_updates = s->cell_updates;
    st->busy_seconds = s->busy; st->hbm_in_use = s->in_use; st->hbm_budget = s->budget;
    st->max_resident = s->max_resident;
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
        if (l.empty()) return 0.0;
        size_t i = (size_t)std::min<double>((double)l.size() - 1, std::ceil(p * l.size()) - 1);
        return l[i];
    };
    st->p50_latency_s = pct(0.50);
    st->p99_latency_s = pct(0.99);
    return s->worker_error ? s->worker_error : BP_OK;
}

void bp_server_destroy(bp_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    delete s;
}

}  // extern "C"

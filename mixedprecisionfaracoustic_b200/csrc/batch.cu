// batch.cu - batched shots (bp_batch): many shots with their own sizes,
// media, sources and receivers advanced by the same persistent launches and
// CUDA-graph replays, with an online autotuner for the persistent grid size
// (CTAs per SM) and the number of steps captured per graph (steps per sync).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "batch.h"

namespace bpk {

std::map<TuneKey, TuneVal>& tune_cache() {
    static std::map<TuneKey, TuneVal> m;
    return m;
}
static std::mutex g_tune_mu;

int BatchCore::init(int device_, cudaStream_t s) {
    device = device_;
    st = s;
    return BP_OK;
}

long long BatchCore::total_cells() const {
    long long c = 0;
    for (auto& s : shots) c += s->cells;
    return c;
}

int BatchCore::rebuild() {
    const int n = (int)shots.size();
    if (n > d_cap) {
        // descriptor blocks come from the arena cache (no cudaMalloc/cudaFree
        // per batch); the old one goes back once no launch can still read it
        if (d_descs) {
            if (st) cudaStreamSynchronize(st);
            arena_release(d_descs, d_bytes);
        }
        d_descs = nullptr;
        d_cap = std::max(n, 2 * d_cap);
        cudaError_t e = arena_alloc((size_t)d_cap * sizeof(ShotDesc), (void**)&d_descs, &d_bytes);
        if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); d_descs = nullptr; d_cap = 0; return BP_ERR_OOM; }
    }
    std::vector<ShotDesc> h(n);
    long long t0 = 0;
    int maxrec = 0;
    long long t0s = 0, t0m = 0;
    for (int i = 0; i < n; i++) {
        h[i] = shots[i]->desc;
        h[i].tile0 = t0;
        h[i].tile0s = t0s;
        h[i].tile0m = t0m;
        h[i].done = 0;
        t0 += shots[i]->ntiles;
        t0s += shots[i]->ntiles_s;
        t0m += shots[i]->ntiles_m;
        maxrec = std::max(maxrec, shots[i]->nurec);
    }
    if (n > 0) {
        cudaError_t e = cudaMemcpyAsync(d_descs, h.data(), n * sizeof(ShotDesc), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // h is a local buffer
        if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    }
    run.post_in_t = true;
    for (auto& sh : shots) run.post_in_t = run.post_in_t && sh->post_in_t;
    run.configure(prec, dim, order, d_descs, n, t0, t0s, t0m, maxrec, st, ctas_per_sm,
                  steps_per_sync > 0 ? steps_per_sync : 32);
    return BP_OK;
}

int BatchCore::advance(int n) {
    if (shots.empty() || n <= 0) return BP_OK;
    int remain = 0;
    for (auto& s : shots) remain = std::max(remain, s->cfg.nt - s->it_host);
    const int m = std::min(n, remain);
    if (m <= 0) return BP_OK;
    cudaError_t e = run.run(m);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    for (auto& s : shots) {
        const int took = std::min(m, s->cfg.nt - s->it_host);
        if (took > 0) cell_updates += (long long)took * s->cells;
        s->it_host += std::max(took, 0);
    }
    return BP_OK;
}

int BatchCore::autotune(int budget_steps) {
    if (shots.empty()) return BP_OK;
    long long cells = total_cells();
    TuneKey key{dim, order, prec, (int)std::floor(std::log2((double)std::max(cells, 1LL)))};
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            if (ctas_per_sm == 0) ctas_per_sm = it->second.ctas_per_sm;
            if (steps_per_sync == 0) steps_per_sync = it->second.steps_per_sync;
            tuned = true;
            return rebuild();
        }
    }
    const int occ = std::min(phase_occupancy(prec, dim, order, true), phase_occupancy(prec, dim, order, false));
    std::vector<int> ctas = {0};
    if (occ >= 2) ctas.push_back(occ / 2 > 0 ? occ / 2 : 1);
    if (occ >= 3) ctas.push_back(1);
    std::vector<int> spss = {8, 32, 128};
    if (ctas_per_sm > 0) ctas = {ctas_per_sm};
    if (steps_per_sync > 0) spss = {steps_per_sync};
    int min_left = 1 << 30;
    for (auto& s : shots) min_left = std::min(min_left, s->cfg.nt - s->it_host);
    const int fixed_c = ctas_per_sm, fixed_s = steps_per_sync;
    double best = 1e30;
    TuneVal bv{fixed_c, fixed_s > 0 ? fixed_s : 32};
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int used = 0;
    for (int c : ctas) {
        for (int sps : spss) {
            const int steps = std::max(sps, 16);
            if (used + 2 * steps > std::min(budget_steps, min_left)) continue;
            ctas_per_sm = c;
            steps_per_sync = sps;
            int rc = rebuild();
            if (rc) { cudaEventDestroy(a); cudaEventDestroy(b); return rc; }
            advance(sps);                          // warm: captures the graph
            cudaEventRecord(a, st);
            rc = advance(steps);
            cudaEventRecord(b, st);
            cudaEventSynchronize(b);
            used += sps + steps;
            if (rc) { cudaEventDestroy(a); cudaEventDestroy(b); return rc; }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            const double per = ms / steps;
            if (per < best) { best = per; bv = TuneVal{c, sps}; }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctas_per_sm = bv.ctas_per_sm;
    steps_per_sync = bv.steps_per_sync;
    tuned = true;
    if (best < 1e30) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_cache()[key] = bv;
    }
    return rebuild();
}

void BatchCore::release() {
    if (st) cudaStreamSynchronize(st);
    run.reset_graph();
    for (auto& s : shots) s->destroy();
    shots.clear();
    if (d_descs) arena_release(d_descs, d_bytes);
    d_descs = nullptr;
    d_cap = 0;
}

}  // namespace bpk

using namespace bpk;

struct bp_batch {
    BatchCore core;
    cudaStream_t st = nullptr;
    bool user_tuned = false;
};

extern "C" {

int bp_batch_create(const bp_config* cfgs, const bp_medium* media, int nshots, const bp_tune* tune, bp_batch** out) {
    if (!cfgs || !media || nshots < 1 || !out) { set_error("bad arguments"); return BP_ERR_ARG; }
    *out = nullptr;
    for (int i = 0; i < nshots; i++) {
        int rc = validate_config(&cfgs[i]);
        if (rc) return rc;
        if (cfgs[i].dim != cfgs[0].dim || cfgs[i].order != cfgs[0].order || cfgs[i].precision != cfgs[0].precision ||
            cfgs[i].device != cfgs[0].device) {
            set_error("all shots of a batch share dim, order, precision and device");
            return BP_ERR_ARG;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfgs[0].device) {
        cudaGetLastError();
        set_error("no CUDA device");
        return BP_ERR_NO_DEVICE;
    }
    cudaSetDevice(cfgs[0].device);
    bp_batch* b = new bp_batch();
    cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    b->core.init(cfgs[0].device, b->st);
    b->core.dim = cfgs[0].dim;
    b->core.order = cfgs[0].order;
    b->core.prec = cfgs[0].precision;
    if (tune) {
        b->core.ctas_per_sm = tune->ctas_per_sm;
        b->core.steps_per_sync = tune->steps_per_sync;
        b->user_tuned = tune->ctas_per_sm > 0 && tune->steps_per_sync > 0;
    }
    for (int i = 0; i < nshots; i++) {
        auto sh = std::make_unique<Shot>();
        bp_config c = cfgs[i];
        c.nsnap = 0;   // batched shots record traces only
        int rc = sh->create(&c, &media[i], b->st);
        if (rc) {
            sh->destroy();
            b->core.release();
            cudaStreamDestroy(b->st);
            delete b;
            return rc;
        }
        b->core.shots.push_back(std::move(sh));
    }
    int rc = b->core.rebuild();
    if (rc) { b->core.release(); cudaStreamDestroy(b->st); delete b; return rc; }
    b->core.tuned = b->user_tuned;
    *out = b;
    return BP_OK;
}

int bp_batch_run(bp_batch* b, int nsteps) {
    if (!b || nsteps < 0) { set_error("bad arguments"); return BP_ERR_ARG; }
    cudaSetDevice(b->core.device);
    if (!b->core.tuned) {
        const int before = (int)(b->core.cell_updates / std::max(1LL, b->core.total_cells()));
        int rc = b->core.autotune(nsteps);
        if (rc) return rc;
        const int used = (int)(b->core.cell_updates / std::max(1LL, b->core.total_cells())) - before;
        nsteps -= std::min(nsteps, std::max(used, 0));
    }
    return b->core.advance(nsteps);
}

int bp_batch_sync(bp_batch* b) {
    if (!b) { set_error("null batch"); return BP_ERR_ARG; }
    cudaError_t e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    for (size_t i = 0; i < b->core.shots.size(); i++) {
        const int bad = b->core.shots[i]->blowup_step(b->st);
        if (bad) {
            set_error("shot " + std::to_string(i) + ": non-finite value recorded at a receiver at step " +
                      std::to_string(bad - 1));
            return BP_ERR_UNSTABLE;
        }
    }
    return BP_OK;
}

int bp_batch_get_traces(bp_batch* b, int shot, int comp, float* host, size_t n) {
    if (!b || !host || shot < 0 || shot >= (int)b->core.shots.size() || comp < 0 || comp >= BP_NTRACE) {
        set_error("bad arguments");
        return BP_ERR_ARG;
    }
    Shot& sh = *b->core.shots[shot];
    const size_t nt = sh.cfg.nt, nr = sh.cfg.nrec;
    if (n < nr * nt) { set_error("host buffer too small"); return BP_ERR_ARG; }
    cudaError_t e = cudaStreamSynchronize(b->st);
    if (e == cudaSuccess) e = sh.copy_traces(comp, host);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    return BP_OK;
}

int bp_batch_get_tune(bp_batch* b, bp_tune* chosen) {
    if (!b || !chosen) { set_error("bad arguments"); return BP_ERR_ARG; }
    memset(chosen, 0, sizeof(*chosen));
    chosen->tile_rows = tile_rows();
    chosen->steps_per_sync = b->core.steps_per_sync;
    chosen->ctas_per_sm = b->core.ctas_per_sm;
    return BP_OK;
}

int bp_batch_cell_updates(bp_batch* b, long long* updates) {
    if (!b || !updates) { set_error("bad arguments"); return BP_ERR_ARG; }
    *updates = b->core.cell_updates;
    return BP_OK;
}

void bp_batch_destroy(bp_batch* b) {
    if (!b) return;
    cudaSetDevice(b->core.device);
    b->core.release();
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

}  // extern "C"

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
    long long t0s = 0, t0m = 0, t0f = 0, t0i = 0;
    int nbands = 0, dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ctas_i = inter_occupancy(prec, dim, order, rounding) * sms;
    bool all_fused = true;
    const TileShape ts = effective_shape();
    for (int i = 0; i < n; i++) {
        h[i] = shots[i]->desc;
        const long long tiles = apply_tile_shape(h[i], dim, prec, ts);
        h[i].tile0 = t0;
        h[i].tile0s = t0s;
        h[i].tile0m = t0m;
        h[i].tile0f = t0f;
        h[i].item0_i = t0i;
        h[i].band0_i = nbands;
        t0i += apply_bands(h[i], dim, tiles, ctas_i);
        nbands += h[i].nbands_i;
        h[i].done = 0;
        t0f += shots[i]->ntiles_f;
        all_fused = all_fused && shots[i]->ntiles_f > 0;
        t0 += tiles;
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
    run.rounding = rounding;
    run.ntiles_f = all_fused ? t0f : 0;
    run.nitems_i = t0i;
    run.nbands_i = nbands;
    run.variant = kernel;
    run.multi_unit = ts.rows * ts.segs > phase_threads() / 32;
    run.indexed = false;
    for (int i = 0; i < n; i++) run.indexed = run.indexed || shots[i]->med_tuples > 0;
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

TileShape BatchCore::effective_shape() const {
    return shape.rows > 0 ? shape : default_tile_shape(dim, prec);
}

// Tile shapes the autotuner tries (the default first).  2D: rows x segments;
// 3D also the split of the rows into y rows x z planes.
static std::vector<TileShape> shape_candidates(int dim, int prec) {
    std::vector<TileShape> c = {default_tile_shape(dim, prec)};
    auto add = [&](int rows, int segs, int tz) {
        TileShape t{rows, segs, tz};
        for (auto& o : c)
            if (o.rows == t.rows && o.segs == t.segs && (dim == 2 || o.tz == t.tz)) return;
        c.push_back(t);
    };
    if (dim == 2) {
        add(4, 2, 1); add(16, 1, 1); add(8, 2, 1); add(4, 1, 1);
    } else {
        add(8, 1, 1); add(8, 1, 2); add(8, 1, 4); add(8, 1, 8); add(16, 1, 4); add(16, 1, 8); add(4, 2, 2);
    }
    return c;
}

int BatchCore::autotune(int budget_steps) {
    if (shots.empty()) return BP_OK;
    long long cells = total_cells();
    TuneKey key{dim, order, prec + 16 * rounding, (int)std::floor(std::log2((double)std::max(cells, 1LL))),
                (int)std::floor(std::log2((double)shots.size()))};
    const bool fix_shape = shape.rows > 0, fix_c = ctas_per_sm > 0, fix_s = steps_per_sync > 0;
    const bool fix_k = kernel != BP_KERNEL_AUTO;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            if (!fix_c) ctas_per_sm = it->second.ctas_per_sm;
            if (!fix_s) steps_per_sync = it->second.steps_per_sync;
            if (!fix_shape) shape = it->second.shape;
            if (!fix_k) kernel = it->second.kernel;
            tuned = true;
            return rebuild();
        }
    }
    int min_left = 1 << 30;
    for (auto& s : shots) min_left = std::min(min_left, s->cfg.nt - s->it_host);
    const int budget = std::min(budget_steps, min_left);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int used = 0;
    double best = 1e30;
    TuneVal bv{ctas_per_sm, fix_s ? steps_per_sync : 32, effective_shape(), fix_k ? kernel : BP_KERNEL_REGISTER};
    // times one candidate; false if it no longer fits the step budget
    auto trial = [&](int c, int sps, TileShape ts, int kern, int* rc) -> bool {
        const int steps = std::max(sps, 16);
        if (used + sps + steps > budget) return false;
        ctas_per_sm = c;
        steps_per_sync = sps;
        shape = ts;
        kernel = kern;
        *rc = rebuild();
        if (*rc) return false;
        advance(sps);                          // warm: captures the graph
        cudaEventRecord(a, st);
        *rc = advance(steps);
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        used += sps + steps;
        if (*rc) return false;
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        const double per = ms / steps;
        if (per < best) { best = per; bv = TuneVal{c, sps, ts, kern}; }
        return true;
    };
    int rc = BP_OK;
    // stage 0: kernel family at the default tile shape: register tiles,
    // interleaved step, and (2D) the fused step kernel
    bool can_fused = fused_supported(prec, dim) && rounding == BP_ROUND_FAST;
    for (auto& s : shots) can_fused = can_fused && s->ntiles_f > 0;
    if (!fix_k) {
        const TuneVal base = bv;
        for (int kern : {BP_KERNEL_REGISTER, BP_KERNEL_INTERLEAVED, BP_KERNEL_FUSED}) {
            if (kern == BP_KERNEL_FUSED && !can_fused) continue;
            if (!trial(base.ctas_per_sm, base.steps_per_sync, base.shape, kern, &rc) && rc) break;
        }
    }
    // stage 1: tile shape of the register kernels (at the current CTA count and 32 steps per sync)
    if (!rc && !fix_shape && bv.kernel == BP_KERNEL_REGISTER)
        for (const TileShape& ts : shape_candidates(dim, prec))
            if (!(best < 1e30 && ts.rows == bv.shape.rows && ts.segs == bv.shape.segs && ts.tz == bv.shape.tz))
                if (!trial(bv.ctas_per_sm, bv.steps_per_sync, ts, bv.kernel, &rc) && rc) break;
    // stage 2: persistent CTAs per SM (register tiles)
    if (!rc && !fix_c && bv.kernel == BP_KERNEL_REGISTER) {
        const int occ = std::min(phase_occupancy(prec, dim, order, true, rounding),
                                 phase_occupancy(prec, dim, order, false, rounding));
        std::vector<int> ctas = {0};
        if (occ >= 2) ctas.push_back(occ / 2 > 0 ? occ / 2 : 1);
        if (occ >= 3) ctas.push_back(1);
        const TuneVal base = bv;
        for (int c : ctas)
            if (!(c == base.ctas_per_sm && best < 1e30))
                if (!trial(c, base.steps_per_sync, base.shape, base.kernel, &rc) && rc) break;
    }
    // stage 3: steps per graph replay
    if (!rc && !fix_s) {
        const TuneVal base = bv;
        for (int sps : {8, 32, 128})
            if (sps != base.steps_per_sync || best >= 1e30)
                if (!trial(base.ctas_per_sm, sps, base.shape, base.kernel, &rc) && rc) break;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    ctas_per_sm = bv.ctas_per_sm;
    steps_per_sync = bv.steps_per_sync;
    shape = bv.shape;
    kernel = bv.kernel;
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

int bp_batch_autotune(bp_batch* b, int budget_steps);

int bp_batch_create(const bp_config* cfgs, const bp_medium* media, int nshots, const bp_tune* tune, bp_batch** out) {
    if (!cfgs || !media || nshots < 1 || !out) { set_error("bad arguments"); return BP_ERR_ARG; }
    *out = nullptr;
    for (int i = 0; i < nshots; i++) {
        int rc = validate_config(&cfgs[i]);
        if (rc) return rc;
        if (cfgs[i].dim != cfgs[0].dim || cfgs[i].order != cfgs[0].order || cfgs[i].precision != cfgs[0].precision ||
            cfgs[i].device != cfgs[0].device || cfgs[i].rounding != cfgs[0].rounding) {
            set_error("all shots of a batch share dim, order, precision, rounding and device");
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
    b->core.rounding = cfgs[0].rounding;
    if (tune) {
        if (tune->tile_rows > 0) {
            TileShape t{tune->tile_rows, tune->tile_segs > 0 ? tune->tile_segs : 1, tune->tile_tz};
            if (!valid_tile_shape(cfgs[0].dim, t)) {
                set_error("bad tile shape: rows 4..32, segs 1..4, tz 1..rows, powers of two");
                cudaStreamDestroy(b->st);
                delete b;
                return BP_ERR_ARG;
            }
            b->core.shape = t;
        }
        if (tune->kernel < BP_KERNEL_AUTO || tune->kernel > BP_KERNEL_INTERLEAVED ||
            (tune->kernel == BP_KERNEL_FUSED && !(fused_supported(cfgs[0].precision, cfgs[0].dim) &&
                                                 cfgs[0].rounding == BP_ROUND_FAST))) {
            set_error("bad kernel family for this batch");
            cudaStreamDestroy(b->st);
            delete b;
            return BP_ERR_ARG;
        }
        b->core.kernel = tune->kernel;
        b->core.ctas_per_sm = tune->ctas_per_sm;
        b->core.steps_per_sync = tune->steps_per_sync;
        b->user_tuned = tune->ctas_per_sm > 0 && tune->steps_per_sync > 0 && tune->tile_rows > 0 &&
                        tune->kernel != BP_KERNEL_AUTO;
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

int bp_batch_run_timed(bp_batch* b, int nsteps, float* ms) {
    if (!b || nsteps < 0 || !ms) { set_error("bad arguments"); return BP_ERR_ARG; }
    cudaSetDevice(b->core.device);
    if (!b->core.tuned) {
        int rc = bp_batch_autotune(b, nsteps);
        if (rc) return rc;
    }
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        set_error("cudaEventCreate failed");
        return BP_ERR_CUDA;
    }
    cudaEventRecord(e0, b->st);
    int rc = b->core.advance(nsteps);
    cudaEventRecord(e1, b->st);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    *ms = t;
    return BP_OK;
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
    TileShape t = b->core.effective_shape();
    if (b->core.dim == 3 && t.tz == 0) t.tz = default_tile_shape(3, b->core.prec).tz;
    chosen->tile_rows = t.rows;
    chosen->tile_segs = t.segs;
    chosen->tile_tz = b->core.dim == 3 ? t.tz : 1;
    chosen->steps_per_sync = b->core.steps_per_sync;
    chosen->ctas_per_sm = b->core.ctas_per_sm;
    chosen->kernel = b->core.run.family();
    return BP_OK;
}

int bp_batch_autotune(bp_batch* b, int budget_steps) {
    if (!b || budget_steps < 0) { set_error("bad arguments"); return BP_ERR_ARG; }
    cudaSetDevice(b->core.device);
    if (b->user_tuned) return BP_OK;
    int rc = b->core.autotune(budget_steps);
    if (rc) return rc;
    b->core.tuned = true;
    return BP_OK;
}

int bp_batch_medium_tuples(bp_batch* b, int shot, int* ntuples) {
    if (!b || !ntuples || shot < 0 || shot >= (int)b->core.shots.size()) { set_error("bad arguments"); return BP_ERR_ARG; }
    *ntuples = b->core.shots[shot]->med_tuples;
    return BP_OK;
}

int bp_batch_algorithmic_bytes(bp_batch* b, double* bytes_per_step) {
    if (!b || !bytes_per_step) { set_error("bad arguments"); return BP_ERR_ARG; }
    double sum = 0;
    for (auto& sh : b->core.shots) {
        double bpc[2];
        algorithmic_bpc(sh->cfg, sh->med_tuples > 0, bpc);
        sum += (bpc[0] + bpc[1]) * (double)sh->cells;
    }
    *bytes_per_step = sum;
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

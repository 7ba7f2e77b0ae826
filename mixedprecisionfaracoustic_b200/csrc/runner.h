// runner.h - issues chunks of time steps for a set of shot descriptors, either
// as direct launches or by replaying a captured CUDA graph of S steps.
//
// Kernel families: the register tile kernels (step.cu: a V-phase and a
// T-phase launch per step, every dim and precision), and for 2D FP32/COMP16
// the fused step kernel (step_fused.cu: one launch per step, steps in pairs,
// an odd last step of a chunk by the tile kernels), the marching kernels
// (step_march.cu) and the bulk-copy staged kernels (step_staged.cu).
#pragma once
#include <cstdlib>

#include "shot.h"

namespace bpk {

struct Runner {
    int prec = 0, dim = 2, order = 2;
    const ShotDesc* d_shots = nullptr;
    int nshots = 0;
    long long ntiles = 0, ntiles_s = 0, ntiles_m = 0;
    int max_rec = 0;
    int grid_v = 1, grid_t = 1, grid_s = 1;
    bool staged = false;
    bool march = false;
    cudaStream_t st = nullptr;
    int graph_steps = 0;               // S; 0 disables graphs
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_failed = false;
    long long launches = 0;            // kernels issued (graph replays count their nodes)
    int* d_err = nullptr;              // set by a staged kernel whose bounded wait expired
    size_t d_err_bytes = 0;            // its block (from the arena cache)
    int variant = BP_KERNEL_AUTO;      // BP_KERNEL_*: which phase-kernel family runs
    bool post_in_t = false;            // every shot's receivers and source lie in cells the T phase visits
    int rounding = BP_ROUND_FAST;      // FP32 BP_ROUND_REFERENCE: PolF32R register kernels only
    bool multi_unit = false;           // the shots' tile shape has more units than a CTA has warps
    bool indexed = false;              // some shot reads an indexed medium (not the marching or staged kernels)
    bool graded = false;               // a variable z grid (PolF32G register kernels only)
    long long ntiles_f = 0;            // tasks of the fused step kernel (0: some shot cannot take it)
    int grid_f = 1;
    bool fused = false;
    long long graph_launches = 0;      // kernels one replay of the captured graph runs
    long long nitems_i = 0;            // work items of the interleaved step kernel
    int nbands_i = 0;                  // band counters of all shots
    int grid_i = 1;
    bool inter = false;
    unsigned long long* d_ctl = nullptr;   // its claim counter and band counters (arena cache)
    size_t d_ctl_bytes = 0, d_ctl_used = 0;

    void configure(int prec_, int dim_, int order_, const ShotDesc* d, int n, long long tiles, long long tiles_s,
                   long long tiles_m, int maxrec, cudaStream_t s, int ctas_per_sm, int steps_per_graph) {
        prec = prec_; dim = dim_; order = order_;
        d_shots = d; nshots = n; ntiles = tiles; ntiles_s = tiles_s; ntiles_m = tiles_m; max_rec = maxrec; st = s;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const bool wide = wide_grid();
        int ov = phase_occupancy(prec, dim, order, true, rounding, wide),
            ot = phase_occupancy(prec, dim, order, false, rounding, wide);
        if (ctas_per_sm > 0) { ov = ov < ctas_per_sm ? ov : ctas_per_sm; ot = ot < ctas_per_sm ? ot : ctas_per_sm; }
        long long gv = (long long)ov * sms, gt = (long long)ot * sms;
        grid_v = (int)(gv < tiles ? gv : (tiles > 0 ? tiles : 1));
        grid_t = (int)(gt < tiles ? gt : (tiles > 0 ? tiles : 1));
        grid_s = (int)(sms < tiles_s ? sms : (tiles_s > 0 ? tiles_s : 1));
        if (fused_supported(prec, dim)) grid_f = fused_occupancy(prec, order) * sms;
        grid_i = inter_occupancy(prec, dim, order, rounding) * sms;
        d_ctl_used = 8 + 4 * (size_t)(nbands_i > 0 ? nbands_i : 1);
        if (d_ctl && d_ctl_bytes < d_ctl_used) { arena_release(d_ctl, d_ctl_bytes); d_ctl = nullptr; }
        if (!d_ctl && nbands_i > 0 &&
            arena_alloc(d_ctl_used < 256 ? 256 : d_ctl_used, (void**)&d_ctl, &d_ctl_bytes) != cudaSuccess)
            d_ctl = nullptr;
        if (!d_err) {
            // from the arena cache: a cudaFree, even of 4 bytes, stalled the
            // host for up to 0.6 s when the simulation was destroyed
            if (arena_alloc(256, (void**)&d_err, &d_err_bytes) == cudaSuccess) cudaMemsetAsync(d_err, 0, sizeof(int), st);
            else d_err = nullptr;
        }
        select_kernels();                  // after the allocations it depends on
        graph_steps = steps_per_graph;
        reset_graph();
    }
    void select_kernels() {
        if (graded) { fused = inter = march = staged = false; return; }
        const bool can_f = fused_supported(prec, dim) && ntiles_f > 0 && rounding == BP_ROUND_FAST;
        fused = can_f && (variant == BP_KERNEL_FUSED || (variant == BP_KERNEL_AUTO && fused_default()));
        const bool can_i = nitems_i > 0 && d_ctl && d_err && !multi_unit;
        inter = !fused && can_i && (variant == BP_KERNEL_INTERLEAVED || (variant == BP_KERNEL_AUTO && inter_default()));
        const bool can_m = march_supported(prec, dim) && ntiles_m > 0 && rounding == BP_ROUND_FAST && !indexed;
        march = !fused && !inter && can_m &&
                (variant == BP_KERNEL_MARCH || (variant == BP_KERNEL_AUTO && march_default()));
        const bool can = staged_supported(prec, dim) && ntiles_s > 0 && rounding == BP_ROUND_FAST && !indexed;
        staged = !fused && !inter && !march && can &&
                 (variant == BP_KERNEL_STAGED || (variant == BP_KERNEL_AUTO && staged_default()));
    }
    int family() const {
        return fused ? BP_KERNEL_FUSED : inter ? BP_KERNEL_INTERLEAVED : march ? BP_KERNEL_MARCH
               : staged ? BP_KERNEL_STAGED : BP_KERNEL_REGISTER;
    }
    void reset_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        graph_failed = false;
    }
    ~Runner() {
        reset_graph();
        if (d_err) arena_release(d_err, d_err_bytes);
        if (d_ctl) arena_release(d_ctl, d_ctl_bytes);
    }

    // The register kernels' T phase records the receivers and injects the
    // next source sample itself where every shot allows it (one launch per
    // step fewer); otherwise, and for the other kernel families, k_post does.
    bool fused_post() const {
#ifdef BP_POST_IN_T
        if (!BP_POST_IN_T) return false;
#endif
        return post_in_t && !march && !staged;
    }
    // large 3D FP32 launches take the looser register caps (PolF32W); the
    // grid's occupancy follows the kernels that run
    // (BP_WIDE_CELLS in the environment moves the threshold, for tests)
    bool wide_grid() const {
        static const long long thr = [] {
            const char* e = std::getenv("BP_WIDE_CELLS");
            return e ? std::atoll(e) : kWideCells;
        }();
        return dim == 3 && prec == BP_PREC_FP32 && rounding == BP_ROUND_FAST && !graded && ntiles * 1024 >= thr;
    }
    // launches of one step of the two-phase kernels
    int launches_per_step() const { return fused_post() ? 2 : 3; }
    cudaError_t phase(bool v, int k) {
        if (march) return launch_phase_march(prec, order, v, d_shots, nshots, ntiles_m, k, st);
        if (staged) return launch_phase_staged(prec, order, v, d_shots, nshots, ntiles_s, k, grid_s, d_err, st);
        return launch_phase(prec, dim, order, v, d_shots, nshots, ntiles, k, v ? grid_v : grid_t, st,
                            (!v && fused_post()) ? 1 : 0, rounding, multi_unit, graded, wide_grid());
    }

    // One step (index k of the chunk) of the two-phase kernels, or of the
    // interleaved kernel (its counters zeroed first).
    cudaError_t tile_step(int k, long long* n) {
        if (inter) {
            cudaError_t e = cudaMemsetAsync(d_ctl, 0, d_ctl_used, st);
            if (e == cudaSuccess)
                e = launch_inter(prec, dim, order, rounding, d_shots, nshots, nitems_i, k, fused_post() ? 1 : 0,
                                 grid_i, d_ctl, d_err, st);
            if (e == cudaSuccess && !fused_post()) e = launch_post(prec, d_shots, nshots, max_rec, k, 1, st);
            *n += fused_post() ? 1 : 2;
            return e;
        }
        cudaError_t e = phase(true, k);
        if (e == cudaSuccess) e = phase(false, k);
        if (e == cudaSuccess && !fused_post()) e = launch_post(prec, d_shots, nshots, max_rec, k, 1, st);
        *n += launches_per_step();
        return e;
    }
    // m steps issued directly (k = 0..m-1), then the step bases advance by m.
    // The fused kernel takes the steps in pairs (copy A -> B -> A); an odd last
    // step runs the two-phase kernels on copy A.  *n receives the launches.
    cudaError_t issue(int m, long long* n) {
        cudaError_t e = cudaSuccess;
        *n = 0;
        for (int k = 0; k < m && e == cudaSuccess;) {
            if (fused && k + 1 < m) {
                e = launch_fused(prec, order, d_shots, nshots, ntiles_f, k, 0, grid_f, st);
                if (e == cudaSuccess) e = launch_fused(prec, order, d_shots, nshots, ntiles_f, k + 1, 1, grid_f, st);
                *n += 2;
                k += 2;
            } else {
                e = tile_step(k, n);
                k += 1;
            }
        }
        if (e == cudaSuccess) e = launch_advance(d_shots, nshots, m, st);
        *n += 1;
        return e;
    }
    cudaError_t issue(int m) {
        long long n = 0;
        cudaError_t e = issue(m, &n);
        launches += n;
        return e;
    }
    cudaError_t ensure_graph() {
        if (exec || graph_failed || graph_steps <= 0) return cudaSuccess;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { graph_failed = true; cudaGetLastError(); return cudaSuccess; }
        cudaError_t ei = issue(graph_steps, &graph_launches);
        e = cudaStreamEndCapture(st, &graph);
        if (ei != cudaSuccess || e != cudaSuccess) { graph_failed = true; cudaGetLastError(); graph = nullptr; return cudaSuccess; }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) { graph_failed = true; exec = nullptr; cudaGetLastError(); }
        return cudaSuccess;
    }
    // Runs m steps: full graph replays of S steps, the remainder directly.
    cudaError_t run(int m) {
        cudaError_t e = cudaSuccess;
        if (graph_steps > 0 && m >= graph_steps) {
            ensure_graph();
            while (exec && m >= graph_steps && e == cudaSuccess) {
                e = cudaGraphLaunch(exec, st);
                launches += graph_launches;
                m -= graph_steps;
            }
        }
        if (m > 0 && e == cudaSuccess) e = issue(m);
        return e;
    }
    // BP_OK, or the error a staged kernel recorded (stream must be synchronised).
    int device_error() const {
        if (!d_err) return BP_OK;
        int h = 0;
        if (cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BP_ERR_CUDA;
        return h;
    }
};

}  // namespace bpk

// shot.h - host-side owner of one shot's device state (used by the single-shot
// bp_sim, the batch and the server).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace bpk {

// launchers (step.cu, precompute.cu, reduce.cu)
// post = 1: the T phase also records the receivers and injects the next source
// sample (every receiver and the source lie in cells the T phase visits)
// rounding = BP_ROUND_REFERENCE (FP32): the PolF32R instantiation; multi: the
// tile shape has more (row, segment) units than a CTA has warps
cudaError_t launch_phase(int prec, int dim, int order, bool vphase, const ShotDesc* d_shots, int nshots,
                         long long ntiles, int k, int grid, cudaStream_t st, int post = 0, int rounding = 0,
                         bool multi = false, bool graded = false, bool wide = false);
// updated cells of a launch from which 3D FP32 takes the large-grid register caps (PolF32W)
constexpr long long kWideCells = 16LL << 20;
cudaError_t launch_post(int prec, const ShotDesc* d_shots, int nshots, int max_rec, int k, int do_record,
                        cudaStream_t st);
cudaError_t launch_inject(int prec, const ShotDesc* d_shots, int nshots, int k, cudaStream_t st);
cudaError_t launch_advance(const ShotDesc* d_shots, int nshots, int n, cudaStream_t st);
cudaError_t launch_snapshot(int prec, const ShotDesc* d_shots, int shot, int f, int slice_y, float* out, int it,
                            cudaStream_t st);
cudaError_t launch_field_f64(int prec, const ShotDesc* d_shots, int f, double* out, cudaStream_t st);
cudaError_t launch_coef(int prec, const ShotDesc* d_shots, int which, float* out, cudaStream_t st);
int phase_threads();
// Tile of the register kernels: `rows` rows (z rows in 2D; in 3D rows/tz y
// rows of tz z planes) x `segs` 128-cell segments along x, taken by the 8 warps
// of a CTA one (row, segment) unit at a time.  Powers of two: rows 4..32,
// segs 1..4, tz 1..rows.  Every shape gives the same results.
struct TileShape {
    int rows = 8, segs = 1, tz = 0;    // tz = 0: the precision's default split
};
TileShape default_tile_shape(int dim, int prec);
bool valid_tile_shape(int dim, const TileShape& t);
// Writes the shape into the descriptor and returns the shot's tile count.
long long apply_tile_shape(ShotDesc& S, int dim, int prec, TileShape t);
// Groups the shot's tiles (current shape, ntiles of them) into the bands of
// the interleaved step kernel, for a launch of `ctas` persistent CTAs; returns
// the shot's work items (2 x ntiles).
long long apply_bands(ShotDesc& S, int dim, long long ntiles, int ctas);
// indexed medium (medium_index.cu): *ntuples = 0 leaves the shot on its arrays
size_t medium_scratch_bytes();
void algorithmic_bpc(const bp_config& c, bool indexed, double bpc[2]);   // sim.cu
cudaError_t build_medium_index(int prec, ShotDesc& S, uint8_t* d_idx, float4* d_tab, void* d_scratch, size_t ncell,
                               int* ntuples, cudaStream_t st);
bool inter_default();            // whether BP_KERNEL_AUTO picks the interleaved kernel
int inter_occupancy(int prec, int dim, int order, int rounding);
// one step of the interleaved kernel; ctl: claim counter (8 bytes) and the
// bands' completion counters, zeroed before the launch; err: timeout flag
cudaError_t launch_inter(int prec, int dim, int order, int rounding, const ShotDesc* d, int nshots, long long nitems,
                         int k, int post, int grid, unsigned long long* ctl, int* err, cudaStream_t st);
int seg_cells();
// TMA-staged 2D phase kernels (step_staged.cu)
bool staged_supported(int prec, int dim);
bool staged_default();           // whether BP_KERNEL_AUTO picks the staged kernels where supported
int staged_tile_rows();
int staged_tile_width();
cudaError_t launch_phase_staged(int prec, int order, bool vphase, const ShotDesc* d, int nshots, long long ntiles,
                                int k, int grid, int* err, cudaStream_t st);
int phase_occupancy(int prec, int dim, int order, bool vphase, int rounding = 0, bool wide = false);
// register-window marching 2D phase kernels (step_march.cu)
bool march_supported(int prec, int dim);
bool march_default();            // whether BP_KERNEL_AUTO picks the marching kernels where supported
int march_cells();
int march_zseg(long long ncol, int nrows, int sms);
cudaError_t launch_phase_march(int prec, int order, bool vphase, const ShotDesc* d, int nshots, long long ntasks,
                               int k, cudaStream_t st);
// fused 2D step kernel (step_fused.cu): one launch per step, state copy par -> 1 - par
bool fused_supported(int prec, int dim);
bool fused_default();            // whether BP_KERNEL_AUTO picks the fused kernel where supported
int fused_cols(int nx);
int fused_zseg(long long ncol, int nrows, int sms);
int fused_occupancy(int prec, int order);
cudaError_t launch_fused(int prec, int order, const ShotDesc* d, int nshots, long long ntasks, int k, int par,
                         int grid, cudaStream_t st);

void host_pml_region(int n, int np, float H, int i, bool* left, bool* right);
cudaError_t launch_profile(int prec, int n, int np, float H, double dt, double v0, double rc, void* b, void* e,
                           void* b2, void* e2, cudaStream_t st);
cudaError_t launch_coefs(int prec, const ShotDesc& S, const float* const* med, int pnx, int pny, int pnz, int np,
                         double dt, int em, cudaStream_t st);
int scan_kr_blocks();
cudaError_t launch_scan_kr(int dim, int nx, int ny, int nz, const float* const* med, int pnx, int pny, int pnz,
                           int np, double* partial, double* out, cudaStream_t st);
int reduce_blocks();
cudaError_t launch_energy(int prec, const ShotDesc* d_shots, double* partial, double* out, cudaStream_t st);
cudaError_t launch_rel_l2(const float* x, const float* ref, long long n, double* partial, double* out,
                          cudaStream_t st);

void set_error(const std::string& msg);

// Arena blocks: reused across shots on a device (see shot.cu).
cudaError_t arena_alloc(size_t bytes, void** ptr, size_t* got);
void arena_release(void* ptr, size_t bytes);
void release_cached_arenas(int device);   // -1: every device
void arm_allocation_failure(long long nth);   // bp_debug_fail_allocation

struct Shot {
    bp_config cfg{};
    std::vector<int> rec_x, rec_y, rec_z, snap_steps;
    std::vector<unsigned> snap_masks;
    std::vector<int> urec_of;          // receiver -> unique receiver cell
    int nurec = 0;
    ShotDesc desc{};                   // host copy of the device descriptor
    ShotDesc* d_desc = nullptr;        // device copy (single-shot runs)
    void* arena = nullptr;
    size_t arena_bytes = 0;            // bytes the plan uses
    size_t arena_alloc_bytes = 0;      // size of the block (a reused cached block may be larger)
    int em = 0, es = 0;
    double kmax = 0, rmax = 0;
    std::vector<float> dyn;            // COMP16 state scale per step
    float* d_snap = nullptr;
    size_t snap_n = 0;                 // floats per snapshot field
    std::vector<long long> snap_off;   // [k * 13 + f] offset in d_snap, -1 if not captured
    double* d_scratch = nullptr;       // reductions
    double* d_out = nullptr;           // 4 doubles
    long long cells = 0;               // updated cells per step
    int it_host = 0;                   // steps issued so far
    long long ntiles = 0;              // tiles of the register kernels (current TileShape)
    long long ntiles_s = 0;            // tiles of the TMA-staged 2D kernels (256 x staged_tile_rows)
    long long ntiles_m = 0;            // tasks of the marching 2D kernels (128 cells x zseg_m rows)
    long long ntiles_f = 0;            // tasks of the fused 2D step kernel (120 cells x zseg_f rows), 0 = none
    long long nitems_i = 0;            // work items of the interleaved step kernel (default tile shape)
    int med_tuples = 0;                // indexed medium: distinct coefficient tuples (0 = per-cell arrays)
    bool post_in_t = false;            // receivers and source all in cells the T phase visits

    // The device regions that make up the shot's evolving state, in a fixed
    // order: wavefields (and COMP16 residuals), CPML memory variables of both
    // phases, recorded traces, captured snapshots.  Everything else in the
    // arena is fixed by the configuration and medium.
    std::vector<std::pair<void*, size_t>> state_regions() const;
    // 1 + the first step whose recorded receiver values were not all finite,
    // 0 if none (synchronises st).
    int blowup_step(cudaStream_t st) const;
    // Seismogram component comp of every receiver (receiver order, nrec x nt)
    // into host memory; the caller has synchronised the shot's stream.
    cudaError_t copy_traces(int comp, float* host) const;

    // Computes the arena size for cfg without allocating (admission control).
    static int plan_bytes(const bp_config* cfg, size_t* bytes);
    int create(const bp_config* cfg, const bp_medium* med, cudaStream_t st);
    void destroy();
};

int validate_config(const bp_config* cfg);

}  // namespace bpk

/*
 * biot.h - C ABI of the B200 staggered-grid Biot poroelastic stepper with CPML.
 *
 * The reference (Zhitao-Zhang/MixedPrecisionFarAcoustic) has no library
 * interface: its "API" is the `main()` of Float/main.cu and Half/main.cu, the
 * signatures of its three kernels (Source Float/main.cu:45, FD_V :64, FD_T
 * :194; Half/main.cu:135,156,270) and the 16 text files it writes.  Each entry
 * point below names the part of that program it replaces.
 *
 * Conventions
 *  - All functions return BP_OK (0) or a positive BP_ERR_* code; none calls
 *    exit().  bp_error_string() maps a code to text; bp_last_error() gives the
 *    detail of the most recent failure on the calling thread.
 *  - The library owns all device memory and one CUDA stream per simulation;
 *    the caller owns every host buffer it passes.
 *  - Grid coordinates named "padded" include the CPML cells: a physical grid of
 *    nx cells becomes nx + 2*npml cells, exactly like NX_ext in the reference
 *    (Float/main.cu:305-307).  Arrays are x fastest: idx = x + y*NXe + z*NXe*NYe.
 *  - One bp_sim per host thread.  A bp_server is internally synchronised.
 */
#ifndef BIOT_B200_H
#define BIOT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define BP_OK 0
#define BP_ERR_ARG 1        /* invalid argument or configuration            */
#define BP_ERR_OOM 2        /* device or host allocation failed             */
#define BP_ERR_CUDA 3       /* a CUDA runtime call failed                   */
#define BP_ERR_CFL 4        /* dt violates the stability limit              */
#define BP_ERR_UNSTABLE 5   /* non-finite values detected in the wavefield   */
#define BP_ERR_TIMEOUT 6    /* a bounded wait ran out                       */
#define BP_ERR_STATE 7      /* call not valid in the object's current state */
#define BP_ERR_NOT_FOUND 8  /* unknown request id / snapshot / component    */
#define BP_ERR_NO_DEVICE 9  /* no CUDA device, or the sm_100a code cannot run */
#define BP_ERR_BUDGET 10    /* request can never fit the HBM budget         */

/* ---- enums ------------------------------------------------------------- */
#define BP_PREC_FP32 0      /* fp32 storage and arithmetic (the Float build)  */
#define BP_PREC_COMP16 1    /* fp16 hi + int8 residual storage, fp32 math     */
#define BP_PREC_FP64 2      /* fp64 storage and arithmetic (accuracy reference) */
#define BP_PREC_CBF16 3     /* compensated bf16 storage: bf16 hi + an unsigned 8-bit
                               residual = the top 24 bits of the fp32 word (rounded
                               to nearest even), fp32 arithmetic as BP_PREC_FP32; no
                               exponent scaling or rescale (bf16 has fp32's range) */

/* How the kernels read the medium (bp_config.medium).  AUTO: when the shot's
 * cells hold at most 256 distinct coefficient tuples (layered, blocky and
 * uniform media), each cell keeps a one-byte index into a table of the
 * decoded tuples, read through L1, in place of its 12 (2D) or 17 (3D)
 * per-cell coefficient arrays; the values, and so the results, are
 * bit-identical, and the coefficient traffic falls from 48 B (FP32) or 36 B
 * (COMP16, CBF16) per cell and step to 2 B.  Shots with more tuples, and FP64
 * shots, read the arrays.  DENSE: always the arrays.  No reference
 * counterpart: the reference reads per-cell arrays (Float/main.cu:106-113,
 * 232-250). */
#define BP_MEDIUM_AUTO 0
#define BP_MEDIUM_DENSE 1

/* FP32 rounding (bp_config.rounding).  FAST divides by H with a reciprocal and
 * one residual step (within one ulp of the IEEE quotient) and forms the CPML
 * memory update in float.  REFERENCE rounds both like the reference's Float
 * build (Float/main.cu:115-158,234-285): the IEEE quotient by H, and psi e +
 * b (e prev + d) with one rounding after the float product psi e, as its
 * double-promoted expression gives.  REFERENCE runs the register tile kernels
 * only and applies to FP32 only. */
#define BP_ROUND_FAST 0
#define BP_ROUND_REFERENCE 1

/* wavefield components, in the order used for bp_get_field / snapshots */
#define BP_F_VUX 0
#define BP_F_VUY 1
#define BP_F_VUZ 2
#define BP_F_VWX 3
#define BP_F_VWY 4
#define BP_F_VWZ 5
#define BP_F_P 6            /* pore pressure ("ss" in the reference)        */
#define BP_F_TXX 7
#define BP_F_TYY 8
#define BP_F_TZZ 9
#define BP_F_TXY 10
#define BP_F_TXZ 11
#define BP_F_TYZ 12
#define BP_NFIELDS 13

/* seismogram components, in the order of the reference's sis* files
 * (sisx=txx, sisz=tzz, sisvu=vux, sisvw=vwx, sisp=p; Float/main.cu:1085-1093) */
#define BP_TR_TXX 0
#define BP_TR_TZZ 1
#define BP_TR_VUX 2
#define BP_TR_VWX 3
#define BP_TR_P 4
#define BP_NTRACE 5

/* source injection mask */
#define BP_SRC_TAU 1        /* add I(t) to txx, tyy, tzz (Float/main.cu:52-57) */
#define BP_SRC_P 2          /* add -I(t) to the pore pressure p              */

/* ---- configuration ----------------------------------------------------- */
typedef struct bp_config {
    int dim;              /* 2 (x-z plane) or 3                                  */
    int nx, ny, nz;       /* physical cells per axis; ny ignored when dim == 2   */
    int npml;             /* CPML width in cells on every face (NP)              */
    int order;            /* spatial order of the staggered stencil: 2 or 4       */
    int precision;        /* BP_PREC_*                                           */
    int nt;               /* time steps the trace buffer holds (NT)              */
    float dx;             /* grid spacing H in metres                            */
    float dt;             /* time step DT in seconds                             */
    float f0;             /* Ricker peak frequency F0 in Hz                      */
    float t0;             /* Ricker delay in s; <= 0 selects 1.2/F0              */
    float pml_v0;         /* CPML reference velocity (4000 in the reference)     */
    float pml_r;          /* CPML target reflection (1e-6 in the reference)      */
    int src_x, src_y, src_z;  /* source cell, padded coordinates                 */
    int src_mask;         /* BP_SRC_* bits                                       */
    int nrec;             /* number of receivers                                 */
    const int* rec_x;     /* receiver cells, padded coordinates (nrec each)      */
    const int* rec_y;     /* ignored when dim == 2                               */
    const int* rec_z;
    int nsnap;            /* number of snapshot steps                            */
    const int* snap_steps;/* step indices `it` after which a snapshot is kept     */
    unsigned snap_fields; /* bitmask of (1u << BP_F_*) captured at every snapshot */
    const unsigned* snap_masks; /* optional per-snapshot masks (nsnap); overrides snap_fields */
    int snap_y;           /* 3D: y index of the stored x-z slice (-1: full volume) */
    int device;           /* CUDA device ordinal                                 */
    int comp_coef_lo;     /* COMP16: 1 = coefficients keep an int8 residual too   */
    int dyn_scale;        /* COMP16: 1 = ramp the state scale 1 -> 16 (Half/main.cu:116-122) */
    int check_cfl;        /* 1 = refuse dt above the stability limit (BP_ERR_CFL) */
    int rounding;         /* FP32: BP_ROUND_FAST (0) or BP_ROUND_REFERENCE (1)   */
    int medium;           /* BP_MEDIUM_AUTO (0) or BP_MEDIUM_DENSE (1), below    */
    int reserved[2];
} bp_config;

/* Cell-centred Biot coefficients over the PHYSICAL grid (nz*ny*nx floats each,
 * x fastest; ny = 1 in 2D).  These are exactly the arrays the reference's
 * create_model() produces (Float/main.cu:1590-1655): bulk density rho, fluid
 * density rhof, Biot moduli M, C, H, H-2mu, shear modulus mu, friction
 * C1 = eta/kappa and mass coupling C2.  The library pads them into the CPML
 * (extmodel, Float/main.cu:1662-1794) and forms the staggered averages and
 * inverses on the GPU in FP64 (Float/main.cu:472-513). */
typedef struct bp_medium {
    const float* rho;
    const float* rhof;
    const float* M;
    const float* C;
    const float* H;
    const float* H2mu;
    const float* mu;
    const float* C1;
    const float* C2;
} bp_medium;

typedef struct bp_sim bp_sim;

/* ---- single shot ------------------------------------------------------- */

/* Replaces main() setup, Float/main.cu:300-1040 (medium padding, staggered
 * averaging, CPML profiles, 93 cudaMalloc + H2D copies) and, for COMP16, the
 * exponent-scaling precompute of Half/main.cu:745-1045.  Copies the medium to
 * the device, runs the FP64 precompute kernels and leaves the state at it=0.
 * The padded grid (row pitch x ny x nz, the pitch being nx + 2 npml rounded up
 * to 32) must hold fewer than 2^31 cells, else BP_ERR_ARG: the kernels address
 * cells with 32-bit offsets.  (At FP32 or FP64 a larger grid would not fit in
 * a B200's memory anyway.) */
int bp_create(const bp_config* cfg, const bp_medium* medium, bp_sim** out);

/* Replaces the time loop body, Float/main.cu:1048-1164: for each of nsteps
 * steps, Source (Float/main.cu:45) -> FD_V (:64) -> FD_T (:194) -> record the
 * five traces (:1085-1093) -> snapshot if `it` is listed (:1094-1163).
 * Asynchronous on the simulation's stream; bp_sync waits. */
int bp_run(bp_sim* sim, int nsteps);
/* Waits for the issued steps.  BP_ERR_UNSTABLE if a recorded receiver value
 * has gone non-finite (the run blew up: dt above the stability limit with
 * check_cfl off, or a broken medium); bp_last_error names the first such step.
 * The same check ends a served request as failed at the next sync point. */
int bp_sync(bp_sim* sim);
/* bp_run bracketed by CUDA events recorded on the simulation's stream; waits
 * and returns the device time of the nsteps steps in *ms. */
int bp_run_timed(bp_sim* sim, int nsteps, float* ms);

/* Steps captured per CUDA graph replay (default 32); 0 issues every step as
 * direct launches. */
int bp_set_graph_steps(bp_sim* sim, int steps);

/* Phase-kernel family: BP_KERNEL_AUTO (the library's choice), BP_KERNEL_REGISTER
 * (register-staged tiles, every dim/precision), BP_KERNEL_STAGED (TMA
 * bulk-copy staged tiles: 2D FP32/COMP16 only, else BP_ERR_ARG) or
 * BP_KERNEL_MARCH (warps marching along z with register windows: 2D
 * FP32/COMP16 only, else BP_ERR_ARG).  All give bit-identical results. */
#define BP_KERNEL_AUTO 0
#define BP_KERNEL_REGISTER 1
#define BP_KERNEL_STAGED 2
#define BP_KERNEL_MARCH 3
#define BP_KERNEL_FUSED 4   /* one launch per step (V, T, record, inject) from one copy
                               of the state into a second one: 2D FP32/COMP16, fast
                               rounding, receivers and source inside the stencil
                               border; steps run in pairs, an odd last step of a
                               bp_run by the register kernels */
#define BP_KERNEL_INTERLEAVED 5 /* one persistent launch per step that interleaves the
                               V and T phases of the register tiles band by band, so
                               the T tiles find the V tiles' data in L2 (every dim
                               and precision; tile shapes of at most 8 units) */
int bp_set_kernel(bp_sim* sim, int variant);
/* The family that runs the steps (BP_KERNEL_REGISTER .. BP_KERNEL_INTERLEAVED). */
int bp_get_kernel(bp_sim* sim, int* variant);

/* Step index of the next step to run (it). */
int bp_get_step(bp_sim* sim, int* it);

/* Seismogram of one component (BP_TR_*): nrec rows of nt floats (row-major,
 * receiver-major), physical units.  n must be >= nrec*nt.  Replaces the
 * sis_* arrays (Float/main.cu:327-338,1085-1093). */
int bp_get_traces(bp_sim* sim, int comp, float* host, size_t n);

/* Snapshot k (index into cfg.snap_steps) of field f (BP_F_*), physical units:
 * the x-z slice at y = snap_y (NZe rows of NXe) or the full padded volume.
 * Replaces txx50..txx300, vux50.. (Float/main.cu:1094-1163). */
int bp_get_snapshot(bp_sim* sim, int k, int field, float* host, size_t n);
/* Elements in one snapshot of this simulation. */
int bp_snapshot_size(bp_sim* sim, size_t* n);

/* Current full padded field f (BP_F_*), in physical units, x fastest.
 * n >= NXe*NYe*NZe.  FP64 simulations are rounded to float. */
int bp_get_field(bp_sim* sim, int field, float* host, size_t n);
/* Same, in double precision (exact for FP64 runs). */
int bp_get_field_f64(bp_sim* sim, int field, double* host, size_t n);

/* Coefficient array `which` as stored on the device, decoded to float over
 * the padded grid (x fastest).  which: 0..9 = V-phase set (rho^-1 x,y,z;
 * rhof; CC1 x,y,z; CC2 x,y,z -- COMP16: 2^-em DT rho^-1 x,y,z; rhof 2^em/DT;
 * Aw x,y,z; Bp x,y,z), 10..16 = T-phase set (C, M, H, H-2mu, mu_xy, mu_xz,
 * mu_yz -- COMP16: times 2^em DT).  Replaces the coefficient dumps the
 * reference keeps commented out (Float/main.cu:514-549). */
int bp_get_coef(bp_sim* sim, int which, float* host, size_t n);

/* Padded extents (NXe, NYe, NZe); NYe = 1 in 2D. */
int bp_get_dims(bp_sim* sim, int* nxe, int* nye, int* nze);

/* Field energy sum over the padded grid of (v_u^2 + v_w^2 + p^2 + tau:tau),
 * physical units, accumulated in FP64 with warp-shuffle reductions. */
int bp_field_energy(bp_sim* sim, double* energy);

/* COMP16 exponent scaling chosen by the precompute (Half/main.cu:745-843):
 * e_m (modulus/inertia exponent), e_s (source exponent) and the fp32 scale
 * the dynamic ramp currently applies (1.0 when off).  Also K_max and R_max. */
int bp_get_scaling(bp_sim* sim, int* em, int* es, float* dyn_scale,
                   double* kmax, double* rmax);

/* Writes the reference program's output files into directory `dir`, in its
 * exact text format (wfile / wfile3d, Float/main.cu:1501-1516,1563-1588):
 * sisx.dat sisz.dat sisvu.dat sisvw.dat sisp.dat (receiver rows x nt steps),
 * one <field><it>.dat per captured snapshot field (e.g. txx500.dat, NZe rows
 * of NXe values of the stored x-z slice) and txx.dat from the current state
 * (Float/main.cu:1187-1222). */
int bp_write_reference_outputs(bp_sim* sim, const char* dir);

/* The same outputs in binary (no counterpart in the reference, whose only
 * format is the text above): traces.bin holds all five components
 * [BP_NTRACE][nrec][nt]; one <field><it>.bin per captured snapshot field
 * ([NZe][NXe] slice or [NZe][NYe][NXe] volume).  Each file is a 32-byte
 * header {char magic[8] = "BPBIN001"; int32 version = 1, dtype = 0 (float32),
 * ndims, dims[3]} followed by the little-endian float32 array, last dimension
 * fastest. */
int bp_write_binary_outputs(bp_sim* sim, const char* dir);

/* Streaming of large receiver sets (no counterpart in the reference): the
 * device keeps one trace per distinct receiver cell; bp_receiver_map gives
 * their count and, if map is not null, the distinct-cell index of each of
 * the nrec receivers.  bp_copy_traces_async enqueues on the simulation's
 * stream, after the steps already issued, the copy of steps [it0, it0 + n)
 * of component comp for every distinct cell into host[nurec][n]; it returns
 * at once (pass page-locked memory for an asynchronous copy) and bp_sync
 * waits for it. */
int bp_receiver_map(bp_sim* sim, int* nurec, int* map);
int bp_copy_traces_async(bp_sim* sim, int comp, int it0, int n, float* host);

/* Checkpoint of the simulation's evolving state (no counterpart in the
 * reference): wavefields, CPML memory variables, traces and snapshots
 * recorded so far, and the step index.  bp_checkpoint_size gives the image
 * size; bp_checkpoint waits for the issued steps and copies the image into
 * host memory; bp_restore loads an image into a simulation created with the
 * same configuration and medium (BP_ERR_ARG otherwise), after which bp_run
 * continues exactly as the checkpointed simulation would have. */
int bp_checkpoint_size(bp_sim* sim, size_t* bytes);
int bp_checkpoint(bp_sim* sim, void* host, size_t bytes);
int bp_restore(bp_sim* sim, const void* host, size_t bytes);

/* Times nsteps steps phase by phase with CUDA events on the simulation's
 * stream and returns the mean device time (ms) of each phase:
 * ms[0] = V phase (velocity + its CPML), ms[1] = T phase (stress, pressure +
 * CPML), ms[2] = record + inject.  The steps are real steps (state advances). */
int bp_profile_phases(bp_sim* sim, int nsteps, float ms[3]);

/* The fused step kernel's mean device time per launch (ms) over nsteps real
 * steps (rounded up to whole pairs), with CUDA events around each launch, and
 * the algorithmic HBM bytes of one fused step per updated cell (every field
 * read once and written once, every coefficient read once).  BP_ERR_ARG where
 * the fused kernel does not apply (3D, FP64, reference rounding). */
int bp_profile_fused(bp_sim* sim, int nsteps, float* ms, double* bytes_per_cell);

/* Algorithmic HBM bytes per updated cell of each phase (the roofline
 * numerator) and the number of updated cells per step.  An indexed medium
 * (BP_MEDIUM_AUTO) counts one index byte per phase for its coefficients. */
int bp_algorithmic_bytes(bp_sim* sim, double bytes_per_cell[2], long long* cells);
/* Variable grid along z (the depth axis).  dz[k], k = 0 .. n-1 with
 * n = nz + 2 npml - 1, is the spacing in metres between padded z rows k and
 * k+1; the z differences of the fields then divide by the local spacing: the
 * forward difference of rows z, z+1 (giving the value at z + 1/2) by dz[z], the
 * backward one of the half rows z - 1/2, z + 1/2 (giving the value at z) by
 * (dz[z-1] + dz[z]) / 2; the x and y spacing stays dx.  No working
 * counterpart in the reference: Float/main.cu:24-25 (NL, m) and :76-89 (h =
 * H/m, h1 = h/m, ..., c1 = 2/(h + H), cc1 = 2/(h + h1), ...) define the
 * constants of such a grid, a spacing that changes by a factor m at a depth,
 * which no computation there uses; this entry point builds that scheme.
 * FP32 with BP_ROUND_FAST at order 2, one shot (not batches or the server),
 * the register tile kernels; the first and last npml + 1 spacings must equal
 * dx (the CPML profiles are the uniform grid's).  Call once, before the first
 * step; with check_cfl, dt is checked against the finest spacing
 * (BP_ERR_CFL).  A checkpoint holds no spacing: set the same one on the
 * simulation it is restored into. */
int bp_set_z_spacing(bp_sim* sim, const double* dz, int n);

/* Distinct coefficient tuples of an indexed medium, 0 where the shot reads
 * the per-cell coefficient arrays (BP_MEDIUM_DENSE, FP64, > 256 tuples). */
int bp_get_medium_tuples(bp_sim* sim, int* ntuples);

/* Kernel launches one step issues (for launch counting): 3 (V phase, T phase,
 * record/inject), or 2 where the T phase records and injects itself. */
int bp_launches_per_step(bp_sim* sim, int* n);
/* Kernel launches this simulation has issued so far (graph replays count
 * every kernel node they contain). */
int bp_launch_count(bp_sim* sim, long long* n);

/* The COMP16 storage codec on the device, over host arrays of n values: the
 * reference's store_ch / load_ch (Half/main.cu:75-100): hi = fp16 RNE(v),
 * lo = int8 residual in units of fp16-ulp(hi)/256 (2^-32 below 2^-14),
 * rounded half away from zero and clamped to +-127; v ~ hi + lo * unit. */
int bp_comp16_encode(const float* host, size_t n, uint16_t* hi, int8_t* lo);
int bp_comp16_decode(const uint16_t* hi, const int8_t* lo, size_t n, float* out);
/* The CBF16 storage codec on the device (BP_PREC_CBF16; no counterpart in the
 * reference, whose compensated format is COMP16's), over host arrays of n <=
 * 2^31 values: the top 24 bits of each fp32 word rounded to nearest even at
 * bit 8 (inf stays inf, a NaN stays a NaN), hi = bits 31..16, lo = bits
 * 15..8; decode: value bits = hi << 16 | lo << 8.  The kernels' own 4-value
 * vector forms, the last n mod 4 values through the scalar ones. */
int bp_cbf16_encode(const float* host, size_t n, uint16_t* hi, uint8_t* lo);
int bp_cbf16_decode(const uint16_t* hi, const uint8_t* lo, size_t n, float* out);

/* Relative L2 difference ||x - ref|| / ||ref|| of two DEVICE float arrays of
 * n elements, accumulated in FP64 with warp-shuffle reductions.  Allocates
 * its reduction scratch on the device for the duration of the call. */
int bp_rel_l2_device(const float* d_x, const float* d_ref, size_t n, double* rel);
/* The same quantity without any device allocation (no counterpart in the
 * reference), for callers that cannot allocate: real-time loops that must not
 * stall on cudaMalloc's implicit synchronisation, and processes that reserve
 * all device memory for their own pool.  The reduction scratch is a fixed 16 KB
 * array in the library's device image, so n is limited to 16,777,216 elements
 * (larger n returns BP_ERR_ARG).  The call is synchronous (legacy default
 * stream, blocking read-back of the result); the inputs must be complete, so
 * synchronise the stream that produces them first.  The first call on a
 * device, with that device current, looks up the array's address; make it
 * before any stream capture begins.  Calls share that array: concurrent calls
 * on one device race and must be serialised. */
int bp_rel_l2_device_noalloc(const float* d_x, const float* d_ref, size_t n, double* rel);
/* Relative L2 seismogram error of component comp of `x` against `ref` (same
 * receivers and nt), computed on the device in FP64. */
int bp_trace_rel_l2(bp_sim* x, bp_sim* ref, int comp, double* rel);

void bp_destroy(bp_sim* sim);

/* Device memory of destroyed simulations, batches and served requests is kept
 * per device for reuse by the next one of a similar size (no counterpart in
 * the reference, which allocates once): a cudaFree of a GB-size block costs
 * 0.4-1 s.  The cache holds at most a quarter of the device's memory (32 GiB
 * at most; environment variable BP_ARENA_CACHE_MB overrides, 0 disables) and
 * is emptied when an allocation fails.  This call returns it to the system
 * for one device, or for all with device = -1. */
int bp_release_cached_memory(int device);

/* Test hook (no counterpart in the reference): the nth device-memory request
 * the library makes from now on (1 = the next one; every arena block, cached
 * or new, counts) fails as if the device were out of memory, so tests can
 * drive the BP_ERR_OOM paths of bp_create, bp_batch_create and the server's
 * admission without exhausting a GPU.  0 disarms.  Process-wide. */
int bp_debug_fail_allocation(int nth);

const char* bp_error_string(int code);
const char* bp_last_error(void);

/* ---- medium builders (host) -------------------------------------------- */

/* The reference's model: a vertical fluid-filled borehole of radius^2 <= 100
 * cells around the x-y centre in a porous formation (create_model,
 * Float/main.cu:1590-1655).  out9 receives 9 arrays of nz*ny*nx floats in the
 * bp_medium order (rho, rhof, M, C, H, H2mu, mu, C1, C2). */
int bp_medium_reference_borehole(int nx, int ny, int nz, float* out9);

/* Biot coefficients of one material given by moduli (Pa), densities (kg/m^3),
 * porosity, tortuosity, viscosity (Pa s), permeability (m^2) and pore-shape
 * factor m (8 in the reference).  out9: rho, rhof, M, C, H, H2mu, mu, C1, C2. */
int bp_biot_from_moduli(double Ks, double Kb, double mu, double Kf,
                        double rhos, double rhof, double phi, double tort,
                        double eta, double kappa, double m_shape, double out9[9]);

/* Stability limit: largest dt for which the scheme is stable on this medium
 * (fast P velocity bound, order-dependent).  vmax receives the bound used. */
int bp_cfl_limit(const bp_config* cfg, const bp_medium* medium, double* dt_max,
                 double* vmax);

/* ---- batched shots (one launch per phase for all shots) ---------------- */
typedef struct bp_batch bp_batch;

typedef struct bp_tune {
    int tile_rows;        /* rows (z, or y*z in 3D) per tile of the register
                             kernels, a power of two 4..32; 0 = autotune      */
    int steps_per_sync;   /* steps captured per CUDA graph launch; 0 = autotune */
    int ctas_per_sm;      /* persistent CTAs per SM; 0 = autotune               */
    int tile_segs;        /* 128-cell x segments per tile, 1..4 (0 = 1)        */
    int tile_tz;          /* 3D: z planes among the tile's rows, 1..tile_rows
                             (0 = the precision's default)                    */
    int kernel;           /* BP_KERNEL_* family; 0 = autotune among the register
                             tiles, the interleaved kernel and (2D) the fused
                             step kernel                                      */
    int reserved[2];
} bp_tune;

/* All shots must share dim, order and precision; sizes, media, sources and
 * receivers may differ.  Every shot runs its own cfg.nt steps. */
int bp_batch_create(const bp_config* cfgs, const bp_medium* media, int nshots,
                    const bp_tune* tune, bp_batch** out);
/* Advances every unfinished shot by up to nsteps steps (async). */
int bp_batch_run(bp_batch* b, int nsteps);
int bp_batch_sync(bp_batch* b);
/* bp_batch_run bracketed by CUDA events on the batch's stream; waits and
 * returns the device time of the steps in *ms (the autotuner, if it still has
 * to run, runs first, outside the timed region). */
int bp_batch_run_timed(bp_batch* b, int nsteps, float* ms);
int bp_batch_get_traces(bp_batch* b, int shot, int comp, float* host, size_t n);
int bp_batch_get_tune(bp_batch* b, bp_tune* chosen);
/* Runs the autotuner now (it otherwise runs inside the first bp_batch_run):
 * times real steps of the batch, at most budget_steps of them, under the
 * candidate kernel families, then (register tiles) tile shapes and persistent
 * CTAs per SM, then steps per sync, and keeps the fastest; results are cached per (dim, order, precision, rounding, grid
 * class) for the process.  The timed steps advance the shots.  No-op when the
 * bp_tune given to bp_batch_create fixed every setting.  (No counterpart in
 * the reference, which has one fixed (16, 8, 1) block, Float/main.cu:26-28.) */
int bp_batch_autotune(bp_batch* b, int budget_steps);
/* Total cell-updates performed so far (all shots). */
int bp_batch_cell_updates(bp_batch* b, long long* updates);
/* Shot `shot`'s indexed-medium tuples (0: per-cell arrays), and the
 * algorithmic HBM bytes of one step of the whole batch (bp_algorithmic_bytes
 * summed over its shots' updated cells). */
int bp_batch_medium_tuples(bp_batch* b, int shot, int* ntuples);
int bp_batch_algorithmic_bytes(bp_batch* b, double* bytes_per_step);
void bp_batch_destroy(bp_batch* b);

/* ---- serving: admission by HBM budget + continuous batching ------------ */
typedef struct bp_server bp_server;

#define BP_REQ_QUEUED 0
#define BP_REQ_RUNNING 1
#define BP_REQ_DONE 2
#define BP_REQ_FAILED 3
#define BP_REQ_CANCELLED 4

typedef struct bp_server_stats {
    long long submitted, admitted, completed, failed, cancelled;
    long long cell_updates;     /* total cell-updates executed               */
    double busy_seconds;        /* wall time with at least one shot resident */
    double p50_latency_s;       /* submit -> done latency percentiles        */
    double p99_latency_s;
    size_t hbm_in_use;          /* bytes of resident shot state              */
    size_t hbm_budget;
    int max_resident;           /* largest number of shots resident at once  */
} bp_server_stats;

/* Device bytes a shot with this configuration occupies while resident (its
 * arena plus the transient medium upload): the cost admission charges. */
int bp_shot_bytes(const bp_config* cfg, size_t* bytes);

/* hbm_budget: bytes of device memory shot state may occupy.
 * steps_per_sync: steps between admission points (0 = 100). */
int bp_server_create(int device, size_t hbm_budget, int steps_per_sync,
                     bp_server** out);
/* Copies cfg/medium; the request waits until its state fits the budget.
 * BP_ERR_BUDGET if it can never fit. */
int bp_server_submit(bp_server* s, const bp_config* cfg, const bp_medium* medium,
                     uint64_t* request_id);
int bp_server_poll(bp_server* s, uint64_t request_id, int* state);
/* Blocks until the request finishes or timeout_s passes (BP_ERR_TIMEOUT). */
int bp_server_wait(bp_server* s, uint64_t request_id, double timeout_s);
int bp_server_cancel(bp_server* s, uint64_t request_id);
/* Traces of a finished request (then released with bp_server_release). */
int bp_server_get_traces(bp_server* s, uint64_t request_id, int comp,
                         float* host, size_t n);
int bp_server_release(bp_server* s, uint64_t request_id);
/* Submit-to-done latency of a finished request, seconds. */
int bp_server_latency(bp_server* s, uint64_t request_id, double* seconds);
int bp_server_get_stats(bp_server* s, bp_server_stats* st);
void bp_server_destroy(bp_server* s);

#ifdef __cplusplus
}
#endif
#endif /* BIOT_B200_H */

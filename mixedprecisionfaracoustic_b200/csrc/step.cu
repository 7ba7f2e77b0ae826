// step.cu - the hot path: velocity phase, stress phase and post-step kernels.
//
// Reference kernels replaced (Zhitao-Zhang/MixedPrecisionFarAcoustic):
//   FD_V   Float/main.cu:64-192,  Half/main.cu:156-268  -> k_vphase
//   FD_T   Float/main.cu:194-295, Half/main.cu:270-371  -> k_tphase
//   Source Float/main.cu:45-59,   Half/main.cu:135-151  -> k_post (inject)
//   trace capture Float/main.cu:1075-1093               -> k_post (record)
//   ScaleHalfArray/ScaleCompressedArray Half/main.cu:102-114: folded into
//   k_vphase/k_tphase as a per-step factor on every old state value.
//
// Work decomposition: a tile is 8 rows x 128 cells of one shot; a CTA of 8
// warps takes one tile at a time (one row per warp, 4 consecutive x cells per
// lane, 16-byte vector accesses along x).  CTAs loop over the tile table of
// all shots of a batch, so one launch advances every shot by one phase.
// Neighbour rows (y, z) are re-read through L1/L2; DRAM sees each array once
// per phase.  The CPML memory variables exist on the slabs only; a chunk
// touches them only when it lies in a slab of that axis.
#include "tile.cuh"

namespace bpk {

template <int DIM, int ORD, class P, bool VPHASE, bool MU>
__global__ void __launch_bounds__(kThreads, (phase_min_blocks<DIM, ORD, P, VPHASE>())) k_phase(const ShotDesc* __restrict__ shots, int nshots,
                                                     long long ntiles, int k, int post) {
    using R = typename P::real;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // The descriptor of the tile's shot is staged in shared memory whenever the
    // shot changes, so the ~100 pointers and extents the chunk code reads are
    // shared-memory broadcasts instead of per-warp global loads.
    __shared__ ShotDesc sdesc;
    int cur = -1;
    bool live = false;
    int it_cur = 0;
    R r = (R)1;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int si = nshots == 1 ? 0 : locate_shot(shots, nshots, t);
        if (si != cur) {                      // uniform across the CTA
            __syncthreads();
            const long long* src = reinterpret_cast<const long long*>(shots + si);
            long long* dst = reinterpret_cast<long long*>(&sdesc);
            for (int w = threadIdx.x; w < (int)(sizeof(ShotDesc) / 8); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            cur = si;
            if constexpr (step_once_per_shot<P>()) {
                // the step index and the COMP16 rescale are fixed for the
                // whole launch: read them once per shot, not once per tile
                const int it = *sdesc.step_base + k;
                it_cur = it;
                live = !sdesc.done && it < sdesc.nt;
                if constexpr (P::prec == BP_PREC_COMP16) r = live ? sdesc.rtab[it] : 1.0f;
            }
        }
        const ShotDesc& S = sdesc;
        int rb, sb;                           // row block and segment block of the tile
        if constexpr (step_once_per_shot<P>()) {
            if (!live) continue;
            const unsigned lt = (unsigned)(t - S.tile0);      // tiles of one shot < 2^32
            const unsigned q = lt / (unsigned)S.nseg_t;
            rb = (int)q;
            sb = (int)(lt - q * (unsigned)S.nseg_t);
        } else {
            const int it = *S.step_base + k;
            if (S.done || it >= S.nt) continue;
            it_cur = it;
            if constexpr (P::prec == BP_PREC_COMP16) r = S.rtab[it];
            const long long lt = t - S.tile0;
            rb = (int)(lt / S.nseg_t);
            sb = (int)(lt % S.nseg_t);
        }
        tile_units<DIM, ORD, P, VPHASE, MU, true>(S, rb, sb, warp, lane, r, it_cur, post);
    }
}

// ---------------------------------------------------------------------------
// Post-step kernel: records the five seismogram components of step it at the
// unique receiver cells, then injects the source sample of step it+1 (the
// reference's Source kernel runs at the top of the next step, so the order
// record(it) -> inject(it+1) -> FD_V(it+1) is unchanged).  The thread that
// records the source cell, if any, injects after its own reads; otherwise
// thread 0 of the shot's first block does.
template <class P>
__global__ void k_post(const ShotDesc* __restrict__ shots, int k, int do_record) {
    const ShotDesc& S = shots[blockIdx.y];
    const int it = *S.step_base + k;
    if (S.done || it >= S.nt) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (do_record && r < S.nrec) record<P>(S, it, r, S.rec_idx[r]);
    const bool owner = (S.src_rec >= 0) ? (r == S.src_rec) : (blockIdx.x == 0 && threadIdx.x == 0);
    if (owner) inject<P>(S, it + 1);
}


// Injection of step it = *step_base + k alone (before the first step).
template <class P>
__global__ void k_inject(const ShotDesc* __restrict__ shots, int nshots, int k) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshots) return;
    const ShotDesc& S = shots[s];
    if (S.done) return;
    inject<P>(S, *S.step_base + k);
}

// Advances the per-shot step base by n after a chunk of n steps.
__global__ void k_advance(const ShotDesc* __restrict__ shots, int nshots, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshots) return;
    const ShotDesc& S = shots[s];
    if (S.done) return;
    int v = *S.step_base + n;
    *S.step_base = v > S.nt ? S.nt : v;
}

// Snapshot: copies field f (physical units) of one shot, either the x-z slice
// at y = sy or the whole padded volume, into a dense float array.
template <class P>
__global__ void k_snapshot(const ShotDesc* __restrict__ shots, int shot, int f, int slice_y, float* out, int it) {
    using R = typename P::real;
    const ShotDesc& S = shots[shot];
    const long long n = slice_y >= 0 ? (long long)S.nx * S.nz : (long long)S.nx * S.ny * S.nz;
    R sc = (R)1;
    if constexpr (P::prec == BP_PREC_COMP16) {
        const bool vel = f <= BP_F_VWZ;
        sc = (vel ? S.out_vel : S.out_stress) / S.dyn[it];
    }
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % S.nx);
        long long rest = q / S.nx;
        int y, z;
        if (slice_y >= 0) { y = slice_y; z = (int)rest; }
        else { y = (int)(rest % S.ny); z = (int)(rest / S.ny); }
        const long long i = x + (long long)y * S.pitch + (long long)z * S.plane;
        out[q] = (float)(P::ld1(S.f[f], S.flo[f], i) * sc);
    }
}

// Full-field read in double precision (physical units) for bp_get_field*.
template <class P>
__global__ void k_field_f64(const ShotDesc* __restrict__ shots, int f, double* out) {
    const ShotDesc& S = shots[0];
    const long long n = (long long)S.nx * S.ny * S.nz;
    double sc = 1.0;
    if constexpr (P::prec == BP_PREC_COMP16) {
        const int it = *S.step_base;
        const int itc = it > 0 ? it - 1 : 0;
        sc = (double)((f <= BP_F_VWZ ? S.out_vel : S.out_stress) / S.dyn[itc < S.nt ? itc : S.nt - 1]);
    }
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % S.nx);
        long long rest = q / S.nx;
        int y = (int)(rest % S.ny), z = (int)(rest / S.ny);
        const long long i = x + (long long)y * S.pitch + (long long)z * S.plane;
        out[q] = (double)P::ld1(S.f[f], S.flo[f], i) * sc;
    }
}

// Coefficient read-back (decoded to float) over the dense padded grid.
template <class P>
__global__ void k_coef(const ShotDesc* __restrict__ shots, int which, float* out) {
    const ShotDesc& S = shots[0];
    const void* p = which < VC_COUNT ? S.vc[which] : S.tc[which - VC_COUNT];
    const int8_t* lo = which < VC_COUNT ? S.vclo[which] : S.tclo[which - VC_COUNT];
    const long long n = (long long)S.nx * S.ny * S.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % S.nx);
        long long rest = q / S.nx;
        int y = (int)(rest % S.ny), z = (int)(rest / S.ny);
        out[q] = p ? (float)P::ld1(p, lo, x + (long long)y * S.pitch + (long long)z * S.plane) : 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Host-side launchers (explicit instantiation over dim x order x precision).

// Shared-memory carveout of the phase kernels, in percent of the SM's unified
// L1/shared storage (their only shared data is the shot descriptor; the rest
// serves as L1 for the neighbour re-reads); -1 leaves the driver's choice.
#ifndef BP_L1_CARVEOUT
#define BP_L1_CARVEOUT -1
#endif
template <int D, int O, class P, bool V, bool M>
static void phase_carveout() {
    if constexpr (BP_L1_CARVEOUT >= 0) {
        static bool set = false;                       // once per kernel
        if (!set) {
            cudaFuncSetAttribute(k_phase<D, O, P, V, M>, cudaFuncAttributePreferredSharedMemoryCarveout, BP_L1_CARVEOUT);
            set = true;
        }
    }
}

template <class P>
struct Launch {
    static cudaError_t phase(int dim, int order, bool v, const ShotDesc* d_shots, int nshots, long long ntiles,
                             int k, int grid, cudaStream_t st, int post, bool multi) {
#define BPK_LAUNCH(D, O)                                                                                        \
    if (dim == D && order == O) {                                                                               \
        if (multi) {                                                                                            \
            if (v) { phase_carveout<D, O, P, true, true>();                                                     \
                     k_phase<D, O, P, true, true><<<grid, kThreads, 0, st>>>(d_shots, nshots, ntiles, k, 0); }  \
            else { phase_carveout<D, O, P, false, true>();                                                      \
                   k_phase<D, O, P, false, true><<<grid, kThreads, 0, st>>>(d_shots, nshots, ntiles, k, post); } \
        } else {                                                                                                \
            if (v) { phase_carveout<D, O, P, true, false>();                                                    \
                     k_phase<D, O, P, true, false><<<grid, kThreads, 0, st>>>(d_shots, nshots, ntiles, k, 0); } \
            else { phase_carveout<D, O, P, false, false>();                                                     \
                   k_phase<D, O, P, false, false><<<grid, kThreads, 0, st>>>(d_shots, nshots, ntiles, k, post); } \
        }                                                                                                       \
        return cudaGetLastError();                                                                              \
    }
        if constexpr (P::graded) {           // the variable z grid: order 2 only
            BPK_LAUNCH(2, 2) BPK_LAUNCH(3, 2)
        } else if constexpr (P::wide) {      // large 3D grids only
            BPK_LAUNCH(3, 2) BPK_LAUNCH(3, 4)
        } else {
            BPK_LAUNCH(2, 2) BPK_LAUNCH(2, 4) BPK_LAUNCH(3, 2) BPK_LAUNCH(3, 4)
        }
#undef BPK_LAUNCH
        return cudaErrorInvalidValue;
    }
};

}  // namespace bpk

// C++ entry points used by the host code (sim.cu, batch.cu).
namespace bpk {
cudaError_t launch_phase(int prec, int dim, int order, bool vphase, const ShotDesc* d_shots, int nshots,
                         long long ntiles, int k, int grid, cudaStream_t st, int post, int rounding, bool multi,
                         bool graded, bool wide) {
    if (wide && dim == 3 && prec == BP_PREC_FP32 && rounding == BP_ROUND_FAST && !graded)
        return Launch<PolF32W>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
    if (graded) {
        if (prec != BP_PREC_FP32 || rounding != BP_ROUND_FAST || order != 2) return cudaErrorInvalidValue;
        return Launch<PolF32G>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
    }
    if (prec == BP_PREC_FP32 && rounding == BP_ROUND_REFERENCE)
        return Launch<PolF32R>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
    if (prec == BP_PREC_FP32)
        return Launch<PolF32>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
    if (prec == BP_PREC_COMP16)
        return Launch<PolC16>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
    if (prec == BP_PREC_CBF16)
        return Launch<PolB24>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
    return Launch<PolF64>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st, post, multi);
}

cudaError_t launch_post(int prec, const ShotDesc* d_shots, int nshots, int max_rec, int k, int do_record,
                        cudaStream_t st) {
    dim3 grid((max_rec + 127) / 128 > 0 ? (max_rec + 127) / 128 : 1, nshots);
    if (prec == BP_PREC_FP32) k_post<PolF32><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    else if (prec == BP_PREC_COMP16) k_post<PolC16><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    else if (prec == BP_PREC_CBF16) k_post<PolB24><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    else k_post<PolF64><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    return cudaGetLastError();
}

cudaError_t launch_inject(int prec, const ShotDesc* d_shots, int nshots, int k, cudaStream_t st) {
    int g = (nshots + 127) / 128;
    if (prec == BP_PREC_FP32) k_inject<PolF32><<<g, 128, 0, st>>>(d_shots, nshots, k);
    else if (prec == BP_PREC_COMP16) k_inject<PolC16><<<g, 128, 0, st>>>(d_shots, nshots, k);
    else if (prec == BP_PREC_CBF16) k_inject<PolB24><<<g, 128, 0, st>>>(d_shots, nshots, k);
    else k_inject<PolF64><<<g, 128, 0, st>>>(d_shots, nshots, k);
    return cudaGetLastError();
}

cudaError_t launch_advance(const ShotDesc* d_shots, int nshots, int n, cudaStream_t st) {
    k_advance<<<(nshots + 127) / 128, 128, 0, st>>>(d_shots, nshots, n);
    return cudaGetLastError();
}

cudaError_t launch_snapshot(int prec, const ShotDesc* d_shots, int shot, int f, int slice_y, float* out, int it,
                            cudaStream_t st) {
    if (prec == BP_PREC_FP32) k_snapshot<PolF32><<<296, 256, 0, st>>>(d_shots, shot, f, slice_y, out, it);
    else if (prec == BP_PREC_COMP16) k_snapshot<PolC16><<<296, 256, 0, st>>>(d_shots, shot, f, slice_y, out, it);
    else if (prec == BP_PREC_CBF16) k_snapshot<PolB24><<<296, 256, 0, st>>>(d_shots, shot, f, slice_y, out, it);
    else k_snapshot<PolF64><<<296, 256, 0, st>>>(d_shots, shot, f, slice_y, out, it);
    return cudaGetLastError();
}

cudaError_t launch_field_f64(int prec, const ShotDesc* d_shots, int f, double* out, cudaStream_t st) {
    if (prec == BP_PREC_FP32) k_field_f64<PolF32><<<296, 256, 0, st>>>(d_shots, f, out);
    else if (prec == BP_PREC_COMP16) k_field_f64<PolC16><<<296, 256, 0, st>>>(d_shots, f, out);
    else if (prec == BP_PREC_CBF16) k_field_f64<PolB24><<<296, 256, 0, st>>>(d_shots, f, out);
    else k_field_f64<PolF64><<<296, 256, 0, st>>>(d_shots, f, out);
    return cudaGetLastError();
}

int phase_occupancy(int prec, int dim, int order, bool vphase, int rounding, bool wide) {
    int n = 0;
    const void* fn = nullptr;
#define BPK_FN(PP, D, O)                                                                   \
    if (dim == D && order == O)                                                            \
        fn = vphase ? (const void*)k_phase<D, O, PP, true, false> : (const void*)k_phase<D, O, PP, false, false>;
    if (wide && dim == 3 && prec == BP_PREC_FP32 && rounding == BP_ROUND_FAST) {
        BPK_FN(PolF32W, 3, 2) BPK_FN(PolF32W, 3, 4)
    } else if (prec == BP_PREC_FP32 && rounding == BP_ROUND_REFERENCE) {
        BPK_FN(PolF32R, 2, 2) BPK_FN(PolF32R, 2, 4) BPK_FN(PolF32R, 3, 2) BPK_FN(PolF32R, 3, 4)
    } else if (prec == BP_PREC_FP32) { BPK_FN(PolF32, 2, 2) BPK_FN(PolF32, 2, 4) BPK_FN(PolF32, 3, 2) BPK_FN(PolF32, 3, 4) }
    else if (prec == BP_PREC_COMP16) { BPK_FN(PolC16, 2, 2) BPK_FN(PolC16, 2, 4) BPK_FN(PolC16, 3, 2) BPK_FN(PolC16, 3, 4) }
    else if (prec == BP_PREC_CBF16) { BPK_FN(PolB24, 2, 2) BPK_FN(PolB24, 2, 4) BPK_FN(PolB24, 3, 2) BPK_FN(PolB24, 3, 4) }
    else { BPK_FN(PolF64, 2, 2) BPK_FN(PolF64, 2, 4) BPK_FN(PolF64, 3, 2) BPK_FN(PolF64, 3, 4) }
#undef BPK_FN
    if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_coef(int prec, const ShotDesc* d_shots, int which, float* out, cudaStream_t st) {
    if (prec == BP_PREC_FP32) k_coef<PolF32><<<296, 256, 0, st>>>(d_shots, which, out);
    else if (prec == BP_PREC_COMP16) k_coef<PolC16><<<296, 256, 0, st>>>(d_shots, which, out);
    else if (prec == BP_PREC_CBF16) k_coef<PolB24><<<296, 256, 0, st>>>(d_shots, which, out);
    else k_coef<PolF64><<<296, 256, 0, st>>>(d_shots, which, out);
    return cudaGetLastError();
}

int phase_threads() { return kThreads; }

static int ilog2(int v) {
    int l = 0;
    while ((1 << (l + 1)) <= v) l++;
    return l;
}
static bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

TileShape default_tile_shape(int dim, int prec) {
    TileShape t;
    t.rows = kWarps;
    t.segs = 1;
    t.tz = dim == 3 ? tile_tz(prec) : 1;
    return t;
}

bool valid_tile_shape(int dim, const TileShape& t) {
    if (!pow2(t.rows) || t.rows < 4 || t.rows > 32 || !pow2(t.segs) || t.segs > 4) return false;
    if (dim == 3 && t.tz != 0 && (!pow2(t.tz) || t.tz > t.rows)) return false;
    return true;
}

long long apply_tile_shape(ShotDesc& S, int dim, int prec, TileShape t) {
    if (dim == 3 && t.tz == 0) t.tz = tile_tz(prec) < t.rows ? tile_tz(prec) : t.rows;
    if (dim == 2) t.tz = 1;
    S.tile_lr = ilog2(t.rows);
    S.tile_ls = ilog2(t.segs);
    S.tile_ltz = ilog2(t.tz);
    S.nseg_t = (S.nseg + t.segs - 1) / t.segs;
    long long blocks;
    if (dim == 3) {
        const int ty = t.rows / t.tz;
        blocks = (long long)((S.ny + ty - 1) / ty) * ((S.nz + t.tz - 1) / t.tz);
    } else {
        blocks = (S.nrows + t.rows - 1) / t.rows;
    }
    return blocks * S.nseg_t;
}
int seg_cells() { return kSegCells; }
}  // namespace bpk

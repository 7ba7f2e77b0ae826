// step_inter.cu - one persistent launch per time step that interleaves the
// velocity and stress phases band by band, so that the stress phase of a band
// finds the velocities and stresses the velocity phase has just touched in L2.
//
// Reference kernels replaced: FD_V (Float/main.cu:64-192, Half/main.cu:156-268)
// and FD_T (Float/main.cu:194-295, Half/main.cu:270-371), with the trace
// capture and Source (Float/main.cu:45-59,1075-1093) in the stress tiles.
//
// The two-phase kernels stream every field through HBM in the V launch and
// again in the T launch: 144 B per cell and step at FP32 in 2D, where one pass
// would need 112.  Here a shot's register tiles are grouped into bands of
// consecutive row blocks, and the work items (one tile of one phase) are
// claimed by the persistent CTAs from one counter in the order
//
//     V(0) .. V(A-1), T(0), V(A), T(1), V(A+1), ..., T(nb-1-A) .. T(nb-1)
//
// with A the lag in bands (sized to the CTAs' in-flight window).  A stress
// tile of band b reads new velocities and old stresses of bands b-1..b+1 and
// overwrites the stresses of band b, which the velocity tiles of bands b-1..b+1
// read: it waits until those three bands' velocity tiles are all done, and
// with A >= 2 they all precede it in the order, so every wait is on work that
// running CTAs have already claimed (a CTA claims its next item while it works
// on the current one, and that next item is never a dependency of the
// current one).  Velocity tiles wait for nothing.  The waits poll a per-band
// completion counter with a bounded number of polls; one that runs out sets
// the error flag (BP_ERR_TIMEOUT at the next sync) and proceeds.
//
// The per-cell arithmetic is the tile kernels' own (tile.cuh), so the results
// are bit-identical to the two-phase kernels.  Loads never take the read-only
// data path here: the arrays a stress tile reads are written by the same launch.
#include "tile.cuh"

namespace bpk {

static_assert(!kReadOnlyPath, "the interleaved kernel reads arrays the same launch writes");

#ifndef BP_INTER_DEFAULT
#define BP_INTER_DEFAULT 0
#endif
// Band height: rows per band in 2D, z planes per band in 3D (whole row blocks).
#ifndef BP_INTER_BAND_ROWS
#define BP_INTER_BAND_ROWS 32
#endif
#ifndef BP_INTER_BAND_PLANES
#define BP_INTER_BAND_PLANES 4
#endif
constexpr long long kInterPolls = 1LL << 22;    // ~1 s of polling before a wait gives up

// Register caps (CTAs per SM the compiler must fit): both phases' code lives
// in one function with the claim loop around it, so the caps sit one step
// looser than the two-phase kernels' where theirs would spill.
#ifndef BP_INTER_MINB_C16
#define BP_INTER_MINB_C16 4
#endif
#ifndef BP_INTER_MINB3
#define BP_INTER_MINB3 2
#endif
template <int DIM, int ORD, class P>
__host__ __device__ constexpr int inter_min_blocks() {
    if (DIM == 3) return P::prec == BP_PREC_FP64 ? 1 : BP_INTER_MINB3;
    if (P::store == BP_PREC_COMP16) return BP_INTER_MINB_C16;
    return phase_min_blocks<DIM, ORD, P, false>();
}

// Binary search of the shot owning item j (item0_i ascending).
__device__ __forceinline__ int locate_shot_i(const ShotDesc* shots, int nshots, long long j) {
    int lo = 0, hi = nshots - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (shots[mid].item0_i <= j) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct InterItem {
    int phase;      // 0: velocity tile, 1: stress tile
    int band, tile; // band of the shot, tile within the band
};

// Item j of a shot (see the header for the order of positions; every
// position holds band_t tiles but those of the last band, band_last).
__device__ __forceinline__ InterItem decode_item(const ShotDesc& S, long long j) {
    const int tpb = S.band_t, nb = S.nbands_i, A = S.lag_i, ntl = S.band_last;
    const int K = nb - A;                              // velocity bands after the first A
    const int pv_last = K == 0 ? nb - 1 : A + 2 * K - 1;   // position of V(nb-1)
    const long long lo = (long long)pv_last * tpb;
    int p, tile;
    if (j < lo) {
        p = (int)(j / tpb);
        tile = (int)(j - (long long)p * tpb);
    } else if (j < lo + ntl) {
        p = pv_last;
        tile = (int)(j - lo);
    } else {
        const long long jj = j - lo - ntl;
        const int q = (int)(jj / tpb);
        p = pv_last + 1 + q;
        tile = (int)(jj - (long long)q * tpb);
    }
    InterItem I;
    I.tile = tile;
    if (p < A) {
        I.phase = 0;
        I.band = p;
    } else {
        const int m = p - A;
        if (m < 2 * K) {
            I.phase = (m & 1) ? 0 : 1;
            I.band = (m & 1) ? A + (m >> 1) : (m >> 1);
        } else {
            I.phase = 1;
            I.band = K + (m - 2 * K);
        }
    }
    return I;
}

template <int DIM, int ORD, class P>
__global__ void __launch_bounds__(kThreads, (inter_min_blocks<DIM, ORD, P>())) k_inter(
    const ShotDesc* __restrict__ shots, int nshots, long long nitems, int k, int post, unsigned long long* claim,
    int* done, int* err) {
    using R = typename P::real;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ ShotDesc sdesc;
    __shared__ long long s_item;
    int cur = -1;
    unsigned long long next = 0;
    if (threadIdx.x == 0) next = atomicAdd(claim, 1ull);
    for (;;) {
        __syncthreads();                               // the previous item is finished by every thread
        if (threadIdx.x == 0) {
            s_item = (long long)next;
            next = atomicAdd(claim, 1ull);             // the item after this one, claimed ahead
        }
        __syncthreads();
        const long long j = s_item;
        if (j >= nitems) break;
        const int si = nshots == 1 ? 0 : locate_shot_i(shots, nshots, j);
        if (si != cur) {
            const long long* src = reinterpret_cast<const long long*>(shots + si);
            long long* dst = reinterpret_cast<long long*>(&sdesc);
            for (int w = threadIdx.x; w < (int)(sizeof(ShotDesc) / 8); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            cur = si;
        }
        const ShotDesc& S = sdesc;
        const int it = *S.step_base + k;
        if (S.done || it >= S.nt) continue;
        R r = (R)1;
        if constexpr (P::prec == BP_PREC_COMP16) r = S.rtab[it];
        const InterItem I = decode_item(S, j - S.item0_i);
        if (I.phase == 1) {
            // the velocity tiles of bands b-1, b, b+1 must all be done
            if (threadIdx.x == 0) {
                for (int bb = I.band - 1; bb <= I.band + 1; bb++) {
                    if (bb < 0 || bb >= S.nbands_i) continue;
                    const int need = bb == S.nbands_i - 1 ? S.band_last : S.band_t;
                    const volatile int* c = done + S.band0_i + bb;
                    const volatile int* ve = err;
                    long long n = 0;
                    // once any wait has given up, the rest give up at once
                    while (*c < need && *ve == 0) {
                        if (++n > kInterPolls) {
                            atomicExch(err, BP_ERR_TIMEOUT);
                            break;
                        }
                        __nanosleep(n < 64 ? 32 : 256);
                    }
                }
                __threadfence();
            }
            __syncthreads();
        }
        const int lt = I.band * S.band_t + I.tile;
        const int rb = lt / S.nseg_t, sb = lt - rb * S.nseg_t;
        if (I.phase == 0) {
            tile_units<DIM, ORD, P, true, false, false>(S, rb, sb, warp, lane, r, it, 0);
            __threadfence();                           // this thread's stores before the count
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(done + S.band0_i + I.band, 1);
        } else {
            tile_units<DIM, ORD, P, false, false, false>(S, rb, sb, warp, lane, r, it, post);
        }
    }
}

// ---------------------------------------------------------------------------
bool inter_default() { return BP_INTER_DEFAULT != 0; }

long long apply_bands(ShotDesc& S, int dim, long long ntiles, int ctas) {
    int rb_per_band;
    if (dim == 3) {
        const int lty = S.tile_lr - S.tile_ltz;
        const int nyb = (S.ny + (1 << lty) - 1) >> lty;
        const int tz = 1 << S.tile_ltz;
        const int bz = (BP_INTER_BAND_PLANES + tz - 1) / tz;
        rb_per_band = bz * nyb;
    } else {
        const int rows = 1 << S.tile_lr;
        rb_per_band = (BP_INTER_BAND_ROWS + rows - 1) / rows;
    }
    const long long tpb = (long long)rb_per_band * S.nseg_t;
    const int nb = (int)((ntiles + tpb - 1) / tpb);
    S.band_t = (int)tpb;
    S.nbands_i = nb;
    S.band_last = (int)(ntiles - (long long)(nb - 1) * tpb);
    // leading velocity bands: at least 2 (so every wait is on earlier items)
    // and enough that the CTAs' in-flight items lie behind the bands a stress
    // tile waits for
    const long long want = (ctas + tpb - 1) / tpb + 2;
    S.lag_i = (int)(nb < want ? nb : want);
    return 2 * ntiles;
}

template <int DIM, int ORD, class P>
static const void* inter_fn() {
    return (const void*)k_inter<DIM, ORD, P>;
}

template <class P>
static const void* inter_fn_of(int dim, int order) {
    if (dim == 2) return order == 2 ? inter_fn<2, 2, P>() : inter_fn<2, 4, P>();
    return order == 2 ? inter_fn<3, 2, P>() : inter_fn<3, 4, P>();
}

static const void* inter_kernel(int prec, int dim, int order, int rounding) {
    if (prec == BP_PREC_FP32 && rounding == BP_ROUND_REFERENCE) return inter_fn_of<PolF32R>(dim, order);
    if (prec == BP_PREC_FP32) return inter_fn_of<PolF32>(dim, order);
    if (prec == BP_PREC_COMP16) return inter_fn_of<PolC16>(dim, order);
    if (prec == BP_PREC_CBF16) return inter_fn_of<PolB24>(dim, order);
    return inter_fn_of<PolF64>(dim, order);
}

int inter_occupancy(int prec, int dim, int order, int rounding) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, inter_kernel(prec, dim, order, rounding), kThreads, 0) !=
        cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_inter(int prec, int dim, int order, int rounding, const ShotDesc* d, int nshots, long long nitems,
                         int k, int post, int grid, unsigned long long* ctl, int* err, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    const void* fn = inter_kernel(prec, dim, order, rounding);
    int* done = reinterpret_cast<int*>(ctl + 1);
    void* args[] = {(void*)&d, (void*)&nshots, (void*)&nitems, (void*)&k, (void*)&post, (void*)&ctl, (void*)&done,
                    (void*)&err};
    return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(kThreads), args, 0, st);
}

}  // namespace bpk

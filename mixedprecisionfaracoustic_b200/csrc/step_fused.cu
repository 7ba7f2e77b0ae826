// step_fused.cu - one whole time step per launch for 2D (x-z) shots, FP32 and
// COMP16: the velocity phase, the stress phase, the trace recording and the
// next source injection, from one copy of the state into the other.
//
// Reference kernels replaced: FD_V (Float/main.cu:64-192, Half/main.cu:156-268),
// FD_T (Float/main.cu:194-295, Half/main.cu:270-371), the trace capture
// (Float/main.cu:1075-1093) and Source (Float/main.cu:45-59), 2D x-z restriction.
//
// Work decomposition: a task is one warp's column of x cells over a segment of
// rows.  The warp's 32 lanes hold 4 consecutive cells each (16-byte vector
// accesses); lanes 1..30 own the column's 120 cells, lanes 0 and 31 are a halo
// whose velocities are computed but not stored, so that the stress update of
// the owned cells has every new velocity it differentiates without waiting for
// the neighbouring columns.  The warp marches down its rows: at row z it forms
// the new velocities (from the old stresses of rows z-HW..z+HW, held decoded in
// register windows), then the new stresses of row z-HW (from the new
// velocities of rows z-2HW..z, also in windows), then records and injects at
// row z-HW.  Each old stress value is loaded and decoded once per step, each
// new velocity is never reloaded, and the stress phase reads no velocity from
// memory: per updated cell the step moves the fields once each way and the
// coefficients once, where the two-phase kernels move the fields three times.
//
// Because columns and segments run in no fixed order, the step reads one copy
// of the state (fields, V-phase memory variables) and writes the other;
// segments recompute the HW velocity rows above and below them, as the halo
// lanes do along x.  Steps run in pairs (copy A -> B -> A), so the state is in
// the first copy between pairs and every other kernel sees it there.  The
// T-phase memory variables are updated in place: only the owner of a cell
// touches them.  The per-cell arithmetic is the two-phase kernels' own
// (v_tail, t_tail, record, inject), so the results are bit-identical to them.
#include "post.cuh"
#include "shot.h"

namespace bpk {

constexpr int kFWarps = 4;
constexpr int kFThreads = kFWarps * 32;
constexpr int kFCols = 120;                   // owned x cells per task (lanes 1..30)
constexpr unsigned kFAll = 0xffffffffu;
// Resident CTAs per SM the fused kernels are register-limited to: at 3 (168
// registers) the order-2 kernels spill 84 (FP32) and 152 (COMP16) bytes; at 4
// (128 registers) 376 and 912; uncapped they take 218-226 registers.
#ifndef BP_FUSED_MINB_F32
#define BP_FUSED_MINB_F32 3
#endif
#ifndef BP_FUSED_MINB_C16
#define BP_FUSED_MINB_C16 3
#endif
// Whether BP_KERNEL_AUTO runs the fused kernel where it applies.
#ifndef BP_FUSED_DEFAULT
#define BP_FUSED_DEFAULT 0
#endif
// Warps per SM the segments are sized for (tasks of a lone shot).
#ifndef BP_FUSED_WARPS_PER_SM
#define BP_FUSED_WARPS_PER_SM 16
#endif

template <class P>
__host__ __device__ constexpr int fused_min_blocks() {
    return P::prec == BP_PREC_FP32 ? BP_FUSED_MINB_F32 : BP_FUSED_MINB_C16;
}

// Binary search of the shot owning task t (tile0f ascending).
__device__ __forceinline__ int locate_shot_f(const ShotDesc* shots, int nshots, long long t) {
    int lo = 0, hi = nshots - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (shots[mid].tile0f <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// A row's 4 cells of one array, or zeros outside the allocation (the halo
// lanes of the first and last columns, rows above and below the grid).
template <class P>
__device__ __forceinline__ void ld_row(const void* p, const int8_t* lo, cidx i, bool in,
                                       typename P::real (&v)[4]) {
    if (in) {
        P::ld4(p, lo, i, v);
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = 0;
    }
}

// The span f(x0 - HW .. x0 + 3 + HW) of one row from the lane's own cells and
// the adjacent lanes' (shuffles).  The outer neighbours of lanes 0 and 31 are
// not available; they only reach the halo cells nobody reads.
template <int ORD, class R>
__device__ __forceinline__ void span_shfl(const R (&c)[4], R (&v)[4 + ORD]) {
    constexpr int HW = ORD / 2;
#pragma unroll
    for (int j = 0; j < 4; j++) v[HW + j] = c[j];
#pragma unroll
    for (int k = 1; k <= HW; k++) {
        v[HW - k] = __shfl_up_sync(kFAll, c[4 - k], 1);
        v[HW + 3 + k] = __shfl_down_sync(kFAll, c[k - 1], 1);
    }
}

template <int N, class R>
__device__ __forceinline__ void wshift(R (&w)[N][4]) {
#pragma unroll
    for (int i = 0; i + 1 < N; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) w[i][j] = w[i + 1][j];
}

// Differences across rows from a window: a[k] = row z + k - HW is w[k - k0]
// for k in [k0, k0 + N) (the stencil reads no other k).
template <int ORD, class P, bool FWD, int N>
__device__ __forceinline__ void dz_win(const typename P::real (&w)[N][4], int k0, const ShotDesc& S,
                                       typename P::real (&d)[4]) {
    using R = typename P::real;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R a[ORD + 1];
#pragma unroll
        for (int k = 0; k <= ORD; k++) a[k] = (k - k0 >= 0 && k - k0 < N) ? w[k - k0][j] : (R)0;
        d[j] = deriv_div<P>(FWD ? rfwd<ORD>(a) : rbwd<ORD>(a), S);
    }
}

template <int ORD, class P, bool FWD>
__device__ __forceinline__ void dx_span(const typename P::real (&c)[4], const ShotDesc& S, typename P::real (&d)[4]) {
    typename P::real v[4 + ORD];
    span_shfl<ORD>(c, v);
#pragma unroll
    for (int j = 0; j < 4; j++) d[j] = deriv_div<P>(FWD ? dfwd<ORD>(v, j) : dbwd<ORD>(v, j), S);
}

// One task: column col (lanes 1..30 own cells [col*120, col*120 + 120)),
// stress rows [za, zb) of step it; par = 0 reads the descriptor's first copy
// of the state and writes the second, par = 1 the other way round.
template <int ORD, class P, bool RS>
__device__ __forceinline__ void fused_task(const ShotDesc& S, int it, typename P::real r, int col, int za, int zb,
                                           int lane, int par) {
    using R = typename P::real;
    constexpr int HW = ORD / 2;
    // window lengths (rows): old stresses txx, txz, tzz, p of rows z-HW .. z,
    // z+HW-1, z+HW, z+HW; new velocities vux, vuz, vwx, vwz of rows z-2HW+1,
    // z-2HW, z-HW, z-2HW .. z (oldest first)
    constexpr int NXX = HW + 1, NXZ = 2 * HW, NZZ = 2 * HW + 1, NP = 2 * HW + 1;
    constexpr int NUX = 2 * HW, NUZ = 2 * HW + 1, NWX = HW + 1, NWZ = 2 * HW + 1;

    void* const* fi = par ? S.fb : S.f;
    int8_t* const* fli = par ? S.flob : S.flo;
    void* const* fo = par ? S.f : S.fb;
    int8_t* const* flo_o = par ? S.flo : S.flob;
    void* const* pvi = par ? S.psiVb : S.psiV;
    void* const* pvo = par ? S.psiV : S.psiVb;

    const int nx = S.nx, nz = S.nz;
    const cidx sz = (cidx)S.plane;
    const int x0 = col * kFCols - 4 + 4 * lane;
    const bool inb = x0 >= 0 && x0 < S.pitch;                       // the lane's cells are allocated
    const bool act = inb && x0 < nx - HW && x0 + 3 >= HW;            // the two-phase kernels' chunk test
    const bool own = act && lane >= 1 && lane <= 30;                 // stores, records, injects
    unsigned mask = 0;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (x0 + j >= HW && x0 + j < nx - HW) mask |= 1u << j;
    auto at = [&](int z) { return (cidx)z * sz + x0; };

    R wxx[NXX][4], wxz[NXZ][4], wzz[NZZ][4], wp[NP][4];
    R vux[NUX][4], vuz[NUZ][4], vwx[NWX][4], vwz[NWZ][4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
        for (int i = 0; i < NXX; i++) wxx[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NXZ; i++) wxz[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NZZ; i++) wzz[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NP; i++) wp[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NUX; i++) vux[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NUZ; i++) vuz[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NWX; i++) vwx[i][j] = 0;
#pragma unroll
        for (int i = 0; i < NWZ; i++) vwz[i][j] = 0;
    }
    const TailOut outV{fo, flo_o, pvi, pvo, false};
    const TailOut outT{fo, flo_o, S.psiT, nullptr, false};
    const int zv0 = za - HW > HW ? za - HW : HW;                     // velocity rows computed
    const int zv1 = zb + HW < nz - HW ? zb + HW : nz - HW;

    for (int z = za - 3 * HW; z < zb + HW; z++) {
        // ---- the newest stress rows of the windows ----
        wshift(wxx); wshift(wxz); wshift(wzz); wshift(wp);
        wshift(vux); wshift(vuz); wshift(vwx); wshift(vwz);
        {
            const int rxx = z, rxz = z + HW - 1, rzz = z + HW;
            ld_row<P>(fi[BP_F_TXX], fli[BP_F_TXX], at(rxx), inb && rxx >= 0 && rxx < nz, wxx[NXX - 1]);
            ld_row<P>(fi[BP_F_TXZ], fli[BP_F_TXZ], at(rxz), inb && rxz >= 0 && rxz < nz, wxz[NXZ - 1]);
            ld_row<P>(fi[BP_F_TZZ], fli[BP_F_TZZ], at(rzz), inb && rzz >= 0 && rzz < nz, wzz[NZZ - 1]);
            ld_row<P>(fi[BP_F_P], fli[BP_F_P], at(rzz), inb && rzz >= 0 && rzz < nz, wp[NP - 1]);
        }
        // ---- velocities of row z (zero on the border rows, never updated) ----
        R nux[4] = {0, 0, 0, 0}, nuz[4] = {0, 0, 0, 0}, nwx[4] = {0, 0, 0, 0}, nwz[4] = {0, 0, 0, 0};
        if (z >= zv0 && z < zv1) {                                  // warp-uniform
            VState<R> V;
            // derivatives of the old stresses (the tile kernels' v_chunk, 2D)
            dx_span<ORD, P, true>(wxx[HW], S, V.x1);                 // txx: D+x
            dx_span<ORD, P, true>(wp[HW], S, V.s1);                  // p: D+x
            dx_span<ORD, P, false>(wxz[HW], S, V.z2);                // txz: D-x
            dz_win<ORD, P, false>(wxz, 0, S, V.x3);                  // txz: D-z, rows z-HW ..
            dz_win<ORD, P, true>(wzz, 0, S, V.z1);                   // tzz: D+z
            dz_win<ORD, P, true>(wp, 0, S, V.s3);                    // p: D+z
            if (act) {
                const cidx c = at(z);
                vcoef4<P, false>(S, VC_RHOF, c, V.rf);
                vcoef4<P, false>(S, VC_RHO_X, c, V.rho_x);
                vcoef4<P, false>(S, VC_CC1_X, c, V.c1_x);
                vcoef4<P, false>(S, VC_CC2_X, c, V.c2_x);
                P::ld4(fi[BP_F_VUX], fli[BP_F_VUX], c, V.vu_x);
                P::ld4(fi[BP_F_VWX], fli[BP_F_VWX], c, V.vw_x);
                vcoef4<P, false>(S, VC_RHO_Z, c, V.rho_z);
                vcoef4<P, false>(S, VC_CC1_Z, c, V.c1_z);
                vcoef4<P, false>(S, VC_CC2_Z, c, V.c2_z);
                P::ld4(fi[BP_F_VUZ], fli[BP_F_VUZ], c, V.vu_z);
                P::ld4(fi[BP_F_VWZ], fli[BP_F_VWZ], c, V.vw_z);
                TailOut o = outV;
                o.store = own && z >= za && z < zb;
                v_tail<2, ORD, P, true, RS>(S, c, x0, 0, z, r, mask, V, o);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    nux[j] = V.vu_x[j]; nuz[j] = V.vu_z[j]; nwx[j] = V.vw_x[j]; nwz[j] = V.vw_z[j];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            vux[NUX - 1][j] = nux[j]; vuz[NUZ - 1][j] = nuz[j];
            vwx[NWX - 1][j] = nwx[j]; vwz[NWZ - 1][j] = nwz[j];
        }
        // ---- stresses of row q = z - HW ----
        const int q = z - HW;
        if (q >= za && q < zb) {                                    // warp-uniform
            TState<R> T;
            dx_span<ORD, P, false>(vux[HW - 1], S, T.uxx);          // vux: D-x at row q
            dx_span<ORD, P, false>(vwx[0], S, T.wx);                // vwx: D-x
            dx_span<ORD, P, true>(vuz[HW], S, T.uzx);               // vuz: D+x
            dz_win<ORD, P, false>(vuz, 0, S, T.uzz);                // vuz: D-z, rows q-HW ..
            dz_win<ORD, P, false>(vwz, 0, S, T.wz);                 // vwz: D-z
            dz_win<ORD, P, true>(vux, 1, S, T.uxz);                 // vux: D+z, rows q-HW+1 ..
            if (own) {                                              // the halo lanes' stresses are not needed
                const cidx c = at(q);
                tcoef4<P, false>(S, TC_C, c, T.cC);
                tcoef4<P, false>(S, TC_M, c, T.cM);
                tcoef4<P, false>(S, TC_H, c, T.cH);
                tcoef4<P, false>(S, TC_H2U, c, T.cH2);
                tcoef4<P, false>(S, TC_MUXZ, c, T.mxz);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    T.op[j] = wp[0][j]; T.oxx[j] = wxx[0][j]; T.ozz[j] = wzz[0][j]; T.oxz[j] = wxz[0][j];
                }
                if constexpr (P::prec == BP_PREC_COMP16 && RS) {
                    scale4(T.op, r); scale4(T.oxx, r); scale4(T.ozz, r); scale4(T.oxz, r);
                }
                TailOut o = outT;
                o.store = true;
                t_tail<2, ORD, P, true, RS>(S, c, x0, 0, q, r, mask, T, o);
                post_chunk<2, P>(S, it, c, x0, 0, q, o);
            }
        }
    }
}

template <int ORD, class P>
__global__ void __launch_bounds__(kFThreads, (fused_min_blocks<P>())) k_fused(const ShotDesc* __restrict__ shots,
                                                                             int nshots, long long ntasks, int k,
                                                                             int par) {
    using R = typename P::real;
    constexpr int HW = ORD / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ ShotDesc sd[kFWarps];
    const long long nwarps = (long long)gridDim.x * kFWarps;
    int cur = -1;
    for (long long t = (long long)blockIdx.x * kFWarps + warp; t < ntasks; t += nwarps) {
        const int si = nshots == 1 ? 0 : locate_shot_f(shots, nshots, t);
        if (si != cur) {                                   // the warp's own copy of its shot's descriptor
            __syncwarp();
            const long long* src = reinterpret_cast<const long long*>(shots + si);
            long long* dst = reinterpret_cast<long long*>(&sd[warp]);
            for (int w = lane; w < (int)(sizeof(ShotDesc) / 8); w += 32) dst[w] = src[w];
            __syncwarp();
            cur = si;
        }
        const ShotDesc& S = sd[warp];
        const int it = *S.step_base + k;
        if (S.done || it >= S.nt) continue;                // warp-uniform
        const unsigned lt = (unsigned)(t - S.tile0f);      // tasks of one shot < 2^32
        const unsigned g = lt / (unsigned)S.ncol_f;
        const int col = (int)(lt - g * (unsigned)S.ncol_f);
        const int za = HW + (int)g * S.zseg_f;
        const int zb = za + S.zseg_f < S.nz - HW ? za + S.zseg_f : S.nz - HW;
        R r = (R)1;
        if constexpr (P::prec == BP_PREC_COMP16) r = S.rtab[it];
        // COMP16: the rescale products only on the steps whose factor is not 1
        if (P::prec == BP_PREC_COMP16 && r != (R)1)
            fused_task<ORD, P, P::prec == BP_PREC_COMP16>(S, it, r, col, za, zb, lane, par);
        else
            fused_task<ORD, P, false>(S, it, r, col, za, zb, lane, par);
    }
}

// ---------------------------------------------------------------------------
bool fused_supported(int prec, int dim) {
    return dim == 2 && (prec == BP_PREC_FP32 || prec == BP_PREC_COMP16 || prec == BP_PREC_CBF16);
}

bool fused_default() { return BP_FUSED_DEFAULT != 0; }

int fused_cols(int nx) { return (nx + kFCols - 1) / kFCols; }

int fused_zseg(long long ncol, int nrows, int sms) {
    // enough tasks for BP_FUSED_WARPS_PER_SM warps on every SM for a lone
    // shot; at least 16 rows, since each segment recomputes 2 HW velocity rows
    const long long want = (long long)sms * BP_FUSED_WARPS_PER_SM;
    const long long nseg = (want + ncol - 1) / ncol;
    const long long L = (nrows + nseg - 1) / (nseg > 0 ? nseg : 1);
    return (int)(L < 16 ? 16 : L);
}

int fused_occupancy(int prec, int order) {
    const void* fn = nullptr;
    if (prec == BP_PREC_FP32) fn = order == 2 ? (const void*)k_fused<2, PolF32> : (const void*)k_fused<4, PolF32>;
    else if (prec == BP_PREC_CBF16) fn = order == 2 ? (const void*)k_fused<2, PolB24> : (const void*)k_fused<4, PolB24>;
    else fn = order == 2 ? (const void*)k_fused<2, PolC16> : (const void*)k_fused<4, PolC16>;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kFThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_fused(int prec, int order, const ShotDesc* d, int nshots, long long ntasks, int k, int par,
                         int grid, cudaStream_t st) {
    if (ntasks <= 0) return cudaSuccess;
    const long long need = (ntasks + kFWarps - 1) / kFWarps;
    const unsigned g = (unsigned)(grid < need ? grid : need);
#define BPK_FUSED(PP, O) k_fused<O, PP><<<g, kFThreads, 0, st>>>(d, nshots, ntasks, k, par)
    if (prec == BP_PREC_FP32) {
        if (order == 2) BPK_FUSED(PolF32, 2);
        else BPK_FUSED(PolF32, 4);
    } else if (prec == BP_PREC_COMP16) {
        if (order == 2) BPK_FUSED(PolC16, 2);
        else BPK_FUSED(PolC16, 4);
    } else if (prec == BP_PREC_CBF16) {
        if (order == 2) BPK_FUSED(PolB24, 2);
        else BPK_FUSED(PolB24, 4);
    } else {
        return cudaErrorInvalidValue;
    }
#undef BPK_FUSED
    return cudaGetLastError();
}

}  // namespace bpk

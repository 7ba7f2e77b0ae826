// step_march.cu - 2D (x-z) phase kernels that march along the slow axis z with
// register windows.
//
// Reference kernels replaced: FD_V (Float/main.cu:64-192, Half/main.cu:156-268)
// and FD_T (Float/main.cu:194-295, Half/main.cu:270-371), 2D x-z restriction.
//
// Work decomposition: a task is one warp's column of 128 x cells (4 per lane,
// 16-byte vector accesses) over a segment of zseg_m rows of one shot.  The
// warp walks its rows in order and keeps, per field that is differentiated
// along z, the rows of the stencil in registers: each row of each array is
// loaded (and, for COMP16, decoded) once per phase instead of once per
// neighbouring row.  x neighbours come from the adjacent lanes by warp
// shuffles; only lanes 0 and 31 load their outer neighbour.  The per-cell
// arithmetic after the derivatives is the tile kernels' own (v_tail, t_tail
// in stencil.cuh), so the results are bit-identical to theirs.
#include "shot.h"
#include "stencil.cuh"

namespace bpk {

constexpr int kMarchWarps = 4;
constexpr int kMarchThreads = kMarchWarps * 32;
constexpr int kMarchCells = 128;                 // x cells per task (4 per lane)
constexpr unsigned kFull = 0xffffffffu;
// Resident CTAs per SM the marching kernels are register-limited to (1 = no
// limit), and the warps per SM the z segments are sized for.  Measured on
// B200 (4040 x 2040, order 2): the lean form below at 8 CTAs (64 registers)
// with 8-row segments was the fastest setting tried (FP32 0.298, COMP16 0.474
// ms per step); the kernel stays slower than the tile kernels (0.221 / 0.394),
// so it is not the default.
#ifndef BP_MARCH_MINB
#define BP_MARCH_MINB 8
#endif
#ifndef BP_MARCH_WARPS_PER_SM
#define BP_MARCH_WARPS_PER_SM 64
#endif
// 1: no look-ahead; the coefficients and old state are loaded by the shared
// tail after the derivatives (as in the tile kernels), which keeps only the
// z windows live across rows.  0: row z+1's loads are all issued before row z
// is computed.
#ifndef BP_MARCH_LEAN
#define BP_MARCH_LEAN 1
#endif

// Binary search of the shot owning task t (tile0m ascending).
__device__ __forceinline__ int locate_shot_m(const ShotDesc* shots, int nshots, long long t) {
    int lo = 0, hi = nshots - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (shots[mid].tile0m <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Raw loads of the 4 cells of a row at flat index i; lanes past the end of
// the row load nothing (their values only reach masked cells through the
// shuffles).
template <class P>
__device__ __forceinline__ typename P::raw4 ldr_row(const void* p, const int8_t* lo, long long i, bool in) {
    return in ? P::ldr4(p, lo, i) : P::zero4();
}

// The outer neighbours of the warp's span of a row, raw: lane 0 loads
// f(x0 - k) and lane 31 f(x0 + 3 + k), k = 1..HW, clamped into the row as the
// tile kernels clamp them; the other lanes take theirs from the adjacent lanes.
template <int ORD, class P>
struct Edges {
    typename P::raw1 e[ORD / 2];
};
template <int ORD, class P>
__device__ __forceinline__ void ldr_edges(const void* p, const int8_t* lo, long long rowbase, int x0, int nx, int lane,
                                          Edges<ORD, P>& E) {
#pragma unroll
    for (int k = 1; k <= ORD / 2; k++) {
        if (lane == 0) E.e[k - 1] = P::ldr1(p, lo, rowbase + (x0 - k < 0 ? 0 : x0 - k));
        else if (lane == 31) E.e[k - 1] = P::ldr1(p, lo, rowbase + (x0 + 3 + k > nx - 1 ? nx - 1 : x0 + 3 + k));
        else E.e[k - 1] = P::zero1();
    }
}

// The span f(x0 - HW .. x0 + 3 + HW) of a row from the lane's own 4 cells,
// the adjacent lanes' cells (shuffles) and the loaded outer neighbours.  Every
// lane of the warp must call it.
template <int ORD, class P>
__device__ __forceinline__ void span_of(const typename P::real (&c)[4], const Edges<ORD, P>& E, int lane,
                                        typename P::real (&v)[4 + ORD]) {
    using R = typename P::real;
    constexpr int HW = ORD / 2;
#pragma unroll
    for (int j = 0; j < 4; j++) v[HW + j] = c[j];
#pragma unroll
    for (int k = 1; k <= HW; k++) {
        R l = __shfl_up_sync(kFull, c[4 - k], 1);
        R rr = __shfl_down_sync(kFull, c[k - 1], 1);
        if (lane == 0) l = P::dec1(E.e[k - 1]);
        if (lane == 31) rr = P::dec1(E.e[k - 1]);
        v[HW - k] = l;
        v[HW + 3 + k] = rr;
    }
}

// Window shift: w[i] = w[i + 1].
template <int N, class R>
__device__ __forceinline__ void shift(R (&w)[N][4]) {
#pragma unroll
    for (int i = 0; i + 1 < N; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) w[i][j] = w[i + 1][j];
}

// D+z from a window of rows z-HW+1 .. z+HW, D-z from rows z-HW .. z+HW-1, in
// the tile kernels' row-array form a[k] = row z + k - HW.
template <int ORD, class P>
__device__ __forceinline__ typename P::real dz_fwd(const typename P::real (&w)[ORD][4], int j, const ShotDesc& S) {
    typename P::real a[ORD + 1];
    a[0] = 0;
#pragma unroll
    for (int k = 1; k <= ORD; k++) a[k] = w[k - 1][j];
    return deriv_div<P>(rfwd<ORD>(a), S);
}
template <int ORD, class P>
__device__ __forceinline__ typename P::real dz_bwd(const typename P::real (&w)[ORD][4], int j, const ShotDesc& S) {
    typename P::real a[ORD + 1];
#pragma unroll
    for (int k = 0; k < ORD; k++) a[k] = w[k][j];
    a[ORD] = 0;
    return deriv_div<P>(rbwd<ORD>(a), S);
}

template <int ORD, class P, bool VPHASE>
__global__ void __launch_bounds__(kMarchThreads, BP_MARCH_MINB) k_march(const ShotDesc* __restrict__ shots, int nshots,
                                                         long long ntasks, int k) {
    using R = typename P::real;
    constexpr int HW = ORD / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ ShotDesc sd[kMarchWarps];
    const long long t = (long long)blockIdx.x * kMarchWarps + warp;
    if (t >= ntasks) return;                          // warp-uniform
    {
        // the warp's own copy of its shot's descriptor (tasks of one CTA may
        // belong to different shots of a batch)
        const int si = nshots == 1 ? 0 : locate_shot_m(shots, nshots, t);
        const long long* src = reinterpret_cast<const long long*>(shots + si);
        long long* dst = reinterpret_cast<long long*>(&sd[warp]);
        for (int w = lane; w < (int)(sizeof(ShotDesc) / 8); w += 32) dst[w] = src[w];
        __syncwarp();
    }
    const ShotDesc& S = sd[warp];
    const int it = *S.step_base + k;
    if (S.done || it >= S.nt) return;
    R r = (R)1;
    if constexpr (P::prec == BP_PREC_COMP16) r = S.rtab[it];
    const unsigned lt = (unsigned)(t - S.tile0m);   // tasks of one shot < 2^32
    const unsigned g = lt / (unsigned)S.ncol_m;
    const int col = (int)(lt - g * (unsigned)S.ncol_m);
    const int zb = HW + (int)g * S.zseg_m;
    const int ze = zb + S.zseg_m < S.nz - HW ? zb + S.zseg_m : S.nz - HW;
    const int x0 = col * kMarchCells + lane * 4;
    const int nx = S.nx;
    const bool in = x0 < nx;                          // the lane's cells lie in the row
    const bool act = x0 < nx - HW && x0 + 3 >= HW;    // the tile kernels' chunk test
    unsigned mask = 0;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (x0 + j >= HW && x0 + j < nx - HW) mask |= 1u << j;
    const long long sz = S.plane;
    auto at = [&](int z) { return (long long)z * sz + x0; };

    if constexpr (VPHASE) {
        // Everything row z reads that is not already in a window, loaded one
        // row ahead: txx(z); the newest window rows p(z+HW), tzz(z+HW),
        // txz(z+HW-1); the outer x neighbours of the spans of txx, p, txz at
        // row z; the V coefficients and old velocities at row z.
        struct Row {
            typename P::raw4 txx, p, zz, xz, rf, rho_x, c1_x, c2_x, vu_x, vw_x, rho_z, c1_z, c2_z, vu_z, vw_z;
            Edges<ORD, P> etxx, ep, exz;
        };
        auto issue_stress = [&](int z, Row& L) {
            const long long c = at(z), rb = (long long)z * sz;
            L.txx = ldr_row<P>(S.f[BP_F_TXX], S.flo[BP_F_TXX], c, in);
            L.p = ldr_row<P>(S.f[BP_F_P], S.flo[BP_F_P], at(z + HW), in);
            L.zz = ldr_row<P>(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], at(z + HW), in);
            L.xz = ldr_row<P>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], at(z + HW - 1), in);
            ldr_edges<ORD, P>(S.f[BP_F_TXX], S.flo[BP_F_TXX], rb, x0, nx, lane, L.etxx);
            ldr_edges<ORD, P>(S.f[BP_F_P], S.flo[BP_F_P], rb, x0, nx, lane, L.ep);
            ldr_edges<ORD, P>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], rb, x0, nx, lane, L.exz);
        };
        auto issue_coef = [&](int z, Row& L) {
            const long long c = at(z);
            L.rf = ldr_row<P>(S.vc[VC_RHOF], S.vclo[VC_RHOF], c, in);
            L.rho_x = ldr_row<P>(S.vc[VC_RHO_X], S.vclo[VC_RHO_X], c, in);
            L.c1_x = ldr_row<P>(S.vc[VC_CC1_X], S.vclo[VC_CC1_X], c, in);
            L.c2_x = ldr_row<P>(S.vc[VC_CC2_X], S.vclo[VC_CC2_X], c, in);
            L.vu_x = ldr_row<P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], c, in);
            L.vw_x = ldr_row<P>(S.f[BP_F_VWX], S.flo[BP_F_VWX], c, in);
            L.rho_z = ldr_row<P>(S.vc[VC_RHO_Z], S.vclo[VC_RHO_Z], c, in);
            L.c1_z = ldr_row<P>(S.vc[VC_CC1_Z], S.vclo[VC_CC1_Z], c, in);
            L.c2_z = ldr_row<P>(S.vc[VC_CC2_Z], S.vclo[VC_CC2_Z], c, in);
            L.vu_z = ldr_row<P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], c, in);
            L.vw_z = ldr_row<P>(S.f[BP_F_VWZ], S.flo[BP_F_VWZ], c, in);
        };
        // windows: p and tzz rows z-HW+1 .. z+HW (D+z), txz rows z-HW .. z+HW-1 (D-z)
        R wp[ORD][4], wzz[ORD][4], wxz[ORD][4];
#pragma unroll
        for (int w = 0; w + 1 < ORD; w++) {
            P::dec4(ldr_row<P>(S.f[BP_F_P], S.flo[BP_F_P], at(zb - HW + 1 + w), in), wp[w]);
            P::dec4(ldr_row<P>(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], at(zb - HW + 1 + w), in), wzz[w]);
            P::dec4(ldr_row<P>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], at(zb - HW + w), in), wxz[w]);
        }
        constexpr bool kLean = BP_MARCH_LEAN;
        Row L;
        if constexpr (!kLean) { issue_stress(zb, L); issue_coef(zb, L); }
        for (int z = zb; z < ze; z++) {
            Row N;
            if constexpr (kLean) issue_stress(z, L);
            else if (z + 1 < ze) { issue_stress(z + 1, N); issue_coef(z + 1, N); }   // next row in flight
            const long long c = at(z);
            R ct[4];
            P::dec4(L.txx, ct);
            P::dec4(L.p, wp[ORD - 1]);
            P::dec4(L.zz, wzz[ORD - 1]);
            P::dec4(L.xz, wxz[ORD - 1]);
            VState<R> V;
            if constexpr (!kLean) {
                P::dec4(L.rf, V.rf);
                P::dec4(L.rho_x, V.rho_x); P::dec4(L.c1_x, V.c1_x); P::dec4(L.c2_x, V.c2_x);
                P::dec4(L.vu_x, V.vu_x); P::dec4(L.vw_x, V.vw_x);
                P::dec4(L.rho_z, V.rho_z); P::dec4(L.c1_z, V.c1_z); P::dec4(L.c2_z, V.c2_z);
                P::dec4(L.vu_z, V.vu_z); P::dec4(L.vw_z, V.vw_z);
            }
            // derivatives of the old stresses (Float/main.cu:115-128)
            R v[4 + ORD];
            span_of<ORD, P>(ct, L.etxx, lane, v);                     // txx: D+x
#pragma unroll
            for (int j = 0; j < 4; j++) V.x1[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
            span_of<ORD, P>(wp[HW - 1], L.ep, lane, v);               // p: D+x
#pragma unroll
            for (int j = 0; j < 4; j++) V.s1[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
            span_of<ORD, P>(wxz[HW], L.exz, lane, v);                 // txz: D-x
#pragma unroll
            for (int j = 0; j < 4; j++) V.z2[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                V.x3[j] = dz_bwd<ORD, P>(wxz, j, S);                   // txz: D-z
                V.z1[j] = dz_fwd<ORD, P>(wzz, j, S);                   // tzz: D+z
                V.s3[j] = dz_fwd<ORD, P>(wp, j, S);                    // p: D+z
            }
            if (act) {
                if (P::prec == BP_PREC_COMP16 && r != (R)1) v_tail<2, ORD, P, !kLean, true>(S, c, x0, 0, z, r, mask, V);
                else v_tail<2, ORD, P, !kLean, false>(S, c, x0, 0, z, r, mask, V);
            }
            shift(wp);
            shift(wzz);
            shift(wxz);
            if constexpr (!kLean) L = N;
        }
    } else {
        // loaded one row ahead: vwx(z); the newest window rows vux(z+HW),
        // vuz(z+HW-1), vwz(z+HW-1); the outer x neighbours of the spans of
        // vux, vwx, vuz at row z; the moduli and old stresses at row z.
        struct Row {
            typename P::raw4 wx, ux, uz, wz, cC, cM, cH, cH2, mxz, op, oxx, ozz, oxz;
            Edges<ORD, P> eux, ewx, euz;
        };
        auto issue_vel = [&](int z, Row& L) {
            const long long c = at(z), rb = (long long)z * sz;
            L.wx = ldr_row<P>(S.f[BP_F_VWX], S.flo[BP_F_VWX], c, in);
            L.ux = ldr_row<P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], at(z + HW), in);
            L.uz = ldr_row<P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], at(z + HW - 1), in);
            L.wz = ldr_row<P>(S.f[BP_F_VWZ], S.flo[BP_F_VWZ], at(z + HW - 1), in);
            ldr_edges<ORD, P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], rb, x0, nx, lane, L.eux);
            ldr_edges<ORD, P>(S.f[BP_F_VWX], S.flo[BP_F_VWX], rb, x0, nx, lane, L.ewx);
            ldr_edges<ORD, P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], rb, x0, nx, lane, L.euz);
        };
        auto issue_coef = [&](int z, Row& L) {
            const long long c = at(z);
            L.cC = ldr_row<P>(S.tc[TC_C], S.tclo[TC_C], c, in);
            L.cM = ldr_row<P>(S.tc[TC_M], S.tclo[TC_M], c, in);
            L.cH = ldr_row<P>(S.tc[TC_H], S.tclo[TC_H], c, in);
            L.cH2 = ldr_row<P>(S.tc[TC_H2U], S.tclo[TC_H2U], c, in);
            L.mxz = ldr_row<P>(S.tc[TC_MUXZ], S.tclo[TC_MUXZ], c, in);
            L.op = ldr_row<P>(S.f[BP_F_P], S.flo[BP_F_P], c, in);
            L.oxx = ldr_row<P>(S.f[BP_F_TXX], S.flo[BP_F_TXX], c, in);
            L.ozz = ldr_row<P>(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], c, in);
            L.oxz = ldr_row<P>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], c, in);
        };
        // windows: vux rows z-HW+1 .. z+HW (D+z); vuz, vwz rows z-HW .. z+HW-1 (D-z)
        R wux[ORD][4], wuz[ORD][4], wwz[ORD][4];
#pragma unroll
        for (int w = 0; w + 1 < ORD; w++) {
            P::dec4(ldr_row<P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], at(zb - HW + 1 + w), in), wux[w]);
            P::dec4(ldr_row<P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], at(zb - HW + w), in), wuz[w]);
            P::dec4(ldr_row<P>(S.f[BP_F_VWZ], S.flo[BP_F_VWZ], at(zb - HW + w), in), wwz[w]);
        }
        constexpr bool kLean = BP_MARCH_LEAN;
        Row L;
        if constexpr (!kLean) { issue_vel(zb, L); issue_coef(zb, L); }
        for (int z = zb; z < ze; z++) {
            Row N;
            if constexpr (kLean) issue_vel(z, L);
            else if (z + 1 < ze) { issue_vel(z + 1, N); issue_coef(z + 1, N); }
            const long long c = at(z);
            R cwx[4];
            P::dec4(L.wx, cwx);
            P::dec4(L.ux, wux[ORD - 1]);
            P::dec4(L.uz, wuz[ORD - 1]);
            P::dec4(L.wz, wwz[ORD - 1]);
            TState<R> T;
            if constexpr (!kLean) {
                P::dec4(L.cC, T.cC); P::dec4(L.cM, T.cM); P::dec4(L.cH, T.cH); P::dec4(L.cH2, T.cH2);
                P::dec4(L.mxz, T.mxz);
                P::dec4(L.op, T.op); P::dec4(L.oxx, T.oxx); P::dec4(L.ozz, T.ozz); P::dec4(L.oxz, T.oxz);
                if (P::prec == BP_PREC_COMP16 && r != (R)1) {    // old state takes this step's rescale
                    scale4(T.op, r); scale4(T.oxx, r); scale4(T.ozz, r); scale4(T.oxz, r);
                }
            }
            // derivatives of this step's velocities (Float/main.cu:236-250)
            R v[4 + ORD];
            span_of<ORD, P>(wux[HW - 1], L.eux, lane, v);             // vux: D-x
#pragma unroll
            for (int j = 0; j < 4; j++) T.uxx[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
            span_of<ORD, P>(cwx, L.ewx, lane, v);                     // vwx: D-x
#pragma unroll
            for (int j = 0; j < 4; j++) T.wx[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
            span_of<ORD, P>(wuz[HW], L.euz, lane, v);                 // vuz: D+x
#pragma unroll
            for (int j = 0; j < 4; j++) T.uzx[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                T.uzz[j] = dz_bwd<ORD, P>(wuz, j, S);                   // vuz: D-z
                T.wz[j] = dz_bwd<ORD, P>(wwz, j, S);                    // vwz: D-z
                T.uxz[j] = dz_fwd<ORD, P>(wux, j, S);                   // vux: D+z
            }
            if (act) {
                if (P::prec == BP_PREC_COMP16 && r != (R)1) t_tail<2, ORD, P, !kLean, true>(S, c, x0, 0, z, r, mask, T);
                else t_tail<2, ORD, P, !kLean, false>(S, c, x0, 0, z, r, mask, T);
            }
            shift(wux);
            shift(wuz);
            shift(wwz);
            if constexpr (!kLean) L = N;
        }
    }
}

bool march_supported(int prec, int dim) { return dim == 2 && (prec == BP_PREC_FP32 || prec == BP_PREC_COMP16); }

bool march_default() { return false; }

int march_cells() { return kMarchCells; }

int march_zseg(long long ncol, int nrows, int sms) {
    // enough tasks for BP_MARCH_WARPS_PER_SM warps on every SM for a lone
    // shot; at least 8 rows so the window prologue stays small
    const long long want = (long long)sms * BP_MARCH_WARPS_PER_SM;
    long long L = (ncol * nrows + want - 1) / want;
    return (int)(L < 8 ? 8 : L);
}

template <int ORD, class P>
static cudaError_t launch_march_t(bool v, const ShotDesc* d, int nshots, long long ntasks, int k, cudaStream_t st) {
    const long long grid = (ntasks + kMarchWarps - 1) / kMarchWarps;
    if (grid <= 0) return cudaSuccess;
    if (v) k_march<ORD, P, true><<<(unsigned)grid, kMarchThreads, 0, st>>>(d, nshots, ntasks, k);
    else k_march<ORD, P, false><<<(unsigned)grid, kMarchThreads, 0, st>>>(d, nshots, ntasks, k);
    return cudaGetLastError();
}

cudaError_t launch_phase_march(int prec, int order, bool vphase, const ShotDesc* d, int nshots, long long ntasks,
                               int k, cudaStream_t st) {
    if (prec == BP_PREC_FP32)
        return order == 2 ? launch_march_t<2, PolF32>(vphase, d, nshots, ntasks, k, st)
                          : launch_march_t<4, PolF32>(vphase, d, nshots, ntasks, k, st);
    if (prec == BP_PREC_COMP16)
        return order == 2 ? launch_march_t<2, PolC16>(vphase, d, nshots, ntasks, k, st)
                          : launch_march_t<4, PolC16>(vphase, d, nshots, ntasks, k, st);
    return cudaErrorInvalidValue;
}

}  // namespace bpk

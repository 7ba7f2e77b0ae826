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
#include "common.cuh"

namespace bpk {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kSegCells = 128;

// Binary search of the shot owning tile t (tile0 ascending).
__device__ __forceinline__ int locate_shot(const ShotDesc* shots, int nshots, long long t) {
    int lo = 0, hi = nshots - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (shots[mid].tile0 <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class P>
__device__ __forceinline__ typename P::real deriv_div(typename P::real a, const ShotDesc& S) {
    // FP32: the reference divides by H.  q = a * (1/H) refined by one residual
    // step, q += (a - q H) * (1/H), with the exact fused residual a - q H,
    // matches the IEEE quotient a / H to within one ulp (equal in all but rare
    // near-tie cases) in 3 instructions instead of a full divide.
    // FP64 divides; COMP16 (own arithmetic) multiplies by 1/H.
    if constexpr (P::prec == BP_PREC_FP64) return a / (typename P::real)S.hd;
    else if constexpr (P::prec == BP_PREC_FP32) {
        const float q = a * S.inv_h;
        return __fmaf_rn(__fmaf_rn(-q, S.h, a), S.inv_h, q);
    } else return a * S.inv_h;
}

// Staggered difference from a span v[j] = f(x0 - HW + j).
template <int ORD, class R>
__device__ __forceinline__ R dfwd(const R* v, int j) {   // at x0+j+1/2
    constexpr int HW = ORD / 2;
    if constexpr (ORD == 2) return v[HW + j + 1] - v[HW + j];
    else return (R)1.125 * (v[HW + j + 1] - v[HW + j]) + (R)(-1.0 / 24.0) * (v[HW + j + 2] - v[HW + j - 1]);
}
template <int ORD, class R>
__device__ __forceinline__ R dbwd(const R* v, int j) {   // at x0+j-1/2
    constexpr int HW = ORD / 2;
    if constexpr (ORD == 2) return v[HW + j] - v[HW + j - 1];
    else return (R)1.125 * (v[HW + j] - v[HW + j - 1]) + (R)(-1.0 / 24.0) * (v[HW + j + 1] - v[HW + j - 2]);
}
// Difference across rows: a[k] = f(row + k - HW) for one cell.
template <int ORD, class R>
__device__ __forceinline__ R rfwd(const R* a) {
    constexpr int HW = ORD / 2;
    if constexpr (ORD == 2) return a[HW + 1] - a[HW];
    else return (R)1.125 * (a[HW + 1] - a[HW]) + (R)(-1.0 / 24.0) * (a[HW + 2] - a[HW - 1]);
}
template <int ORD, class R>
__device__ __forceinline__ R rbwd(const R* a) {
    constexpr int HW = ORD / 2;
    if constexpr (ORD == 2) return a[HW] - a[HW - 1];
    else return (R)1.125 * (a[HW] - a[HW - 1]) + (R)(-1.0 / 24.0) * (a[HW + 1] - a[HW - 2]);
}

// Load f(x0 - HW .. x0 + 3 + HW) of one row; x neighbours clamped into the row
// (clamped values only feed cells that are never updated).
template <int ORD, class P>
__device__ __forceinline__ void load_span(const void* p, const int8_t* lo, long long rowbase, int x0, int nx,
                                          typename P::real (&v)[4 + ORD]) {
    constexpr int HW = ORD / 2;
    typename P::real c[4];
    P::ld4(p, lo, rowbase + x0, c);
#pragma unroll
    for (int j = 0; j < 4; j++) v[HW + j] = c[j];
#pragma unroll
    for (int k = 1; k <= HW; k++) {
        int xl = x0 - k; xl = xl < 0 ? 0 : xl;
        int xr = x0 + 3 + k; xr = xr > nx - 1 ? nx - 1 : xr;
        v[HW - k] = P::ld1(p, lo, rowbase + xl);
        v[HW + 3 + k] = P::ld1(p, lo, rowbase + xr);
    }
}

// Load the 4 cells of rows row-HW .. row+HW (offsets along y or z).
template <int ORD, class P>
__device__ __forceinline__ void load_rows(const void* p, const int8_t* lo, long long c, long long stride,
                                          typename P::real (&a)[ORD + 1][4]) {
    constexpr int HW = ORD / 2;
#pragma unroll
    for (int k = 0; k <= ORD; k++) P::ld4(p, lo, c + (long long)(k - HW) * stride, a[k]);
}

template <class R>
__device__ __forceinline__ void scale4(R (&v)[4], R r) {
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] *= r;
}

// CPML memory update of one derivative slot for a 4-cell chunk
// (Float/main.cu:130-158):  ψ = ψ e + b (e prev + ∂),  prev = ∂,  ∂ += ψ,
// with b = -DT d / 2 precomputed.  The x axis has per-cell tables; the y and z
// axes one value per chunk.  Old ψ/prev are multiplied by the state rescale r.
template <class R>
__device__ __forceinline__ void cpml_x(R (&d)[4], R* psi, R* prev, const R* b, const R* e, int x0, R r) {
    R ps[4], pv[4];
#pragma unroll
    for (int j = 0; j < 4; j++) { ps[j] = psi[j] * r; pv[j] = prev[j] * r; }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R ee = e[x0 + j], bb = b[x0 + j];
        R np = ps[j] * ee + bb * (ee * pv[j] + d[j]);
        ps[j] = np;
        pv[j] = d[j];
        d[j] = d[j] + np;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) { psi[j] = ps[j]; prev[j] = pv[j]; }
}
template <class R>
__device__ __forceinline__ void cpml_s(R (&d)[4], R* psi, R* prev, R bb, R ee, R r) {
    R ps[4], pv[4];
#pragma unroll
    for (int j = 0; j < 4; j++) { ps[j] = psi[j] * r; pv[j] = prev[j] * r; }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R np = ps[j] * ee + bb * (ee * pv[j] + d[j]);
        ps[j] = np;
        pv[j] = d[j];
        d[j] = d[j] + np;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) { psi[j] = ps[j]; prev[j] = pv[j]; }
}

// Vector access helpers for the memory variables (ψ in fp32 or fp64).
template <class R>
struct PsiIO {
    __device__ __forceinline__ static void ld(const R* p, R (&v)[4]) {
        if constexpr (sizeof(R) == 4) {
            float4 t = *reinterpret_cast<const float4*>(p);
            v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
        } else {
            double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
        }
    }
    __device__ __forceinline__ static void st(R* p, const R (&v)[4]) {
        if constexpr (sizeof(R) == 4) {
            *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
            reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
        }
    }
};

// One derivative slot of one axis: memory variables k (ψ) and NS+k (prev) of
// the (phase, axis) slab array; fwd selects the half-grid profile.
template <int NS, class R>
__device__ __forceinline__ void cpml_slot(R (&d)[4], void* base, long long cells, int k, long long sidx,
                                          bool xaxis, int pos, int x0, const void* pb, const void* pe, R r) {
    R* ps = static_cast<R*>(base) + (long long)k * cells + sidx;
    R* pv = static_cast<R*>(base) + (long long)(NS + k) * cells + sidx;
    R psv[4], pvv[4];
    PsiIO<R>::ld(ps, psv);
    PsiIO<R>::ld(pv, pvv);
    const R* b = static_cast<const R*>(pb);
    const R* e = static_cast<const R*>(pe);
    if (xaxis) cpml_x<R>(d, psv, pvv, b, e, x0, r);
    else cpml_s<R>(d, psv, pvv, b[pos], e[pos], r);
    PsiIO<R>::st(ps, psv);
    PsiIO<R>::st(pv, pvv);
}

// Slab memory-variable index of a chunk for one axis, or -1 outside the slab.
__device__ __forceinline__ long long slab_index(const ShotDesc& S, int axis, int x0, int y, int z) {
    const Slab& sl = S.slab[axis];
    if (axis == 0) {
        int sx = sl.index(x0);
        if (sx < 0) return -1;
        return ((long long)z * S.ny + y) * sl.width + sx;
    } else if (axis == 1) {
        int sy = sl.index(y);
        if (sy < 0) return -1;
        return ((long long)z * sl.width + sy) * S.pitch + x0;
    } else {
        int sz = sl.index(z);
        if (sz < 0) return -1;
        return ((long long)sz * S.ny + y) * S.pitch + x0;
    }
}

// ---------------------------------------------------------------------------
// V phase for one 4-cell chunk: FD_V (Float/main.cu:103-191).
template <int DIM, int ORD, class P>
__device__ __forceinline__ void v_chunk(const ShotDesc& S, int x0, int y, int z, typename P::real r,
                                        unsigned mask) {
    using R = typename P::real;
    const long long sy = S.pitch, sz = S.plane;
    const long long c = x0 + (long long)y * sy + (long long)z * sz;
    const long long row = c - x0;

    // ---- derivatives of the old stresses (x1..s3, Float/main.cu:115-128) ----
    R x1[4], x3[4], s1[4], z1[4], z2[4], s3[4];
    R x2[4], y1[4], y2[4], y3[4], s2[4], z3[4];
    {
        R v[4 + ORD];
        load_span<ORD, P>(S.f[BP_F_TXX], S.flo[BP_F_TXX], row, x0, S.nx, v);       // txx: D+x
#pragma unroll
        for (int j = 0; j < 4; j++) x1[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
        load_span<ORD, P>(S.f[BP_F_P], S.flo[BP_F_P], row, x0, S.nx, v);           // p: D+x
#pragma unroll
        for (int j = 0; j < 4; j++) s1[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
        load_span<ORD, P>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], row, x0, S.nx, v);       // txz: D-x
#pragma unroll
        for (int j = 0; j < 4; j++) z2[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
        R a[ORD + 1][4];
        load_rows<ORD, P>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], c, sz, a);               // txz: D-z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            x3[j] = deriv_div<P>(rbwd<ORD>(t), S); }
        load_rows<ORD, P>(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], c, sz, a);               // tzz: D+z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            z1[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        load_rows<ORD, P>(S.f[BP_F_P], S.flo[BP_F_P], c, sz, a);                   // p: D+z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            s3[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        if constexpr (DIM == 3) {
            load_span<ORD, P>(S.f[BP_F_TXY], S.flo[BP_F_TXY], row, x0, S.nx, v);   // txy: D-x
#pragma unroll
            for (int j = 0; j < 4; j++) y2[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
            load_rows<ORD, P>(S.f[BP_F_TXY], S.flo[BP_F_TXY], c, sy, a);           // txy: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                x2[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_TYY], S.flo[BP_F_TYY], c, sy, a);           // tyy: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                y1[j] = deriv_div<P>(rfwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_TYZ], S.flo[BP_F_TYZ], c, sz, a);           // tyz: D-z
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                y3[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_TYZ], S.flo[BP_F_TYZ], c, sy, a);           // tyz: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                z3[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_P], S.flo[BP_F_P], c, sy, a);               // p: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                s2[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        }
    }
    // the rescale factor applies to old stresses: scale their derivatives
    if constexpr (P::prec == BP_PREC_COMP16) {
        scale4(x1, r); scale4(s1, r); scale4(z2, r); scale4(x3, r); scale4(z1, r); scale4(s3, r);
        if constexpr (DIM == 3) { scale4(x2, r); scale4(y1, r); scale4(y2, r); scale4(y3, r); scale4(s2, r); scale4(z3, r); }
    }
    // masked cells (never updated) feed zero derivatives into the memory variables
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (!(mask >> j & 1u)) {
            x1[j] = 0; s1[j] = 0; z2[j] = 0; x3[j] = 0; z1[j] = 0; s3[j] = 0;
            if constexpr (DIM == 3) { x2[j] = 0; y1[j] = 0; y2[j] = 0; y3[j] = 0; s2[j] = 0; z3[j] = 0; }
        }

    // ---- CPML memory variables on the slabs (Float/main.cu:130-158) ----
    {
        constexpr int NS = DIM == 3 ? 4 : 3;
        long long si = slab_index(S, 0, x0, y, z);
        if (si >= 0) {
            void* B = S.psiV[0];
            const long long n = S.slab_cells[0];
            cpml_slot<NS, R>(x1, B, n, 0, si, true, x0, x0, S.pb2[0], S.pe2[0], r);
            cpml_slot<NS, R>(s1, B, n, 1, si, true, x0, x0, S.pb2[0], S.pe2[0], r);
            cpml_slot<NS, R>(z2, B, n, 2, si, true, x0, x0, S.pb[0], S.pe[0], r);
            if constexpr (DIM == 3) cpml_slot<NS, R>(y2, B, n, 3, si, true, x0, x0, S.pb[0], S.pe[0], r);
        }
        if constexpr (DIM == 3) {
            si = slab_index(S, 1, x0, y, z);
            if (si >= 0) {
                void* B = S.psiV[1];
                const long long n = S.slab_cells[1];
                cpml_slot<NS, R>(x2, B, n, 0, si, false, y, x0, S.pb[1], S.pe[1], r);
                cpml_slot<NS, R>(y1, B, n, 1, si, false, y, x0, S.pb2[1], S.pe2[1], r);
                cpml_slot<NS, R>(s2, B, n, 2, si, false, y, x0, S.pb2[1], S.pe2[1], r);
                cpml_slot<NS, R>(z3, B, n, 3, si, false, y, x0, S.pb[1], S.pe[1], r);
            }
        }
        si = slab_index(S, 2, x0, y, z);
        if (si >= 0) {
            void* B = S.psiV[2];
            const long long n = S.slab_cells[2];
            cpml_slot<NS, R>(x3, B, n, 0, si, false, z, x0, S.pb[2], S.pe[2], r);
            cpml_slot<NS, R>(z1, B, n, 1, si, false, z, x0, S.pb2[2], S.pe2[2], r);
            cpml_slot<NS, R>(s3, B, n, 2, si, false, z, x0, S.pb2[2], S.pe2[2], r);
            if constexpr (DIM == 3) cpml_slot<NS, R>(y3, B, n, 3, si, false, z, x0, S.pb[2], S.pe[2], r);
        }
    }

    // ---- stress divergence per axis ----
    R sumx[4], sumz[4], sumy[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (DIM == 3) {
            sumx[j] = x1[j] + x2[j] + x3[j];
            sumy[j] = y1[j] + y2[j] + y3[j];
            sumz[j] = z1[j] + z2[j] + z3[j];
        } else {
            sumx[j] = x1[j] + x3[j];
            sumz[j] = z1[j] + z2[j];
        }
    }

    // ---- velocity updates per axis (Float/main.cu:106-113,160-190) ----
    R rf[4];
    P::ld4(S.vc[VC_RHOF], S.vclo[VC_RHOF], c, rf);
    auto axis_update = [&](const R (&sum)[4], const R (&dp)[4], int fu, int fw, int crho, int ccc1, int ccc2) {
        R rho[4], c1[4], c2[4], vu[4], vw[4];
        P::ld4(S.vc[crho], S.vclo[crho], c, rho);
        P::ld4(S.vc[ccc1], S.vclo[ccc1], c, c1);
        P::ld4(S.vc[ccc2], S.vclo[ccc2], c, c2);
        P::ld4(S.f[fu], S.flo[fu], c, vu);
        P::ld4(S.f[fw], S.flo[fw], c, vw);
        R nu[4], nw[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) {
                // Half/main.cu:256-262 with Bt = (rhof rho^-1) Bp formed here
                R wo = vw[j] * r, uo = vu[j] * r;
                R rr = rf[j] * rho[j];                    // rhof * rho^-1
                R wn = c1[j] * wo - (rr * c2[j]) * sum[j] - c2[j] * dp[j];
                nw[j] = wn;
                nu[j] = uo + rho[j] * sum[j] - rr * (wn - wo);
            } else {
                R wo = vw[j];
                R wn = (c1[j] == (R)0) ? (R)0
                                       : (wo * c2[j] - S.dtr<R>() * (rf[j] * rho[j] * sum[j] + dp[j])) / c1[j];
                nw[j] = wn;
                nu[j] = vu[j] + S.dtr<R>() * rho[j] * sum[j] - rf[j] * rho[j] * (wn - wo);
            }
            if (!(mask >> j & 1u)) { nw[j] = vw[j]; nu[j] = vu[j]; }
        }
        P::st4(S.f[fw], S.flo[fw], c, nw);
        P::st4(S.f[fu], S.flo[fu], c, nu);
    };
    axis_update(sumx, s1, BP_F_VUX, BP_F_VWX, VC_RHO_X, VC_CC1_X, VC_CC2_X);
    if constexpr (DIM == 3) axis_update(sumy, s2, BP_F_VUY, BP_F_VWY, VC_RHO_Y, VC_CC1_Y, VC_CC2_Y);
    axis_update(sumz, s3, BP_F_VUZ, BP_F_VWZ, VC_RHO_Z, VC_CC1_Z, VC_CC2_Z);
}

// ---------------------------------------------------------------------------
// T phase for one 4-cell chunk: FD_T (Float/main.cu:232-294).
template <int DIM, int ORD, class P>
__device__ __forceinline__ void t_chunk(const ShotDesc& S, int x0, int y, int z, typename P::real r,
                                        unsigned mask) {
    using R = typename P::real;
    const long long sy = S.pitch, sz = S.plane;
    const long long c = x0 + (long long)y * sy + (long long)z * sz;
    const long long row = c - x0;

    R uxx[4], uzz[4], wx[4], wz[4], uxz[4], uzx[4];
    R uyy[4], wy[4], uxy[4], uyx[4], uyz[4], uzy[4];
    {
        R v[4 + ORD];
        R a[ORD + 1][4];
        load_span<ORD, P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], row, x0, S.nx, v);       // vux: D-x
#pragma unroll
        for (int j = 0; j < 4; j++) uxx[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
        load_span<ORD, P>(S.f[BP_F_VWX], S.flo[BP_F_VWX], row, x0, S.nx, v);       // vwx: D-x
#pragma unroll
        for (int j = 0; j < 4; j++) wx[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
        load_span<ORD, P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], row, x0, S.nx, v);       // vuz: D+x
#pragma unroll
        for (int j = 0; j < 4; j++) uzx[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
        load_rows<ORD, P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], c, sz, a);               // vuz: D-z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            uzz[j] = deriv_div<P>(rbwd<ORD>(t), S); }
        load_rows<ORD, P>(S.f[BP_F_VWZ], S.flo[BP_F_VWZ], c, sz, a);               // vwz: D-z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            wz[j] = deriv_div<P>(rbwd<ORD>(t), S); }
        load_rows<ORD, P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], c, sz, a);               // vux: D+z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            uxz[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        if constexpr (DIM == 3) {
            load_span<ORD, P>(S.f[BP_F_VUY], S.flo[BP_F_VUY], row, x0, S.nx, v);   // vuy: D+x
#pragma unroll
            for (int j = 0; j < 4; j++) uyx[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
            load_rows<ORD, P>(S.f[BP_F_VUY], S.flo[BP_F_VUY], c, sy, a);           // vuy: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uyy[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_VWY], S.flo[BP_F_VWY], c, sy, a);           // vwy: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                wy[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_VUX], S.flo[BP_F_VUX], c, sy, a);           // vux: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uxy[j] = deriv_div<P>(rfwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_VUY], S.flo[BP_F_VUY], c, sz, a);           // vuy: D+z
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uyz[j] = deriv_div<P>(rfwd<ORD>(t), S); }
            load_rows<ORD, P>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], c, sy, a);           // vuz: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uzy[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (!(mask >> j & 1u)) {
            uxx[j] = 0; wx[j] = 0; uzx[j] = 0; uzz[j] = 0; wz[j] = 0; uxz[j] = 0;
            if constexpr (DIM == 3) { uyx[j] = 0; uyy[j] = 0; wy[j] = 0; uxy[j] = 0; uyz[j] = 0; uzy[j] = 0; }
        }

    // ---- CPML (Float/main.cu:252-285).  The velocities are this step's, but the
    // stored ψ/prev of this phase are old state and take the rescale r ----
    {
        constexpr int NS = DIM == 3 ? 4 : 3;
        long long si = slab_index(S, 0, x0, y, z);
        if (si >= 0) {
            void* B = S.psiT[0];
            const long long n = S.slab_cells[0];
            cpml_slot<NS, R>(uxx, B, n, 0, si, true, x0, x0, S.pb[0], S.pe[0], r);
            cpml_slot<NS, R>(wx, B, n, 1, si, true, x0, x0, S.pb[0], S.pe[0], r);
            cpml_slot<NS, R>(uzx, B, n, 2, si, true, x0, x0, S.pb2[0], S.pe2[0], r);
            if constexpr (DIM == 3) cpml_slot<NS, R>(uyx, B, n, 3, si, true, x0, x0, S.pb2[0], S.pe2[0], r);
        }
        if constexpr (DIM == 3) {
            si = slab_index(S, 1, x0, y, z);
            if (si >= 0) {
                void* B = S.psiT[1];
                const long long n = S.slab_cells[1];
                cpml_slot<NS, R>(uyy, B, n, 0, si, false, y, x0, S.pb[1], S.pe[1], r);
                cpml_slot<NS, R>(wy, B, n, 1, si, false, y, x0, S.pb[1], S.pe[1], r);
                cpml_slot<NS, R>(uxy, B, n, 2, si, false, y, x0, S.pb2[1], S.pe2[1], r);
                cpml_slot<NS, R>(uzy, B, n, 3, si, false, y, x0, S.pb2[1], S.pe2[1], r);
            }
        }
        si = slab_index(S, 2, x0, y, z);
        if (si >= 0) {
            void* B = S.psiT[2];
            const long long n = S.slab_cells[2];
            cpml_slot<NS, R>(uzz, B, n, 0, si, false, z, x0, S.pb[2], S.pe[2], r);
            cpml_slot<NS, R>(wz, B, n, 1, si, false, z, x0, S.pb[2], S.pe[2], r);
            cpml_slot<NS, R>(uxz, B, n, 2, si, false, z, x0, S.pb2[2], S.pe2[2], r);
            if constexpr (DIM == 3) cpml_slot<NS, R>(uyz, B, n, 3, si, false, z, x0, S.pb2[2], S.pe2[2], r);
        }
    }

    // ---- pressure and stress updates (Float/main.cu:287-293) ----
    R cC[4], cM[4], cH[4], cH2[4];
    P::ld4(S.tc[TC_C], S.tclo[TC_C], c, cC);
    P::ld4(S.tc[TC_M], S.tclo[TC_M], c, cM);
    P::ld4(S.tc[TC_H], S.tclo[TC_H], c, cH);
    P::ld4(S.tc[TC_H2U], S.tclo[TC_H2U], c, cH2);
    const R dt = S.dtr<R>();
    auto old4 = [&](int f, R (&v)[4]) {
        P::ld4(S.f[f], S.flo[f], c, v);
        if constexpr (P::prec == BP_PREC_COMP16) scale4(v, r);
    };
    auto store4 = [&](int f, R (&nv)[4], const R (&ov)[4]) {
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (!(mask >> j & 1u)) nv[j] = ov[j];
        P::st4(S.f[f], S.flo[f], c, nv);
    };
    R o[4], n[4];
    if constexpr (DIM == 3) {
        old4(BP_F_P, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] - cC[j] * (uxx[j] + uyy[j] + uzz[j]) - cM[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] - dt * (cC[j] * (uxx[j] + uyy[j] + uzz[j]) + cM[j] * (wx[j] + wy[j] + wz[j]));
        }
        store4(BP_F_P, n, o);
        old4(BP_F_TXX, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * (uyy[j] + uzz[j]) + cH[j] * uxx[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * (uyy[j] + uzz[j]) + cH[j] * uxx[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        store4(BP_F_TXX, n, o);
        old4(BP_F_TYY, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * (uxx[j] + uzz[j]) + cH[j] * uyy[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * (uxx[j] + uzz[j]) + cH[j] * uyy[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        store4(BP_F_TYY, n, o);
        old4(BP_F_TZZ, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * (uxx[j] + uyy[j]) + cH[j] * uzz[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * (uxx[j] + uyy[j]) + cH[j] * uzz[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        store4(BP_F_TZZ, n, o);
        R mu[4];
        P::ld4(S.tc[TC_MUXY], S.tclo[TC_MUXY], c, mu);
        old4(BP_F_TXY, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = o[j] + mu[j] * (uxy[j] + uyx[j]);
            else n[j] = o[j] + mu[j] * dt * (uxy[j] + uyx[j]);
        }
        store4(BP_F_TXY, n, o);
        P::ld4(S.tc[TC_MUYZ], S.tclo[TC_MUYZ], c, mu);
        old4(BP_F_TYZ, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = o[j] + mu[j] * (uyz[j] + uzy[j]);
            else n[j] = o[j] + mu[j] * dt * (uyz[j] + uzy[j]);
        }
        store4(BP_F_TYZ, n, o);
        P::ld4(S.tc[TC_MUXZ], S.tclo[TC_MUXZ], c, mu);
        old4(BP_F_TXZ, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = o[j] + mu[j] * (uxz[j] + uzx[j]);
            else n[j] = o[j] + mu[j] * dt * (uxz[j] + uzx[j]);
        }
        store4(BP_F_TXZ, n, o);
    } else {
        old4(BP_F_P, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] - cC[j] * (uxx[j] + uzz[j]) - cM[j] * (wx[j] + wz[j]);
            else
                n[j] = o[j] - dt * (cC[j] * (uxx[j] + uzz[j]) + cM[j] * (wx[j] + wz[j]));
        }
        store4(BP_F_P, n, o);
        old4(BP_F_TXX, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * uzz[j] + cH[j] * uxx[j] + cC[j] * (wx[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * uzz[j] + cH[j] * uxx[j] + cC[j] * (wx[j] + wz[j]));
        }
        store4(BP_F_TXX, n, o);
        old4(BP_F_TZZ, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * uxx[j] + cH[j] * uzz[j] + cC[j] * (wx[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * uxx[j] + cH[j] * uzz[j] + cC[j] * (wx[j] + wz[j]));
        }
        store4(BP_F_TZZ, n, o);
        R mu[4];
        P::ld4(S.tc[TC_MUXZ], S.tclo[TC_MUXZ], c, mu);
        old4(BP_F_TXZ, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = o[j] + mu[j] * (uxz[j] + uzx[j]);
            else n[j] = o[j] + mu[j] * dt * (uxz[j] + uzx[j]);
        }
        store4(BP_F_TXZ, n, o);
    }
}

// ---------------------------------------------------------------------------
// Tile loop shared by both phases.
template <int DIM, int ORD, class P, bool VPHASE>
__global__ void __launch_bounds__(kThreads) k_phase(const ShotDesc* __restrict__ shots, int nshots,
                                                     long long ntiles, int k) {
    using R = typename P::real;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // The descriptor of the tile's shot is staged in shared memory whenever the
    // shot changes, so the ~100 pointers and extents the chunk code reads are
    // shared-memory broadcasts instead of per-warp global loads.
    __shared__ ShotDesc sdesc;
    int cur = -1;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int si = nshots == 1 ? 0 : locate_shot(shots, nshots, t);
        if (si != cur) {                      // uniform across the CTA
            __syncthreads();
            const long long* src = reinterpret_cast<const long long*>(shots + si);
            long long* dst = reinterpret_cast<long long*>(&sdesc);
            for (int w = threadIdx.x; w < (int)(sizeof(ShotDesc) / 8); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            cur = si;
        }
        const ShotDesc& S = sdesc;
        const int it = *S.step_base + k;
        if (S.done || it >= S.nt) continue;
        const long long lt = t - S.tile0;
        const int seg = (int)(lt % S.nseg);
        const int row = (int)(lt / S.nseg) * kWarps + warp;
        if (row >= S.nrows) continue;
        int y, z;
        if constexpr (DIM == 3) { y = row % S.ny; z = row / S.ny; }
        else { y = 0; z = row; }
        const int hw = ORD / 2;
        if (z < hw || z >= S.nz - hw) continue;
        if (DIM == 3 && (y < hw || y >= S.ny - hw)) continue;
        const int x0 = seg * kSegCells + lane * 4;
        if (x0 >= S.nx - hw || x0 + 3 < hw) continue;
        unsigned mask = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (x0 + j >= hw && x0 + j < S.nx - hw) mask |= 1u << j;
        R r = (R)1;
        if constexpr (P::prec == BP_PREC_COMP16) r = S.rtab[it];
        if constexpr (VPHASE) v_chunk<DIM, ORD, P>(S, x0, y, z, r, mask);
        else t_chunk<DIM, ORD, P>(S, x0, y, z, r, mask);
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
__device__ __forceinline__ typename P::real read_phys(const ShotDesc& S, int f, long long i, typename P::real sc) {
    return P::ld1(S.f[f], S.flo[f], i) * sc;
}

template <class P>
__device__ __forceinline__ void inject(const ShotDesc& S, int it) {
    using R = typename P::real;
    if (!S.src_idx_valid || it >= S.nt) return;
    const long long i = S.src_idx;
    R I;
    if constexpr (P::prec == BP_PREC_FP64) I = static_cast<const double*>(S.wavelet)[it];
    else I = static_cast<const float*>(S.wavelet)[it];
    // COMP16: the sample enters at the scale the state has when it is added
    // (that of step it-1); step it's rescale factor then carries it to dyn[it].
    if constexpr (P::prec == BP_PREC_COMP16) I = I * S.inj_scale * (it > 0 ? S.dyn[it - 1] : 1.0f);
    if (S.src_mask & BP_SRC_TAU) {
        P::st1(S.f[BP_F_TXX], S.flo[BP_F_TXX], i, P::ld1(S.f[BP_F_TXX], S.flo[BP_F_TXX], i) + I);
        if (S.dim == 3) P::st1(S.f[BP_F_TYY], S.flo[BP_F_TYY], i, P::ld1(S.f[BP_F_TYY], S.flo[BP_F_TYY], i) + I);
        P::st1(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], i, P::ld1(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], i) + I);
    }
    if (S.src_mask & BP_SRC_P) P::st1(S.f[BP_F_P], S.flo[BP_F_P], i, P::ld1(S.f[BP_F_P], S.flo[BP_F_P], i) - I);
}

template <class P>
__global__ void k_post(const ShotDesc* __restrict__ shots, int k, int do_record) {
    using R = typename P::real;
    const ShotDesc& S = shots[blockIdx.y];
    const int it = *S.step_base + k;
    if (S.done || it >= S.nt) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (do_record && r < S.nrec && it < S.nt) {
        const long long i = S.rec_idx[r];
        R ss = (R)1, sv = (R)1;
        if constexpr (P::prec == BP_PREC_COMP16) {
            const float d = 1.0f / S.dyn[it];
            ss = S.out_stress * d;
            sv = S.out_vel * d;
        }
        R v[BP_NTRACE];
        v[BP_TR_TXX] = read_phys<P>(S, BP_F_TXX, i, ss);
        v[BP_TR_TZZ] = read_phys<P>(S, BP_F_TZZ, i, ss);
        v[BP_TR_VUX] = read_phys<P>(S, BP_F_VUX, i, sv);
        v[BP_TR_VWX] = read_phys<P>(S, BP_F_VWX, i, sv);
        v[BP_TR_P] = read_phys<P>(S, BP_F_P, i, ss);
        const long long cs = (long long)S.nrec * S.nt;
#pragma unroll
        for (int q = 0; q < BP_NTRACE; q++) {
            S.traces[q * cs + (long long)r * S.nt + it] = (float)v[q];
            if constexpr (P::prec == BP_PREC_FP64) S.traces64[q * cs + (long long)r * S.nt + it] = v[q];
        }
    }
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
template <class P>
struct Launch {
    static cudaError_t phase(int dim, int order, bool v, const ShotDesc* d_shots, int nshots, long long ntiles,
                             int k, int grid, cudaStream_t st) {
#define BPK_LAUNCH(D, O)                                                                              \
    if (dim == D && order == O) {                                                                     \
        if (v) k_phase<D, O, P, true><<<grid, kThreads, 0, st>>>(d_shots, nshots, ntiles, k);         \
        else k_phase<D, O, P, false><<<grid, kThreads, 0, st>>>(d_shots, nshots, ntiles, k);          \
        return cudaGetLastError();                                                                    \
    }
        BPK_LAUNCH(2, 2) BPK_LAUNCH(2, 4) BPK_LAUNCH(3, 2) BPK_LAUNCH(3, 4)
#undef BPK_LAUNCH
        return cudaErrorInvalidValue;
    }
};

}  // namespace bpk

// C++ entry points used by the host code (sim.cu, batch.cu).
namespace bpk {
cudaError_t launch_phase(int prec, int dim, int order, bool vphase, const ShotDesc* d_shots, int nshots,
                         long long ntiles, int k, int grid, cudaStream_t st) {
    if (prec == BP_PREC_FP32) return Launch<PolF32>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st);
    if (prec == BP_PREC_COMP16) return Launch<PolC16>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st);
    return Launch<PolF64>::phase(dim, order, vphase, d_shots, nshots, ntiles, k, grid, st);
}

cudaError_t launch_post(int prec, const ShotDesc* d_shots, int nshots, int max_rec, int k, int do_record,
                        cudaStream_t st) {
    dim3 grid((max_rec + 127) / 128 > 0 ? (max_rec + 127) / 128 : 1, nshots);
    if (prec == BP_PREC_FP32) k_post<PolF32><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    else if (prec == BP_PREC_COMP16) k_post<PolC16><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    else k_post<PolF64><<<grid, 128, 0, st>>>(d_shots, k, do_record);
    return cudaGetLastError();
}

cudaError_t launch_inject(int prec, const ShotDesc* d_shots, int nshots, int k, cudaStream_t st) {
    int g = (nshots + 127) / 128;
    if (prec == BP_PREC_FP32) k_inject<PolF32><<<g, 128, 0, st>>>(d_shots, nshots, k);
    else if (prec == BP_PREC_COMP16) k_inject<PolC16><<<g, 128, 0, st>>>(d_shots, nshots, k);
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
    else k_snapshot<PolF64><<<296, 256, 0, st>>>(d_shots, shot, f, slice_y, out, it);
    return cudaGetLastError();
}

cudaError_t launch_field_f64(int prec, const ShotDesc* d_shots, int f, double* out, cudaStream_t st) {
    if (prec == BP_PREC_FP32) k_field_f64<PolF32><<<296, 256, 0, st>>>(d_shots, f, out);
    else if (prec == BP_PREC_COMP16) k_field_f64<PolC16><<<296, 256, 0, st>>>(d_shots, f, out);
    else k_field_f64<PolF64><<<296, 256, 0, st>>>(d_shots, f, out);
    return cudaGetLastError();
}

int phase_occupancy(int prec, int dim, int order, bool vphase) {
    int n = 0;
    const void* fn = nullptr;
#define BPK_FN(PP, D, O)                                                                   \
    if (dim == D && order == O)                                                            \
        fn = vphase ? (const void*)k_phase<D, O, PP, true> : (const void*)k_phase<D, O, PP, false>;
    if (prec == BP_PREC_FP32) { BPK_FN(PolF32, 2, 2) BPK_FN(PolF32, 2, 4) BPK_FN(PolF32, 3, 2) BPK_FN(PolF32, 3, 4) }
    else if (prec == BP_PREC_COMP16) { BPK_FN(PolC16, 2, 2) BPK_FN(PolC16, 2, 4) BPK_FN(PolC16, 3, 2) BPK_FN(PolC16, 3, 4) }
    else { BPK_FN(PolF64, 2, 2) BPK_FN(PolF64, 2, 4) BPK_FN(PolF64, 3, 2) BPK_FN(PolF64, 3, 4) }
#undef BPK_FN
    if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_coef(int prec, const ShotDesc* d_shots, int which, float* out, cudaStream_t st) {
    if (prec == BP_PREC_FP32) k_coef<PolF32><<<296, 256, 0, st>>>(d_shots, which, out);
    else if (prec == BP_PREC_COMP16) k_coef<PolC16><<<296, 256, 0, st>>>(d_shots, which, out);
    else k_coef<PolF64><<<296, 256, 0, st>>>(d_shots, which, out);
    return cudaGetLastError();
}

int phase_threads() { return kThreads; }
int tile_rows() { return kWarps; }
int seg_cells() { return kSegCells; }
}  // namespace bpk

// stencil.cuh - per-chunk stencil arithmetic shared by the phase kernels:
// staggered differences, the division by H, span/row loads, the CPML memory
// update, and the tails of FD_V / FD_T (rescale, mask, CPML, update, store)
// that both the tile kernels (step.cu) and the marching kernels
// (step_march.cu) call, so both produce bit-identical results.
#pragma once
#include "common.cuh"

namespace bpk {

template <class P>
__device__ __forceinline__ typename P::real deriv_div(typename P::real a, const ShotDesc& S) {
    // FP32: the reference divides by H.  q = a * (1/H) refined by one residual
    // step, q += (a - q H) * (1/H), with the exact fused residual a - q H,
    // matches the IEEE quotient a / H to within one ulp (equal in all but rare
    // near-tie cases) in 3 instructions instead of a full divide.
    // FP64 divides; COMP16 (own arithmetic) multiplies by 1/H.  PolF32R takes
    // the IEEE quotient like the reference; a zero dividend (the quiet grid
    // ahead of the wavefront), which sends the divide routine down its slow
    // path, gives the same signed zero as a product.
    if constexpr (P::prec == BP_PREC_FP64) return a / (typename P::real)S.hd;
    else if constexpr (P::prec == BP_PREC_FP32 && P::exact) return a == 0.0f ? a * S.inv_h : __fdiv_rn(a, S.h);
    else if constexpr (P::prec == BP_PREC_FP32) {
        const float q = a * S.inv_h;
        return __fmaf_rn(__fmaf_rn(-q, S.h, a), S.inv_h, q);
    } else return a * S.inv_h;
}

// A difference along z divided by the row spacing: H on a uniform grid
// (deriv_div), the row's factor on a variable one (PolF32G; FWD: the forward
// difference of rows z, z+1, else the backward one of rows z-1, z).
template <class P, bool FWD>
__device__ __forceinline__ typename P::real deriv_z(typename P::real a, const ShotDesc& S, int z) {
    if constexpr (P::graded) return __fmul_rn(a, S.zf[FWD ? z : S.nz + z]);   // never contracted into a later add
    else return deriv_div<P>(a, S);
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
template <int ORD, class P, bool NC = kReadOnlyPath>
__device__ __forceinline__ void load_span(const void* p, const int8_t* lo, cidx rowbase, int x0, int nx,
                                          typename P::real (&v)[4 + ORD]) {
    constexpr int HW = ORD / 2;
    typename P::real c[4];
    P::template ld4<NC>(p, lo, rowbase + x0, c);
#pragma unroll
    for (int j = 0; j < 4; j++) v[HW + j] = c[j];
#pragma unroll
    for (int k = 1; k <= HW; k++) {
        int xl = x0 - k; xl = xl < 0 ? 0 : xl;
        int xr = x0 + 3 + k; xr = xr > nx - 1 ? nx - 1 : xr;
        v[HW - k] = P::template ld1<NC>(p, lo, rowbase + xl);
        v[HW + 3 + k] = P::template ld1<NC>(p, lo, rowbase + xr);
    }
}

// Load the 4 cells of rows row-HW .. row+HW (offsets along y or z).
template <int ORD, class P, bool NC = kReadOnlyPath>
__device__ __forceinline__ void load_rows(const void* p, const int8_t* lo, cidx c, cidx stride,
                                          typename P::real (&a)[ORD + 1][4]) {
    constexpr int HW = ORD / 2;
#pragma unroll
    for (int k = 0; k <= ORD; k++) P::template ld4<NC>(p, lo, c + (k - HW) * stride, a[k]);
}

// Product by the COMP16 rescale factor, never fused into a neighbouring add:
// the kernels skip it when the factor is exactly 1 (all steps but one in a
// hundred), and x * 1 == x only holds if no FMA ever absorbs the product.
template <class R>
__device__ __forceinline__ R mulr(R x, R r) {
    if constexpr (sizeof(R) == 4) return __fmul_rn(x, r);
    else return __dmul_rn(x, r);
}
template <class R>
__device__ __forceinline__ void scale4(R (&v)[4], R r) {
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = mulr(v[j], r);
}

// New ψ of one cell: ψ e + b (e prev + ∂).  EX (FP32 only): e prev + ∂ fused,
// then added times b to the float product ψ e with one rounding, as the
// reference's double-promoted expression rounds it (Float/main.cu:130-158).
template <bool EX, class R>
__device__ __forceinline__ R cpml_psi(R ps, R pv, R d, R bb, R ee) {
    if constexpr (EX) return __fmaf_rn(bb, __fmaf_rn(ee, pv, d), __fmul_rn(ps, ee));
    else return ps * ee + bb * (ee * pv + d);
}

// CPML memory update of one derivative slot for a 4-cell chunk
// (Float/main.cu:130-158):  ψ = ψ e + b (e prev + ∂),  prev = ∂,  ∂ += ψ,
// with b = -DT d / 2 precomputed.  The x axis has per-cell tables; the y and z
// axes one value per chunk.  Old ψ/prev are multiplied by the state rescale r.
template <bool RS, class R, bool EX = false>
__device__ __forceinline__ void cpml_x(R (&d)[4], R* psi, R* prev, const R* b, const R* e, int x0, R r) {
    R ps[4], pv[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        ps[j] = RS ? mulr(psi[j], r) : psi[j];
        pv[j] = RS ? mulr(prev[j], r) : prev[j];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R ee = e[x0 + j], bb = b[x0 + j];
        R np = cpml_psi<EX>(ps[j], pv[j], d[j], bb, ee);
        ps[j] = np;
        pv[j] = d[j];
        d[j] = d[j] + np;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) { psi[j] = ps[j]; prev[j] = pv[j]; }
}
template <bool RS, class R, bool EX = false>
__device__ __forceinline__ void cpml_s(R (&d)[4], R* psi, R* prev, R bb, R ee, R r) {
    R ps[4], pv[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        ps[j] = RS ? mulr(psi[j], r) : psi[j];
        pv[j] = RS ? mulr(prev[j], r) : prev[j];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R np = cpml_psi<EX>(ps[j], pv[j], d[j], bb, ee);
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
template <int NS, bool RS, class R, bool EX = false>
__device__ __forceinline__ void cpml_slot(R (&d)[4], void* base, long long cells, int k, cidx sidx,
                                          bool xaxis, int pos, int x0, const void* pb, const void* pe, R r,
                                          void* out = nullptr, bool st = true) {
    R* ps = static_cast<R*>(base) + (long long)k * cells + sidx;
    R* pv = static_cast<R*>(base) + (long long)(NS + k) * cells + sidx;
    R psv[4], pvv[4];
    PsiIO<R>::ld(ps, psv);
    PsiIO<R>::ld(pv, pvv);
    const R* b = static_cast<const R*>(pb);
    const R* e = static_cast<const R*>(pe);
    if (xaxis) cpml_x<RS, R, EX>(d, psv, pvv, b, e, x0, r);
    else cpml_s<RS, R, EX>(d, psv, pvv, b[pos], e[pos], r);
    if (out) {       // double-buffered memory variables: the new values go to `out`
        ps = static_cast<R*>(out) + (long long)k * cells + sidx;
        pv = static_cast<R*>(out) + (long long)(NS + k) * cells + sidx;
    }
    if (st) {
        PsiIO<R>::st(ps, psv);
        PsiIO<R>::st(pv, pvv);
    }
}

// Slab memory-variable index of a chunk for one axis, or -1 outside the slab.
__device__ __forceinline__ cidx slab_index(const ShotDesc& S, int axis, int x0, int y, int z) {
    const Slab& sl = S.slab[axis];
    if (axis == 0) {
        int sx = sl.index(x0);
        if (sx < 0) return -1;
        return (z * S.ny + y) * sl.width + sx;
    } else if (axis == 1) {
        int sy = sl.index(y);
        if (sy < 0) return -1;
        return (z * sl.width + sy) * S.pitch + x0;
    } else {
        int sz = sl.index(z);
        if (sz < 0) return -1;
        return (sz * S.ny + y) * S.pitch + x0;
    }
}

// ---------------------------------------------------------------------------
// Everything of the V phase after the stress derivatives: COMP16 rescale,
// masking, CPML memory variables, divergence, the velocity updates and their
// stores.  PRE: the caller has already loaded the coefficients and old
// velocities into V (the marching kernel); otherwise they are loaded here.
// RS: old state is multiplied by the COMP16 rescale r; the kernels pass false
// when r is exactly 1, which gives the same bits without the products.
// Where a phase tail stores: the field arrays (and COMP16 residuals) of the
// new state, and the memory variables it reads (psi_in) and writes (psi_out).
// In place, the single-buffered kernels' case, everything is the descriptor's
// own; the fused step kernel (step_fused.cu) reads one copy of the state and
// writes the other, and computes without storing on its halo cells.
struct TailOut {
    void* const* f;
    int8_t* const* flo;
    void* const* psi_in;
    void* const* psi_out;        // nullptr: in place
    bool store;                  // false: compute only (the fused kernel's halo cells)
    __device__ __forceinline__ static TailOut v_of(const ShotDesc& S) { return TailOut{S.f, S.flo, S.psiV, nullptr, true}; }
    __device__ __forceinline__ static TailOut t_of(const ShotDesc& S) { return TailOut{S.f, S.flo, S.psiT, nullptr, true}; }
};

// Coefficients of a chunk: from the per-cell arrays, or from the tuple table
// of an indexed medium (float policies only; FP64 shots are never indexed).
template <class P>
__device__ __forceinline__ bool med_on(const ShotDesc& S) {
    if constexpr (sizeof(typename P::real) == 4) return S.med_idx != nullptr;
    else return false;
}
// Component q of group g of the chunk's four tuples.
template <class R>
__device__ __forceinline__ void med_comp4(const ShotDesc& S, unsigned ids, int g, int q, R (&o)[4]) {
    float4 t[4];
    med_group4(S, ids, g, t);
#pragma unroll
    for (int j = 0; j < 4; j++) o[j] = (R)(q == 0 ? t[j].x : q == 1 ? t[j].y : q == 2 ? t[j].z : t[j].w);
}
// One V-phase coefficient (VCoef k) of the chunk at c.
template <class P, bool NC = kReadOnlyPath>
__device__ __forceinline__ void vcoef4(const ShotDesc& S, int k, cidx c, typename P::real (&o)[4]) {
    if (med_on<P>(S)) {
        const int g = (k == VC_RHO_Y || k == VC_CC1_Y || k == VC_CC2_Y) ? MED_V_Y
                      : (k == VC_RHO_Z || k == VC_CC1_Z || k == VC_CC2_Z) ? MED_V_Z : MED_V_X;
        const int q = k == VC_RHOF ? 3 : (k == VC_RHO_X || k == VC_RHO_Y || k == VC_RHO_Z) ? 0
                      : (k == VC_CC1_X || k == VC_CC1_Y || k == VC_CC1_Z) ? 1 : 2;
        med_comp4(S, med_ids(S, c), g, q, o);
        return;
    }
    P::template ld4<NC>(S.vc[k], S.vclo[k], c, o);
}
// One T-phase coefficient (TCoef k) of the chunk at c.
template <class P, bool NC = kReadOnlyPath>
__device__ __forceinline__ void tcoef4(const ShotDesc& S, int k, cidx c, typename P::real (&o)[4]) {
    if (med_on<P>(S)) {
        const int g = (k == TC_C || k == TC_M || k == TC_H || k == TC_H2U) ? MED_T_A : MED_T_B;
        const int q = (k == TC_C || k == TC_MUXZ) ? 0 : (k == TC_M || k == TC_MUXY) ? 1
                      : (k == TC_H || k == TC_MUYZ) ? 2 : 3;
        med_comp4(S, med_ids(S, c), g, q, o);
        return;
    }
    P::template ld4<NC>(S.tc[k], S.tclo[k], c, o);
}

template <class R>
struct VState {
    R x1[4], x3[4], s1[4], z1[4], z2[4], s3[4];       // derivatives (2D and 3D)
    R x2[4], y1[4], y2[4], y3[4], s2[4], z3[4];       // 3D only
    R rf[4], rho_x[4], c1_x[4], c2_x[4], vu_x[4], vw_x[4], rho_z[4], c1_z[4], c2_z[4], vu_z[4], vw_z[4];
    R rho_y[4], c1_y[4], c2_y[4], vu_y[4], vw_y[4];
    unsigned mids;                 // indexed medium: the chunk's four tuple indices (set before the tail)
};

// On return V's old-velocity members (vu_*, vw_*) hold the new velocities as a
// later load of the stored values returns them.
template <int DIM, int ORD, class P, bool PRE, bool RS, bool NC = kReadOnlyPath>
__device__ __forceinline__ void v_tail(const ShotDesc& S, cidx c, int x0, int y, int z, typename P::real r,
                                       unsigned mask, VState<typename P::real>& V, const TailOut& O) {
    using R = typename P::real;
    auto &x1 = V.x1, &x3 = V.x3, &s1 = V.s1, &z1 = V.z1, &z2 = V.z2, &s3 = V.s3;
    auto &x2 = V.x2, &y1 = V.y1, &y2 = V.y2, &y3 = V.y3, &s2 = V.s2, &z3 = V.z3;
    auto &rf = V.rf, &rho_x = V.rho_x, &c1_x = V.c1_x, &c2_x = V.c2_x, &vu_x = V.vu_x, &vw_x = V.vw_x;
    auto &rho_z = V.rho_z, &c1_z = V.c1_z, &c2_z = V.c2_z, &vu_z = V.vu_z, &vw_z = V.vw_z;
    auto &rho_y = V.rho_y, &c1_y = V.c1_y, &c2_y = V.c2_y, &vu_y = V.vu_y, &vw_y = V.vw_y;
    const bool med = med_on<P>(S);
    auto load_axis = [&](int fu, int fw, int crho, int ccc1, int ccc2, R (&rho)[4], R (&c1)[4], R (&c2)[4],
                         R (&vu)[4], R (&vw)[4]) {
        if (med) {
            // one group per cell: (rho, cc1, cc2, rhof) of this axis
            const int g = crho == VC_RHO_X ? MED_V_X : crho == VC_RHO_Y ? MED_V_Y : MED_V_Z;
            float4 t[4];
            med_group4(S, V.mids, g, t);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                rho[j] = (R)t[j].x; c1[j] = (R)t[j].y; c2[j] = (R)t[j].z;
                if (g == MED_V_X) rf[j] = (R)t[j].w;
            }
        } else {
            P::template ld4<NC>(S.vc[crho], S.vclo[crho], c, rho);
            P::template ld4<NC>(S.vc[ccc1], S.vclo[ccc1], c, c1);
            P::template ld4<NC>(S.vc[ccc2], S.vclo[ccc2], c, c2);
        }
        P::ld4(S.f[fu], S.flo[fu], c, vu);
        P::ld4(S.f[fw], S.flo[fw], c, vw);
    };
    // the rescale factor applies to old stresses: scale their derivatives
    if constexpr (P::prec == BP_PREC_COMP16 && RS) {
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
        cidx si = slab_index(S, 0, x0, y, z);
        if (si >= 0) {
            void* B = O.psi_in[0];
            void* Bo = O.psi_out ? O.psi_out[0] : nullptr;
            const long long n = S.slab_cells[0];
            cpml_slot<NS, RS, R, P::exact>(x1, B, n, 0, si, true, x0, x0, S.pb2[0], S.pe2[0], r, Bo, O.store);
            cpml_slot<NS, RS, R, P::exact>(s1, B, n, 1, si, true, x0, x0, S.pb2[0], S.pe2[0], r, Bo, O.store);
            cpml_slot<NS, RS, R, P::exact>(z2, B, n, 2, si, true, x0, x0, S.pb[0], S.pe[0], r, Bo, O.store);
            if constexpr (DIM == 3) cpml_slot<NS, RS, R, P::exact>(y2, B, n, 3, si, true, x0, x0, S.pb[0], S.pe[0], r, Bo, O.store);
        }
        if constexpr (DIM == 3) {
            si = slab_index(S, 1, x0, y, z);
            if (si >= 0) {
                void* B = O.psi_in[1];
                void* Bo = O.psi_out ? O.psi_out[1] : nullptr;
                const long long n = S.slab_cells[1];
                cpml_slot<NS, RS, R, P::exact>(x2, B, n, 0, si, false, y, x0, S.pb[1], S.pe[1], r, Bo, O.store);
                cpml_slot<NS, RS, R, P::exact>(y1, B, n, 1, si, false, y, x0, S.pb2[1], S.pe2[1], r, Bo, O.store);
                cpml_slot<NS, RS, R, P::exact>(s2, B, n, 2, si, false, y, x0, S.pb2[1], S.pe2[1], r, Bo, O.store);
                cpml_slot<NS, RS, R, P::exact>(z3, B, n, 3, si, false, y, x0, S.pb[1], S.pe[1], r, Bo, O.store);
            }
        }
        si = slab_index(S, 2, x0, y, z);
        if (si >= 0) {
            void* B = O.psi_in[2];
            void* Bo = O.psi_out ? O.psi_out[2] : nullptr;
            const long long n = S.slab_cells[2];
            cpml_slot<NS, RS, R, P::exact>(x3, B, n, 0, si, false, z, x0, S.pb[2], S.pe[2], r, Bo, O.store);
            cpml_slot<NS, RS, R, P::exact>(z1, B, n, 1, si, false, z, x0, S.pb2[2], S.pe2[2], r, Bo, O.store);
            cpml_slot<NS, RS, R, P::exact>(s3, B, n, 2, si, false, z, x0, S.pb2[2], S.pe2[2], r, Bo, O.store);
            if constexpr (DIM == 3) cpml_slot<NS, RS, R, P::exact>(y3, B, n, 3, si, false, z, x0, S.pb[2], S.pe[2], r, Bo, O.store);
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
    auto axis_update = [&](const R (&sum)[4], const R (&dp)[4], int fu, int fw, const R (&rho)[4],
                           const R (&c1)[4], const R (&c2)[4], R (&vu)[4], R (&vw)[4]) {
        R nu[4], nw[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) {
                // Half/main.cu:256-262 with Bt = (rhof rho^-1) Bp formed here
                const R wo = RS ? mulr(vw[j], r) : vw[j], uo = RS ? mulr(vu[j], r) : vu[j];
                R rr = rf[j] * rho[j];                    // rhof * rho^-1
                R wn = c1[j] * wo - (rr * c2[j]) * sum[j] - c2[j] * dp[j];
                nw[j] = wn;
                nu[j] = uo + rho[j] * sum[j] - rr * (wn - wo);
            } else {
                R wo = vw[j];
                // IEEE division; a zero dividend (the whole quiet grid ahead of
                // the wavefront) takes the divide routine's slow path, so its
                // exact result, a zero with the quotient's sign, is formed by a
                // product instead: 7-15 % off the V phase, bit-identical.
                const R num = wo * c2[j] - S.dtr<R>() * (rf[j] * rho[j] * sum[j] + dp[j]);
                const R wn = (c1[j] == (R)0) ? (R)0 : (num == (R)0 ? num * c1[j] : num / c1[j]);
                nw[j] = wn;
                nu[j] = vu[j] + S.dtr<R>() * rho[j] * sum[j] - rf[j] * rho[j] * (wn - wo);
            }
            if (!(mask >> j & 1u)) { nw[j] = vw[j]; nu[j] = vu[j]; }
        }
        P::st4_rt(O.f[fw], O.flo[fw], c, nw, O.store);
        P::st4_rt(O.f[fu], O.flo[fu], c, nu, O.store);
#pragma unroll
        for (int j = 0; j < 4; j++) { vw[j] = nw[j]; vu[j] = nu[j]; }
    };
    if constexpr (!PRE) {
        if (!med) P::template ld4<NC>(S.vc[VC_RHOF], S.vclo[VC_RHOF], c, rf);   // indexed: with the x group
        load_axis(BP_F_VUX, BP_F_VWX, VC_RHO_X, VC_CC1_X, VC_CC2_X, rho_x, c1_x, c2_x, vu_x, vw_x);
    }
    axis_update(sumx, s1, BP_F_VUX, BP_F_VWX, rho_x, c1_x, c2_x, vu_x, vw_x);
    if constexpr (DIM == 3) {
        if constexpr (!PRE) load_axis(BP_F_VUY, BP_F_VWY, VC_RHO_Y, VC_CC1_Y, VC_CC2_Y, rho_y, c1_y, c2_y, vu_y, vw_y);
        axis_update(sumy, s2, BP_F_VUY, BP_F_VWY, rho_y, c1_y, c2_y, vu_y, vw_y);
    }
    if constexpr (!PRE) load_axis(BP_F_VUZ, BP_F_VWZ, VC_RHO_Z, VC_CC1_Z, VC_CC2_Z, rho_z, c1_z, c2_z, vu_z, vw_z);
    axis_update(sumz, s3, BP_F_VUZ, BP_F_VWZ, rho_z, c1_z, c2_z, vu_z, vw_z);
}

template <int DIM, int ORD, class P, bool PRE, bool RS, bool NC = kReadOnlyPath>
__device__ __forceinline__ void v_tail(const ShotDesc& S, cidx c, int x0, int y, int z, typename P::real r,
                                       unsigned mask, VState<typename P::real>& V) {
    v_tail<DIM, ORD, P, PRE, RS, NC>(S, c, x0, y, z, r, mask, V, TailOut::v_of(S));
}

// ---------------------------------------------------------------------------
// Everything of the T phase after the velocity derivatives: masking, CPML
// memory variables, the pressure and stress updates and their stores.  PRE:
// the caller has already loaded the moduli and the old stresses into T, the
// latter multiplied by the COMP16 rescale (the marching kernel).
template <class R>
struct TState {
    R uxx[4], uzz[4], wx[4], wz[4], uxz[4], uzx[4];   // derivatives (2D and 3D)
    R uyy[4], wy[4], uxy[4], uyx[4], uyz[4], uzy[4];   // 3D only
    R cC[4], cM[4], cH[4], cH2[4], mxz[4], op[4], oxx[4], ozz[4], oxz[4];
    R mxy[4], myz[4], oyy[4], oxy[4], oyz[4];
    unsigned mids;                 // indexed medium: the chunk's four tuple indices (set before the tail)
};

// On return T's old-stress members (op, oxx, ...) hold the new values.
template <int DIM, int ORD, class P, bool PRE, bool RS, bool NC = kReadOnlyPath>
__device__ __forceinline__ void t_tail(const ShotDesc& S, cidx c, int x0, int y, int z, typename P::real r,
                                       unsigned mask, TState<typename P::real>& T, const TailOut& O) {
    using R = typename P::real;
    auto &uxx = T.uxx, &uzz = T.uzz, &wx = T.wx, &wz = T.wz, &uxz = T.uxz, &uzx = T.uzx;
    auto &uyy = T.uyy, &wy = T.wy, &uxy = T.uxy, &uyx = T.uyx, &uyz = T.uyz, &uzy = T.uzy;
    auto &cC = T.cC, &cM = T.cM, &cH = T.cH, &cH2 = T.cH2, &mxz = T.mxz;
    auto &op = T.op, &oxx = T.oxx, &ozz = T.ozz, &oxz = T.oxz;
    auto &mxy = T.mxy, &myz = T.myz, &oyy = T.oyy, &oxy = T.oxy, &oyz = T.oyz;
    auto load_state = [&]() {
        if (med_on<P>(S)) {
            const unsigned ids = T.mids;
            float4 a[4], b[4];
            med_group4(S, ids, MED_T_A, a);
            med_group4(S, ids, MED_T_B, b);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                cC[j] = (R)a[j].x; cM[j] = (R)a[j].y; cH[j] = (R)a[j].z; cH2[j] = (R)a[j].w; mxz[j] = (R)b[j].x;
                if constexpr (DIM == 3) { mxy[j] = (R)b[j].y; myz[j] = (R)b[j].z; }
            }
        } else {
            P::template ld4<NC>(S.tc[TC_C], S.tclo[TC_C], c, cC);
            P::template ld4<NC>(S.tc[TC_M], S.tclo[TC_M], c, cM);
            P::template ld4<NC>(S.tc[TC_H], S.tclo[TC_H], c, cH);
            P::template ld4<NC>(S.tc[TC_H2U], S.tclo[TC_H2U], c, cH2);
            P::template ld4<NC>(S.tc[TC_MUXZ], S.tclo[TC_MUXZ], c, mxz);
            if constexpr (DIM == 3) {
                P::template ld4<NC>(S.tc[TC_MUXY], S.tclo[TC_MUXY], c, mxy);
                P::template ld4<NC>(S.tc[TC_MUYZ], S.tclo[TC_MUYZ], c, myz);
            }
        }
        P::ld4(S.f[BP_F_P], S.flo[BP_F_P], c, op);
        P::ld4(S.f[BP_F_TXX], S.flo[BP_F_TXX], c, oxx);
        P::ld4(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], c, ozz);
        P::ld4(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], c, oxz);
        if constexpr (DIM == 3) {
            P::ld4(S.f[BP_F_TYY], S.flo[BP_F_TYY], c, oyy);
            P::ld4(S.f[BP_F_TXY], S.flo[BP_F_TXY], c, oxy);
            P::ld4(S.f[BP_F_TYZ], S.flo[BP_F_TYZ], c, oyz);
        }
        if constexpr (P::prec == BP_PREC_COMP16 && RS) {     // old state takes this step's rescale
            scale4(op, r); scale4(oxx, r); scale4(ozz, r); scale4(oxz, r);
            if constexpr (DIM == 3) { scale4(oyy, r); scale4(oxy, r); scale4(oyz, r); }
        }
    };
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
        cidx si = slab_index(S, 0, x0, y, z);
        if (si >= 0) {
            void* B = O.psi_in[0];
            const long long n = S.slab_cells[0];
            cpml_slot<NS, RS, R, P::exact>(uxx, B, n, 0, si, true, x0, x0, S.pb[0], S.pe[0], r, nullptr, O.store);
            cpml_slot<NS, RS, R, P::exact>(wx, B, n, 1, si, true, x0, x0, S.pb[0], S.pe[0], r, nullptr, O.store);
            cpml_slot<NS, RS, R, P::exact>(uzx, B, n, 2, si, true, x0, x0, S.pb2[0], S.pe2[0], r, nullptr, O.store);
            if constexpr (DIM == 3) cpml_slot<NS, RS, R, P::exact>(uyx, B, n, 3, si, true, x0, x0, S.pb2[0], S.pe2[0], r, nullptr, O.store);
        }
        if constexpr (DIM == 3) {
            si = slab_index(S, 1, x0, y, z);
            if (si >= 0) {
                void* B = O.psi_in[1];
                const long long n = S.slab_cells[1];
                cpml_slot<NS, RS, R, P::exact>(uyy, B, n, 0, si, false, y, x0, S.pb[1], S.pe[1], r, nullptr, O.store);
                cpml_slot<NS, RS, R, P::exact>(wy, B, n, 1, si, false, y, x0, S.pb[1], S.pe[1], r, nullptr, O.store);
                cpml_slot<NS, RS, R, P::exact>(uxy, B, n, 2, si, false, y, x0, S.pb2[1], S.pe2[1], r, nullptr, O.store);
                cpml_slot<NS, RS, R, P::exact>(uzy, B, n, 3, si, false, y, x0, S.pb2[1], S.pe2[1], r, nullptr, O.store);
            }
        }
        si = slab_index(S, 2, x0, y, z);
        if (si >= 0) {
            void* B = O.psi_in[2];
            const long long n = S.slab_cells[2];
            cpml_slot<NS, RS, R, P::exact>(uzz, B, n, 0, si, false, z, x0, S.pb[2], S.pe[2], r, nullptr, O.store);
            cpml_slot<NS, RS, R, P::exact>(wz, B, n, 1, si, false, z, x0, S.pb[2], S.pe[2], r, nullptr, O.store);
            cpml_slot<NS, RS, R, P::exact>(uxz, B, n, 2, si, false, z, x0, S.pb2[2], S.pe2[2], r, nullptr, O.store);
            if constexpr (DIM == 3) cpml_slot<NS, RS, R, P::exact>(uyz, B, n, 3, si, false, z, x0, S.pb2[2], S.pe2[2], r, nullptr, O.store);
        }
    }

    // ---- pressure and stress updates (Float/main.cu:287-293) ----
    if constexpr (!PRE) load_state();
    const R dt = S.dtr<R>();
    auto finish = [&](int f, R (&nv)[4], R (&ov)[4]) {
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (!(mask >> j & 1u)) nv[j] = ov[j];
        if (O.store) P::st4(O.f[f], O.flo[f], c, nv);
#pragma unroll
        for (int j = 0; j < 4; j++) ov[j] = nv[j];
    };
    R n[4];
    if constexpr (DIM == 3) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = op[j] - cC[j] * (uxx[j] + uyy[j] + uzz[j]) - cM[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = op[j] - dt * (cC[j] * (uxx[j] + uyy[j] + uzz[j]) + cM[j] * (wx[j] + wy[j] + wz[j]));
        }
        finish(BP_F_P, n, op);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = oxx[j] + cH2[j] * (uyy[j] + uzz[j]) + cH[j] * uxx[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = oxx[j] + dt * (cH2[j] * (uyy[j] + uzz[j]) + cH[j] * uxx[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        finish(BP_F_TXX, n, oxx);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = oyy[j] + cH2[j] * (uxx[j] + uzz[j]) + cH[j] * uyy[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = oyy[j] + dt * (cH2[j] * (uxx[j] + uzz[j]) + cH[j] * uyy[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        finish(BP_F_TYY, n, oyy);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = ozz[j] + cH2[j] * (uxx[j] + uyy[j]) + cH[j] * uzz[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = ozz[j] + dt * (cH2[j] * (uxx[j] + uyy[j]) + cH[j] * uzz[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        finish(BP_F_TZZ, n, ozz);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = oxy[j] + mxy[j] * (uxy[j] + uyx[j]);
            else n[j] = oxy[j] + mxy[j] * dt * (uxy[j] + uyx[j]);
        }
        finish(BP_F_TXY, n, oxy);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = oyz[j] + myz[j] * (uyz[j] + uzy[j]);
            else n[j] = oyz[j] + myz[j] * dt * (uyz[j] + uzy[j]);
        }
        finish(BP_F_TYZ, n, oyz);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = oxz[j] + mxz[j] * (uxz[j] + uzx[j]);
            else n[j] = oxz[j] + mxz[j] * dt * (uxz[j] + uzx[j]);
        }
        finish(BP_F_TXZ, n, oxz);
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = op[j] - cC[j] * (uxx[j] + uzz[j]) - cM[j] * (wx[j] + wz[j]);
            else
                n[j] = op[j] - dt * (cC[j] * (uxx[j] + uzz[j]) + cM[j] * (wx[j] + wz[j]));
        }
        finish(BP_F_P, n, op);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = oxx[j] + cH2[j] * uzz[j] + cH[j] * uxx[j] + cC[j] * (wx[j] + wz[j]);
            else
                n[j] = oxx[j] + dt * (cH2[j] * uzz[j] + cH[j] * uxx[j] + cC[j] * (wx[j] + wz[j]));
        }
        finish(BP_F_TXX, n, oxx);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = ozz[j] + cH2[j] * uxx[j] + cH[j] * uzz[j] + cC[j] * (wx[j] + wz[j]);
            else
                n[j] = ozz[j] + dt * (cH2[j] * uxx[j] + cH[j] * uzz[j] + cC[j] * (wx[j] + wz[j]));
        }
        finish(BP_F_TZZ, n, ozz);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16) n[j] = oxz[j] + mxz[j] * (uxz[j] + uzx[j]);
            else n[j] = oxz[j] + mxz[j] * dt * (uxz[j] + uzx[j]);
        }
        finish(BP_F_TXZ, n, oxz);
    }
}

template <int DIM, int ORD, class P, bool PRE, bool RS, bool NC = kReadOnlyPath>
__device__ __forceinline__ void t_tail(const ShotDesc& S, cidx c, int x0, int y, int z, typename P::real r,
                                       unsigned mask, TState<typename P::real>& T) {
    t_tail<DIM, ORD, P, PRE, RS, NC>(S, c, x0, y, z, r, mask, T, TailOut::t_of(S));
}

}  // namespace bpk

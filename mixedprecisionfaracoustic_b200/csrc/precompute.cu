// precompute.cu - FP64 set-up kernels run once per shot on the GPU.
//
// Replaces the reference's host precompute:
//   extmodel edge padding          Float/main.cu:387-399,1662-1794
//   staggered averaging            Float/main.cu:472-513
//   CC1/CC2 friction denominators  Float/main.cu:106-113 (per step in FD_V)
//   CPML profiles                  Float/main.cu:570-654
//   COMP16 exponent scan, Aw/Bp/Bt and scaled moduli  Half/main.cu:745-1045
// Every quantity is formed in double precision from the float medium and
// rounded once into the storage type of the precision policy.
#include <cmath>

#include "common.cuh"

namespace bpk {

struct MediumDev {                 // device copies of the 9 cell-centred arrays
    const float* a[9];             // rho, rhof, M, C, H, H2mu, mu, C1, C2
    int nx, ny, nz;                // physical extents (ny = 1 in 2D)
    int np;                        // CPML width
};
enum { MD_RHO, MD_RHOF, MD_M, MD_C, MD_H, MD_H2MU, MD_MU, MD_C1, MD_C2 };

// extmodel: the padded array is the physical one clamped to its edges.
__device__ __forceinline__ double padded(const MediumDev& m, int k, int x, int y, int z) {
    int px = min(max(x - m.np, 0), m.nx - 1);
    int py = m.ny > 1 ? min(max(y - m.np, 0), m.ny - 1) : 0;
    int pz = min(max(z - m.np, 0), m.nz - 1);
    return (double)m.a[k][(size_t)px + (size_t)py * m.nx + (size_t)pz * m.nx * m.ny];
}

// Harmonic average of four shear moduli, 0 if any is 0 (Float/main.cu:480-491).
__device__ __forceinline__ double harm4(double a, double b, double c, double d) {
    if (a == 0.0 || b == 0.0 || c == 0.0 || d == 0.0) return 0.0;
    return 1.0 / (0.25 * (1.0 / a + 1.0 / b + 1.0 / c + 1.0 / d));
}

struct FaceCoef {                  // one face direction of one cell, FP64
    double rho_inv, C1, C2, Q;
};
__device__ __forceinline__ FaceCoef face(const MediumDev& m, int x, int y, int z, int ax) {
    int x1 = x + (ax == 0), y1 = y + (ax == 1), z1 = z + (ax == 2);
    FaceCoef f;
    f.rho_inv = 2.0 / (padded(m, MD_RHO, x, y, z) + padded(m, MD_RHO, x1, y1, z1));
    f.C1 = 0.5 * (padded(m, MD_C1, x, y, z) + padded(m, MD_C1, x1, y1, z1));
    f.C2 = 0.5 * (padded(m, MD_C2, x, y, z) + padded(m, MD_C2, x1, y1, z1));
    double rf = padded(m, MD_RHOF, x, y, z);
    f.Q = f.C2 - rf * rf * f.rho_inv;
    return f;
}

struct CellCoef {
    FaceCoef fc[3];
    double rhof, C, M, H, H2u, mu;
    double muxy, muxz, muyz;
};
__device__ __forceinline__ CellCoef cell_coef(const MediumDev& m, int dim, int x, int y, int z) {
    CellCoef c;
    c.fc[0] = face(m, x, y, z, 0);
    c.fc[2] = face(m, x, y, z, 2);
    if (dim == 3) c.fc[1] = face(m, x, y, z, 1);
    else c.fc[1] = FaceCoef{0, 0, 0, 0};
    c.rhof = padded(m, MD_RHOF, x, y, z);
    c.C = padded(m, MD_C, x, y, z);
    c.M = padded(m, MD_M, x, y, z);
    c.H = padded(m, MD_H, x, y, z);
    c.H2u = padded(m, MD_H2MU, x, y, z);
    c.mu = padded(m, MD_MU, x, y, z);
    c.muxz = harm4(c.mu, padded(m, MD_MU, x + 1, y, z), padded(m, MD_MU, x, y, z + 1),
                   padded(m, MD_MU, x + 1, y, z + 1));
    if (dim == 3) {
        c.muyz = harm4(c.mu, padded(m, MD_MU, x, y + 1, z), padded(m, MD_MU, x, y, z + 1),
                       padded(m, MD_MU, x, y + 1, z + 1));
        c.muxy = harm4(c.mu, padded(m, MD_MU, x + 1, y, z), padded(m, MD_MU, x, y + 1, z),
                       padded(m, MD_MU, x + 1, y + 1, z));
    } else {
        c.muyz = c.muxy = 0.0;
    }
    return c;
}

template <class P>
__device__ __forceinline__ void put(void* p, int8_t* lo, long long i, double v) {
    if constexpr (P::prec == BP_PREC_FP64) static_cast<double*>(p)[i] = v;
    else if constexpr (P::prec == BP_PREC_FP32) static_cast<float*>(p)[i] = (float)v;
    else {
        if (lo) {
            __half h; int8_t l;
            encode_ch((float)v, h, l);
            static_cast<__half*>(p)[i] = h;
            lo[i] = l;
        } else {
            static_cast<__half*>(p)[i] = __float2half_rn((float)v);
        }
    }
}

// ---- FP32: the reference's own float arithmetic (Float/main.cu:480-509 and
// the per-step CC1/CC2 of :106-113), reproduced bit for bit with explicit
// round-to-nearest intrinsics (no contraction), so the FP32 path starts from
// exactly the coefficients the Float build uses.
__device__ __forceinline__ float padf(const MediumDev& m, int k, int x, int y, int z) {
    return (float)padded(m, k, x, y, z);
}
__device__ __forceinline__ float ref_harm4(float a, float b, float c, float d) {
    if (a == 0.0f || b == 0.0f || c == 0.0f || d == 0.0f) return 0.0f;
    const float s = __fadd_rn(__fadd_rn(__fadd_rn(__fdiv_rn(1.0f, a), __fdiv_rn(1.0f, b)), __fdiv_rn(1.0f, c)),
                              __fdiv_rn(1.0f, d));
    return (float)__ddiv_rn(1.0, __dmul_rn(0.25, (double)s));
}
struct Ref32Face {
    float rho_x, c1, c2;
};
__device__ __forceinline__ Ref32Face ref32_face(const MediumDev& m, int x, int y, int z, int ax) {
    const int x1 = x + (ax == 0), y1 = y + (ax == 1), z1 = z + (ax == 2);
    Ref32Face f;
    f.rho_x = __fdiv_rn(2.0f, __fadd_rn(padf(m, MD_RHO, x, y, z), padf(m, MD_RHO, x1, y1, z1)));
    f.c1 = (float)__dmul_rn(0.5, (double)__fadd_rn(padf(m, MD_C1, x, y, z), padf(m, MD_C1, x1, y1, z1)));
    f.c2 = (float)__dmul_rn(0.5, (double)__fadd_rn(padf(m, MD_C2, x, y, z), padf(m, MD_C2, x1, y1, z1)));
    return f;
}
// CC1 = 0.5*C1*DT + C2 - rhof*rhof*rho (double sum, float product);
// CC2 = (C2 - rhof*rhof*rho) [float] - 0.5*C1*DT [double]; CC1 = 0 marks C1 == 0.
__device__ __forceinline__ void ref32_cc(float c1, float c2, float rhof, float rho, float DT, float& cc1, float& cc2) {
    const float rr = __fmul_rn(__fmul_rn(rhof, rhof), rho);
    const double h = __dmul_rn(__dmul_rn(0.5, (double)c1), (double)DT);
    cc1 = c1 == 0.0f ? 0.0f : (float)__dsub_rn(__dadd_rn(h, (double)c2), (double)rr);
    cc2 = (float)__dsub_rn((double)__fsub_rn(c2, rr), h);
}

// P: PolF32 stores the float coefficients, PolB24 their compensated-bf16 form.
template <class P>
__global__ void k_coefs_ref32(ShotDesc S, MediumDev m, float DT) {
    const long long n = (long long)S.nx * S.ny * S.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % S.nx);
        const long long rest = q / S.nx;
        const int y = (int)(rest % S.ny), z = (int)(rest / S.ny);
        const long long i = x + (long long)y * S.pitch + (long long)z * S.plane;
        const bool inner = x >= 1 && x < S.nx - 1 && z >= 1 && z < S.nz - 1 && (S.dim == 2 || (y >= 1 && y < S.ny - 1));
        const float rhof = padf(m, MD_RHOF, x, y, z);
        auto vc = [&](int k, float v) { P::st1(S.vc[k], S.vclo[k], i, v); };
        auto tc = [&](int k, float v) { P::st1(S.tc[k], S.tclo[k], i, v); };
        vc(VC_RHOF, rhof);
        tc(TC_C, padf(m, MD_C, x, y, z));
        tc(TC_M, padf(m, MD_M, x, y, z));
        tc(TC_H, padf(m, MD_H, x, y, z));
        tc(TC_H2U, padf(m, MD_H2MU, x, y, z));
        if (!inner) continue;   // outer cells are never updated: coefficients stay 0
        const int rho_slot[3] = {VC_RHO_X, VC_RHO_Y, VC_RHO_Z};
        const int c1_slot[3] = {VC_CC1_X, VC_CC1_Y, VC_CC1_Z};
        const int c2_slot[3] = {VC_CC2_X, VC_CC2_Y, VC_CC2_Z};
        for (int a = 0; a < 3; a++) {
            if (a == 1 && S.dim == 2) continue;
            const Ref32Face f = ref32_face(m, x, y, z, a);
            float cc1, cc2;
            ref32_cc(f.c1, f.c2, rhof, f.rho_x, DT, cc1, cc2);
            vc(rho_slot[a], f.rho_x);
            vc(c1_slot[a], cc1);
            vc(c2_slot[a], cc2);
        }
        const float mu = padf(m, MD_MU, x, y, z);
        tc(TC_MUXZ, ref_harm4(mu, padf(m, MD_MU, x + 1, y, z), padf(m, MD_MU, x, y, z + 1), padf(m, MD_MU, x + 1, y, z + 1)));
        if (S.dim == 3) {
            tc(TC_MUYZ, ref_harm4(mu, padf(m, MD_MU, x, y + 1, z), padf(m, MD_MU, x, y, z + 1), padf(m, MD_MU, x, y + 1, z + 1)));
            tc(TC_MUXY, ref_harm4(mu, padf(m, MD_MU, x + 1, y, z), padf(m, MD_MU, x, y + 1, z), padf(m, MD_MU, x + 1, y + 1, z)));
        }
    }
}

// Coefficient arrays of one shot (FP64 precompute, COMP16 and FP64 paths).
// The averaging runs over the reference's range 1..N-2 (Float/main.cu:473-477);
// other cells keep 0.  For COMP16, em/scales come from the exponent scan
// (k_scan_kr + host rounding).
template <class P>
__global__ void k_coefs(ShotDesc S, MediumDev m, double dt, int em) {
    const long long n = (long long)S.nx * S.ny * S.nz;
    const double sm = ldexp(1.0, em), ism = ldexp(1.0, -em);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % S.nx);
        long long rest = q / S.nx;
        int y = (int)(rest % S.ny), z = (int)(rest / S.ny);
        const long long i = x + (long long)y * S.pitch + (long long)z * S.plane;
        bool inner = x >= 1 && x < S.nx - 1 && z >= 1 && z < S.nz - 1 && (S.dim == 2 || (y >= 1 && y < S.ny - 1));
        CellCoef c;
        if (inner) c = cell_coef(m, S.dim, x, y, z);
        else {
            c = CellCoef{};
            c.rhof = padded(m, MD_RHOF, x, y, z);
            c.C = padded(m, MD_C, x, y, z);
            c.M = padded(m, MD_M, x, y, z);
            c.H = padded(m, MD_H, x, y, z);
            c.H2u = padded(m, MD_H2MU, x, y, z);
        }
        const int rho_slot[3] = {VC_RHO_X, VC_RHO_Y, VC_RHO_Z};
        const int c1_slot[3] = {VC_CC1_X, VC_CC1_Y, VC_CC1_Z};
        const int c2_slot[3] = {VC_CC2_X, VC_CC2_Y, VC_CC2_Z};
        for (int a = 0; a < 3; a++) {
            if (a == 1 && S.dim == 2) continue;
            const FaceCoef& f = c.fc[a];
            double v_rho, v_c1, v_c2;
            if constexpr (P::prec == BP_PREC_COMP16) {
                // Half/main.cu:986-1012: Aw = (Q - C1 DT/2)/(Q + C1 DT/2),
                // Bp = 2^-em DT / (Q + C1 DT/2); zero where C1 == 0 or Q ~ 0.
                double denom = f.Q + 0.5 * f.C1 * dt;
                bool ok = f.C1 != 0.0 && fabs(f.Q) > 1e-12 && fabs(denom) > 1e-12;
                v_rho = ism * dt * f.rho_inv;
                v_c1 = ok ? (f.Q - 0.5 * f.C1 * dt) / denom : 0.0;
                v_c2 = ok ? ism * dt / denom : 0.0;
            } else {
                v_rho = f.rho_inv;
                v_c1 = f.C1 == 0.0 ? 0.0 : f.Q + 0.5 * f.C1 * dt;   // CC1, 0 = "C1 == 0"
                v_c2 = f.Q - 0.5 * f.C1 * dt;                       // CC2
            }
            put<P>(S.vc[rho_slot[a]], S.vclo[rho_slot[a]], i, v_rho);
            put<P>(S.vc[c1_slot[a]], S.vclo[c1_slot[a]], i, v_c1);
            put<P>(S.vc[c2_slot[a]], S.vclo[c2_slot[a]], i, v_c2);
        }
        double t_scale = 1.0, rf = c.rhof;
        if constexpr (P::prec == BP_PREC_COMP16) {
            t_scale = sm * dt;          // moduli carry 2^em DT (Half/main.cu:1023-1029)
            rf = c.rhof * sm / dt;      // rhof 2^em / DT, so rhof rho^-1 = RHOF * RHO_a
        }
        put<P>(S.vc[VC_RHOF], S.vclo[VC_RHOF], i, rf);
        put<P>(S.tc[TC_C], S.tclo[TC_C], i, t_scale * c.C);
        put<P>(S.tc[TC_M], S.tclo[TC_M], i, t_scale * c.M);
        put<P>(S.tc[TC_H], S.tclo[TC_H], i, t_scale * c.H);
        put<P>(S.tc[TC_H2U], S.tclo[TC_H2U], i, t_scale * c.H2u);
        put<P>(S.tc[TC_MUXZ], S.tclo[TC_MUXZ], i, t_scale * c.muxz);
        if (S.dim == 3) {
            put<P>(S.tc[TC_MUXY], S.tclo[TC_MUXY], i, t_scale * c.muxy);
            put<P>(S.tc[TC_MUYZ], S.tclo[TC_MUYZ], i, t_scale * c.muyz);
        }
    }
}

// ---------------------------------------------------------------------------
// K_max / R_max scan of Half/main.cu:745-790 in FP64 with warp-shuffle max
// reductions; one partial pair per block into `partial` (scratch).
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_scan_kr(int dim, int nx, int ny, int nz, MediumDev m, double* partial) {
    const long long n = (long long)nx * ny * nz;
    double kmax = 0.0, rmax = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % nx);
        long long rest = q / nx;
        int y = (int)(rest % ny), z = (int)(rest / ny);
        bool inner = x >= 1 && x < nx - 1 && z >= 1 && z < nz - 1 && (dim == 2 || (y >= 1 && y < ny - 1));
        double H = padded(m, MD_H, x, y, z), H2u = padded(m, MD_H2MU, x, y, z);
        double C = padded(m, MD_C, x, y, z), M = padded(m, MD_M, x, y, z), mu = padded(m, MD_MU, x, y, z);
        kmax = fmax(kmax, fmax(fmax(fabs(H), fabs(H2u)), fmax(fmax(fabs(C), fabs(M)), fabs(mu))));
        if (!inner) continue;
        CellCoef c = cell_coef(m, dim, x, y, z);
        kmax = fmax(kmax, fmax(fabs(c.muxz), fmax(fabs(c.muxy), fabs(c.muyz))));
        for (int a = 0; a < 3; a++) {
            if (a == 1 && dim == 2) continue;
            const FaceCoef& f = c.fc[a];
            if (f.rho_inv > 0.0) rmax = fmax(rmax, f.rho_inv);
            if (f.C1 != 0.0 && fabs(f.Q) > 1e-12) {
                rmax = fmax(rmax, 1.0 / fabs(f.Q));
                rmax = fmax(rmax, fabs(c.rhof * f.rho_inv / f.Q));
            }
        }
    }
    __shared__ double sk[32], sr[32];
    kmax = warp_max(kmax);
    rmax = warp_max(rmax);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sk[w] = kmax; sr[w] = rmax; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        kmax = l < nw ? sk[l] : 0.0;
        rmax = l < nw ? sr[l] : 0.0;
        kmax = warp_max(kmax);
        rmax = warp_max(rmax);
        if (l == 0) { partial[2 * blockIdx.x] = kmax; partial[2 * blockIdx.x + 1] = rmax; }
    }
}

__global__ void k_reduce_max2(const double* partial, int n, double* out) {
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a = fmax(a, partial[2 * i]);
        b = fmax(b, partial[2 * i + 1]);
    }
    __shared__ double sa[32], sb[32];
    a = warp_max(a);
    b = warp_max(b);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        a = l < nw ? sa[l] : 0.0;
        b = l < nw ? sb[l] : 0.0;
        a = warp_max(a);
        b = warp_max(b);
        if (l == 0) { out[0] = a; out[1] = b; }
    }
}

// ---------------------------------------------------------------------------
// CPML profile tables of one axis (Float/main.cu:570-654).  The membership of
// a cell in the left/right absorbing region uses the reference's float
// arithmetic (x = i*H, xoleft = NP*H, xoright = (N-1)*H - NP*H), so the set of
// damped cells is identical; the damping values are formed in FP64.
struct PmlGeom {
    int n, np;
    float H;
};
__host__ __device__ inline void pml_region(const PmlGeom& g, int i, bool& left, bool& right) {
#ifdef __CUDA_ARCH__
    float DP = __fmul_rn((float)g.np, g.H);
    float oright = __fsub_rn(__fmul_rn((float)(g.n - 1), g.H), DP);
    float x = __fmul_rn((float)i, g.H);
    float xend = __fmul_rn((float)g.n, g.H);
#else
    volatile float DP = (float)g.np * g.H;
    volatile float t = (float)(g.n - 1) * g.H;
    volatile float oright = t - DP;
    volatile float x = (float)i * g.H;
    volatile float xend = (float)g.n * g.H;
#endif
    left = x >= 0.0f && x < DP;
    right = x >= oright && x < xend;
}

template <class R>
__global__ void k_profile(PmlGeom g, double dt, double v0, double rc, R* b, R* e, R* b2, R* e2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    bool left, right;
    pml_region(g, i, left, right);
    const float DPf = __fmul_rn((float)g.np, g.H);
    const double DP = DPf, H = g.H;
    const double oleft = DPf;
    const double oright = (double)__fsub_rn(__fmul_rn((float)(g.n - 1), g.H), DPf);
    const double x = (double)i * H;     // exact cell position; only the region test uses float x
    const double d0 = 3.0 * v0 * log(1.0 / rc) / (2.0 * DP);
    double d = 0.0, d2 = 0.0;
    if (left) {
        double a = (oleft - x) / DP, c = (oleft - x - 0.5 * H) / DP;
        d = d0 * a * a;
        d2 = d0 * c * c;
    }
    if (right) {
        double a = (x - oright) / DP, c = (x + 0.5 * H - oright) / DP;
        d = d0 * a * a;
        d2 = d0 * c * c;
    }
    b[i] = (R)(-0.5 * dt * d);
    e[i] = (R)exp(-d * dt);
    b2[i] = (R)(-0.5 * dt * d2);
    e2[i] = (R)exp(-d2 * dt);
}

// FP32 tables exactly as the reference's host code forms them
// (Float/main.cu:599-651): float positions and differences, double pow/exp
// intermediates rounded to float, e = exp(float(-d DT)).  The FP32 path stores
// b = float(-DT d) / 2, the double factor FD_V/FD_T apply (Float/main.cu:130).
// Explicit _rn intrinsics keep the compiler from fusing any of it.
__device__ __forceinline__ float ref_expf(float a) { return (float)exp((double)a); }
__global__ void k_profile_ref32(PmlGeom g, float DT, float v0, float RC, float* b, float* e, float* b2, float* e2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    bool left, right;
    pml_region(g, i, left, right);
    const float H = g.H;
    const float DP = __fmul_rn((float)g.np, H);
    const float oleft = DP;
    const float oright = __fsub_rn(__fmul_rn((float)(g.n - 1), H), DP);
    const float x = __fmul_rn((float)i, H);
    const float d0 = (float)__ddiv_rn(__dmul_rn(__dmul_rn(3.0, (double)v0), log(__ddiv_rn(1.0, (double)RC))),
                                      __dmul_rn(2.0, (double)DP));
    float d = 0.0f, d2 = 0.0f;
    if (left) {
        const float t = __fdiv_rn(__fsub_rn(oleft, x), DP);
        const double u = __ddiv_rn(__dsub_rn((double)__fsub_rn(oleft, x), __dmul_rn(0.5, (double)H)), (double)DP);
        d = (float)__dmul_rn((double)d0, __dmul_rn((double)t, (double)t));
        d2 = (float)__dmul_rn((double)d0, __dmul_rn(u, u));
    }
    if (right) {
        const float t = __fdiv_rn(__fsub_rn(x, oright), DP);
        const double u = __ddiv_rn(__dsub_rn(__dadd_rn((double)x, __dmul_rn(0.5, (double)H)), (double)oright), (double)DP);
        d = (float)__dmul_rn((double)d0, __dmul_rn((double)t, (double)t));
        d2 = (float)__dmul_rn((double)d0, __dmul_rn(u, u));
    }
    const float ed = (left || right) ? ref_expf(__fmul_rn(-d, DT)) : 1.0f;
    const float ed2 = (left || right) ? ref_expf(__fmul_rn(-d2, DT)) : 1.0f;
    b[i] = __fmul_rn(__fmul_rn(-DT, d), 0.5f);
    e[i] = ed;
    b2[i] = __fmul_rn(__fmul_rn(-DT, d2), 0.5f);
    e2[i] = ed2;
}

// ---------------------------------------------------------------------------
// Host launchers
void host_pml_region(int n, int np, float H, int i, bool* left, bool* right) {
    PmlGeom g{n, np, H};
    bool l, r;
    pml_region(g, i, l, r);
    *left = l;
    *right = r;
}

cudaError_t launch_profile(int prec, int n, int np, float H, double dt, double v0, double rc, void* b, void* e,
                           void* b2, void* e2, cudaStream_t st) {
    PmlGeom g{n, np, H};
    int grid = (n + 255) / 256;
    if (prec == BP_PREC_FP32 || prec == BP_PREC_CBF16)
        k_profile_ref32<<<grid, 256, 0, st>>>(g, (float)dt, (float)v0, (float)rc, (float*)b, (float*)e, (float*)b2,
                                              (float*)e2);
    else if (prec == BP_PREC_FP64)
        k_profile<double><<<grid, 256, 0, st>>>(g, dt, v0, rc, (double*)b, (double*)e, (double*)b2, (double*)e2);
    else
        k_profile<float><<<grid, 256, 0, st>>>(g, dt, v0, rc, (float*)b, (float*)e, (float*)b2, (float*)e2);
    return cudaGetLastError();
}

cudaError_t launch_coefs(int prec, const ShotDesc& S, const float* const* med, int pnx, int pny, int pnz, int np,
                         double dt, int em, cudaStream_t st) {
    MediumDev m;
    for (int k = 0; k < 9; k++) m.a[k] = med[k];
    m.nx = pnx; m.ny = pny; m.nz = pnz; m.np = np;
    const int grid = 148 * 8;
    if (prec == BP_PREC_FP32) k_coefs_ref32<PolF32><<<grid, 256, 0, st>>>(S, m, (float)dt);
    else if (prec == BP_PREC_CBF16) k_coefs_ref32<PolB24><<<grid, 256, 0, st>>>(S, m, (float)dt);
    else if (prec == BP_PREC_COMP16) k_coefs<PolC16><<<grid, 256, 0, st>>>(S, m, dt, em);
    else k_coefs<PolF64><<<grid, 256, 0, st>>>(S, m, dt, em);
    return cudaGetLastError();
}

// partial: scratch of 2 * nblocks doubles; out: 2 doubles (device).
int scan_kr_blocks() { return 148 * 4; }
cudaError_t launch_scan_kr(int dim, int nx, int ny, int nz, const float* const* med, int pnx, int pny, int pnz,
                           int np, double* partial, double* out, cudaStream_t st) {
    MediumDev m;
    for (int k = 0; k < 9; k++) m.a[k] = med[k];
    m.nx = pnx; m.ny = pny; m.nz = pnz; m.np = np;
    const int nb = scan_kr_blocks();
    k_scan_kr<<<nb, 256, 0, st>>>(dim, nx, ny, nz, m, partial);
    k_reduce_max2<<<1, 1024, 0, st>>>(partial, nb, out);
    return cudaGetLastError();
}

}  // namespace bpk

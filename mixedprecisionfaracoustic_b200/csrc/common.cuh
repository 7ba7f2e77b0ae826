// common.cuh - device-side data layout, precision policies and helpers shared
// by the precompute, step and reduction kernels.
//
// HBM layout of one shot ("padded" grid nx x ny x nz, ny = 1 in 2D):
//   * every field / coefficient is a separate array, x fastest, with a row
//     pitch rounded up to 32 elements so 4-cell chunks are 16-byte aligned
//     (FP32) and every row starts on a 128-byte boundary;
//     index(x, y, z) = x + y * pitch + z * pitch * ny.
//   * CPML memory variables (ψ and the previous derivative, 2 per derivative
//     slot) exist only on the absorbing slabs of their axis (the reference
//     keeps 48 full-volume arrays, Float/main.cu:707-755).
//   * COMP16 fields are two arrays: fp16 "hi" and int8 residual "lo".
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/biot.h"

namespace bpk {

// V-phase coefficient slots (FP32/FP64: reference-shaped; COMP16: scaled set)
//  FP32/FP64: RHO_X,Y,Z = rho^-1 on faces (Float/main.cu:499-501), RHOF cell,
//             CC1_X..Z, CC2_X..Z = C2 - rhof^2 rho^-1 +/- C1 DT/2 (:106-113),
//             CC1 = 0 marks a face with C1 == 0 (vw forced to 0, :160-185).
//  COMP16:    RHO_* = 2^-em DT rho^-1, RHOF = rhof 2^em / DT, CC1_* = Aw,
//             CC2_* = Bp (Half/main.cu:986-1012); Bt = rhof rho^-1 Bp in-kernel.
enum VCoef { VC_RHO_X, VC_RHO_Y, VC_RHO_Z, VC_RHOF, VC_CC1_X, VC_CC1_Y, VC_CC1_Z,
             VC_CC2_X, VC_CC2_Y, VC_CC2_Z, VC_COUNT };
// T-phase coefficients: C, M, H, H-2mu at the cell; harmonic mu on edges
// (Float/main.cu:480-491).  COMP16 stores 2^em DT times each (Half :1023-1029).
enum TCoef { TC_C, TC_M, TC_H, TC_H2U, TC_MUXY, TC_MUXZ, TC_MUYZ, TC_COUNT };

// CPML slab of one axis: cells [0, lo) and [hi0, n) carry memory variables.
struct Slab {
    int lo;      // cells [0, lo)
    int hi0;     // cells [hi0, n)
    int width;   // lo + (n - hi0), x axis rounded up to a multiple of 4
    __host__ __device__ int index(int i) const {
        return i < lo ? i : (i >= hi0 ? lo + (i - hi0) : -1);
    }
};

// Offset of a cell (or of a slab memory variable) within one array.  Every
// array of a shot holds fewer than 2^31 elements (validate_config bounds the
// padded grid), so the phase kernels index with 32-bit integers: one
// wide multiply-add forms each address, where 64-bit offsets cost several
// instructions per access (1-5 % of the step, measured on B200).
using cidx = int;

struct ShotDesc {
    int dim, order, hw;           // hw = order / 2 = untouched border cells
    int nx, ny, nz;               // padded extents
    int pitch;                    // row pitch (elements)
    long long plane;              // pitch * ny
    int nseg;                     // 128-cell x segments per row
    int nrows;                    // rows per shot: ny * nz (3D) or nz (2D)
    long long tile0;              // first tile index of this shot in the batch
    // tile shape of the register kernels (TileShape): 2^tile_lr rows (3D:
    // 2^(tile_lr - tile_ltz) y rows of 2^tile_ltz z planes) x 2^tile_ls
    // 128-cell segments; nseg_t = tiles per row block along x
    int tile_lr, tile_ls, tile_ltz, nseg_t;
    int nt;                       // trace length
    int src_idx_valid;
    long long src_idx;            // flat index of the source cell
    int src_mask;
    int nrec;
    const long long* rec_idx;     // flat indices
    float* traces;                // [BP_NTRACE][nrec][nt]
    double* traces64;             // FP64 runs: [BP_NTRACE][nrec][nt]
    const void* wavelet;          // source samples per step (float or double)
    const float* dyn;             // COMP16: state scale during step it (nt entries)
    float out_stress, out_vel;    // COMP16: 2^-es, 2^(em-es) (divided by dyn at use)
    float inj_scale;              // COMP16: 2^es
    float dt;                     // DT (FP32/COMP16)
    double dtd;                   // DT (FP64)
    float inv_h;                  // 1/H (COMP16 multiplies; FP32/FP64 divide by H like the reference)
    float h;                      // H
    double hd;
    void* f[BP_NFIELDS];          // field arrays (hi for COMP16)
    int8_t* flo[BP_NFIELDS];      // COMP16 residuals
    void* vc[VC_COUNT];
    int8_t* vclo[VC_COUNT];
    void* tc[TC_COUNT];
    int8_t* tclo[TC_COUNT];
    // CPML: per axis tables of length n (b = -DT d / 2, e = exp(-d DT)) on the
    // integer (b, e) and half (b2, e2) grids, and the slab memory variables.
    const void* pb[3];
    const void* pe[3];
    const void* pb2[3];
    const void* pe2[3];
    Slab slab[3];
    void* psiV[3];                // per axis: [2*nslot][slab cells] (ψ then prev)
    void* psiT[3];
    long long slab_cells[3];
    int done;                     // batch: slot empty or retired, skip its tiles
    int* step_base;               // device: step index `it` of step k=0 of the current chunk
    const float* rtab;            // COMP16: per-step factor applied to old state (dyn[it]/dyn[it-1])
    int src_rec;                  // receiver index that owns the source cell, or -1
    long long tile0s;             // first tile of this shot in the TMA-staged 2D tiling
    int nseg_s;                   // 256-cell segments per row in that tiling
    int* blowup;                  // first step (+1) with a non-finite recorded value, 0 = none
    int ncol_m;                   // marching 2D kernels: 128-cell columns per row
    long long tile0m;             // first task of this shot in the marching tiling
    int zseg_m;                   // rows per marching task
    int pad_m;
    // receivers by row, for the T phase that records them itself: the unique
    // receivers of row key (3D: z * ny + y, 2D: z) are rec_xu[rec_row[key] ..
    // rec_row[key + 1]), sorted by x, each as (x, unique receiver index)
    const int* rec_row;
    const int2* rec_xu;
    // second copy of the state for the fused step kernel (2D FP32/COMP16): the
    // fields (and residuals) and the V-phase memory variables; steps alternate
    // between the two copies in pairs, so the first copy is current between
    // pairs.  Tasks: columns of 120 cells x segments of zseg_f rows.
    void* fb[BP_NFIELDS];
    int8_t* flob[BP_NFIELDS];
    void* psiVb[3];
    long long tile0f;             // first task of this shot in the fused tiling
    int ncol_f, zseg_f, nzs_f, pad_f;
    // the interleaved step kernel (step_inter.cu): the shot's register tiles
    // grouped into bands of band_t consecutive tiles (whole row blocks; the
    // last band holds band_last), and its V and T work items in the order
    // V(0) .. V(lag_i - 1), then T(0), V(lag_i), T(1), V(lag_i + 1), ..., then
    // the remaining T; item0_i = the shot's first item, band0_i = its first
    // band counter
    long long item0_i;
    int band_t, nbands_i, lag_i, band_last, band0_i, pad_i;
    // indexed medium (FP32, COMP16, CBF16): when a shot's cells hold at most
    // 256 distinct coefficient tuples, med_idx gives each cell the index of its
    // tuple (one byte, at the cell's offset) and ctab holds the tuples decoded,
    // kMedRow float4 groups each (MedGroup); null: the per-cell arrays above
    const uint8_t* med_idx;
    const float4* ctab;
    int med_tuples, pad_med;
    // variable grid along z (PolF32G): fwd factors of rows 0..nz-1, then bwd
    // factors; null on a uniform grid
    const float* zf;
    template <class R>
    __device__ __forceinline__ R dtr() const { return sizeof(R) == 8 ? (R)dtd : (R)dt; }
};

// Groups of one indexed-medium tuple, as float4 (x, y, z, w):
//   V_X = (rho_x, cc1_x, cc2_x, rhof), V_Y / V_Z = (rho, cc1, cc2, 0) of that
//   axis, T_A = (C, M, H, H2mu), T_B = (mu_xz, mu_xy, mu_yz, 0).
enum MedGroup { MED_V_X, MED_V_Y, MED_V_Z, MED_T_A, MED_T_B, kMedRow };
constexpr int kMedMaxTuples = 256;

// The four indices of the chunk at cell offset c (a multiple of 4).
__device__ __forceinline__ unsigned med_ids(const ShotDesc& S, cidx c) {
    return __ldg(reinterpret_cast<const unsigned*>(S.med_idx + c));
}
// Group g of the tuple of the chunk's cell j.
__device__ __forceinline__ float4 med_group(const ShotDesc& S, unsigned ids, int j, int g) {
    return __ldg(S.ctab + ((ids >> (8 * j)) & 0xffu) * kMedRow + g);
}
// Group g of the chunk's four tuples: one load when the four cells share a
// tuple (a layered medium's rows, the bulk of a blocky one), else four.
__device__ __forceinline__ void med_group4(const ShotDesc& S, unsigned ids, int g, float4 (&t)[4]) {
    const unsigned id0 = ids & 0xffu;
    if (ids == id0 * 0x01010101u) {
        const float4 u = __ldg(S.ctab + id0 * kMedRow + g);
        t[0] = u; t[1] = u; t[2] = u; t[3] = u;
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++) t[j] = med_group(S, ids, j, g);
    }
}

// Steps are issued in chunks; step k of a chunk of shot s has index
// it = *step_base + k.  Reading the base from device memory lets one captured
// CUDA graph serve every chunk: k_advance moves the bases after each chunk.

// ---------------------------------------------------------------------------
// Compensated FP16 codec (the reference's store_ch / load_ch,
// Half/main.cu:59-100): value ~ hi + lo * u(hi), u = fp16 ulp(hi) / 256
// = 2^(e-19) with e the frexp exponent of |hi|, and u = 2^-32 for |hi| < 2^-14;
// for the biased fp16 exponent E of hi that is u = 2^(max(E, 1) - 33).
//
// Both directions work from the float value of hi: its exponent field masked
// out, m = 2^(E-15) for a normal hi, is clamped below to 2^-14 (zero and
// subnormal hi, E = 0) and above to 2^15 (inf / NaN hi, where the scale only
// has to stay finite), so u = 2^-18 m and 1/u = 2^18 / m are exact powers of
// two formed by integer operations on the float bits.  Checked bit for bit
// against the direct exponent-field form over all 2^24 (hi, lo) pairs and all
// 2^32 float inputs; this form takes 6 instead of 9 instructions per decode.
__device__ __forceinline__ unsigned half_scale_bits(float hf) {
    unsigned m = __float_as_uint(hf) & 0x7f800000u;
    m = m > 0x38800000u ? m : 0x38800000u;
    return m < 0x47000000u ? m : 0x47000000u;
}
__device__ __forceinline__ float decode_ch(__half hi, int8_t lo) {
    const float hf = __half2float(hi);
    // lo * 2^-18, exact: the int8 added to the bits of 48.0f (ulp 2^-18) minus 48
    const float lof = __int_as_float(0x42400000 + (int)lo) - 48.0f;
    return fmaf(lof, __uint_as_float(half_scale_bits(hf)), hf);   // hi + lo u, exact
}
__device__ __forceinline__ void encode_ch(float v, __half& hi, int8_t& lo) {
    const __half h = __float2half_rn(v);
    const float hf = __half2float(h);
    const float uinv = __uint_as_float(0x88000000u - half_scale_bits(hf));   // 1/u = 2^18 / m
    const float scaled = (v - hf) * uinv;                                      // exact
    int q = __float2int_rz(scaled + copysignf(0.5f, scaled));   // round half away from zero
    q = q > 127 ? 127 : (q < -127 ? -127 : q);
    hi = h;
    lo = (int8_t)q;
}

// Loads of arrays that no thread writes while the kernel runs (the fields a
// phase differentiates and the coefficients) may take the read-only data path
// (__ldg).  Measured on B200, bit-identical either way: the 2D FP32 T phase
// 2.7 % faster, the 3D order-4 FP32 V phase 4 % slower, COMP16 and the large 3D
// grid unchanged; so off by default.
#ifndef BP_NC_LOADS
#define BP_NC_LOADS 0
#endif
constexpr bool kReadOnlyPath = BP_NC_LOADS;
template <bool NC, class T>
__device__ __forceinline__ T ldv(const T* p) {
    if constexpr (NC) return __ldg(p);
    else return *p;
}

// ---------------------------------------------------------------------------
// Precision policies: storage of fields/coefficients and the arithmetic type.
struct PolF32 {
    using real = float;
    static constexpr int prec = BP_PREC_FP32;
    static constexpr int store = BP_PREC_FP32;   // storage format (PolB24: BP_PREC_CBF16)
    static constexpr bool exact = false;      // reference rounding (PolF32R)
    static constexpr bool graded = false;     // variable z spacing (PolF32G)
    static constexpr bool wide = false;       // 3D register caps for large grids (PolF32W)
    template <bool NC = false>
    __device__ __forceinline__ static void ld4(const void* p, const int8_t*, cidx i, real (&v)[4]) {
        float4 t = ldv<NC>(reinterpret_cast<const float4*>(static_cast<const float*>(p) + i));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    template <bool NC = false>
    __device__ __forceinline__ static real ld1(const void* p, const int8_t*, cidx i) {
        return ldv<NC>(static_cast<const float*>(p) + i);
    }
    __device__ __forceinline__ static void st4(void* p, int8_t*, cidx i, const real (&v)[4]) {
        *reinterpret_cast<float4*>(static_cast<float*>(p) + i) = make_float4(v[0], v[1], v[2], v[3]);
    }
    __device__ __forceinline__ static void st1(void* p, int8_t*, cidx i, real v) {
        static_cast<float*>(p)[i] = v;
    }
    // store (if st) and leave in v the value a later load returns
    __device__ __forceinline__ static void st4_rt(void* p, int8_t* lo, cidx i, real (&v)[4], bool st) {
        if (st) st4(p, lo, i, v);
    }
    // raw (undecoded) loads, for kernels that issue loads well before use
    using raw4 = float4;
    using raw1 = float;
    __device__ __forceinline__ static raw4 ldr4(const void* p, const int8_t*, cidx i) {
        return *reinterpret_cast<const float4*>(static_cast<const float*>(p) + i);
    }
    __device__ __forceinline__ static raw1 ldr1(const void* p, const int8_t*, cidx i) {
        return static_cast<const float*>(p)[i];
    }
    __device__ __forceinline__ static raw4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ __forceinline__ static raw1 zero1() { return 0.f; }
    __device__ __forceinline__ static void dec4(const raw4& t, real (&v)[4]) {
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    __device__ __forceinline__ static real dec1(raw1 t) { return t; }
};

struct PolF64 {
    using real = double;
    static constexpr int prec = BP_PREC_FP64;
    static constexpr int store = BP_PREC_FP64;
    static constexpr bool exact = false;
    static constexpr bool wide = false;
    static constexpr bool graded = false;
    template <bool NC = false>
    __device__ __forceinline__ static void ld4(const void* p, const int8_t*, cidx i, real (&v)[4]) {
        const double2* q = reinterpret_cast<const double2*>(static_cast<const double*>(p) + i);
        double2 a = ldv<NC>(q), b = ldv<NC>(q + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    template <bool NC = false>
    __device__ __forceinline__ static real ld1(const void* p, const int8_t*, cidx i) {
        return ldv<NC>(static_cast<const double*>(p) + i);
    }
    __device__ __forceinline__ static void st4(void* p, int8_t*, cidx i, const real (&v)[4]) {
        double2* q = reinterpret_cast<double2*>(static_cast<double*>(p) + i);
        q[0] = make_double2(v[0], v[1]);
        q[1] = make_double2(v[2], v[3]);
    }
    __device__ __forceinline__ static void st1(void* p, int8_t*, cidx i, real v) {
        static_cast<double*>(p)[i] = v;
    }
    __device__ __forceinline__ static void st4_rt(void* p, int8_t* lo, cidx i, real (&v)[4], bool st) {
        if (st) st4(p, lo, i, v);
    }
    struct raw4 { double2 a, b; };
    using raw1 = double;
    __device__ __forceinline__ static raw4 ldr4(const void* p, const int8_t*, cidx i) {
        const double2* q = reinterpret_cast<const double2*>(static_cast<const double*>(p) + i);
        return raw4{q[0], q[1]};
    }
    __device__ __forceinline__ static raw1 ldr1(const void* p, const int8_t*, cidx i) {
        return static_cast<const double*>(p)[i];
    }
    __device__ __forceinline__ static raw4 zero4() { return raw4{make_double2(0, 0), make_double2(0, 0)}; }
    __device__ __forceinline__ static raw1 zero1() { return 0.0; }
    __device__ __forceinline__ static void dec4(const raw4& t, real (&v)[4]) {
        v[0] = t.a.x; v[1] = t.a.y; v[2] = t.b.x; v[3] = t.b.y;
    }
    __device__ __forceinline__ static real dec1(raw1 t) { return t; }
};

// FP32 with the reference Float build's rounding where PolF32 rounds
// differently (bp_config.rounding = BP_ROUND_REFERENCE): the division by H is
// the IEEE quotient (PolF32: reciprocal plus one residual step, within one
// ulp), and the CPML memory update psi e + b (e prev + d) adds b (e prev + d)
// to the float product psi e with one rounding, which is what the reference's
// double-promoted expression gives (Float/main.cu:130-158,252-285: float
// psi e, the double product 0.5 fl(-DT d) (e prev + d), one rounding of the
// double sum to float).  Same storage as PolF32.
struct PolF32R : PolF32 {
    static constexpr bool exact = true;
};

// FP32 on a variable grid along z (bp_set_z_spacing): the z differences are
// multiplied by per-row factors, fwd[z] = 1/dz[z] for the forward difference
// from rows z, z+1 and bwd[z] = 2/(dz[z-1] + dz[z]) for the backward one from
// the half rows z-1/2, z+1/2 (S.zf); x and y differences as PolF32.
struct PolF32G : PolF32 {
    static constexpr bool graded = true;
};

// FP32 on large 3D grids: the same arithmetic as PolF32 under looser register
// caps (tile.cuh, phase_min_blocks), chosen at launch by the grid's size.
struct PolF32W : PolF32 {
    static constexpr bool wide = true;
};

// Compensated BF16 storage (BP_PREC_CBF16): each value is the top 24 bits of
// its fp32 word, rounded to nearest even at bit 8, kept as the bf16 "hi" half
// (bits 31..16) and an unsigned 8-bit residual "lo" (bits 15..8): value bits =
// hi << 16 | lo << 8.  16 significant bits (relative rounding <= 2^-17), the
// fp32 exponent range, so no exponent scaling or rescale; decoding places two
// bytes.  Arithmetic is FP32's (PolF32's prec), storage 3 bytes per value like
// COMP16.
// The rounded word in place: bits 31..8 hold the 24-bit value, bits 7..0
// are don't-care (the stores take bytes 1..3 of it).
__device__ __forceinline__ unsigned b24_round_word(float v) {
    const unsigned b = __float_as_uint(v);
    if ((b & 0x7f800000u) == 0x7f800000u) return b | ((b & 0x007fffffu) ? 0x100u : 0u);   // inf / nan
    return b + 0x7fu + ((b >> 8) & 1u);                                                  // RNE at bit 8
}

struct PolB24 : PolF32 {
    static constexpr int store = BP_PREC_CBF16;
    // Decoding and packing are byte moves (__byte_perm): value j of a 4-cell
    // group is [0, lo_j, hi_j.lo, hi_j.hi] from the low byte up.
    template <bool NC = false>
    __device__ __forceinline__ static void ld4(const void* p, const int8_t* lo, cidx i, real (&v)[4]) {
        const uint2 h = ldv<NC>(reinterpret_cast<const uint2*>(static_cast<const uint16_t*>(p) + i));
        const unsigned l = ldv<NC>(reinterpret_cast<const unsigned*>(lo + i));
        const unsigned y = l << 8, y2 = l >> 8;        // [0, l0, l1, l2], [l1, l2, l3, 0]
        v[0] = __uint_as_float(__byte_perm(h.x, y, 0x1054));
        v[1] = __uint_as_float(__byte_perm(h.x, y, 0x3264));
        v[2] = __uint_as_float(__byte_perm(h.y, y, 0x1074));
        v[3] = __uint_as_float(__byte_perm(h.y, y2, 0x3267));
    }
    template <bool NC = false>
    __device__ __forceinline__ static real ld1(const void* p, const int8_t* lo, cidx i) {
        const unsigned h = ldv<NC>(static_cast<const uint16_t*>(p) + i);
        const unsigned l = (unsigned char)ldv<NC>(reinterpret_cast<const signed char*>(lo) + i);
        return __uint_as_float(__byte_perm(h, l, 0x1042));
    }
    __device__ __forceinline__ static void st4(void* p, int8_t* lo, cidx i, const real (&v)[4]) {
        unsigned w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) w[j] = b24_round_word(v[j]);
        *reinterpret_cast<uint2*>(static_cast<uint16_t*>(p) + i) =
            make_uint2(__byte_perm(w[0], w[1], 0x7632), __byte_perm(w[2], w[3], 0x7632));
        *reinterpret_cast<unsigned*>(lo + i) =
            __byte_perm(__byte_perm(w[0], w[1], 0x0051), __byte_perm(w[2], w[3], 0x0051), 0x5410);
    }
    __device__ __forceinline__ static void st1(void* p, int8_t* lo, cidx i, real v) {
        const unsigned w = b24_round_word(v);
        static_cast<uint16_t*>(p)[i] = (uint16_t)(w >> 16);
        lo[i] = (int8_t)(unsigned char)((w >> 8) & 0xffu);
    }
    __device__ __forceinline__ static void st4_rt(void* p, int8_t* lo, cidx i, real (&v)[4], bool st) {
        if (st) st4(p, lo, i, v);
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = __uint_as_float(b24_round_word(v[j]) & 0xffffff00u);
    }
    // (the raw-load interface of PolF32 does not apply; the marching and staged
    // kernels, its only users, do not take this storage)
};

// COMP16: fp16 hi (8 bytes per 4 cells) + int8 lo (4 bytes per 4 cells).
// A null lo pointer means "hi only" (used for fp16-only coefficient storage).
struct PolC16 {
    using real = float;
    static constexpr int prec = BP_PREC_COMP16;
    static constexpr int store = BP_PREC_COMP16;
    static constexpr bool exact = false;
    static constexpr bool wide = false;
    static constexpr bool graded = false;
    template <bool NC = false>
    __device__ __forceinline__ static void ld4(const void* p, const int8_t* lo, cidx i, real (&v)[4]) {
        uint2 h = ldv<NC>(reinterpret_cast<const uint2*>(static_cast<const __half*>(p) + i));
        __half2 h01 = *reinterpret_cast<__half2*>(&h.x);
        __half2 h23 = *reinterpret_cast<__half2*>(&h.y);
        __half hs[4] = {__low2half(h01), __high2half(h01), __low2half(h23), __high2half(h23)};
        if (lo) {
            char4 l = ldv<NC>(reinterpret_cast<const char4*>(lo + i));
            v[0] = decode_ch(hs[0], l.x); v[1] = decode_ch(hs[1], l.y);
            v[2] = decode_ch(hs[2], l.z); v[3] = decode_ch(hs[3], l.w);
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) v[j] = __half2float(hs[j]);
        }
    }
    template <bool NC = false>
    __device__ __forceinline__ static real ld1(const void* p, const int8_t* lo, cidx i) {
        __half h = ldv<NC>(static_cast<const __half*>(p) + i);
        return lo ? decode_ch(h, ldv<NC>(reinterpret_cast<const signed char*>(lo) + i)) : __half2float(h);
    }
    __device__ __forceinline__ static void st4(void* p, int8_t* lo, cidx i, const real (&v)[4]) {
        __half hs[4];
        int8_t ls[4];
#pragma unroll
        for (int j = 0; j < 4; j++) encode_ch(v[j], hs[j], ls[j]);
        uint2 h;
        __half2 a = __halves2half2(hs[0], hs[1]), b = __halves2half2(hs[2], hs[3]);
        h.x = *reinterpret_cast<unsigned*>(&a);
        h.y = *reinterpret_cast<unsigned*>(&b);
        *reinterpret_cast<uint2*>(static_cast<__half*>(p) + i) = h;
        *reinterpret_cast<char4*>(lo + i) = make_char4(ls[0], ls[1], ls[2], ls[3]);
    }
    __device__ __forceinline__ static void st1(void* p, int8_t* lo, cidx i, real v) {
        __half h;
        int8_t l;
        encode_ch(v, h, l);
        static_cast<__half*>(p)[i] = h;
        lo[i] = l;
    }
    // store (if st) and leave in v the decoded stored value, as a later load returns it
    __device__ __forceinline__ static void st4_rt(void* p, int8_t* lo, cidx i, real (&v)[4], bool st) {
        __half hs[4];
        int8_t ls[4];
#pragma unroll
        for (int j = 0; j < 4; j++) encode_ch(v[j], hs[j], ls[j]);
        if (st) {
            uint2 h;
            __half2 a = __halves2half2(hs[0], hs[1]), b = __halves2half2(hs[2], hs[3]);
            h.x = *reinterpret_cast<unsigned*>(&a);
            h.y = *reinterpret_cast<unsigned*>(&b);
            *reinterpret_cast<uint2*>(static_cast<__half*>(p) + i) = h;
            *reinterpret_cast<char4*>(lo + i) = make_char4(ls[0], ls[1], ls[2], ls[3]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = decode_ch(hs[j], ls[j]);
    }
    // raw loads: the fp16 words and the residual bytes (zero residuals where
    // the array has none, which decodes to the same value as hi alone)
    struct raw4 { uint2 h; char4 l; };
    struct raw1 { __half h; int8_t l; };
    __device__ __forceinline__ static raw4 ldr4(const void* p, const int8_t* lo, cidx i) {
        raw4 t;
        t.h = *reinterpret_cast<const uint2*>(static_cast<const __half*>(p) + i);
        t.l = lo ? *reinterpret_cast<const char4*>(lo + i) : make_char4(0, 0, 0, 0);
        return t;
    }
    __device__ __forceinline__ static raw1 ldr1(const void* p, const int8_t* lo, cidx i) {
        raw1 t;
        t.h = static_cast<const __half*>(p)[i];
        t.l = lo ? lo[i] : (int8_t)0;
        return t;
    }
    __device__ __forceinline__ static raw4 zero4() {
        raw4 t;
        t.h = make_uint2(0u, 0u);
        t.l = make_char4(0, 0, 0, 0);
        return t;
    }
    __device__ __forceinline__ static raw1 zero1() {
        raw1 t;
        t.h = __ushort_as_half((unsigned short)0);
        t.l = 0;
        return t;
    }
    __device__ __forceinline__ static void dec4(const raw4& t, real (&v)[4]) {
        __half2 h01 = *reinterpret_cast<const __half2*>(&t.h.x);
        __half2 h23 = *reinterpret_cast<const __half2*>(&t.h.y);
        v[0] = decode_ch(__low2half(h01), t.l.x); v[1] = decode_ch(__high2half(h01), t.l.y);
        v[2] = decode_ch(__low2half(h23), t.l.z); v[3] = decode_ch(__high2half(h23), t.l.w);
    }
    __device__ __forceinline__ static real dec1(const raw1& t) { return decode_ch(t.h, t.l); }
};

}  // namespace bpk

namespace bpk {
static_assert(sizeof(ShotDesc) % 8 == 0, "ShotDesc is copied to shared memory in 8-byte words");
static_assert(alignof(ShotDesc) == 8, "ShotDesc alignment");
}  // namespace bpk

// tile.cuh - the register tile kernels' work units, shared by the two-phase
// kernels (step.cu) and the interleaved step kernel (step_inter.cu): the
// V-phase and T-phase arithmetic of one 4-cell chunk (whole or one output
// group at a time), the tile geometry, and the per-tile unit loop.
//
// Reference kernels: FD_V Float/main.cu:64-192, Half/main.cu:156-268; FD_T
// Float/main.cu:194-295, Half/main.cu:270-371.
#pragma once
#include "post.cuh"
#include "shot.h"

namespace bpk {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kSegCells = 128;
// 3D tiles: the 8 rows of a tile are 8/TZ consecutive y rows of TZ consecutive
// z planes, so the z neighbours of most rows are rows of the same tile (2D
// tiles are 8 consecutive z rows).  Measured on B200 (192^3, 200^3 order 4,
// 552 x 552 x 424; all shapes bit-identical): FP32 is fastest with 1 x 8
// (up to 8 % over 8 x 1), COMP16 with 4 x 2.
__host__ __device__ constexpr int tile_tz(int prec) {
    return prec == BP_PREC_FP32 ? 8 : (prec == BP_PREC_COMP16 ? 2 : 1);
}

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

#ifndef BP_RS_SPLIT
#define BP_RS_SPLIT 1
#endif
// Resident CTAs per SM the 2D phase kernels are register-limited to (1 = no
// limit).  Measured on B200 for the 4040 x 2040 order-2 grid: FP32 is fastest
// at 3 (80 registers, no spills); COMP16, whose decode/encode chains leave it
// latency-bound, at 6 (40 registers) for both phases, the T phase in grouped
// form (below), both with some spilled values; FP64 at 2 (128 registers;
// uncapped it takes ~150, one CTA per SM, and runs 40 % slower).
#ifndef BP_MINB_F32
#define BP_MINB_F32 3
#endif
#ifndef BP_MINB_C16
#define BP_MINB_C16 6
#endif
#ifndef BP_MINB_C16_V
#define BP_MINB_C16_V 6
#endif
#ifndef BP_MINB_F64
#define BP_MINB_F64 2
#endif
// 3D: uncapped, the kernels take 128-169 registers (1-2 CTAs per SM); capped
// at 3 CTAs (80 registers, ~130 bytes spilled) the 192^3 order-2 and 200^3
// order-4 FP32 steps run 1.75-2.1x faster on B200.  COMP16, taken one output
// group at a time (v_chunk_g/t_chunk_g, next to no spills), is fastest at 4 CTAs
// (64 registers) on the 552 x 552 x 424 and 200^3 grids; FP64 at 2 (128
// registers; uncapped it takes 196-240, one CTA per SM).
#ifndef BP_MINB3_F32
#define BP_MINB3_F32 3
#endif
// 3D FP32 on large grids (PolF32W, from kWideCells updated cells of a launch):
// 2 CTAs (128 registers, no spills) for the T phase and the order-2 V phase,
// measured on B200: the 552 x 552 x 424 order-2 step 5 % faster (16,716 ->
// 17,507 Mcell-updates/s) and the uniform 300^3 order-2 T phase 15 % faster,
// while the 192^3 order-2 reference run (7 M cells) is 13 % slower (26 % with
// reference rounding) and keeps 3; the order-4 V phase keeps 3 everywhere
// (12 % slower at 2)
#ifndef BP_MINB3_F32_WIDE
#define BP_MINB3_F32_WIDE 2
#endif
#ifndef BP_MINB3_C16
#define BP_MINB3_C16 4
#endif
#ifndef BP_MINB3_F64
#define BP_MINB3_F64 2
#endif
// Compensated-BF16 storage (FP32 arithmetic, 3-byte values, a two-instruction
// decode): its own caps.
#ifndef BP_MINB_B24
#define BP_MINB_B24 3
#endif
#ifndef BP_MINB_B24_V
#define BP_MINB_B24_V 3
#endif
#ifndef BP_MINB3_B24
#define BP_MINB3_B24 3
#endif
template <int DIM, int ORD, class P, bool VPHASE>
__host__ __device__ constexpr int phase_min_blocks() {
    if (P::store == BP_PREC_CBF16) return DIM == 3 ? BP_MINB3_B24 : (VPHASE ? BP_MINB_B24_V : BP_MINB_B24);
    if (DIM == 3 && P::prec == BP_PREC_FP32 && P::wide) return (VPHASE && ORD == 4) ? BP_MINB3_F32 : BP_MINB3_F32_WIDE;
    if (DIM == 3) return P::prec == BP_PREC_FP32 ? BP_MINB3_F32 : P::prec == BP_PREC_COMP16 ? BP_MINB3_C16 : BP_MINB3_F64;
    return P::prec == BP_PREC_FP32 ? BP_MINB_F32
                                   : P::prec == BP_PREC_COMP16 ? (VPHASE ? BP_MINB_C16_V : BP_MINB_C16) : BP_MINB_F64;
}
// How a tile learns its step index: 1 = once per shot per launch, 0 = a read
// of the step counter per tile (measured faster for FP32 at 80 registers).
#ifndef BP_TILE_LOOP_F32
#define BP_TILE_LOOP_F32 0
#endif
#ifndef BP_TILE_LOOP_C16
#define BP_TILE_LOOP_C16 1
#endif
template <class P>
__host__ __device__ constexpr bool step_once_per_shot() {
    return P::prec == BP_PREC_COMP16 ? BP_TILE_LOOP_C16 : P::prec == BP_PREC_FP32 ? BP_TILE_LOOP_F32 : 1;
}

// Phases whose neighbour-field and coefficient loads take the read-only path
// (bit 0 = V, bit 1 = T), for the whole-chunk form of FP32.  Measured on B200:
// the T phase 2.5 % faster in 2D (4040 x 2040) and 1-2 % in 3D (192^3, 200^3
// order 4, 552 x 552 x 424); the V phase unchanged in 2D, up to 4 % slower in 3D.
#ifndef BP_NC_F32_2D
#define BP_NC_F32_2D 2
#endif
#ifndef BP_NC_F32_3D
#define BP_NC_F32_3D 2
#endif
template <int DIM, class P, bool VPHASE>
__host__ __device__ constexpr bool read_only_loads() {
    return kReadOnlyPath ||
           (P::prec == BP_PREC_FP32 && (((DIM == 2 ? BP_NC_F32_2D : BP_NC_F32_3D) >> (VPHASE ? 0 : 1)) & 1));
}

// ---------------------------------------------------------------------------
// V phase for one 4-cell chunk: FD_V (Float/main.cu:103-191).
// NCOK = false: no read-only-path loads (the interleaved step kernel reads
// arrays that the same launch writes)
template <int DIM, int ORD, class P, bool RS, bool NCOK = true>
__device__ __forceinline__ void v_chunk(const ShotDesc& S, int x0, int y, int z, typename P::real r,
                                        unsigned mask) {
    using R = typename P::real;
    const cidx sy = S.pitch, sz = S.plane;
    const cidx c = x0 + y * sy + z * sz;
    const cidx row = c - x0;

    VState<R> V;
    // an indexed medium's tuple indices first: their load overlaps the field loads
    if (med_on<P>(S)) V.mids = med_ids(S, c);
    auto &x1 = V.x1, &x3 = V.x3, &s1 = V.s1, &z1 = V.z1, &z2 = V.z2, &s3 = V.s3;
    auto &x2 = V.x2, &y1 = V.y1, &y2 = V.y2, &y3 = V.y3, &s2 = V.s2, &z3 = V.z3;

    // ---- derivatives of the old stresses (x1..s3, Float/main.cu:115-128) ----
    {
        R v[4 + ORD];
        load_span<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TXX], S.flo[BP_F_TXX], row, x0, S.nx, v);       // txx: D+x
#pragma unroll
        for (int j = 0; j < 4; j++) x1[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
        load_span<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_P], S.flo[BP_F_P], row, x0, S.nx, v);           // p: D+x
#pragma unroll
        for (int j = 0; j < 4; j++) s1[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
        load_span<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], row, x0, S.nx, v);       // txz: D-x
#pragma unroll
        for (int j = 0; j < 4; j++) z2[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
        R a[ORD + 1][4];
        load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TXZ], S.flo[BP_F_TXZ], c, sz, a);               // txz: D-z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            x3[j] = deriv_z<P, false>(rbwd<ORD>(t), S, z); }
        load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TZZ], S.flo[BP_F_TZZ], c, sz, a);               // tzz: D+z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            z1[j] = deriv_z<P, true>(rfwd<ORD>(t), S, z); }
        load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_P], S.flo[BP_F_P], c, sz, a);                   // p: D+z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            s3[j] = deriv_z<P, true>(rfwd<ORD>(t), S, z); }
        if constexpr (DIM == 3) {
            load_span<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TXY], S.flo[BP_F_TXY], row, x0, S.nx, v);   // txy: D-x
#pragma unroll
            for (int j = 0; j < 4; j++) y2[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
            load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TXY], S.flo[BP_F_TXY], c, sy, a);           // txy: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                x2[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TYY], S.flo[BP_F_TYY], c, sy, a);           // tyy: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                y1[j] = deriv_div<P>(rfwd<ORD>(t), S); }
            load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TYZ], S.flo[BP_F_TYZ], c, sz, a);           // tyz: D-z
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                y3[j] = deriv_z<P, false>(rbwd<ORD>(t), S, z); }
            load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_TYZ], S.flo[BP_F_TYZ], c, sy, a);           // tyz: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                z3[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P, (read_only_loads<DIM, P, true>() && NCOK)>(S.f[BP_F_P], S.flo[BP_F_P], c, sy, a);               // p: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                s2[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        }
    }
    v_tail<DIM, ORD, P, false, RS, (read_only_loads<DIM, P, true>() && NCOK)>(S, c, x0, y, z, r, mask, V);
}

// ---------------------------------------------------------------------------
// T phase for one 4-cell chunk: FD_T (Float/main.cu:232-294).
template <int DIM, int ORD, class P, bool RS, bool NCOK = true>
__device__ __forceinline__ void t_chunk(const ShotDesc& S, int x0, int y, int z, typename P::real r,
                                        unsigned mask) {
    using R = typename P::real;
    const cidx sy = S.pitch, sz = S.plane;
    const cidx c = x0 + y * sy + z * sz;
    const cidx row = c - x0;

    TState<R> T;
    if (med_on<P>(S)) T.mids = med_ids(S, c);
    auto &uxx = T.uxx, &uzz = T.uzz, &wx = T.wx, &wz = T.wz, &uxz = T.uxz, &uzx = T.uzx;
    auto &uyy = T.uyy, &wy = T.wy, &uxy = T.uxy, &uyx = T.uyx, &uyz = T.uyz, &uzy = T.uzy;

    {
        R v[4 + ORD];
        R a[ORD + 1][4];
        load_span<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUX], S.flo[BP_F_VUX], row, x0, S.nx, v);       // vux: D-x
#pragma unroll
        for (int j = 0; j < 4; j++) uxx[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
        load_span<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VWX], S.flo[BP_F_VWX], row, x0, S.nx, v);       // vwx: D-x
#pragma unroll
        for (int j = 0; j < 4; j++) wx[j] = deriv_div<P>(dbwd<ORD>(v, j), S);
        load_span<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], row, x0, S.nx, v);       // vuz: D+x
#pragma unroll
        for (int j = 0; j < 4; j++) uzx[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
        load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], c, sz, a);               // vuz: D-z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            uzz[j] = deriv_z<P, false>(rbwd<ORD>(t), S, z); }
        load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VWZ], S.flo[BP_F_VWZ], c, sz, a);               // vwz: D-z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            wz[j] = deriv_z<P, false>(rbwd<ORD>(t), S, z); }
        load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUX], S.flo[BP_F_VUX], c, sz, a);               // vux: D+z
#pragma unroll
        for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
            for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
            uxz[j] = deriv_z<P, true>(rfwd<ORD>(t), S, z); }
        if constexpr (DIM == 3) {
            load_span<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUY], S.flo[BP_F_VUY], row, x0, S.nx, v);   // vuy: D+x
#pragma unroll
            for (int j = 0; j < 4; j++) uyx[j] = deriv_div<P>(dfwd<ORD>(v, j), S);
            load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUY], S.flo[BP_F_VUY], c, sy, a);           // vuy: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uyy[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VWY], S.flo[BP_F_VWY], c, sy, a);           // vwy: D-y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                wy[j] = deriv_div<P>(rbwd<ORD>(t), S); }
            load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUX], S.flo[BP_F_VUX], c, sy, a);           // vux: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uxy[j] = deriv_div<P>(rfwd<ORD>(t), S); }
            load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUY], S.flo[BP_F_VUY], c, sz, a);           // vuy: D+z
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uyz[j] = deriv_z<P, true>(rfwd<ORD>(t), S, z); }
            load_rows<ORD, P, (read_only_loads<DIM, P, false>() && NCOK)>(S.f[BP_F_VUZ], S.flo[BP_F_VUZ], c, sy, a);           // vuz: D+y
#pragma unroll
            for (int j = 0; j < 4; j++) { R t[ORD + 1];
#pragma unroll
                for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
                uzy[j] = deriv_div<P>(rfwd<ORD>(t), S); }
        }
    }
    t_tail<DIM, ORD, P, false, RS, (read_only_loads<DIM, P, false>() && NCOK)>(S, c, x0, y, z, r, mask, T);
}

// ---------------------------------------------------------------------------
// Chunks taken one output group at a time.  v_chunk/t_chunk form all the
// derivatives of a chunk before the CPML and the updates: twelve in 3D, so 48
// values (96 in FP64) are live at once and the capped kernels spill.  Here each
// velocity component (and each shear stress, then the normal stresses and
// the pressure) loads, differences, CPML-corrects and stores only what it
// needs.  Every element goes through the same operations in the same order
// as in v_tail/t_tail, so the results are bit-identical.
// Which phases take this form, per dimension and precision (bit 0 = V, bit 1
// = T).  Measured on B200 (3D: 192^3 and 552 x 552 x 424 order 2, 200^3
// order 4; 2D: 4040 x 2040 order 2): 3D COMP16 both (12-16 % off the step,
// its spills gone); 2D COMP16 the T phase (13 % off it, the V phase 2 %
// slower grouped); FP64 the 3D T phase (with 2 CTAs per SM, 25-30 % off the
// 3D step); FP32 neither (10-20 % slower, its latency-bound phases losing the
// loads they had in flight).
#ifndef BP_GROUP3_C16
#define BP_GROUP3_C16 3
#endif
#ifndef BP_GROUP3_F32
#define BP_GROUP3_F32 0
#endif
#ifndef BP_GROUP3_F64
#define BP_GROUP3_F64 2
#endif
#ifndef BP_GROUP2_C16
#define BP_GROUP2_C16 2
#endif
#ifndef BP_GROUP2_F32
#define BP_GROUP2_F32 0
#endif
#ifndef BP_GROUP2_F64
#define BP_GROUP2_F64 0
#endif
template <int DIM, class P, bool VPHASE>
__host__ __device__ constexpr bool grouped() {
    const int m = DIM == 3 ? (P::prec == BP_PREC_COMP16 ? BP_GROUP3_C16 : P::prec == BP_PREC_FP32 ? BP_GROUP3_F32 : BP_GROUP3_F64)
                           : (P::prec == BP_PREC_COMP16 ? BP_GROUP2_C16 : P::prec == BP_PREC_FP32 ? BP_GROUP2_F32 : BP_GROUP2_F64);
    return (m >> (VPHASE ? 0 : 1)) & 1;
}

// Difference along x of one field at the chunk (span load), divided by H.
template <int ORD, class P, bool FWD>
__device__ __forceinline__ void d_span(const ShotDesc& S, int f, cidx row, int x0,
                                       typename P::real (&d)[4]) {
    typename P::real v[4 + ORD];
    load_span<ORD, P>(S.f[f], S.flo[f], row, x0, S.nx, v);
#pragma unroll
    for (int j = 0; j < 4; j++) d[j] = deriv_div<P>(FWD ? dfwd<ORD>(v, j) : dbwd<ORD>(v, j), S);
}
// Difference across rows (y or z) of one field at the chunk, divided by H.
template <int ORD, class P, bool FWD>
__device__ __forceinline__ void d_rows(const ShotDesc& S, int f, cidx c, cidx stride,
                                       typename P::real (&d)[4]) {
    static_assert(!P::graded, "the grouped forms take a uniform grid (FP32 runs the whole-chunk form)");
    using R = typename P::real;
    R a[ORD + 1][4];
    load_rows<ORD, P>(S.f[f], S.flo[f], c, stride, a);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R t[ORD + 1];
#pragma unroll
        for (int k = 0; k <= ORD; k++) t[k] = a[k][j];
        d[j] = deriv_div<P>(FWD ? rfwd<ORD>(t) : rbwd<ORD>(t), S);
    }
}
// Masked cells feed zero derivatives into the memory variables.
template <class R>
__device__ __forceinline__ void mask0(R (&d)[4], unsigned mask) {
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (!(mask >> j & 1u)) d[j] = 0;
}
// CPML of one derivative on the slab of `axis` (slot k, half-grid profile if
// half); nothing outside that slab.  Slabs hold 3 slots per phase in 2D, 4 in 3D.
template <int DIM, bool RS, class R, bool EX = false>
__device__ __forceinline__ void cpml_g(const ShotDesc& S, void* const (&psi)[3], int axis, int k, bool half,
                                       cidx si, int x0, int y, int z, R (&d)[4], R r) {
    if (si < 0) return;
    const void* pb = half ? S.pb2[axis] : S.pb[axis];
    const void* pe = half ? S.pe2[axis] : S.pe[axis];
    cpml_slot<DIM == 3 ? 4 : 3, RS, R, EX>(d, psi[axis], S.slab_cells[axis], k, si, axis == 0,
                                        axis == 0 ? x0 : (axis == 1 ? y : z), x0, pb, pe, r);
}

// One velocity component AX (0 = x, 1 = y, 2 = z) of the V phase
// (Float/main.cu:103-191 for that component).
template <int DIM, int ORD, class P, bool RS, int AX>
__device__ __forceinline__ void v_comp(const ShotDesc& S, cidx c, cidx row, int x0, int y, int z,
                                       typename P::real r, unsigned mask, const typename P::real (&rf)[4]) {
    using R = typename P::real;
    const cidx sy = S.pitch, sz = S.plane;
    // dx, dy, dz: the stress derivatives summed into this component (dy in 3D
    // only); dp: the pressure derivative along AX.  Slots as in v_tail.
    R dx[4], dy[4], dz[4], dp[4];
    if constexpr (AX == 0) {
        d_span<ORD, P, true>(S, BP_F_TXX, row, x0, dx);                          // x1
        if constexpr (DIM == 3) d_rows<ORD, P, false>(S, BP_F_TXY, c, sy, dy);   // x2
        d_rows<ORD, P, false>(S, BP_F_TXZ, c, sz, dz);                           // x3
        d_span<ORD, P, true>(S, BP_F_P, row, x0, dp);                            // s1
    } else if constexpr (AX == 1) {
        d_span<ORD, P, false>(S, BP_F_TXY, row, x0, dx);                         // y2
        d_rows<ORD, P, true>(S, BP_F_TYY, c, sy, dy);                            // y1
        d_rows<ORD, P, false>(S, BP_F_TYZ, c, sz, dz);                           // y3
        d_rows<ORD, P, true>(S, BP_F_P, c, sy, dp);                              // s2
    } else {
        d_span<ORD, P, false>(S, BP_F_TXZ, row, x0, dx);                         // z2
        if constexpr (DIM == 3) d_rows<ORD, P, false>(S, BP_F_TYZ, c, sy, dy);   // z3
        d_rows<ORD, P, true>(S, BP_F_TZZ, c, sz, dz);                            // z1
        d_rows<ORD, P, true>(S, BP_F_P, c, sz, dp);                              // s3
    }
    if constexpr (P::prec == BP_PREC_COMP16 && RS) {
        scale4(dx, r); scale4(dz, r); scale4(dp, r);
        if constexpr (DIM == 3) scale4(dy, r);
    }
    mask0(dx, mask); mask0(dz, mask); mask0(dp, mask);
    if constexpr (DIM == 3) mask0(dy, mask);
    void* const psi[3] = {S.psiV[0], S.psiV[1], S.psiV[2]};
    const cidx s0 = slab_index(S, 0, x0, y, z), s2 = slab_index(S, 2, x0, y, z);
    const cidx s1 = DIM == 3 ? slab_index(S, 1, x0, y, z) : -1;
    if constexpr (AX == 0) {
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 0, true, s0, x0, y, z, dx, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 1, true, s0, x0, y, z, dp, r);
        if constexpr (DIM == 3) cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 0, false, s1, x0, y, z, dy, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 0, false, s2, x0, y, z, dz, r);
    } else if constexpr (AX == 1) {
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 3, false, s0, x0, y, z, dx, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 1, true, s1, x0, y, z, dy, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 2, true, s1, x0, y, z, dp, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 3, false, s2, x0, y, z, dz, r);
    } else {
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 2, false, s0, x0, y, z, dx, r);
        if constexpr (DIM == 3) cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 3, false, s1, x0, y, z, dy, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 1, true, s2, x0, y, z, dz, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 2, true, s2, x0, y, z, dp, r);
    }
    // the divergence in v_tail's summation order: x1 (+x2) +x3, y1+y2+y3, z1+z2 (+z3)
    R sum[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (DIM == 2) sum[j] = AX == 0 ? dx[j] + dz[j] : dz[j] + dx[j];
        else if constexpr (AX == 0) sum[j] = dx[j] + dy[j] + dz[j];
        else if constexpr (AX == 1) sum[j] = dy[j] + dx[j] + dz[j];
        else sum[j] = dz[j] + dx[j] + dy[j];
    }
    constexpr int fu = AX == 0 ? BP_F_VUX : AX == 1 ? BP_F_VUY : BP_F_VUZ;
    constexpr int fw = AX == 0 ? BP_F_VWX : AX == 1 ? BP_F_VWY : BP_F_VWZ;
    constexpr int crho = AX == 0 ? VC_RHO_X : AX == 1 ? VC_RHO_Y : VC_RHO_Z;
    constexpr int cc1 = AX == 0 ? VC_CC1_X : AX == 1 ? VC_CC1_Y : VC_CC1_Z;
    constexpr int cc2 = AX == 0 ? VC_CC2_X : AX == 1 ? VC_CC2_Y : VC_CC2_Z;
    R rho[4], c1[4], c2[4], vu[4], vw[4], nu[4], nw[4];
    vcoef4<P>(S, crho, c, rho);
    vcoef4<P>(S, cc1, c, c1);
    vcoef4<P>(S, cc2, c, c2);
    P::ld4(S.f[fu], S.flo[fu], c, vu);
    P::ld4(S.f[fw], S.flo[fw], c, vw);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (P::prec == BP_PREC_COMP16) {
            const R wo = RS ? mulr(vw[j], r) : vw[j], uo = RS ? mulr(vu[j], r) : vu[j];
            R rr = rf[j] * rho[j];
            R wn = c1[j] * wo - (rr * c2[j]) * sum[j] - c2[j] * dp[j];
            nw[j] = wn;
            nu[j] = uo + rho[j] * sum[j] - rr * (wn - wo);
        } else {
            R wo = vw[j];
            const R num = wo * c2[j] - S.dtr<R>() * (rf[j] * rho[j] * sum[j] + dp[j]);
            const R wn = (c1[j] == (R)0) ? (R)0 : (num == (R)0 ? num * c1[j] : num / c1[j]);
            nw[j] = wn;
            nu[j] = vu[j] + S.dtr<R>() * rho[j] * sum[j] - rf[j] * rho[j] * (wn - wo);
        }
        if (!(mask >> j & 1u)) { nw[j] = vw[j]; nu[j] = vu[j]; }
    }
    P::st4(S.f[fw], S.flo[fw], c, nw);
    P::st4(S.f[fu], S.flo[fu], c, nu);
}

template <int DIM, int ORD, class P, bool RS>
__device__ __forceinline__ void v_chunk_g(const ShotDesc& S, int x0, int y, int z, typename P::real r,
                                          unsigned mask) {
    using R = typename P::real;
    const cidx c = x0 + y * S.pitch + z * (cidx)S.plane;
    const cidx row = c - x0;
    R rf[4];
    vcoef4<P>(S, VC_RHOF, c, rf);
    v_comp<DIM, ORD, P, RS, 0>(S, c, row, x0, y, z, r, mask, rf);
    if constexpr (DIM == 3) v_comp<DIM, ORD, P, RS, 1>(S, c, row, x0, y, z, r, mask, rf);
    v_comp<DIM, ORD, P, RS, 2>(S, c, row, x0, y, z, r, mask, rf);
}

// Old value of a stress field at the chunk, with this step's rescale.
template <class P, bool RS>
__device__ __forceinline__ void ld_old(const ShotDesc& S, int f, cidx c, typename P::real r,
                                       typename P::real (&o)[4]) {
    P::ld4(S.f[f], S.flo[f], c, o);
    if constexpr (P::prec == BP_PREC_COMP16 && RS) scale4(o, r);
}
template <class P>
__device__ __forceinline__ void st_new(const ShotDesc& S, int f, cidx c, unsigned mask,
                                       typename P::real (&nv)[4], const typename P::real (&ov)[4]) {
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (!(mask >> j & 1u)) nv[j] = ov[j];
    P::st4(S.f[f], S.flo[f], c, nv);
}

// One shear stress of the T phase: SH 0 = txy, 1 = tyz (3D only), 2 = txz
// (Float/main.cu:232-294 for that stress).
template <int DIM, int ORD, class P, bool RS, int SH>
__device__ __forceinline__ void t_shear(const ShotDesc& S, cidx c, cidx row, int x0, int y, int z,
                                        typename P::real r, unsigned mask, void* const (&psi)[3]) {
    using R = typename P::real;
    const cidx sy = S.pitch, sz = S.plane;
    R a[4], b[4];    // the two derivatives, in the order of the update's sum
    if constexpr (SH == 0) {
        d_rows<ORD, P, true>(S, BP_F_VUX, c, sy, a);        // uxy
        d_span<ORD, P, true>(S, BP_F_VUY, row, x0, b);      // uyx
    } else if constexpr (SH == 1) {
        d_rows<ORD, P, true>(S, BP_F_VUY, c, sz, a);        // uyz
        d_rows<ORD, P, true>(S, BP_F_VUZ, c, sy, b);        // uzy
    } else {
        d_rows<ORD, P, true>(S, BP_F_VUX, c, sz, a);        // uxz
        d_span<ORD, P, true>(S, BP_F_VUZ, row, x0, b);      // uzx
    }
    mask0(a, mask); mask0(b, mask);
    if constexpr (SH == 0) {
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 3, true, slab_index(S, 0, x0, y, z), x0, y, z, b, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 2, true, slab_index(S, 1, x0, y, z), x0, y, z, a, r);
    } else if constexpr (SH == 1) {
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 3, true, slab_index(S, 1, x0, y, z), x0, y, z, b, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 3, true, slab_index(S, 2, x0, y, z), x0, y, z, a, r);
    } else {
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 2, true, slab_index(S, 0, x0, y, z), x0, y, z, b, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 2, true, slab_index(S, 2, x0, y, z), x0, y, z, a, r);
    }
    constexpr int f = SH == 0 ? BP_F_TXY : SH == 1 ? BP_F_TYZ : BP_F_TXZ;
    constexpr int cm = SH == 0 ? TC_MUXY : SH == 1 ? TC_MUYZ : TC_MUXZ;
    R mu[4], o[4], n[4];
    tcoef4<P>(S, cm, c, mu);
    ld_old<P, RS>(S, f, c, r, o);
    const R dt = S.dtr<R>();
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (P::prec == BP_PREC_COMP16) n[j] = o[j] + mu[j] * (a[j] + b[j]);
        else n[j] = o[j] + mu[j] * dt * (a[j] + b[j]);
    }
    st_new<P>(S, f, c, mask, n, o);
}

template <int DIM, int ORD, class P, bool RS>
__device__ __forceinline__ void t_chunk_g(const ShotDesc& S, int x0, int y, int z, typename P::real r,
                                          unsigned mask) {
    using R = typename P::real;
    const cidx sy = S.pitch, sz = S.plane;
    const cidx c = x0 + y * sy + z * sz;
    const cidx row = c - x0;
    void* const psi[3] = {S.psiT[0], S.psiT[1], S.psiT[2]};
    if constexpr (DIM == 3) {
        t_shear<DIM, ORD, P, RS, 0>(S, c, row, x0, y, z, r, mask, psi);
        t_shear<DIM, ORD, P, RS, 1>(S, c, row, x0, y, z, r, mask, psi);
    }
    t_shear<DIM, ORD, P, RS, 2>(S, c, row, x0, y, z, r, mask, psi);

    // normal stresses and pressure: the divergence derivatives (uyy, wy in 3D)
    R uxx[4], uyy[4], uzz[4], wx[4], wy[4], wz[4];
    d_span<ORD, P, false>(S, BP_F_VUX, row, x0, uxx);
    d_span<ORD, P, false>(S, BP_F_VWX, row, x0, wx);
    if constexpr (DIM == 3) {
        d_rows<ORD, P, false>(S, BP_F_VUY, c, sy, uyy);
        d_rows<ORD, P, false>(S, BP_F_VWY, c, sy, wy);
    }
    d_rows<ORD, P, false>(S, BP_F_VUZ, c, sz, uzz);
    d_rows<ORD, P, false>(S, BP_F_VWZ, c, sz, wz);
    mask0(uxx, mask); mask0(wx, mask); mask0(uzz, mask); mask0(wz, mask);
    if constexpr (DIM == 3) { mask0(uyy, mask); mask0(wy, mask); }
    {
        const cidx s0 = slab_index(S, 0, x0, y, z);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 0, false, s0, x0, y, z, uxx, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 0, 1, false, s0, x0, y, z, wx, r);
        if constexpr (DIM == 3) {
            const cidx s1 = slab_index(S, 1, x0, y, z);
            cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 0, false, s1, x0, y, z, uyy, r);
            cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 1, 1, false, s1, x0, y, z, wy, r);
        }
        const cidx s2 = slab_index(S, 2, x0, y, z);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 0, false, s2, x0, y, z, uzz, r);
        cpml_g<DIM, RS, typename P::real, P::exact>(S, psi, 2, 1, false, s2, x0, y, z, wz, r);
    }
    R cC[4], cM[4], cH[4], cH2[4], o[4], n[4];
    const R dt = S.dtr<R>();
    tcoef4<P>(S, TC_C, c, cC);
    tcoef4<P>(S, TC_M, c, cM);
    ld_old<P, RS>(S, BP_F_P, c, r, o);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (DIM == 3) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] - cC[j] * (uxx[j] + uyy[j] + uzz[j]) - cM[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] - dt * (cC[j] * (uxx[j] + uyy[j] + uzz[j]) + cM[j] * (wx[j] + wy[j] + wz[j]));
        } else {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] - cC[j] * (uxx[j] + uzz[j]) - cM[j] * (wx[j] + wz[j]);
            else
                n[j] = o[j] - dt * (cC[j] * (uxx[j] + uzz[j]) + cM[j] * (wx[j] + wz[j]));
        }
    }
    st_new<P>(S, BP_F_P, c, mask, n, o);
    tcoef4<P>(S, TC_H, c, cH);
    tcoef4<P>(S, TC_H2U, c, cH2);
    ld_old<P, RS>(S, BP_F_TXX, c, r, o);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (DIM == 3) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * (uyy[j] + uzz[j]) + cH[j] * uxx[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * (uyy[j] + uzz[j]) + cH[j] * uxx[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        } else {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * uzz[j] + cH[j] * uxx[j] + cC[j] * (wx[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * uzz[j] + cH[j] * uxx[j] + cC[j] * (wx[j] + wz[j]));
        }
    }
    st_new<P>(S, BP_F_TXX, c, mask, n, o);
    if constexpr (DIM == 3) {
        ld_old<P, RS>(S, BP_F_TYY, c, r, o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * (uxx[j] + uzz[j]) + cH[j] * uyy[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * (uxx[j] + uzz[j]) + cH[j] * uyy[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        }
        st_new<P>(S, BP_F_TYY, c, mask, n, o);
    }
    ld_old<P, RS>(S, BP_F_TZZ, c, r, o);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if constexpr (DIM == 3) {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * (uxx[j] + uyy[j]) + cH[j] * uzz[j] + cC[j] * (wx[j] + wy[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * (uxx[j] + uyy[j]) + cH[j] * uzz[j] + cC[j] * (wx[j] + wy[j] + wz[j]));
        } else {
            if constexpr (P::prec == BP_PREC_COMP16)
                n[j] = o[j] + cH2[j] * uxx[j] + cH[j] * uzz[j] + cC[j] * (wx[j] + wz[j]);
            else
                n[j] = o[j] + dt * (cH2[j] * uxx[j] + cH[j] * uzz[j] + cC[j] * (wx[j] + wz[j]));
        }
    }
    st_new<P>(S, BP_F_TZZ, c, mask, n, o);
}

// ---------------------------------------------------------------------------
// The (row, segment) units of tile (rb, sb) of shot S in one phase (it: the
// step index, r: the COMP16 rescale factor of that step).  post (T phase
// only): each chunk also records the receivers in its cells and, if it holds
// the source cell, injects the next source sample, in place of the post-step
// kernel k_post.
template <int DIM, int ORD, class P, bool VPHASE, bool MU, bool NCOK>
__device__ __forceinline__ void tile_units(const ShotDesc& S, int rb, int sb, int warp, int lane, typename P::real r,
                                           int it, int post) {
    using R = typename P::real;
    // the tile's (row, segment) units, warp w taking units w, w + 8, ...;
    // consecutive warps take consecutive rows
    const int lr = S.tile_lr, units = 1 << (lr + S.tile_ls);
    auto unit = [&](int u) {
        const int ri = u & ((1 << lr) - 1);
        const int seg = (sb << S.tile_ls) + (u >> lr);
        if (seg >= S.nseg) return;
        int y, z;
        if constexpr (DIM == 3) {
            const int ltz = S.tile_ltz, lty = lr - ltz;
            const int nyb = (S.ny + (1 << lty) - 1) >> lty;
            const int zb = rb / nyb, yb = rb - zb * nyb;
            y = (yb << lty) + (ri & ((1 << lty) - 1));
            z = (zb << ltz) + (ri >> lty);
            if (y >= S.ny || z >= S.nz) return;
        } else {
            const int row = (rb << lr) + ri;
            if (row >= S.nrows) return;
            y = 0;
            z = row;
        }
        const int hw = ORD / 2;
        if (z < hw || z >= S.nz - hw) return;
        if (DIM == 3 && (y < hw || y >= S.ny - hw)) return;
        const int x0 = seg * kSegCells + lane * 4;
        if (x0 >= S.nx - hw || x0 + 3 < hw) return;
        unsigned mask = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (x0 + j >= hw && x0 + j < S.nx - hw) mask |= 1u << j;
        // COMP16: the rescale products only on the steps whose factor is not
        // exactly 1 (a uniform branch; the products are never fused, so both
        // forms give the same bits when r == 1)
        if constexpr (grouped<DIM, P, VPHASE>()) {
            if (P::prec == BP_PREC_COMP16 && (r != (R)1 || !BP_RS_SPLIT)) {
                if constexpr (VPHASE) v_chunk_g<DIM, ORD, P, P::prec == BP_PREC_COMP16>(S, x0, y, z, r, mask);
                else t_chunk_g<DIM, ORD, P, P::prec == BP_PREC_COMP16>(S, x0, y, z, r, mask);
            } else {
                if constexpr (VPHASE) v_chunk_g<DIM, ORD, P, false>(S, x0, y, z, r, mask);
                else t_chunk_g<DIM, ORD, P, false>(S, x0, y, z, r, mask);
            }
        } else if (P::prec == BP_PREC_COMP16 && (r != (R)1 || !BP_RS_SPLIT)) {
            if constexpr (VPHASE) v_chunk<DIM, ORD, P, P::prec == BP_PREC_COMP16, NCOK>(S, x0, y, z, r, mask);
            else t_chunk<DIM, ORD, P, P::prec == BP_PREC_COMP16, NCOK>(S, x0, y, z, r, mask);
        } else {
            if constexpr (VPHASE) v_chunk<DIM, ORD, P, false, NCOK>(S, x0, y, z, r, mask);
            else t_chunk<DIM, ORD, P, false, NCOK>(S, x0, y, z, r, mask);
        }
        if constexpr (!VPHASE)
            if (post) post_chunk<DIM, P>(S, it, x0 + y * (cidx)S.pitch + z * (cidx)S.plane, x0, y, z);
    };
    // MU: tiles of more units than warps (16-row or 8 x 2 tiles); the
    // one-unit form keeps no loop state live across the chunk code, which
    // costs the 2D FP32 V phase its spill-free 80 registers otherwise
    if constexpr (MU) {
        for (int u = warp; u < units; u += kWarps) unit(u);
    } else {
        if (warp < units) unit(warp);
    }
}

}  // namespace bpk

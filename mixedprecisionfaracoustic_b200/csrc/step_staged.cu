// step_staged.cu - 2D x-z phase kernels with TMA bulk-copy staging.
//
// The same FD_V / FD_T arithmetic as step.cu (Float/main.cu:64-295,
// Half/main.cu:156-371), restructured for B200 memory parallelism: a
// persistent CTA (one per SM, 16 warps) walks a tile table; one thread issues
// cp.async.bulk copies (TMA, completion on an mbarrier) of every row span the
// next tile reads into a shared-memory stage while all warps compute the
// current tile from the other stage.  Bytes in flight no longer depend on
// registers, so the phase streams at HBM speed for both FP32 and the
// compensated FP16 layout (whose separate hi/lo arrays halve the bytes per
// load instruction of a register-staged kernel).
//
// Tile: 256 cells along x by TR rows along z.  Spans of arrays that are
// differentiated along x carry 16 cells of halo on each side (16-byte aligned
// for 4-, 2- and 1-byte elements); rows above/below come as extra spans.
// Copies are clipped to [0, pitch) and to existing rows; cells whose stencil
// would touch a clipped region are exactly the never-updated border cells.
// Every mbarrier wait is bounded: on expiry the CTA records an error code in
// global memory, drains its outstanding copies (bounded) and returns.
#include "common.cuh"

namespace bpk {

constexpr int kSW = 256;          // tile width (cells)
constexpr int kHalo = 16;         // x halo cells on each side of a halo span
constexpr int kSThreads = 512;    // 16 warps
constexpr unsigned kWaitLimit = 1u << 22;

// ---- PTX wrappers ---------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false if the phase did not complete within the limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    for (unsigned n = 0; n < kWaitLimit; n++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (n > 64) __nanosleep(64);
    }
    return false;
}

// ---- stage layout -----------------------------------------------------------
// One staged array: descriptor field index (fields, V or T coefficients), x
// halo or not, rows [r0, r1] relative to the tile's first row.
struct SArr {
    int kind;     // 0 field, 1 V coefficient, 2 T coefficient
    int idx;
    int halo;
    int r0, r1;
};

template <int ORD, bool V>
struct Arrays {
    static constexpr int HW = ORD / 2;
    static constexpr int N = V ? 15 : 13;
    __host__ __device__ static constexpr SArr get(int i, int TR) {
        const int L = TR - 1;
        if (V) {
            switch (i) {
                case 0: return {0, BP_F_TXX, 1, 0, L};
                case 1: return {0, BP_F_P, 1, -(HW - 1), L + HW};
                case 2: return {0, BP_F_TXZ, 1, -HW, L + HW - 1};
                case 3: return {0, BP_F_TZZ, 0, -(HW - 1), L + HW};
                case 4: return {0, BP_F_VUX, 0, 0, L};
                case 5: return {0, BP_F_VUZ, 0, 0, L};
                case 6: return {0, BP_F_VWX, 0, 0, L};
                case 7: return {0, BP_F_VWZ, 0, 0, L};
                case 8: return {1, VC_RHO_X, 0, 0, L};
                case 9: return {1, VC_RHO_Z, 0, 0, L};
                case 10: return {1, VC_RHOF, 0, 0, L};
                case 11: return {1, VC_CC1_X, 0, 0, L};
                case 12: return {1, VC_CC1_Z, 0, 0, L};
                case 13: return {1, VC_CC2_X, 0, 0, L};
                default: return {1, VC_CC2_Z, 0, 0, L};
            }
        } else {
            switch (i) {
                case 0: return {0, BP_F_VUX, 1, -(HW - 1), L + HW};
                case 1: return {0, BP_F_VWX, 1, 0, L};
                case 2: return {0, BP_F_VUZ, 1, -HW, L + HW - 1};
                case 3: return {0, BP_F_VWZ, 0, -HW, L + HW - 1};
                case 4: return {0, BP_F_P, 0, 0, L};
                case 5: return {0, BP_F_TXX, 0, 0, L};
                case 6: return {0, BP_F_TZZ, 0, 0, L};
                case 7: return {0, BP_F_TXZ, 0, 0, L};
                case 8: return {2, TC_C, 0, 0, L};
                case 9: return {2, TC_M, 0, 0, L};
                case 10: return {2, TC_H, 0, 0, L};
                case 11: return {2, TC_H2U, 0, 0, L};
                default: return {2, TC_MUXZ, 0, 0, L};
            }
        }
    }
};

// Element size of the main array and of the residual array (0 = none).
template <class P>
struct Elem {
    static constexpr int hi = P::prec == BP_PREC_COMP16 ? 2 : (P::prec == BP_PREC_FP64 ? 8 : 4);
    static constexpr int lo = P::prec == BP_PREC_COMP16 ? 1 : 0;
};

__host__ __device__ constexpr int span_cells(int halo) { return halo ? kSW + 2 * kHalo : kSW; }

// Bytes of one stage (every array gets space for a residual span when the
// policy has one, used or not, so all shots of a batch share the layout).
template <int ORD, class P, bool V>
__host__ __device__ constexpr unsigned stage_bytes(int TR) {
    unsigned b = 0;
    for (int i = 0; i < Arrays<ORD, V>::N; i++) {
        SArr a = Arrays<ORD, V>::get(i, TR);
        const unsigned rows = a.r1 - a.r0 + 1;
        b += rows * span_cells(a.halo) * (Elem<P>::hi + Elem<P>::lo);
    }
    return (b + 127u) & ~127u;
}

struct SPtrs {                    // where array i of a stage lives
    unsigned off_hi, off_lo;      // byte offsets in the stage
};

template <int ORD, class P, bool V>
__device__ __forceinline__ SPtrs stage_offsets(int i, int TR) {
    unsigned b = 0;
    SPtrs p{0, 0};
#pragma unroll
    for (int k = 0; k < Arrays<ORD, V>::N; k++) {
        const SArr a = Arrays<ORD, V>::get(k, TR);
        const unsigned rows = a.r1 - a.r0 + 1, cells = span_cells(a.halo);
        if (k == i) {
            p.off_hi = b;
            p.off_lo = b + rows * cells * Elem<P>::hi;
        }
        b += rows * cells * (Elem<P>::hi + Elem<P>::lo);
    }
    return p;
}

// Total staged rows of a tile (over all arrays).
template <int ORD, bool V>
__host__ __device__ constexpr int total_rows(int TR) {
    int n = 0;
    for (int i = 0; i < Arrays<ORD, V>::N; i++) {
        const SArr a = Arrays<ORD, V>::get(i, TR);
        n += a.r1 - a.r0 + 1;
    }
    return n;
}

__device__ __forceinline__ const void* arr_ptr(const ShotDesc& S, const SArr& a, const int8_t** lo) {
    if (a.kind == 0) { *lo = S.flo[a.idx]; return S.f[a.idx]; }
    if (a.kind == 1) { *lo = S.vclo[a.idx]; return S.vc[a.idx]; }
    *lo = S.tclo[a.idx];
    return S.tc[a.idx];
}

// Tile t of the staged tiling -> shot, x0, z0.  Returns false for tiles of
// finished or empty shots (no copies are issued and nothing is computed).
__device__ __forceinline__ bool decode_tile(const ShotDesc* shots, int nshots, long long t, int k, int TR,
                                            int& si, int& x0, int& z0) {
    int lo = 0, hi = nshots - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (shots[mid].tile0s <= t) lo = mid;
        else hi = mid - 1;
    }
    si = lo;
    const ShotDesc& S = shots[si];
    const long long lt = t - S.tile0s;
    x0 = (int)(lt % S.nseg_s) * kSW;
    z0 = (int)(lt / S.nseg_s) * TR;
    const int it = *S.step_base + k;
    return !S.done && it < S.nt;
}

// The bulk copies of one tile, spread over the 32 lanes of the producer warp:
// lane l takes staged rows q = l, l+32, ... of the flattened (array, row)
// list.  With issue = false it only returns the lane's byte count (the
// warp-summed count is armed on the mbarrier before any copy is issued).
template <int ORD, class P, bool V, int TR>
__device__ __forceinline__ unsigned tile_copies_lane(const ShotDesc& S, int x0, int z0, unsigned char* stage,
                                                     uint64_t* bar, int lane, bool issue) {
    constexpr int NR = total_rows<ORD, V>(TR);
    unsigned total = 0;
    for (int q = lane; q < NR; q += 32) {
        int i = 0, base = 0;
        bool found = false;
#pragma unroll
        for (int k = 0; k < Arrays<ORD, V>::N; k++) {      // which array holds flat row q
            const SArr a = Arrays<ORD, V>::get(k, TR);
            const int rows = a.r1 - a.r0 + 1;
            if (!found) {
                if (q < base + rows) { i = k; found = true; }
                else base += rows;
            }
        }
        const SArr a = Arrays<ORD, V>::get(i, TR);
        const int r = a.r0 + (q - base);
        const int z = z0 + r;
        if (z < 0 || z >= S.nz) continue;
        const int cells = span_cells(a.halo);
        const int xs = a.halo ? x0 - kHalo : x0;       // first cell of the span
        const int c0 = xs < 0 ? -xs : 0;               // cells clipped on the left
        const int c1 = xs + cells > S.pitch ? S.pitch - xs : cells;
        if (c1 <= c0) continue;
        const int8_t* lo;
        const void* hi = arr_ptr(S, a, &lo);
        const SPtrs sp = stage_offsets<ORD, P, V>(i, TR);
        const long long g = (long long)z * S.pitch + xs + c0;   // first copied cell
        const unsigned nb = (unsigned)(c1 - c0);
        const unsigned rowoff = (unsigned)(r - a.r0) * cells;
        total += nb * Elem<P>::hi;
        if (issue)
            bulk_g2s(stage + sp.off_hi + (rowoff + c0) * Elem<P>::hi,
                     static_cast<const unsigned char*>(hi) + g * Elem<P>::hi, nb * Elem<P>::hi, bar);
        if (Elem<P>::lo && lo) {
            total += nb * Elem<P>::lo;
            if (issue)
                bulk_g2s(stage + sp.off_lo + (rowoff + c0) * Elem<P>::lo,
                         reinterpret_cast<const unsigned char*>(lo) + g * Elem<P>::lo, nb * Elem<P>::lo, bar);
        }
    }
    return total;
}

// Warp 0 arms `bar` with the tile's byte count and issues its copies.
template <int ORD, class P, bool V, int TR>
__device__ __forceinline__ void produce_tile(const ShotDesc& G, int x0, int z0, unsigned char* stage, uint64_t* bar,
                                             int lane) {
    fence_proxy_async();   // earlier generic reads of this stage before the async-proxy writes
    unsigned bytes = tile_copies_lane<ORD, P, V, TR>(G, x0, z0, stage, bar, lane, false);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
    __syncwarp();
    tile_copies_lane<ORD, P, V, TR>(G, x0, z0, stage, bar, lane, true);
}

// Reads of staged values.
template <class P>
struct SView {
    const unsigned char* hi;
    const unsigned char* lo;   // null when the residual span was not copied
    int row0, cells, xoff;
    __device__ __forceinline__ typename P::real at(int r, int c) const {
        const int i = (r - row0) * cells + c + xoff;
        if constexpr (P::prec == BP_PREC_COMP16) {
            const __half h = reinterpret_cast<const __half*>(hi)[i];
            return lo ? decode_ch(h, reinterpret_cast<const int8_t*>(lo)[i]) : __half2float(h);
        } else {
            return reinterpret_cast<const typename P::real*>(hi)[i];
        }
    }
};

template <int ORD, class P, bool V>
__device__ __forceinline__ SView<P> view(const ShotDesc& S, const unsigned char* stage, int i, int TR) {
    const SArr a = Arrays<ORD, V>::get(i, TR);
    const SPtrs sp = stage_offsets<ORD, P, V>(i, TR);
    const int8_t* lo;
    arr_ptr(S, a, &lo);
    SView<P> v;
    v.hi = stage + sp.off_hi;
    v.lo = (Elem<P>::lo && lo) ? stage + sp.off_lo : nullptr;
    v.row0 = a.r0;
    v.cells = span_cells(a.halo);
    v.xoff = a.halo ? kHalo : 0;
    return v;
}

template <int ORD, class P>
__device__ __forceinline__ typename P::real dx_fwd(const SView<P>& v, int r, int c) {
    using R = typename P::real;
    if constexpr (ORD == 2) return v.at(r, c + 1) - v.at(r, c);
    else return (R)1.125 * (v.at(r, c + 1) - v.at(r, c)) + (R)(-1.0 / 24.0) * (v.at(r, c + 2) - v.at(r, c - 1));
}
template <int ORD, class P>
__device__ __forceinline__ typename P::real dx_bwd(const SView<P>& v, int r, int c) {
    using R = typename P::real;
    if constexpr (ORD == 2) return v.at(r, c) - v.at(r, c - 1);
    else return (R)1.125 * (v.at(r, c) - v.at(r, c - 1)) + (R)(-1.0 / 24.0) * (v.at(r, c + 1) - v.at(r, c - 2));
}
template <int ORD, class P>
__device__ __forceinline__ typename P::real dz_fwd(const SView<P>& v, int r, int c) {
    using R = typename P::real;
    if constexpr (ORD == 2) return v.at(r + 1, c) - v.at(r, c);
    else return (R)1.125 * (v.at(r + 1, c) - v.at(r, c)) + (R)(-1.0 / 24.0) * (v.at(r + 2, c) - v.at(r - 1, c));
}
template <int ORD, class P>
__device__ __forceinline__ typename P::real dz_bwd(const SView<P>& v, int r, int c) {
    using R = typename P::real;
    if constexpr (ORD == 2) return v.at(r, c) - v.at(r - 1, c);
    else return (R)1.125 * (v.at(r, c) - v.at(r - 1, c)) + (R)(-1.0 / 24.0) * (v.at(r + 1, c) - v.at(r - 2, c));
}

template <class P>
__device__ __forceinline__ typename P::real ddiv(typename P::real a, const ShotDesc& S) {
    if constexpr (P::prec == BP_PREC_FP32) {
        const float q = a * S.inv_h;
        return __fmaf_rn(__fmaf_rn(-q, S.h, a), S.inv_h, q);
    } else {
        return a * S.inv_h;
    }
}

// CPML memory update of one cell (Float/main.cu:130): ψ = ψe + b(e prev + ∂).
__device__ __forceinline__ float cpml1(float d, float* psi, float* prev, float b, float e, float r) {
    const float ps = *psi * r, pv = *prev * r;
    const float np = ps * e + b * (e * pv + d);
    *psi = np;
    *prev = d;
    return d + np;
}

template <class P>
__device__ __forceinline__ void st_field(const ShotDesc& S, int f, long long i, typename P::real v) {
    P::st1(S.f[f], S.flo[f], i, v);
}

// ---- the kernel --------------------------------------------------------------
template <int ORD, class P, bool V, int TR, int NST>
__global__ void __launch_bounds__(kSThreads, 1) k_phase_staged(const ShotDesc* __restrict__ shots, int nshots,
                                                                long long ntiles, int k, int* err) {
    using R = typename P::real;
    static_assert(P::prec != BP_PREC_FP64, "FP64 runs the register kernel");
    static_assert(NST >= 2 && NST <= 4, "2..4 stages");
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr unsigned SB = stage_bytes<ORD, P, V>(TR);
    // stage q lives at smem + q * SB; its mbarrier at bars[q]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + NST * SB);
    __shared__ ShotDesc sdesc;
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int q = 0; q < NST; q++) mbar_init(&bars[q], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();

    unsigned par = 0;                    // bit q: parity of the next completion of stage q
    unsigned armed = 0;                  // bit q: stage q has copies outstanding
    // prologue: the first NST-1 tiles of this CTA
    for (int q = 0; q < NST - 1; q++) {
        const long long tq = blockIdx.x + (long long)q * gridDim.x;
        int a = 0, b = 0, c = 0;
        if (tq < ntiles && decode_tile(shots, nshots, tq, k, TR, a, b, c)) {
            if (tid < 32) produce_tile<ORD, P, V, TR>(shots[a], b, c, smem + q * SB, &bars[q], tid);
            armed |= 1u << q;
        }
    }
    int cur_shot = -1;
    int s = 0;                           // stage of the current tile
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, s = (s + 1 == NST ? 0 : s + 1)) {
        // prefetch tile t + (NST-1) grid strides into the stage consumed last
        // iteration (protected by the barrier that ended it)
        const long long tn = t + (long long)(NST - 1) * gridDim.x;
        const int sn = s == 0 ? NST - 1 : s - 1;
        int sin = 0, x0n = 0, z0n = 0;
        if (tn < ntiles && decode_tile(shots, nshots, tn, k, TR, sin, x0n, z0n)) {
            if (tid < 32) produce_tile<ORD, P, V, TR>(shots[sin], x0n, z0n, smem + sn * SB, &bars[sn], tid);
            armed |= 1u << sn;
        }
        int si = 0, x0 = 0, z0 = 0;
        const bool act = decode_tile(shots, nshots, t, k, TR, si, x0, z0);
        if (act && si != cur_shot) {     // stage the descriptor of this tile's shot
            const long long* src = reinterpret_cast<const long long*>(shots + si);
            long long* dst = reinterpret_cast<long long*>(&sdesc);
            for (int w = tid; w < (int)(sizeof(ShotDesc) / 8); w += blockDim.x) dst[w] = src[w];
        }
        __syncthreads();                 // sdesc ready
        if (act) {
            if (!mbar_wait_bounded(&bars[s], (par >> s) & 1u)) s_abort = 1;
            else { par ^= 1u << s; armed &= ~(1u << s); }
        }
        __syncthreads();
        if (s_abort) break;
        if (act) {
            cur_shot = si;
            const ShotDesc& S = sdesc;
            const int it = *S.step_base + k;
            R rr = (R)1;
            if constexpr (P::prec == BP_PREC_COMP16) rr = S.rtab[it];
            const int c = tid & (kSW - 1);
            const int x = x0 + c;
            const int hw = ORD / 2;
            const bool xok = x >= hw && x < S.nx - hw;
            constexpr int RPT = TR / (kSThreads / kSW);      // rows per thread
            const int rbase = (tid / kSW) * RPT;
            const unsigned char* st = smem + s * SB;
#pragma unroll 1
            for (int q = 0; q < RPT; q++) {
                const int r = rbase + q;
                const int z = z0 + r;
                if (!xok || z < hw || z >= S.nz - hw) continue;
                const long long gi = (long long)z * S.pitch + x;
                if constexpr (V) {
                    const SView<P> txx = view<ORD, P, V>(S, st, 0, TR), pp = view<ORD, P, V>(S, st, 1, TR);
                    const SView<P> txz = view<ORD, P, V>(S, st, 2, TR), tzz = view<ORD, P, V>(S, st, 3, TR);
                    R x1 = ddiv<P>(dx_fwd<ORD, P>(txx, r, c), S), s1 = ddiv<P>(dx_fwd<ORD, P>(pp, r, c), S);
                    R z2 = ddiv<P>(dx_bwd<ORD, P>(txz, r, c), S), x3 = ddiv<P>(dz_bwd<ORD, P>(txz, r, c), S);
                    R z1 = ddiv<P>(dz_fwd<ORD, P>(tzz, r, c), S), s3 = ddiv<P>(dz_fwd<ORD, P>(pp, r, c), S);
                    if constexpr (P::prec == BP_PREC_COMP16) { x1 *= rr; s1 *= rr; z2 *= rr; x3 *= rr; z1 *= rr; s3 *= rr; }
                    // CPML on the slabs (slots as in step.cu: x {x1, s1, z2}, z {x3, z1, s3})
                    const int sx = S.slab[0].index(x);
                    if (sx >= 0) {
                        float* B = static_cast<float*>(S.psiV[0]);
                        const long long n = S.slab_cells[0], j = (long long)z * S.slab[0].width + sx;
                        const float* b = static_cast<const float*>(S.pb[0]); const float* e = static_cast<const float*>(S.pe[0]);
                        const float* b2 = static_cast<const float*>(S.pb2[0]); const float* e2 = static_cast<const float*>(S.pe2[0]);
                        x1 = cpml1(x1, B + j, B + 3 * n + j, b2[x], e2[x], rr);
                        s1 = cpml1(s1, B + n + j, B + 4 * n + j, b2[x], e2[x], rr);
                        z2 = cpml1(z2, B + 2 * n + j, B + 5 * n + j, b[x], e[x], rr);
                    }
                    const int sz = S.slab[2].index(z);
                    if (sz >= 0) {
                        float* B = static_cast<float*>(S.psiV[2]);
                        const long long n = S.slab_cells[2], j = (long long)sz * S.pitch + x;
                        const float* b = static_cast<const float*>(S.pb[2]); const float* e = static_cast<const float*>(S.pe[2]);
                        const float* b2 = static_cast<const float*>(S.pb2[2]); const float* e2 = static_cast<const float*>(S.pe2[2]);
                        x3 = cpml1(x3, B + j, B + 3 * n + j, b[z], e[z], rr);
                        z1 = cpml1(z1, B + n + j, B + 4 * n + j, b2[z], e2[z], rr);
                        s3 = cpml1(s3, B + 2 * n + j, B + 5 * n + j, b2[z], e2[z], rr);
                    }
                    const R sumx = x1 + x3, sumz = z1 + z2;
                    const R rf = view<ORD, P, V>(S, st, 10, TR).at(r, c);
                    // x: vux (4), vwx (6), rho_x (8), cc1_x (11), cc2_x (13); z: vuz (5), vwz (7), 9, 12, 14
#pragma unroll
                    for (int ax = 0; ax < 2; ax++) {
                        const R sum = ax ? sumz : sumx, dp = ax ? s3 : s1;
                        const R rho = view<ORD, P, V>(S, st, ax ? 9 : 8, TR).at(r, c);
                        const R c1 = view<ORD, P, V>(S, st, ax ? 12 : 11, TR).at(r, c);
                        const R c2 = view<ORD, P, V>(S, st, ax ? 14 : 13, TR).at(r, c);
                        const R vu = view<ORD, P, V>(S, st, ax ? 5 : 4, TR).at(r, c);
                        const R vw = view<ORD, P, V>(S, st, ax ? 7 : 6, TR).at(r, c);
                        R nw, nu;
                        if constexpr (P::prec == BP_PREC_COMP16) {
                            const R wo = vw * rr, uo = vu * rr, rrho = rf * rho;
                            nw = c1 * wo - (rrho * c2) * sum - c2 * dp;
                            nu = uo + rho * sum - rrho * (nw - wo);
                        } else {
                            nw = (c1 == (R)0) ? (R)0 : (vw * c2 - S.dt * (rf * rho * sum + dp)) / c1;
                            nu = vu + S.dt * rho * sum - rf * rho * (nw - vw);
                        }
                        st_field<P>(S, ax ? BP_F_VWZ : BP_F_VWX, gi, nw);
                        st_field<P>(S, ax ? BP_F_VUZ : BP_F_VUX, gi, nu);
                    }
                } else {
                    const SView<P> vux = view<ORD, P, V>(S, st, 0, TR), vwx = view<ORD, P, V>(S, st, 1, TR);
                    const SView<P> vuz = view<ORD, P, V>(S, st, 2, TR), vwz = view<ORD, P, V>(S, st, 3, TR);
                    R uxx = ddiv<P>(dx_bwd<ORD, P>(vux, r, c), S), wx = ddiv<P>(dx_bwd<ORD, P>(vwx, r, c), S);
                    R uzx = ddiv<P>(dx_fwd<ORD, P>(vuz, r, c), S), uzz = ddiv<P>(dz_bwd<ORD, P>(vuz, r, c), S);
                    R wz = ddiv<P>(dz_bwd<ORD, P>(vwz, r, c), S), uxz = ddiv<P>(dz_fwd<ORD, P>(vux, r, c), S);
                    const int sx = S.slab[0].index(x);
                    if (sx >= 0) {
                        float* B = static_cast<float*>(S.psiT[0]);
                        const long long n = S.slab_cells[0], j = (long long)z * S.slab[0].width + sx;
                        const float* b = static_cast<const float*>(S.pb[0]); const float* e = static_cast<const float*>(S.pe[0]);
                        const float* b2 = static_cast<const float*>(S.pb2[0]); const float* e2 = static_cast<const float*>(S.pe2[0]);
                        uxx = cpml1(uxx, B + j, B + 3 * n + j, b[x], e[x], rr);
                        wx = cpml1(wx, B + n + j, B + 4 * n + j, b[x], e[x], rr);
                        uzx = cpml1(uzx, B + 2 * n + j, B + 5 * n + j, b2[x], e2[x], rr);
                    }
                    const int sz = S.slab[2].index(z);
                    if (sz >= 0) {
                        float* B = static_cast<float*>(S.psiT[2]);
                        const long long n = S.slab_cells[2], j = (long long)sz * S.pitch + x;
                        const float* b = static_cast<const float*>(S.pb[2]); const float* e = static_cast<const float*>(S.pe[2]);
                        const float* b2 = static_cast<const float*>(S.pb2[2]); const float* e2 = static_cast<const float*>(S.pe2[2]);
                        uzz = cpml1(uzz, B + j, B + 3 * n + j, b[z], e[z], rr);
                        wz = cpml1(wz, B + n + j, B + 4 * n + j, b[z], e[z], rr);
                        uxz = cpml1(uxz, B + 2 * n + j, B + 5 * n + j, b2[z], e2[z], rr);
                    }
                    const R cC = view<ORD, P, V>(S, st, 8, TR).at(r, c), cM = view<ORD, P, V>(S, st, 9, TR).at(r, c);
                    const R cH = view<ORD, P, V>(S, st, 10, TR).at(r, c), cH2 = view<ORD, P, V>(S, st, 11, TR).at(r, c);
                    const R mu = view<ORD, P, V>(S, st, 12, TR).at(r, c);
                    R op = view<ORD, P, V>(S, st, 4, TR).at(r, c), oxx = view<ORD, P, V>(S, st, 5, TR).at(r, c);
                    R ozz = view<ORD, P, V>(S, st, 6, TR).at(r, c), oxz = view<ORD, P, V>(S, st, 7, TR).at(r, c);
                    R np, nxx, nzz, nxz;
                    if constexpr (P::prec == BP_PREC_COMP16) {
                        op *= rr; oxx *= rr; ozz *= rr; oxz *= rr;
                        np = op - cC * (uxx + uzz) - cM * (wx + wz);
                        nxx = oxx + cH2 * uzz + cH * uxx + cC * (wx + wz);
                        nzz = ozz + cH2 * uxx + cH * uzz + cC * (wx + wz);
                        nxz = oxz + mu * (uxz + uzx);
                    } else {
                        const R dt = S.dt;
                        np = op - dt * (cC * (uxx + uzz) + cM * (wx + wz));
                        nxx = oxx + dt * (cH2 * uzz + cH * uxx + cC * (wx + wz));
                        nzz = ozz + dt * (cH2 * uxx + cH * uzz + cC * (wx + wz));
                        nxz = oxz + mu * dt * (uxz + uzx);
                    }
                    st_field<P>(S, BP_F_P, gi, np);
                    st_field<P>(S, BP_F_TXX, gi, nxx);
                    st_field<P>(S, BP_F_TZZ, gi, nzz);
                    st_field<P>(S, BP_F_TXZ, gi, nxz);
                }
            }
        }
        __syncthreads();                 // stage s fully read before it is refilled
    }
    if (s_abort) {
        // record the failure and drain copies still in flight (bounded) before exiting
        if (tid == 0) {
            atomicExch(err, BP_ERR_TIMEOUT);
            for (int q = 0; q < NST; q++)
                if (armed >> q & 1u) mbar_wait_bounded(&bars[q], (par >> q) & 1u);
        }
        __syncthreads();
    }
}

// ---- host side ---------------------------------------------------------------
template <int ORD, class P, bool V, int TR, int NST>
static cudaError_t launch_one(const ShotDesc* d, int nshots, long long ntiles, int k, int grid, int* err,
                              cudaStream_t st) {
    const unsigned smem = NST * stage_bytes<ORD, P, V>(TR) + NST * sizeof(uint64_t);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_phase_staged<ORD, P, V, TR, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    k_phase_staged<ORD, P, V, TR, NST><<<grid, kSThreads, smem, st>>>(d, nshots, ntiles, k, err);
    return cudaGetLastError();
}

constexpr int kTR = 4;
constexpr int kStages = 3;   // prefetch distance 2 tiles; 3 x 73 KB (FP32 order 4 V) fits in 227 KB

int staged_tile_rows() { return kTR; }
int staged_tile_width() { return kSW; }

bool staged_supported(int prec, int dim) { return dim == 2 && (prec == BP_PREC_FP32 || prec == BP_PREC_COMP16); }
bool staged_default() { return false; }

cudaError_t launch_phase_staged(int prec, int order, bool vphase, const ShotDesc* d, int nshots, long long ntiles,
                                int k, int grid, int* err, cudaStream_t st) {
#define BPS(O, PP)                                                                                       \
    if (order == O) return vphase ? launch_one<O, PP, true, kTR, kStages>(d, nshots, ntiles, k, grid, err, st) \
                                  : launch_one<O, PP, false, kTR, kStages>(d, nshots, ntiles, k, grid, err, st);
    if (prec == BP_PREC_FP32) { BPS(2, PolF32) BPS(4, PolF32) }
    if (prec == BP_PREC_COMP16) { BPS(2, PolC16) BPS(4, PolC16) }
#undef BPS
    return cudaErrorInvalidValue;
}

}  // namespace bpk

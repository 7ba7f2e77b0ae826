// post.cuh - what follows a step's stress update at the receivers and the
// source: recording the five seismogram components (Float/main.cu:1085-1093)
// and injecting the next source sample (Source, Float/main.cu:45-59), for one
// cell or for the cells of one 4-cell chunk.  Shared by the post-step kernel
// and the T phases of the tile kernels (step.cu) and by the fused step kernel
// (step_fused.cu).
#pragma once
#include "stencil.cuh"

namespace bpk {

template <class P>
__device__ __forceinline__ typename P::real read_phys(const TailOut& F, int f, long long i, typename P::real sc) {
    return P::ld1(F.f[f], F.flo[f], i) * sc;
}

// The state arrays these helpers read and write are F's (the descriptor's own
// for the single-buffered kernels; the new state's for the fused kernel).
template <class P>
__device__ __forceinline__ void inject(const ShotDesc& S, int it, const TailOut& F) {
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
        P::st1(F.f[BP_F_TXX], F.flo[BP_F_TXX], i, P::ld1(F.f[BP_F_TXX], F.flo[BP_F_TXX], i) + I);
        if (S.dim == 3) P::st1(F.f[BP_F_TYY], F.flo[BP_F_TYY], i, P::ld1(F.f[BP_F_TYY], F.flo[BP_F_TYY], i) + I);
        P::st1(F.f[BP_F_TZZ], F.flo[BP_F_TZZ], i, P::ld1(F.f[BP_F_TZZ], F.flo[BP_F_TZZ], i) + I);
    }
    if (S.src_mask & BP_SRC_P) P::st1(F.f[BP_F_P], F.flo[BP_F_P], i, P::ld1(F.f[BP_F_P], F.flo[BP_F_P], i) - I);
}
template <class P>
__device__ __forceinline__ void inject(const ShotDesc& S, int it) { inject<P>(S, it, TailOut::t_of(S)); }

// Records step it's five components at unique receiver r, cell i.
template <class P>
__device__ __forceinline__ void record(const ShotDesc& S, int it, int r, long long i, const TailOut& F) {
    using R = typename P::real;
    R ss = (R)1, sv = (R)1;
    if constexpr (P::prec == BP_PREC_COMP16) {
        const float d = 1.0f / S.dyn[it];
        ss = S.out_stress * d;
        sv = S.out_vel * d;
    }
    R v[BP_NTRACE];
    v[BP_TR_TXX] = read_phys<P>(F, BP_F_TXX, i, ss);
    v[BP_TR_TZZ] = read_phys<P>(F, BP_F_TZZ, i, ss);
    v[BP_TR_VUX] = read_phys<P>(F, BP_F_VUX, i, sv);
    v[BP_TR_VWX] = read_phys<P>(F, BP_F_VWX, i, sv);
    v[BP_TR_P] = read_phys<P>(F, BP_F_P, i, ss);
    const long long cs = (long long)S.nrec * S.nt;
    bool finite = true;
#pragma unroll
    for (int q = 0; q < BP_NTRACE; q++) {
        S.traces[q * cs + (long long)r * S.nt + it] = (float)v[q];
        if constexpr (P::prec == BP_PREC_FP64) S.traces64[q * cs + (long long)r * S.nt + it] = v[q];
        finite = finite && isfinite(v[q]);
    }
    // blow-up detection: the first step whose recorded values are not all
    // finite (step + 1; 0 = none), read by the host at its next sync
    if (!finite) atomicCAS(S.blowup, 0, it + 1);
}
template <class P>
__device__ __forceinline__ void record(const ShotDesc& S, int it, int r, long long i) {
    record<P>(S, it, r, i, TailOut::t_of(S));
}

// k_post's work for the cells of one T-phase chunk (c = flat index of cell
// x0), after the chunk's stores: the chunk's receivers, found by a binary
// search of its row's x-sorted list, read back the values this thread has just
// written (the velocities are not written in the T phase), so the recorded
// values are k_post's; then the source, if its cell is here.  The receiver on
// the source cell, if any, is recorded before the injection, as in k_post.
// The recording and injection, out of line: only the few chunks that hold a
// receiver or the source call it, and the phase kernels keep their registers.
template <class P>
__device__ __noinline__ void post_cells(const ShotDesc& S, int it, cidx c, int x0, int lo, int end, TailOut F) {
    if (lo < end) {
        int hi = end;
        while (lo < hi) {                       // first receiver with x >= x0
            const int mid = (lo + hi) >> 1;
            if (S.rec_xu[mid].x < x0) lo = mid + 1;
            else hi = mid;
        }
        for (; lo < end; lo++) {
            const int2 xu = S.rec_xu[lo];
            if (xu.x >= x0 + 4) break;
            record<P>(S, it, xu.y, (long long)c + (xu.x - x0), F);
        }
    }
    if (S.src_idx_valid && S.src_idx >= c && S.src_idx < (long long)c + 4) inject<P>(S, it + 1, F);
}

template <int DIM, class P>
__device__ __forceinline__ void post_chunk(const ShotDesc& S, int it, cidx c, int x0, int y, int z, const TailOut& F) {
    const int key = DIM == 3 ? z * S.ny + y : z;
    const int lo = S.rec_row[key], end = S.rec_row[key + 1];
    const bool src = S.src_idx_valid && S.src_idx >= c && S.src_idx < (long long)c + 4;
    if (lo < end || src) post_cells<P>(S, it, c, x0, lo, end, F);
}
template <int DIM, class P>
__device__ __forceinline__ void post_chunk(const ShotDesc& S, int it, cidx c, int x0, int y, int z) {
    post_chunk<DIM, P>(S, it, c, x0, y, z, TailOut::t_of(S));
}

}  // namespace bpk

// medium_index.cu - the indexed medium: a shot whose cells hold at most 256
// distinct coefficient tuples (layered, blocky and uniform media) gets a
// one-byte index per cell and a table of the decoded tuples, which the phase
// kernels read in place of the per-cell coefficient arrays (BP_MEDIUM_AUTO).
//
// No reference counterpart: the reference keeps one array per coefficient
// (Float/main.cu:106-113 forms the staggered values per cell, FD_T reads its
// moduli per cell at :232-250).  The table holds exactly the values a load
// from those arrays decodes, so the kernels' results are bit-identical.
//
// Built on the device after the coefficient precompute, in three passes over
// the cells:
//   1. hash each cell's tuple (the decoded values' bits) into an
//      open-addressing table of kSlots keys; the first cell of each key is its
//      representative; more than 256 keys stops the build (the shot reads the
//      arrays);
//   2. (host) number the keys in slot order;
//   3. write each cell's number, checking that its tuple equals its
//      representative's bit for bit (a hash collision stops the build), and
//      decode the representatives into the table.
#include <cstring>
#include <string>
#include <vector>

#include "shot.h"

namespace bpk {

constexpr int kSlots = 4096;               // keys, a power of two well above 256

// The tuple of cell i in table order (MedGroup): 5 groups of 4 values.
template <class P>
__device__ __forceinline__ void med_tuple(const ShotDesc& S, cidx i, float (&t)[4 * kMedRow]) {
    auto v = [&](int k) -> float { return S.vc[k] ? (float)P::ld1(S.vc[k], S.vclo[k], i) : 0.0f; };
    auto m = [&](int k) -> float { return S.tc[k] ? (float)P::ld1(S.tc[k], S.tclo[k], i) : 0.0f; };
    t[0] = v(VC_RHO_X); t[1] = v(VC_CC1_X); t[2] = v(VC_CC2_X); t[3] = v(VC_RHOF);
    t[4] = v(VC_RHO_Y); t[5] = v(VC_CC1_Y); t[6] = v(VC_CC2_Y); t[7] = 0.0f;
    t[8] = v(VC_RHO_Z); t[9] = v(VC_CC1_Z); t[10] = v(VC_CC2_Z); t[11] = 0.0f;
    t[12] = m(TC_C); t[13] = m(TC_M); t[14] = m(TC_H); t[15] = m(TC_H2U);
    t[16] = m(TC_MUXZ); t[17] = m(TC_MUXY); t[18] = m(TC_MUYZ); t[19] = 0.0f;
}

__device__ __forceinline__ unsigned long long med_hash(const float (&t)[4 * kMedRow]) {
    unsigned long long h = 0x243f6a8885a308d3ull;
#pragma unroll
    for (int q = 0; q < 4 * kMedRow; q++) {
        h ^= (unsigned long long)__float_as_uint(t[q]) + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        h *= 0xbf58476d1ce4e5b9ull;
        h ^= h >> 31;
    }
    return h ? h : 1ull;                   // 0 marks an empty slot
}

struct MedScratch {
    unsigned long long keys[kSlots];
    int reps[kSlots];                      // representative cell of each key
    int ids[kSlots];                       // key -> tuple number (host-filled)
    int count, overflow, collide, pad;
};

// Cell q of the nx x ny x nz extent (x fastest) -> its offset.
__device__ __forceinline__ cidx med_cell(const ShotDesc& S, long long q) {
    const int x = (int)(q % S.nx);
    const long long r = q / S.nx;
    const int y = (int)(r % S.ny), z = (int)(r / S.ny);
    return (cidx)(x + (long long)y * S.pitch + (long long)z * S.plane);
}

template <class P>
__global__ void k_med_hash(const ShotDesc S, MedScratch* M) {
    const long long n = (long long)S.nx * S.ny * S.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        if (*(volatile int*)&M->overflow) return;
        const cidx i = med_cell(S, q);
        float t[4 * kMedRow];
        med_tuple<P>(S, i, t);
        const unsigned long long h = med_hash(t);
        unsigned slot = (unsigned)h & (kSlots - 1);
        bool placed = false;
        for (int probe = 0; probe < kSlots && !placed; probe++) {
            unsigned long long k = *(volatile unsigned long long*)&M->keys[slot];
            if (k == 0) {
                k = atomicCAS(&M->keys[slot], 0ull, h);
                if (k == 0) {                              // a new key: this cell represents it
                    M->reps[slot] = i;
                    if (atomicAdd(&M->count, 1) >= kMedMaxTuples) atomicExch(&M->overflow, 1);
                    placed = true;
                    break;
                }
            }
            if (k == h) { placed = true; break; }
            slot = (slot + 1) & (kSlots - 1);
        }
        if (!placed) atomicExch(&M->overflow, 1);
    }
}

template <class P>
__global__ void k_med_index(const ShotDesc S, MedScratch* M, uint8_t* idx) {
    const long long n = (long long)S.nx * S.ny * S.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const cidx i = med_cell(S, q);
        float t[4 * kMedRow];
        med_tuple<P>(S, i, t);
        const unsigned long long h = med_hash(t);
        unsigned slot = (unsigned)h & (kSlots - 1);
        int probe = 0;
        while (M->keys[slot] != h && probe < kSlots) { slot = (slot + 1) & (kSlots - 1); probe++; }
        if (probe == kSlots) { atomicExch(&M->collide, 1); continue; }
        float u[4 * kMedRow];
        med_tuple<P>(S, M->reps[slot], u);
        bool same = true;
#pragma unroll
        for (int k = 0; k < 4 * kMedRow; k++) same = same && __float_as_uint(t[k]) == __float_as_uint(u[k]);
        if (!same) atomicExch(&M->collide, 1);
        idx[i] = (uint8_t)M->ids[slot];
    }
}

template <class P>
__global__ void k_med_table(const ShotDesc S, const int* reps, int n, float4* tab) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    float t[4 * kMedRow];
    med_tuple<P>(S, reps[id], t);
    for (int g = 0; g < kMedRow; g++) tab[id * kMedRow + g] = make_float4(t[4 * g], t[4 * g + 1], t[4 * g + 2], t[4 * g + 3]);
}

size_t medium_scratch_bytes() { return sizeof(MedScratch); }

template <class P>
static cudaError_t med_build(ShotDesc& S, uint8_t* d_idx, float4* d_tab, void* d_scratch, size_t ncell, int* ntuples,
                             cudaStream_t st) {
    *ntuples = 0;
    MedScratch* M = static_cast<MedScratch*>(d_scratch);
    cudaError_t e = cudaMemsetAsync(M, 0, sizeof(MedScratch), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_idx, 0, ncell, st);
    const int blocks = 148 * 8;
    if (e == cudaSuccess) {
        k_med_hash<P><<<blocks, 256, 0, st>>>(S, M);
        e = cudaGetLastError();
    }
    // the keys, their representatives and the flags back to the host
    std::vector<unsigned long long> keys(kSlots);
    std::vector<int> reps(kSlots);
    int flags[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(keys.data(), M->keys, sizeof(M->keys), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(reps.data(), M->reps, sizeof(M->reps), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, &M->count, sizeof(flags), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (flags[1] || flags[0] > kMedMaxTuples || flags[0] < 1) return cudaSuccess;   // too many tuples: dense
    std::vector<int> ids(kSlots, 0), rep_of(kSlots, 0);
    int n = 0;
    for (int s = 0; s < kSlots; s++)
        if (keys[s]) { ids[s] = n; rep_of[n] = reps[s]; n++; }
    if (n != flags[0] || n > kMedMaxTuples) return cudaSuccess;
    int* d_reps = M->reps;                 // reused: rep of each tuple number, after the index pass
    e = cudaMemcpyAsync(M->ids, ids.data(), sizeof(M->ids), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_med_index<P><<<blocks, 256, 0, st>>>(S, M, d_idx);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_reps, rep_of.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_med_table<P><<<(n + 127) / 128, 128, 0, st>>>(S, d_reps, n, d_tab);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, &M->count, sizeof(flags), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (flags[2]) return cudaSuccess;      // a hash collision: dense
    *ntuples = n;
    return cudaSuccess;
}

cudaError_t build_medium_index(int prec, ShotDesc& S, uint8_t* d_idx, float4* d_tab, void* d_scratch, size_t ncell,
                               int* ntuples, cudaStream_t st) {
    *ntuples = 0;
    if (prec == BP_PREC_FP32) return med_build<PolF32>(S, d_idx, d_tab, d_scratch, ncell, ntuples, st);
    if (prec == BP_PREC_COMP16) return med_build<PolC16>(S, d_idx, d_tab, d_scratch, ncell, ntuples, st);
    if (prec == BP_PREC_CBF16) return med_build<PolB24>(S, d_idx, d_tab, d_scratch, ncell, ntuples, st);
    return cudaSuccess;                    // FP64: the arrays
}

}  // namespace bpk

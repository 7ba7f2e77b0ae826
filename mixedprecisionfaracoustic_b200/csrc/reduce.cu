// reduce.cu - FP64 reductions: field energy and relative L2 error.
//
// Both accumulate in double precision per thread, reduce each warp with
// __shfl_xor_sync, each block through shared memory, write one partial per
// block into a scratch array and finish with a single-block pass, so the
// result does not depend on scheduling (no floating-point atomics).
#include "common.cuh"

namespace bpk {

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread; thread 0 returns the totals.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
    __shared__ double sh[NV][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = wsum(v[k]);
    if (l == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k][w] = v[k];
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            v[k] = l < nw ? sh[k][l] : 0.0;
            v[k] = wsum(v[k]);
        }
    }
}

template <class P>
__global__ void k_energy(const ShotDesc* __restrict__ shots, double* partial) {
    const ShotDesc& S = shots[0];
    const long long n = (long long)S.nx * S.ny * S.nz;
    double sv = 1.0, ss = 1.0;
    if constexpr (P::prec == BP_PREC_COMP16) {
        const int it = *S.step_base;
        const int itc = it > 0 ? (it - 1 < S.nt ? it - 1 : S.nt - 1) : 0;
        sv = (double)S.out_vel / S.dyn[itc];
        ss = (double)S.out_stress / S.dyn[itc];
    }
    double acc[1] = {0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % S.nx);
        long long rest = q / S.nx;
        int y = (int)(rest % S.ny), z = (int)(rest / S.ny);
        const long long i = x + (long long)y * S.pitch + (long long)z * S.plane;
        double e = 0.0;
#pragma unroll
        for (int f = 0; f < BP_NFIELDS; f++) {
            if (S.f[f] == nullptr) continue;
            double v = (double)P::ld1(S.f[f], S.flo[f], i) * (f <= BP_F_VWZ ? sv : ss);
            e += v * v;
        }
        acc[0] += e;
    }
    block_sum<1>(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

template <int NV>
__global__ void k_finish(const double* partial, int nblocks, double* out) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] += partial[(long long)i * NV + k];
    block_sum<NV>(v);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) out[k] = v[k];
}

// sum (x - ref)^2 and sum ref^2 over n floats
__global__ void k_rel_l2(const float* __restrict__ x, const float* __restrict__ ref, long long n, double* partial) {
    double v[2] = {0.0, 0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        double a = x[q], b = ref[q];
        v[0] += (a - b) * (a - b);
        v[1] += b * b;
    }
    block_sum<2>(v);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = v[0]; partial[2 * blockIdx.x + 1] = v[1]; }
}

int reduce_blocks() { return 148 * 2; }

cudaError_t launch_energy(int prec, const ShotDesc* d_shots, double* partial, double* out, cudaStream_t st) {
    const int nb = reduce_blocks();
    if (prec == BP_PREC_FP32) k_energy<PolF32><<<nb, 256, 0, st>>>(d_shots, partial);
    else if (prec == BP_PREC_COMP16) k_energy<PolC16><<<nb, 256, 0, st>>>(d_shots, partial);
    else if (prec == BP_PREC_CBF16) k_energy<PolB24><<<nb, 256, 0, st>>>(d_shots, partial);
    else k_energy<PolF64><<<nb, 256, 0, st>>>(d_shots, partial);
    k_finish<1><<<1, 1024, 0, st>>>(partial, nb, out);
    return cudaGetLastError();
}

// partial: 2 * reduce_blocks() doubles, out: 2 doubles (device)
cudaError_t launch_rel_l2(const float* x, const float* ref, long long n, double* partial, double* out,
                          cudaStream_t st) {
    const int nb = reduce_blocks();
    k_rel_l2<<<nb, 256, 0, st>>>(x, ref, n, partial);
    k_finish<2><<<1, 1024, 0, st>>>(partial, nb, out);
    return cudaGetLastError();
}

}  // namespace bpk

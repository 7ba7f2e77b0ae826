// codec.cu - the compensated FP16 codec run on the device over host arrays.
//
// bp_comp16_encode / bp_comp16_decode apply the same encode_ch / decode_ch
// the COMP16 kernels use (the reference's store_ch / load_ch,
// Half/main.cu:75-100) to caller data, for verification and for callers that
// want to produce or read COMP16 state themselves.
#include <string>

#include "shot.h"

namespace bpk {

__global__ void k_encode(const float* __restrict__ v, long long n, __half* hi, int8_t* lo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        encode_ch(v[i], hi[i], lo[i]);
}
__global__ void k_decode(const __half* __restrict__ hi, const int8_t* __restrict__ lo, long long n, float* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = decode_ch(hi[i], lo[i]);
}

}  // namespace bpk

using namespace bpk;

extern "C" {

int bp_comp16_encode(const float* host, size_t n, uint16_t* hi, int8_t* lo) {
    if (!host || !hi || !lo) { set_error("bad arguments"); return BP_ERR_ARG; }
    if (n == 0) return BP_OK;
    char* d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * 7);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return e == cudaErrorMemoryAllocation ? BP_ERR_OOM : BP_ERR_NO_DEVICE; }
    float* dv = (float*)d;
    __half* dh = (__half*)(d + n * 4);
    int8_t* dl = (int8_t*)(d + n * 6);
    e = cudaMemcpy(dv, host, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) { k_encode<<<296, 256>>>(dv, (long long)n, dh, dl); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaMemcpy(hi, dh, n * 2, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(lo, dl, n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    return BP_OK;
}

int bp_comp16_decode(const uint16_t* hi, const int8_t* lo, size_t n, float* out) {
    if (!hi || !lo || !out) { set_error("bad arguments"); return BP_ERR_ARG; }
    if (n == 0) return BP_OK;
    char* d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * 7);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return e == cudaErrorMemoryAllocation ? BP_ERR_OOM : BP_ERR_NO_DEVICE; }
    float* dv = (float*)d;
    __half* dh = (__half*)(d + n * 4);
    int8_t* dl = (int8_t*)(d + n * 6);
    e = cudaMemcpy(dh, hi, n * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dl, lo, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) { k_decode<<<296, 256>>>(dh, dl, (long long)n, dv); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaMemcpy(out, dv, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    return BP_OK;
}

}  // extern "C"

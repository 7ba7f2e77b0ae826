// codec.cu - the compensated storage codecs run on the device over host arrays.
//
// bp_comp16_encode / bp_comp16_decode apply the same encode_ch / decode_ch
// the COMP16 kernels use (the reference's store_ch / load_ch,
// Half/main.cu:75-100) to caller data, for verification and for callers that
// want to produce or read COMP16 state themselves.  bp_cbf16_encode /
// bp_cbf16_decode do the same with the CBF16 kernels' 4-value vector forms
// (PolB24::st4 / ld4) and, for a tail of n mod 4 values, the scalar ones.
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

// one thread per group of 4 values (the kernels' vector forms), the tail scalar
__global__ void k_encode_b24(const float* __restrict__ v, long long n, uint16_t* hi, int8_t* lo) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g * 4 < n; g += (long long)gridDim.x * blockDim.x) {
        const long long i = g * 4;
        if (i + 4 <= n) {
            float w[4] = {v[i], v[i + 1], v[i + 2], v[i + 3]};
            PolB24::st4(hi, lo, (cidx)i, w);
        } else {
            for (long long j = i; j < n; j++) PolB24::st1(hi, lo, (cidx)j, v[j]);
        }
    }
}
__global__ void k_decode_b24(const uint16_t* __restrict__ hi, const int8_t* __restrict__ lo, long long n, float* out) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g * 4 < n; g += (long long)gridDim.x * blockDim.x) {
        const long long i = g * 4;
        if (i + 4 <= n) {
            float w[4];
            PolB24::ld4(hi, lo, (cidx)i, w);
            for (int j = 0; j < 4; j++) out[i + j] = w[j];
        } else {
            for (long long j = i; j < n; j++) out[j] = PolB24::ld1(hi, lo, (cidx)j);
        }
    }
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

static int b24_io(bool enc, const float* v, size_t n, uint16_t* hi, int8_t* lo, float* out) {
    if (n == 0) return BP_OK;
    if (n > ((size_t)1 << 31)) { set_error("more than 2^31 values"); return BP_ERR_ARG; }   // cidx offsets
    char* d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * 7 + 16);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return e == cudaErrorMemoryAllocation ? BP_ERR_OOM : BP_ERR_NO_DEVICE; }
    float* dv = (float*)d;                         // n * 4 bytes
    uint16_t* dh = (uint16_t*)(d + n * 4);         // n * 2, 8-byte aligned when n % 4 == 0
    int8_t* dl = (int8_t*)(d + n * 6);             // n
    if (n % 4) {                                   // keep the vector accesses aligned
        dh = (uint16_t*)(d + ((n * 4 + 15) & ~(size_t)15));
        dl = (int8_t*)((char*)dh + ((n * 2 + 15) & ~(size_t)15));
    }
    if (enc) {
        e = cudaMemcpy(dv, v, n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) { k_encode_b24<<<296, 256>>>(dv, (long long)n, dh, dl); e = cudaGetLastError(); }
        if (e == cudaSuccess) e = cudaMemcpy(hi, dh, n * 2, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(lo, dl, n, cudaMemcpyDeviceToHost);
    } else {
        e = cudaMemcpy(dh, hi, n * 2, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dl, lo, n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) { k_decode_b24<<<296, 256>>>(dh, dl, (long long)n, dv); e = cudaGetLastError(); }
        if (e == cudaSuccess) e = cudaMemcpy(out, dv, n * 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    return BP_OK;
}

int bp_cbf16_encode(const float* host, size_t n, uint16_t* hi, uint8_t* lo) {
    if (!host || !hi || !lo) { set_error("bad arguments"); return BP_ERR_ARG; }
    return b24_io(true, host, n, hi, (int8_t*)lo, nullptr);
}

int bp_cbf16_decode(const uint16_t* hi, const uint8_t* lo, size_t n, float* out) {
    if (!hi || !lo || !out) { set_error("bad arguments"); return BP_ERR_ARG; }
    return b24_io(false, nullptr, n, const_cast<uint16_t*>(hi), (int8_t*)const_cast<uint8_t*>(lo), out);
}

}  // extern "C"

// noalloc.cu - relative L2 difference of two device arrays without any
// device allocation.
//
// bp_rel_l2_device allocates its reduction scratch with cudaMalloc on every
// call.  Some callers cannot allow that: real-time loops that must not stall
// on the implicit device synchronisation cudaMalloc/cudaFree can bring, and
// processes that hand all device memory to their own pool up front, where a
// cudaMalloc fails.  This variant keeps its scratch in a fixed array that lives
// in the library's device image instead.
//
// Scratch: one (sum of squared differences, sum of squared reference values)
// partial pair per block, at most kMaxBlocks blocks, plus the final pair: about
// 16 KB per GPU that loads the library, held until the process exits.  Each
// block covers up to kPerBlock elements, so the largest accepted n is
// kMaxBlocks * kPerBlock = 16,777,216; larger inputs are rejected with
// BP_ERR_ARG.
//
// The call is synchronous: both kernels run on the legacy default stream and
// the result comes back by a blocking cudaMemcpy, so the function returns once
// the value is known.  Work still running on other streams (the library's own
// streams are created non-blocking) is not ordered before it: the inputs must
// be complete, so synchronise the stream that produces them first.
//
// Every call on a device shares that one array, which keeps the last call's
// contents.  Nothing in it needs to start at zero: each call writes every
// partial it reads and then the final pair.  Two calls whose kernels overlap
// on the GPU (calls from different host threads without ordering) race on the
// array and may return wrong results; serialise them.
//
// The device address of the array is looked up with cudaGetSymbolAddress once
// per device, by the first call made while that device is current; make that
// first call before any stream capture begins on the device.
#include <cmath>
#include <mutex>
#include <string>

#include "shot.h"

namespace bpk {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kMaxBlocks = 1024;
constexpr long long kPerBlock = 16384;            // 64 elements per thread
constexpr long long kMaxElems = kMaxBlocks * kPerBlock;

static __device__ __align__(256) double g_rel_l2_scratch[2 * kMaxBlocks + 2];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums (a-b)^2 and b^2 over this block's slice into partial[2*block ..].
__global__ void k_rel_l2_partials(const float* __restrict__ x, const float* __restrict__ ref, long long n,
                                  double* partial) {
    __shared__ double sh[2][kNoAllocThreads / 32];
    double d = 0.0, r = 0.0;
    const long long beg = (long long)blockIdx.x * kPerBlock;
    const long long end = beg + kPerBlock < n ? beg + kPerBlock : n;
    for (long long q = beg + threadIdx.x; q < end; q += blockDim.x) {
        const double a = x[q], b = ref[q];
        d += (a - b) * (a - b);
        r += b * b;
    }
    d = wsum(d);
    r = wsum(r);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[0][w] = d; sh[1][w] = r; }
    __syncthreads();
    if (w == 0) {
        d = l < kNoAllocThreads / 32 ? sh[0][l] : 0.0;
        r = l < kNoAllocThreads / 32 ? sh[1][l] : 0.0;
        d = wsum(d);
        r = wsum(r);
        if (l == 0) { partial[2 * blockIdx.x] = d; partial[2 * blockIdx.x + 1] = r; }
    }
}

// One block: totals of the first nblocks partial pairs into out[0..1].
__global__ void k_rel_l2_total(const double* __restrict__ partial, int nblocks, double* out) {
    __shared__ double sh[2][32];
    double d = 0.0, r = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        d += partial[2 * i];
        r += partial[2 * i + 1];
    }
    d = wsum(d);
    r = wsum(r);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[0][w] = d; sh[1][w] = r; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        d = l < nw ? sh[0][l] : 0.0;
        r = l < nw ? sh[1][l] : 0.0;
        d = wsum(d);
        r = wsum(r);
        if (l == 0) { out[0] = d; out[1] = r; }
    }
}

// Device address of the scratch array on the current device (looked up once).
int scratch_for_current_device(double** ptr) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e)); return BP_ERR_NO_DEVICE; }
    if (dev < 0 || dev >= kMaxDevices) { set_error("device ordinal beyond the scratch table"); return BP_ERR_ARG; }
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_rel_l2_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            return BP_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *ptr = g_scratch_ptr[dev];
    return BP_OK;
}

}  // namespace
}  // namespace bpk

using namespace bpk;

extern "C" int bp_rel_l2_device_noalloc(const float* d_x, const float* d_ref, size_t n, double* rel) {
    if (!d_x || !d_ref || !rel) { set_error("bad arguments"); return BP_ERR_ARG; }
    if (n == 0) { set_error("empty input"); return BP_ERR_ARG; }
    if ((long long)n > kMaxElems) {
        set_error("n = " + std::to_string(n) + " exceeds the no-allocation limit of " + std::to_string(kMaxElems) +
                  " elements (use bp_rel_l2_device)");
        return BP_ERR_ARG;
    }
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    const int nblocks = (int)(((long long)n + kPerBlock - 1) / kPerBlock);
    k_rel_l2_partials<<<nblocks, kNoAllocThreads>>>(d_x, d_ref, (long long)n, scratch);
    k_rel_l2_total<<<1, 1024>>>(scratch, nblocks, scratch + 2 * kMaxBlocks);
    double h[2] = {0.0, 0.0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, scratch + 2 * kMaxBlocks, sizeof h, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    *rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
    return BP_OK;
}

// Allocation-free variant of the statistics reduction.
//
// The solver's statistics (the maxima of |a|, |v|, |u| written to
// stats-*.bin) reduce per-block partial results in a device scratch buffer
// that each handle allocates when it is created.  Some callers cannot
// allocate device memory at the point where they want such a reduction:
// code running while a memory pool is frozen or its budget is exhausted,
// code inside allocation-sensitive regions of a host framework, or callers
// that must not touch the CUDA allocator at all.  sord_vector_max_noalloc
// computes the same maximum of w0^2 + w1^2 + w2^2 over a region of a
// caller-owned field, keeping its partial results in a file-scope
// __device__ array instead:
//
//   * the array holds kNoAllocBlocks (1024) partial maxima, 4 KiB; every GPU
//     that loads this library holds one copy until the process exits;
//   * each block strides over the region, so the number of blocks (and
//     therefore the partials used) never exceeds 1024; regions of 2^31
//     elements or more, or non-positive extents, are rejected;
//   * every call shares the array and overwrites the partials it uses
//     (nothing in it has to start at zero); calls that overlap on the GPU
//     (concurrent streams, or host threads racing on one device) race on
//     the array and must be serialised by the caller;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress while that device is current and caches it; make
//     that first call before any stream capture on the device.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/sordgpu.h"

namespace {

constexpr int kNoAllocBlocks = 1024;
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned g_noalloc_partials[kNoAllocBlocks];

unsigned* g_partials_ptr[kMaxDevices] = {};
std::mutex g_partials_mutex;

// Non-negative floats order like their bit patterns; NaN (0x7fc00000)
// sorts above +Inf, so a NaN anywhere wins the maximum.
__device__ __forceinline__ unsigned max_bits(unsigned a, unsigned b) { return a > b ? a : b; }

__global__ void k_vmax_partials(const float* __restrict__ w0, const float* __restrict__ w1, const float* __restrict__ w2,
                                int n0, int n1, int a0, int a1, int a2, int c0, int c1, int c2, unsigned* partials) {
    const long long m0 = c0, m1 = c1, cnt = m0 * m1 * (long long)c2;
    unsigned best = 0u;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        const int j = a0 + (int)(t % m0), k = a1 + (int)((t / m0) % m1), l = a2 + (int)(t / (m0 * m1));
        const long long q = (long long)(j - 1) + (long long)n0 * ((long long)(k - 1) + (long long)n1 * (long long)(l - 1));
        const float v = w0[q] * w0[q] + w1[q] * w1[q] + w2[q] * w2[q];
        best = max_bits(best, v != v ? 0x7fc00000u : __float_as_uint(v));
    }
    __shared__ unsigned s[kNoAllocThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max_bits(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        best = threadIdx.x < kNoAllocThreads / 32 ? s[threadIdx.x] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max_bits(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (threadIdx.x == 0) partials[blockIdx.x] = best;
    }
}

__global__ void k_vmax_final(const unsigned* partials, int nblocks, float* out) {
    unsigned best = 0u;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) best = max_bits(best, partials[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max_bits(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ unsigned s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        best = threadIdx.x < (int)(blockDim.x >> 5) ? s[threadIdx.x] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max_bits(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (threadIdx.x == 0) out[0] = __uint_as_float(best);
    }
}

}  // namespace

namespace sordgpu {
void set_global_error(const char* msg);  // api.cu: message of sord_last_error(NULL)
}

namespace {
int set_error(int code, const char* msg) {
    sordgpu::set_global_error(msg);
    return code;
}
}  // namespace

extern "C" int sord_vector_max_noalloc(const float* w0, const float* w1, const float* w2, const int* nm, const int* i1,
                                       const int* i2, float* out, void* stream) {
    if (!w0 || !w1 || !w2 || !nm || !i1 || !i2 || !out) return set_error(SORD_E_PARAM, "null argument");
    long long cnt = 1;
    int c[3];
    for (int d = 0; d < 3; d++) {
        if (nm[d] < 1) return set_error(SORD_E_PARAM, "field extents must be positive");
        if (i1[d] < 1 || i2[d] > nm[d] || i2[d] < i1[d]) return set_error(SORD_E_PARAM, "region outside the field");
        c[d] = i2[d] - i1[d] + 1;
        cnt *= c[d];
    }
    if (cnt >= (1LL << 31)) return set_error(SORD_E_PARAM, "region too large: at most 2^31 - 1 elements");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return set_error(SORD_E_CUDA, "no current CUDA device");
    unsigned* partials;
    {
        std::lock_guard<std::mutex> lock(g_partials_mutex);
        if (!g_partials_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
            if (e != cudaSuccess || !p) return set_error(SORD_E_CUDA, cudaGetErrorString(e));
            g_partials_ptr[dev] = (unsigned*)p;
        }
        partials = g_partials_ptr[dev];
    }
    long long want = (cnt + kNoAllocThreads - 1) / kNoAllocThreads;
    int nb = (int)(want < kNoAllocBlocks ? want : kNoAllocBlocks);
    cudaStream_t st = (cudaStream_t)stream;
    // each launch reports its own status: an error the caller left pending
    // from an earlier launch stays the caller's (no cudaGetLastError here)
    int n0 = nm[0], n1 = nm[1], a0 = i1[0], a1 = i1[1], a2 = i1[2], c0 = c[0], c1 = c[1], c2 = c[2];
    void* pargs[] = {(void*)&w0, (void*)&w1, (void*)&w2, &n0, &n1, &a0, &a1, &a2, &c0, &c1, &c2, (void*)&partials};
    cudaError_t e = cudaLaunchKernel((const void*)k_vmax_partials, dim3(nb), dim3(kNoAllocThreads), pargs, 0, st);
    if (e != cudaSuccess) return set_error(SORD_E_CUDA, cudaGetErrorString(e));
    const unsigned* cpart = partials;
    void* fargs[] = {(void*)&cpart, &nb, (void*)&out};
    e = cudaLaunchKernel((const void*)k_vmax_final, dim3(1), dim3(kNoAllocThreads), fargs, 0, st);
    if (e != cudaSuccess) return set_error(SORD_E_CUDA, cudaGetErrorString(e));
    return SORD_OK;
}

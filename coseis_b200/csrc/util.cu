// Device helpers used by setup, field I/O and statistics: fills, set_halo
// (utilities.f90:103-117), region reductions, vector/tensor norms
// (utilities.f90:120-165) and rinvert (utilities.f90:40-49).
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <utility>

#include "sord.cuh"

namespace sordgpu {

static unsigned grid_for(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

__global__ void k_fill(float* p, long long n, float v) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) p[q] = v;
}
__global__ void k_copy(float* d, const float* s, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) d[q] = s[q];
}
__global__ void k_rinvert(float* p, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        float v = p[q];
        if (v != 0.0f) p[q] = 1.0f / v;
    }
}

struct Box {
    int n[3];
    int i3[3], i4[3];
};

// f = r outside [i1, i2] on axes with extent > 1
__global__ void k_set_halo(float* f, Box b, float r) {
    long long n = (long long)b.n[0] * b.n[1] * b.n[2];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int j = (int)(q % b.n[0]) + 1, k = (int)((q / b.n[0]) % b.n[1]) + 1, l = (int)(q / ((long long)b.n[0] * b.n[1])) + 1;
        bool h = (b.n[0] > 1 && (j < b.i3[0] || j > b.i4[0])) || (b.n[1] > 1 && (k < b.i3[1] || k > b.i4[1])) ||
                 (b.n[2] > 1 && (l < b.i3[2] || l > b.i4[2]));
        if (h) f[q] = r;
    }
}

// max / min / sum over region [i1, i2] (inclusive, 1-based) of a field
__global__ void k_reduce(const float* f, Box b, int mode, double* out) {
    long long n0 = b.i4[0] - b.i3[0] + 1, n1 = b.i4[1] - b.i3[1] + 1, n2 = b.i4[2] - b.i3[2] + 1;
    long long n = n0 * n1 * n2;
    double acc = mode == 0 ? -HUGE_VAL : mode == 1 ? HUGE_VAL : 0.0;
    bool nan = false;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int j = b.i3[0] + (int)(t % n0), k = b.i3[1] + (int)((t / n0) % n1), l = b.i3[2] + (int)(t / (n0 * n1));
        float v = f[(j - 1) + (long long)b.n[0] * ((k - 1) + (long long)b.n[1] * (l - 1))];
        if (v != v) nan = true;
        if (mode == 0) acc = fmax(acc, (double)v);
        else if (mode == 1) acc = fmin(acc, (double)v);
        else acc += (double)v;
    }
    __shared__ double sm[256];
    __shared__ int snan;
    if (threadIdx.x == 0) snan = 0;
    __syncthreads();
    if (nan) snan = 1;
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            double a = sm[threadIdx.x], c = sm[threadIdx.x + s];
            sm[threadIdx.x] = mode == 0 ? fmax(a, c) : mode == 1 ? fmin(a, c) : a + c;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = sm[0];
        out[2 * blockIdx.x + 1] = snan ? 1.0 : 0.0;
    }
}

__global__ void k_vnorm(float* dst, const float* a, const float* b, const float* c, Box bx, int d0, int d1, int d2, long long sy, long long sz) {
    long long n0 = (bx.i4[0] - bx.i3[0]) / d0 + 1, n1 = (bx.i4[1] - bx.i3[1]) / d1 + 1, n2 = (bx.i4[2] - bx.i3[2]) / d2 + 1;
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return;
    long long n = n0 * n1 * n2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int j = bx.i3[0] + d0 * (int)(t % n0), k = bx.i3[1] + d1 * (int)((t / n0) % n1), l = bx.i3[2] + d2 * (int)(t / (n0 * n1));
        long long q = (j - 1) + sy * (k - 1) + sz * (l - 1);
        dst[q] = a[q] * a[q] + b[q] * b[q] + c[q] * c[q];
    }
}
__global__ void k_tnorm(float* dst, const float* a0, const float* a1, const float* a2, const float* b0, const float* b1,
                        const float* b2, Box bx, int d0, int d1, int d2, long long sy, long long sz) {
    long long n0 = (bx.i4[0] - bx.i3[0]) / d0 + 1, n1 = (bx.i4[1] - bx.i3[1]) / d1 + 1, n2 = (bx.i4[2] - bx.i3[2]) / d2 + 1;
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return;
    long long n = n0 * n1 * n2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int j = bx.i3[0] + d0 * (int)(t % n0), k = bx.i3[1] + d1 * (int)((t / n0) % n1), l = bx.i3[2] + d2 * (int)(t / (n0 * n1));
        long long q = (j - 1) + sy * (k - 1) + sz * (l - 1);
        dst[q] = (a0[q] * a0[q] + a1[q] * a1[q] + a2[q] * a2[q]) + 2.0f * (b0[q] * b0[q] + b1[q] * b1[q] + b2[q] * b2[q]);
    }
}

void dev_fill(Solver& s, float* p, long long n, float v) {
    if (n <= 0) return;
    k_fill<<<grid_for(n), 256, 0, s.stream>>>(p, n, v);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}
void dev_copy(Solver& s, float* d, const float* src, long long n) {
    if (n <= 0) return;
    k_copy<<<grid_for(n), 256, 0, s.stream>>>(d, src, n);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}
void dev_rinvert(Solver& s, float* p, long long n) {
    if (n <= 0) return;
    k_rinvert<<<grid_for(n), 256, 0, s.stream>>>(p, n);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}
void dev_set_halo(Solver& s, FieldView f, float r, const int* i1, const int* i2) {
    Box b;
    for (int i = 0; i < 3; i++) {
        b.n[i] = f.n[i];
        b.i3[i] = std::min(i1[i], f.n[i] + 1);
        b.i4[i] = std::max(i2[i], 0);
    }
    long long n = (long long)f.n[0] * f.n[1] * f.n[2];
    k_set_halo<<<grid_for(n), 256, 0, s.stream>>>(f.p, b, r);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

static double reduce(Solver& s, FieldView f, const int* i1, const int* i2, int mode, bool* nan) {
    Box b;
    long long n = 1;
    for (int i = 0; i < 3; i++) {
        b.n[i] = f.n[i];
        b.i3[i] = std::max(i1[i], 1);
        b.i4[i] = std::min(i2[i], f.n[i]);
        if (b.i4[i] < b.i3[i]) n = 0;
        else n *= (b.i4[i] - b.i3[i] + 1);
    }
    if (nan) *nan = false;
    if (n == 0) return mode == 0 ? -HUGE_VAL : mode == 1 ? HUGE_VAL : 0.0;
    unsigned nb = (unsigned)std::min<long long>((n + 255) / 256, 1024);
    double* d = (double*)s.d.red + kRedReduce;
    k_reduce<<<nb, 256, 0, s.stream>>>(f.p, b, mode, d);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
    std::vector<double> h(2 * nb);
    SORD_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    double acc = mode == 0 ? -HUGE_VAL : mode == 1 ? HUGE_VAL : 0.0;
    for (unsigned i = 0; i < nb; i++) {
        double v = h[2 * i];
        if (nan && h[2 * i + 1] != 0.0) *nan = true;
        acc = mode == 0 ? std::max(acc, v) : mode == 1 ? std::min(acc, v) : acc + v;
    }
    return acc;
}
float dev_reduce_max(Solver& s, FieldView f, const int* i1, const int* i2) {
    bool nan;
    double v = reduce(s, f, i1, i2, 0, &nan);
    return nan ? NAN : (float)v;
}
float dev_reduce_min(Solver& s, FieldView f, const int* i1, const int* i2) {
    bool nan;
    double v = reduce(s, f, i1, i2, 1, &nan);
    return nan ? NAN : (float)v;
}
double dev_reduce_sum_d(Solver& s, FieldView f, const int* i1, const int* i2) { return reduce(s, f, i1, i2, 2, nullptr); }

void dev_vector_norm(Solver& s, float* dst, float* const w[3], const int* i1, const int* i2, const int* di) {
    Box b;
    for (int i = 0; i < 3; i++) { b.n[i] = s.g.nm[i]; b.i3[i] = i1[i]; b.i4[i] = i2[i]; }
    long long n = (long long)s.g.nv;
    k_vnorm<<<grid_for(n), 256, 0, s.stream>>>(dst, w[0], w[1], w[2], b, di[0], di[1], di[2], s.g.sy, s.g.sz);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}
void dev_tensor_norm(Solver& s, float* dst, float* const a[3], float* const bb[3], const int* i1, const int* i2, const int* di) {
    Box b;
    for (int i = 0; i < 3; i++) { b.n[i] = s.g.nm[i]; b.i3[i] = i1[i]; b.i4[i] = i2[i]; }
    long long n = (long long)s.g.nv;
    k_tnorm<<<grid_for(n), 256, 0, s.stream>>>(dst, a[0], a[1], a[2], bb[0], bb[1], bb[2], b, di[0], di[1], di[2], s.g.sy, s.g.sz);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

// Raise a kernel's dynamic shared-memory limit once per device; safe when
// several host threads launch on one or more devices (each thread remembers
// what it has seen, so the shared set is consulted once per thread).
void smem_limit(const void* func, int bytes) {
    static std::mutex m;
    static std::set<std::pair<int, const void*>> done;
    thread_local std::set<std::pair<int, const void*>> seen;
    int dev = 0;
    SORD_CUDA(cudaGetDevice(&dev));
    if (seen.count({dev, func})) return;
    std::lock_guard<std::mutex> lock(m);
    if (!done.count({dev, func})) {
        SORD_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        done.insert({dev, func});
    }
    seen.insert({dev, func});
}

// ------------------------------------------------------------ memory
// Device memory of a handle comes from the device's default memory pool in
// stream order (cudaMallocAsync / cudaFreeAsync on the handle's stream):
// unlike cudaMalloc and cudaFree, neither call synchronises the device, so
// handles that run concurrently (an ensemble) do not serialise each other's
// setup and teardown.  While any handle is alive the pool keeps freed
// memory for the next allocation; when the last one goes it is trimmed.
// Returning tens of GB to the driver takes up to seconds, so the trim runs
// on a helper thread and the destroying call returns at once; the next
// handle created on that device, and the exit of the process (an atexit
// handler, registered after the CUDA runtime's own and so run before it),
// wait for it.
static std::mutex g_mem_m;
static std::map<int, int> g_live;             // device -> live handles
static std::map<int, std::thread> g_trim;     // device -> trim in progress

static void trim_join_locked(int device) {
    auto it = g_trim.find(device);
    if (it != g_trim.end() && it->second.joinable()) it->second.join();
}

static void trim_join_all() {
    std::lock_guard<std::mutex> lock(g_mem_m);
    for (auto& t : g_trim)
        if (t.second.joinable()) t.second.join();
}

void mem_attach(int device) {
    std::lock_guard<std::mutex> lock(g_mem_m);
    trim_join_locked(device);
    if (g_live[device]++ == 0) {
        cudaMemPool_t pool;
        SORD_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = ~0ull;
        SORD_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
}

// Wait for a pending trim on `device`; with no live handle there, return
// the pool's unused memory to the driver now.
void mem_trim(int device) {
    std::lock_guard<std::mutex> lock(g_mem_m);
    trim_join_locked(device);
    if (g_live[device] == 0) {
        cudaMemPool_t pool;
        SORD_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        SORD_CUDA(cudaMemPoolTrimTo(pool, 0));
    }
}

void mem_detach(int device) {
    static std::once_flag at_exit;
    std::lock_guard<std::mutex> lock(g_mem_m);
    if (--g_live[device] == 0) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = 0;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            std::call_once(at_exit, [] { std::atexit(trim_join_all); });
            trim_join_locked(device);
            g_trim[device] = std::thread([device, pool] {
                cudaSetDevice(device);
                cudaMemPoolTrimTo(pool, 0);
            });
        }
    }
}

cudaError_t dev_malloc(Solver& s, void** p, size_t bytes) {
    return cudaMallocAsync(p, bytes > 0 ? bytes : 4, s.stream);
}

void dev_free(Solver& s, void* p) {
    if (p) cudaFreeAsync(p, s.stream);
}

// Pinned host buffers, kept for reuse by later handles: cudaMallocHost
// synchronises the device, so a buffer is allocated only when no free one
// is large enough.
static std::multimap<size_t, void*> g_pin_free;
static std::map<void*, size_t> g_pin_size;

void* pinned_get(size_t bytes) {
    std::lock_guard<std::mutex> lock(g_mem_m);
    auto it = g_pin_free.lower_bound(bytes);
    if (it != g_pin_free.end()) {
        void* p = it->second;
        g_pin_free.erase(it);
        return p;
    }
    void* p = nullptr;
    SORD_CUDA(cudaMallocHost(&p, bytes));
    g_pin_size[p] = bytes;
    return p;
}

void pinned_put(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_mem_m);
    auto it = g_pin_size.find(p);
    if (it == g_pin_size.end()) return;
    g_pin_free.insert({it->second, p});
}

}  // namespace sordgpu

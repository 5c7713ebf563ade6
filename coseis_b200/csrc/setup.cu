// Setup on the device: every coefficient the step kernels read.
//
//   init_grid          grid_generation.f90:6-200
//   init_material      material_model.f90:6-171
//   init_pml           boundary_pml.f90:7-82
//   init_finite_source kinematic_source.f90:10-63
//   resample_material  material_resample.f90:6-55
// plus the check that selects the rectilinear fast path: every real cell's
// support-operator brackets equal those of one reference cell, bit for bit,
// so the fast path computes exactly what the general operator would.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "sord.cuh"
#include "stencil.cuh"

namespace sordgpu {

static unsigned gfor(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : b);
}
#define LAUNCH_CHECK(s) do { (s).launches++; SORD_CUDA(cudaGetLastError()); } while (0)

// Counter hash replacing Fortran random_number (same function as the oracle).
__device__ __forceinline__ unsigned long long d_splitmix(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float d_urand(unsigned long long call, unsigned long long idx) {
    unsigned long long h = d_splitmix(d_splitmix(call * 0x100000001B3ull + 0x5151) ^ idx);
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------ grid
// xx(i,:,:,c) = dx(c) * (i + nnoff(c) - 1) on the node range, shifted by one
// node past the fault (grid_generation.f90:22-33).
__global__ void k_grid(Geom g, float* x0, float* x1, float* x2, int shift_axis, int shift_from) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int p[3] = {(int)(q % g.sy) + 1, (int)((q / g.sy) % g.nm[1]) + 1, (int)(q / g.sz) + 1};
        float* X[3] = {x0, x1, x2};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float v = 0.f;
            if (p[c] >= g.i1node[c] && p[c] <= g.i2node[c]) {
                int off = (c == shift_axis && p[c] >= shift_from) ? 2 : 1;
                v = g.dx[c] * (float)(p[c] + g.nnoff[c] - off);
            }
            X[c][q] = v;
        }
    }
}

// gridnoise (grid_generation.f90:41-62): xx += amp*(rand - 0.5), zero outside
// [i1pml+1, i2pml-1] and [i1bc+1, i2bc-1] and on the two fault planes.
__global__ void k_gridnoise(Geom g, float* x0, float* x1, float* x2, unsigned long long call, float amp, int fault_axis,
                            int f1, int f2) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int p[3] = {(int)(q % g.sy) + 1, (int)((q / g.sy) % g.nm[1]) + 1, (int)(q / g.sz) + 1};
        bool zero = false;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (g.nm[d] > 1 && (p[d] < g.i1pml[d] + 1 || p[d] > g.i2pml[d] - 1)) zero = true;
            if (g.nm[d] > 1 && (p[d] < g.i1bc[d] + 1 || p[d] > g.i2bc[d] - 1)) zero = true;
        }
        if (fault_axis >= 0 && p[fault_axis] >= f1 && p[fault_axis] <= f2) zero = true;
        float* X[3] = {x0, x1, x2};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float w = amp * (d_urand(call, (unsigned long long)q + (unsigned long long)c * g.nv) - 0.5f);
            if (zero) w = 0.f;
            X[c][q] = X[c][q] + w;
        }
    }
}

// rexpand (grid_generation.f90:65-100): add a per-plane offset along axis d
__global__ void k_plane_add(Geom g, float* x, int d, int p, float sft) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int c = d == 0 ? (int)(q % g.sy) + 1 : d == 1 ? (int)((q / g.sy) % g.nm[1]) + 1 : (int)(q / g.sz) + 1;
        if (c == p) x[q] = x[q] + sft;
    }
}

__global__ void k_affine(Geom g, float* x0, float* x1, float* x2, float m0, float m1, float m2, float m3, float m4,
                         float m5, float m6, float m7, float m8) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        float a = x0[q], b = x1[q], c = x2[q];
        x0[q] = m0 * a + m1 * b + m2 * c;
        x1[q] = m3 * a + m4 * b + m5 * c;
        x2[q] = m6 * a + m7 * b + m8 * c;
    }
}

// cell volume: vc = diff_nc(x_3, 3) on the cell range (grid_generation.f90:184-193)
__global__ void k_volume(Geom g, const float* x0, const float* x1, const float* x2, float* vc) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int j = (int)(q % g.sy) + 1, k = (int)((q / g.sy) % g.nm[1]) + 1, l = (int)(q / g.sz) + 1;
        bool in = j >= g.i1cell[0] && j <= g.i2cell[0] && k >= g.i1cell[1] && k <= g.i2cell[1] && l >= g.i1cell[2] &&
                  l <= g.i2cell[2];
        float v = 0.f;
        if (in) {
            const float* X_[3] = {x0, x1, x2};
            float X[3][8];
            for (int c = 0; c < 3; c++)
                for (int n = 0; n < 8; n++) X[c][n] = X_[c][q + (n & 1) + ((n >> 1) & 1) * g.sy + ((n >> 2) & 1) * g.sz];
            float B[8], F[8];
            brackets_nc(X, 2, B);
            for (int t = 0; t < 8; t++) F[t] = X[2][term_corner(t)];
            v = stencil8(F, B, g.h);
            if (g.ifn && (g.ifn == 1 ? j : g.ifn == 2 ? k : l) == g.irup) v = 0.f;
        }
        vc[q] = v;
    }
}

// cell centres (grid_generation.f90:127-132): 8-point average, 0 elsewhere
__global__ void k_average(Geom g, float* dst, const float* src, int a1, int a2, int b1, int b2, int c1, int c2, int d) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int j = (int)(q % g.sy) + 1, k = (int)((q / g.sy) % g.nm[1]) + 1, l = (int)(q / g.sz) + 1;
        if (j >= a1 && j <= a2 && k >= b1 && k <= b2 && l >= c1 && l <= c2) {
            long long dj = d, dk = d * g.sy, dl = d * g.sz;
            dst[q] = 0.125f * (src[q] + src[q + dj + dk + dl] + src[q + dk + dl] + src[q + dj] + src[q + dj + dl] +
                               src[q + dk] + src[q + dj + dk] + src[q + dl]);
        } else {
            // set_halo(f2, 0, i1, i2) applies on axes of extent > 1 only
            bool h = (g.nm[0] > 1 && (j < a1 || j > a2)) || (g.nm[1] > 1 && (k < b1 || k > b2)) || (g.nm[2] > 1 && (l < c1 || l > c2));
            if (h) dst[q] = 0.f;
        }
    }
}

// ------------------------------------------------------------ material
__global__ void k_rlimits(float* f, long long n, float fmin, float fmax) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        float v = f[q];
        if (fmin > 0.f && fmax > 0.f) v = fmaxf(fminf(v, fmax), fmin);
        else if (fmin > 0.f) v = fmaxf(v, fmin);
        else if (fmax > 0.f) v = fminf(v, fmax);
        f[q] = v;
    }
}
__global__ void k_vdamp(float* gam, const float* vs, long long n, float vdamp) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        gam[q] = vs[q] == 0.f ? 0.f : vdamp / vs[q];
}
// mu = rho vs^2, lam = rho vp^2 - 2 mu, yy = Poisson ratio (material_model.f90:272-287)
__global__ void k_moduli(long long n, const float* mr, const float* s1, const float* s2, float* lam, float* mu, float* yy) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        float m = mr[q] * s2[q] * s2[q];
        float la = mr[q] * s1[q] * s1[q] - 2.0f * m;
        mu[q] = m;
        lam[q] = la;
        float r = la + m;
        yy[q] = r == 0.f ? 0.f : 0.5f * la / r;
    }
}
// hourglass constant (material_model.f90:324-338)
__global__ void k_hgconst(long long n, const float* lam, const float* mu, float* yy, float s) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        float r = lam[q] + 2.0f * mu[q];
        yy[q] = r == 0.f ? 0.f : mu[q] * (lam[q] + mu[q]) * s / r;
    }
}
__global__ void k_mul(float* d, const float* a, const float* b, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) d[q] = a[q] * b[q];
}
__global__ void k_scale(float* d, const float* a, float s, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) d[q] = a[q] * s;
}
__global__ void k_zero_plane(Geom g, float* f, int axis, int p) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int c = axis == 0 ? (int)(q % g.sy) + 1 : axis == 1 ? (int)((q / g.sy) % g.nm[1]) + 1 : (int)(q / g.sz) + 1;
        if (c == p) f[q] = 0.f;
    }
}

// ------------------------------------------------------------ rectilinear check
// Brackets of a reference cell / node (one thread) and a comparison of every
// real cell against them; cells on the fault plane (zero volume) and halo
// cells are excluded (their stress is identically zero).
__global__ void k_ref_brackets(Geom g, const float* x0, const float* x1, const float* x2, int jc, int kc, int lc, int jn,
                               int kn, int ln, float* out) {
    const float* X_[3] = {x0, x1, x2};
    long long q = g.idx(jc, kc, lc);
    float X[3][8];
    for (int c = 0; c < 3; c++)
        for (int n = 0; n < 8; n++) X[c][n] = X_[c][q + (n & 1) + ((n >> 1) & 1) * g.sy + ((n >> 2) & 1) * g.sz];
    for (int a = 0; a < 3; a++) brackets_nc(X, a, out + 8 * a);
    long long qn = g.idx(jn, kn, ln);
    auto XN = [&](int c, int m) -> float {
        int dj = m % 3 - 1, dk = (m / 3) % 3 - 1, dl = m / 9 - 1;
        return X_[c][qn + dj + dk * g.sy + dl * g.sz];
    };
    for (int a = 0; a < 3; a++) brackets_cn(XN, a, out + 24 + 8 * a);
}

// Mismatch bits are gathered per thread (a direction already found to differ
// is not tested again) and merged with one atomic per warp.
__global__ void k_rect_check(Geom g, const float* x0, const float* x1, const float* x2, const float* ref, unsigned* bad) {
    const float* X_[3] = {x0, x1, x2};
    unsigned m = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int p[3] = {(int)(q % g.sy) + 1, (int)((q / g.sy) % g.nm[1]) + 1, (int)(q / g.sz) + 1};
        // cell test
        bool cell = true;
        for (int d = 0; d < 3; d++) cell = cell && p[d] >= g.i1cell[d] && p[d] <= g.i2cell[d];
        if (g.ifn && p[g.ifn - 1] == g.irup) cell = false;
        if (cell) {
            float X[3][8];
            for (int c = 0; c < 3; c++)
                for (int n = 0; n < 8; n++) X[c][n] = X_[c][q + (n & 1) + ((n >> 1) & 1) * g.sy + ((n >> 2) & 1) * g.sz];
            for (int a = 0; a < 3; a++) {
                if (m & (1u << a)) continue;
                float B[8];
                brackets_nc(X, a, B);
                for (int t = 0; t < 8; t++)
                    if (!(B[t] == ref[8 * a + t])) m |= 1u << a;
            }
        }
        // node test: terms whose cell is real and off the fault plane
        bool node = true;
        for (int d = 0; d < 3; d++) node = node && p[d] >= g.i1node[d] && p[d] <= g.i2node[d];
        if (node) {
            auto XN = [&](int c, int m) -> float {
                int dj = m % 3 - 1, dk = (m / 3) % 3 - 1, dl = m / 9 - 1;
                return X_[c][q + dj + dk * g.sy + dl * g.sz];
            };
            const int ct[8] = {-1, 0, -1, 0, -1, 0, -1, 0}, kt[8] = {-1, -1, -1, -1, 0, 0, 0, 0}, lt[8] = {-1, -1, 0, 0, -1, -1, 0, 0};
            for (int a = 0; a < 3; a++) {
                if (m & (8u << a)) continue;
                float B[8];
                brackets_cn(XN, a, B);
                for (int t = 0; t < 8; t++) {
                    int c[3] = {p[0] + ct[t], p[1] + kt[t], p[2] + lt[t]};
                    bool real = true;
                    for (int d = 0; d < 3; d++) real = real && c[d] >= g.i1cell[d] && c[d] <= g.i2cell[d];
                    if (g.ifn && c[g.ifn - 1] == g.irup) real = false;
                    if (real && !(B[t] == ref[24 + 8 * a + t])) m |= 8u << a;
                }
            }
        }
    }
    m = __reduce_or_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicOr(bad, m);
}

// terrain mesh test: x depends on j only and y on k only (bit 64 if not)
__global__ void k_terrain_check(Geom g, const float* x0, const float* x1, const float* x1d, const float* y1d, unsigned* bad) {
    unsigned m = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int j = (int)(q % g.sy) + 1, k = (int)((q / g.sy) % g.nm[1]) + 1;
        if (!(x0[q] == x1d[j - 1]) || !(x1[q] == y1d[k - 1])) m = 64u;
    }
    m = __reduce_or_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicOr(bad, m);
}
__global__ void k_line(const float* src, float* dst, int n, long long stride, long long base) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[base + stride * i];
}

// ------------------------------------------------------------ host side
static float powi_f(float x, int n) {
    if (n < 0) return 1.0f / powi_f(x, -n);
    float r = 1.0f, b = x;
    bool first = true;
    while (n) {
        if (n & 1) { r = first ? b : r * b; first = false; }
        n >>= 1;
        if (n) b = b * b;
    }
    return r;
}
static long ipow_l(long x, int n) { long r = 1; for (int i = 0; i < n; i++) r *= x; return r; }

static FieldView vol(Solver& s, float* p) {
    FieldView f;
    f.p = p;
    for (int i = 0; i < 3; i++) f.n[i] = s.g.nm[i];
    return f;
}

static void alloc(Solver& s, float** p, long long n) {
    cudaError_t e = dev_malloc(s, (void**)p, sizeof(float) * (size_t)(n > 0 ? n : 1));
    if (e != cudaSuccess) throw SordError(SORD_E_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    SORD_CUDA(cudaMemsetAsync(*p, 0, sizeof(float) * (size_t)(n > 0 ? n : 1), s.stream));
}

// setup.f90:6-84 for the serial block
static void setup_dimensions(Solver& s) {
    Params& P = s.prm;
    Geom& g = s.g;
    for (int i = 0; i < 3; i++) { g.dx[i] = P.delta[i]; g.nn[i] = P.shape[i]; }
    g.dt = P.delta[3];
    s.nt = std::max(P.shape[3], 0);
    char c = P.faultnormal.size() > 1 ? P.faultnormal[1] : ' ';
    int ifn;
    switch (c) {
        case 'o': ifn = 0; break;
        case 'x': ifn = 1; break;
        case 'y': ifn = 2; break;
        case 'z': ifn = 3; break;
        default: throw SordError(SORD_E_PARAM, "Error in faultnormal");
    }
    const bool part = s.nparts != 1;
    if (!part && P.nproc3[0] * P.nproc3[1] * P.nproc3[2] != 1)
        throw SordError(SORD_E_PARAM, "a run split by nproc3 needs sord_create_part for each part");
    if (part) {
        // a run split along l (sord_create_part)
        if (P.nproc3[0] != 1 || P.nproc3[1] != 1 || P.nproc3[2] < 1)
            throw SordError(SORD_E_PARAM, "partitioned runs split l only: nproc3 must be [1, 1, P]");
        if (ifn) throw SordError(SORD_E_PARAM, "partitioned runs take no fault");
        if (P.gridnoise > 0.f) throw SordError(SORD_E_PARAM, "partitioned runs take no gridnoise (random per process)");
        for (const IoOp& io : s.ops)
            if (io.op.find('~') != std::string::npos)
                throw SordError(SORD_E_PARAM, "partitioned runs take no random ('~') field ops (random per process)");
    }
    for (int i = 0; i < 3; i++) {
        if (g.nn[i] < 1) throw SordError(SORD_E_PARAM, "Error in shape");
        g.nhalo[i] = 1;
    }
    if (ifn) g.nhalo[ifn - 1] = 2;
    for (int i = 0; i < 3; i++) {
        // setup.f90:33-38 and 48-50: planes per part and this part's offset
        int nl3 = std::max(g.nn[i], g.nhalo[i]), ip3 = 0;
        if (part && i == 2) {
            nl3 = std::max((g.nn[i] - 1) / P.nproc3[2] + 1, g.nhalo[i]);
            const int nproc = (g.nn[i] - 1) / nl3 + 1;
            if (s.part >= nproc)
                throw SordError(SORD_E_PARAM, "part " + std::to_string(s.part) + " beyond the " + std::to_string(nproc) +
                                                  " parts that nproc3 gives for " + std::to_string(g.nn[i]) + " planes");
            s.nparts = nproc;
            ip3 = s.part;
            // the PML of an l face, and one plane more, inside the first
            // or last part (the PML memories are kept per face)
            const int near = P.i1pml[2], far = P.i2pml[2], last0 = nl3 * (nproc - 1) + 1;
            if ((near >= 1 && nl3 < near + 1) || (far <= g.nn[2] && last0 > far - 1))
                throw SordError(SORD_E_PARAM, "partitioned runs need the PML of each l face and one plane more "
                                              "inside the first and last part (" + std::to_string(nl3) +
                                              " planes per part)");
        }
        g.nnoff[i] = nl3 * ip3 - g.nhalo[i];
        int nl = std::min(nl3, g.nn[i] - g.nnoff[i] - g.nhalo[i]);
        g.nm[i] = nl + 2 * g.nhalo[i];
        g.i1bc[i] = 1 - g.nnoff[i];
        g.i2bc[i] = g.nn[i] - g.nnoff[i];
        g.i1core[i] = 1 + g.nhalo[i];
        g.i2core[i] = g.nm[i] - g.nhalo[i];
        g.i1node[i] = std::max(g.i1bc[i], 2);
        g.i2node[i] = std::min(g.i2bc[i], g.nm[i] - 1);
        g.i1cell[i] = std::max(g.i1bc[i], 1);
        g.i2cell[i] = std::min(g.i2bc[i] - 1, g.nm[i] - 1);
        g.i1pml[i] = P.i1pml[i] - g.nnoff[i];
        g.i2pml[i] = P.i2pml[i] - g.nnoff[i];
    }
    g.irup = 0;
    if (ifn) {
        g.irup = (int)std::floor(P.hypocenter[ifn - 1] + 0.000001f) - g.nnoff[ifn - 1] + 1;
        if (g.irup + 1 < g.i1core[ifn - 1] || g.irup > g.i2core[ifn - 1]) ifn = 0;
    }
    g.ifn = ifn;
    g.npml = P.npml;
    g.sy = g.nm[0];
    g.sz = (long long)g.nm[0] * g.nm[1];
    g.nv = g.sz * g.nm[2];
    float prod = g.dx[0] * g.dx[1] * g.dx[2];
    g.h = prod >= 0.f ? 1.0f / 12.0f : -(1.0f / 12.0f);
}

static void allocate_arrays(Solver& s) {
    long long nv = s.g.nv;
    Device& d = s.d;
    // the volume fields: one zeroed block, each field at a 256-byte boundary
    float** const fields[29] = {&d.x[0], &d.x[1], &d.x[2], &d.v[0], &d.v[1], &d.v[2], &d.u[0], &d.u[1], &d.u[2],
                                &d.w1n[0], &d.w1n[1], &d.w1n[2], &d.sd[0], &d.sd[1], &d.sd[2], &d.so[0], &d.so[1],
                                &d.so[2], &d.vc, &d.mr, &d.lam, &d.mu, &d.gam, &d.yy, &d.s1, &d.s2,
                                &d.vb[0], &d.vb[1], &d.vb[2]};
    const size_t pitch = ((size_t)std::max(nv, 1LL) + 63) / 64 * 64;  // floats
    const size_t total = pitch * (29 + 3);                            // + ub[3]
    d.vol_plain = sizeof(float) * total >= ((size_t)4 << 30);
    cudaError_t e = d.vol_plain ? cudaMalloc(&d.vol, sizeof(float) * total) : dev_malloc(s, &d.vol, sizeof(float) * total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        d.vol = nullptr;
        throw SordError(SORD_E_NOMEM, std::string("device memory for the volume fields: ") + cudaGetErrorString(e));
    }
    SORD_CUDA(cudaMemsetAsync(d.vol, 0, sizeof(float) * total, s.stream));
    float* base = (float*)d.vol;
    for (int i = 0; i < 29; i++) *fields[i] = base + (size_t)i * pitch;
    for (int i = 0; i < 3; i++) d.ub[i] = base + (size_t)(29 + i) * pitch;
    alloc(s, &d.red, kRedFloats);
    const char* fz = getenv("SORD_FUSED");
    s.use_fused = !(fz && fz[0] == '0');
    const char* ar = getenv("SORD_ARITHMETIC");
    s.arith = (ar && std::strcmp(ar, "fast") == 0) ? 1 : 0;
    SORD_CUDA(dev_malloc(s, (void**)&d.inj, sizeof(Inject) * kInjectSlots * kInjectRing * kMaxInject));
    s.hinj = (Inject*)pinned_get(sizeof(Inject) * kInjectSlots * kInjectRing * kMaxInject);
}

static void init_grid(Solver& s) {
    Geom& g = s.g;
    Device& d = s.d;
    Params& P = s.prm;
    char fc = P.faultnormal.size() > 1 ? P.faultnormal[1] : ' ';
    int axis = fc == 'x' ? 0 : fc == 'y' ? 1 : fc == 'z' ? 2 : -1;
    // grid_generation.f90:28 uses i1 = max(i1core, irup + 1) with irup of setup
    int irup_raw = 0;
    if (axis >= 0) irup_raw = (int)std::floor(P.hypocenter[axis] + 0.000001f) - g.nnoff[axis] + 1;
    int from = axis >= 0 ? std::max(g.i1core[axis], irup_raw + 1) : 0;
    k_grid<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.x[0], d.x[1], d.x[2], axis, from);
    LAUNCH_CHECK(s);
    field_io(s, "<", "x", vol(s, d.x[0]));
    field_io(s, "<", "y", vol(s, d.x[1]));
    field_io(s, "<", "z", vol(s, d.x[2]));
    if (P.gridnoise > 0.f) {
        unsigned long long call = s.rng_calls++;
        float amp = std::sqrt(g.dx[0] * g.dx[0] + g.dx[1] * g.dx[1] + g.dx[2] * g.dx[2]) * P.gridnoise;
        int f1 = axis >= 0 ? std::max(g.i1core[axis], irup_raw) : 0;
        int f2 = axis >= 0 ? std::min(g.i2core[axis], irup_raw + 1) : -1;
        k_gridnoise<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.x[0], d.x[1], d.x[2], call, amp, axis, f1, f2);
        LAUNCH_CHECK(s);
    }
    if (P.rexpand > 1.0f) {
        for (int dd = 0; dd < 3; dd++) {
            int e1 = P.n1expand[dd] - g.nnoff[dd], e2 = g.nn[dd] - P.n2expand[dd] + 1 - g.nnoff[dd];
            for (int p = g.i1node[dd]; p <= std::min(g.i2node[dd], e1); p++) {
                int i = e1 - p;
                float sft = g.dx[dd] * ((float)(i + 1) - (powi_f(P.rexpand, i + 1) - 1.0f) / (P.rexpand - 1.0f));
                k_plane_add<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.x[dd], dd, p, sft);
                LAUNCH_CHECK(s);
            }
            for (int p = std::max(g.i1node[dd], e2); p <= g.i2node[dd]; p++) {
                int i = p - e2;
                float sft = g.dx[dd] * ((float)(i + 1) - (powi_f(P.rexpand, i + 1) - 1.0f) / (P.rexpand - 1.0f));
                k_plane_add<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.x[dd], dd, p, -sft);
                LAUNCH_CHECK(s);
            }
        }
    }
    const float* m = P.affine;
    k_affine<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.x[0], d.x[1], d.x[2], m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
    LAUNCH_CHECK(s);
    {
        int bc[3] = {4, 4, 4}, a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = g.i1bc[i] - 1; a2[i] = g.i2bc[i] + 1; }
        float* X[3] = {d.x[0], d.x[1], d.x[2]};
        launch_vector_bc(s, X, bc, bc, a1, a2);
        // a partitioned run takes the coordinates of its halo planes from
        // its neighbours (the volume and bracket stencils of its halo cells
        // read them)
        halo_exchange(s, X, 3);
    }
    field_io(s, ">", "x", vol(s, d.x[0]));
    field_io(s, ">", "y", vol(s, d.x[1]));
    field_io(s, ">", "z", vol(s, d.x[2]));
    const char* cn[3] = {"xc", "yc", "zc"};
    for (int c = 0; c < 3; c++)
        if (field_active(s, cn[c], '>')) {
            k_average<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.s1, d.x[c], g.i1cell[0], g.i2cell[0], g.i1cell[1], g.i2cell[1],
                                                        g.i1cell[2], g.i2cell[2], 1);
            LAUNCH_CHECK(s);
            field_io(s, ">", cn[c], vol(s, d.s1));
        }
    k_volume<<<gfor(g.nv), 256, 0, s.stream>>>(g, d.x[0], d.x[1], d.x[2], d.vc);
    LAUNCH_CHECK(s);
    int one[3] = {1, 1, 1};
    float mn = dev_reduce_min(s, vol(s, d.vc), one, g.nm);
    field_io(s, ">", "vc", vol(s, d.vc));
    if (mn < 0.f) throw SordError(SORD_E_NEGVOL, "Negative cell volume. Wrong sign in dx or problem with mesh.");
}

static void init_material(Solver& s) {
    Geom& g = s.g;
    Device& d = s.d;
    Params& P = s.prm;
    long long nv = g.nv;
    dev_fill(s, d.mr, nv, 0.f);
    dev_fill(s, d.lam, nv, 0.f);
    dev_fill(s, d.mu, nv, 0.f);
    dev_fill(s, d.gam, nv, 0.f);
    field_io(s, "<", "rho", vol(s, d.mr));
    field_io(s, "<", "vp", vol(s, d.lam));
    field_io(s, "<", "vs", vol(s, d.mu));
    field_io(s, "<", "gam", vol(s, d.gam));
    dev_copy(s, d.s1, d.lam, nv);
    dev_copy(s, d.s2, d.mu, nv);
    k_rlimits<<<gfor(nv), 256, 0, s.stream>>>(d.mr, nv, P.rho_min, P.rho_max); LAUNCH_CHECK(s);
    k_rlimits<<<gfor(nv), 256, 0, s.stream>>>(d.s1, nv, P.vp_min, P.vp_max); LAUNCH_CHECK(s);
    k_rlimits<<<gfor(nv), 256, 0, s.stream>>>(d.s2, nv, P.vs_min, P.vs_max); LAUNCH_CHECK(s);
    if (P.vdamp > 0.f) { k_vdamp<<<gfor(nv), 256, 0, s.stream>>>(d.gam, d.s2, nv, P.vdamp); LAUNCH_CHECK(s); }
    k_rlimits<<<gfor(nv), 256, 0, s.stream>>>(d.gam, nv, P.gam_min, P.gam_max); LAUNCH_CHECK(s);
    dev_set_halo(s, vol(s, d.mr), 0.f, g.i1cell, g.i2cell);
    dev_set_halo(s, vol(s, d.s1), 0.f, g.i1cell, g.i2cell);
    dev_set_halo(s, vol(s, d.s2), 0.f, g.i1cell, g.i2cell);
    dev_set_halo(s, vol(s, d.gam), 0.f, g.i1cell, g.i2cell);
    k_moduli<<<gfor(nv), 256, 0, s.stream>>>(nv, d.mr, d.s1, d.s2, d.lam, d.mu, d.yy); LAUNCH_CHECK(s);
    int a1[3], a2[3];
    for (int i = 0; i < 3; i++) { a1[i] = std::max(g.i1core[i], g.i1bc[i]); a2[i] = std::min(g.i2core[i], g.i2bc[i] - 1); }
    float* arrs[7] = {d.mr, d.s1, d.s2, d.gam, d.lam, d.mu, d.yy};
    float maxg[14];
    for (int q = 0; q < 7; q++) {
        maxg[q] = -dev_reduce_min(s, vol(s, arrs[q]), a1, a2);
        maxg[q + 7] = dev_reduce_max(s, vol(s, arrs[q]), a1, a2);
    }
    {
        // extrema over all parts of a partitioned run (material_model.f90:138)
        double mg[14];
        for (int q = 0; q < 14; q++) mg[q] = maxg[q];
        all_reduce(s, mg, 14, 0);
        for (int q = 0; q < 14; q++) maxg[q] = (float)mg[q];
    }
    field_io(s, ">", "rho", vol(s, d.mr));
    field_io(s, ">", "vp", vol(s, d.s1));
    field_io(s, ">", "vs", vol(s, d.s2));
    field_io(s, ">", "gam", vol(s, d.gam));
    field_io(s, ">", "lam", vol(s, d.lam));
    field_io(s, ">", "mu", vol(s, d.mu));
    field_io(s, ">", "nu", vol(s, d.yy));
    float sc = std::sqrt((g.dx[0] * g.dx[0] + g.dx[1] * g.dx[1] + g.dx[2] * g.dx[2]) / 3.0f) / 12.0f;
    k_hgconst<<<gfor(nv), 256, 0, s.stream>>>(nv, d.lam, d.mu, d.yy, sc); LAUNCH_CHECK(s);
    if (P.vpml <= 0.f) {
        float vmn = -maxg[2], vmx = maxg[8];
        P.vpml = 2.0f * vmn * vmx / (vmn + vmx);
    }
    float vmx = maxg[8];
    float r = g.dx[0] * g.dx[0] + g.dx[1] * g.dx[1] + g.dx[2] * g.dx[2];
    float cfl1 = g.dt * vmx * std::sqrt(3.0f / r);
    float cfl2 = g.dt * vmx * 3.0f / std::sqrt(r);
    FILE* fp = s.part == 0 ? fopen(s.path("material.json").c_str(), "w") : nullptr;
    if (fp) {
        fprintf(fp, "{\n");
        fprintf(fp, "    \"cfl\": [%.9g, %.9g],\n", (double)cfl1, (double)cfl2);
        const char* nm_[7] = {"rho", "vp", "vs", "gam", "lam", "mu", "nu"};
        for (int q = 0; q < 7; q++)
            fprintf(fp, "    \"%s\": [%.9g, %.9g]%s\n", nm_[q], (double)-maxg[q], (double)maxg[q + 7], q < 6 ? "," : "");
        fprintf(fp, "}\n");
        fclose(fp);
    }
    for (int q = 0; q < 7; q++)
        if (maxg[q] > 0.f) throw SordError(SORD_E_CFL, "negative moduli");
    if (cfl2 > 1.0f) throw SordError(SORD_E_CFL, "Courant condition not satisfied!");
}

static void init_pml(Solver& s) {
    Geom& g = s.g;
    Params& P = s.prm;
    int np = P.npml;
    if (np < 1) {
        for (int i = 0; i < 6; i++) {
            s.d.slabs.p[i] = s.d.slabs.g[i] = s.d.gb[i] = nullptr;
            s.d.slabs.tp[i] = s.d.slabs.tg[i] = 0;
        }
        alloc(s, &s.d.pmlc, 4);
        return;
    }
    s.dn1.assign(np, 0.f); s.dn2.assign(np, 0.f); s.dc1.assign(np, 0.f); s.dc2.assign(np, 0.f);
    float c1 = 8.0f / 15.0f, c2 = -3.0f / 100.0f, c3 = 1.0f / 1500.0f, tune = 3.5f;
    float r = g.dx[0] * g.dx[0] + g.dx[1] * g.dx[1] + g.dx[2] * g.dx[2];
    float damp = tune * P.vpml / std::sqrt(r / 3.0f) * (c1 + (c2 + c3 * (float)np) * (float)np) / (float)ipow_l(np, P.ppml);
    for (int i = 1; i <= np; i++) {
        float dampn = damp * (float)ipow_l(i, P.ppml);
        float dampc = damp * (float)(ipow_l(i, P.ppml) + ipow_l(i - 1, P.ppml)) * 0.5f;
        int p = np - i;
        s.dn1[p] = -(2.0f * dampn) / (2.0f + g.dt * dampn);
        s.dc1[p] = (2.0f - g.dt * dampc) / (2.0f + g.dt * dampc);
        s.dn2[p] = 2.0f / (2.0f + g.dt * dampn);
        s.dc2[p] = 2.0f * g.dt / (2.0f + g.dt * dampc);
    }
    std::vector<float> h(4 * np);
    for (int i = 0; i < np; i++) { h[i] = s.dn1[i]; h[np + i] = s.dn2[i]; h[2 * np + i] = s.dc1[i]; h[3 * np + i] = s.dc2[i]; }
    alloc(s, &s.d.pmlc, 4 * np);
    SORD_CUDA(cudaMemcpyAsync(s.d.pmlc, h.data(), sizeof(float) * 4 * np, cudaMemcpyHostToDevice, s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    Slabs& sl = s.d.slabs;
    for (int a = 0; a < 3; a++) {
        int tpn = std::min(g.i2node[a], g.i1pml[a]) - g.i1node[a] + 1;
        int tpf = g.i2node[a] - std::max(g.i1node[a], g.i2pml[a]) + 1;
        int tgn = std::min(g.i2cell[a], g.i1pml[a]) - g.i1cell[a] + 1;
        int tgf = g.i2cell[a] - std::max(g.i1cell[a], g.i2pml[a] - 1) + 1;
        sl.tp[a] = std::max(tpn, 0); sl.tp[3 + a] = std::max(tpf, 0);
        sl.tg[a] = std::max(tgn, 0); sl.tg[3 + a] = std::max(tgf, 0);
        long long other = g.nv / g.nm[a];
        for (int side = 0; side < 2; side++) {
            int sidx = side * 3 + a;
            alloc(s, &sl.p[sidx], other * sl.tp[sidx] * 3);
            alloc(s, &sl.g[sidx], other * sl.tg[sidx] * 3);
            alloc(s, &s.d.gb[sidx], other * sl.tg[sidx] * 3);
        }
    }
}

static void read_floats(Solver& s, const std::string& fn, std::vector<float>& v, int n) {
    v.assign(n, 0.f);
    FILE* fp = fopen(s.path(fn).c_str(), "rb");
    if (!fp) throw SordError(SORD_E_IO, "cannot open " + fn);
    size_t got = fread(v.data(), sizeof(float), n, fp);
    fclose(fp);
    if (got != (size_t)n) throw SordError(SORD_E_IO, "short read " + fn);
}

// kinematic_source.f90:10-63 (host: the source list drives per-step injections)
static void init_finite_source(Solver& s) {
    Params& P = s.prm;
    Geom& g = s.g;
    if (P.nsource == 0) return;
    int n = std::abs(P.nsource);
    read_floats(s, "source-xi1.bin", s.src_xi[0], n);
    read_floats(s, "source-xi2.bin", s.src_xi[1], n);
    read_floats(s, "source-xi3.bin", s.src_xi[2], n);
    bool force = P.source == "force";
    for (int i = 0; i < 3; i++) {
        bool lo = true, hi = true;
        for (auto& x : s.src_xi[i]) {
            x = force ? x - (float)g.nnoff[i] : x - 0.5f - (float)g.nnoff[i];
            int a = force ? g.i1node[i] : g.i1cell[i], b = force ? g.i2node[i] : g.i2cell[i];
            lo = lo && x < (float)(-1 + a);
            hi = hi && x > (float)(1 + b);
        }
        if (lo || hi) { P.nsource = 0; return; }
    }
    if (force) {
        read_floats(s, "source-w11.bin", s.src_w1[0], n);
        read_floats(s, "source-w12.bin", s.src_w1[1], n);
        read_floats(s, "source-w13.bin", s.src_w1[2], n);
    } else {
        read_floats(s, "source-w11.bin", s.src_w1[0], n);
        read_floats(s, "source-w22.bin", s.src_w1[1], n);
        read_floats(s, "source-w33.bin", s.src_w1[2], n);
        read_floats(s, "source-w23.bin", s.src_w2[0], n);
        read_floats(s, "source-w31.bin", s.src_w2[1], n);
        read_floats(s, "source-w12.bin", s.src_w2[2], n);
    }
    read_floats(s, "source-t0.bin", s.src_t0, n);
    read_floats(s, "source-dt.bin", s.src_dt, n);
    {
        s.src_nt.assign(n, 0);
        FILE* fp = fopen(s.path("source-nt.bin").c_str(), "rb");
        if (!fp) throw SordError(SORD_E_IO, "cannot open source-nt.bin");
        size_t got = fread(s.src_nt.data(), sizeof(int), n, fp);
        fclose(fp);
        if (got != (size_t)n) throw SordError(SORD_E_IO, "short read source-nt.bin");
    }
    long tot = 0;
    for (int v : s.src_nt) tot += v;
    if (tot) read_floats(s, "source-history.bin", s.src_history, (int)tot);
}

static void resample_material(Solver& s) {
    Geom& g = s.g;
    Device& d = s.d;
    Params& P = s.prm;
    long long nv = g.nv;
    k_mul<<<gfor(nv), 256, 0, s.stream>>>(d.s2, d.mr, d.vc, nv); LAUNCH_CHECK(s);
    k_average<<<gfor(nv), 256, 0, s.stream>>>(g, d.mr, d.s2, g.i1node[0], g.i2node[0], g.i1node[1], g.i2node[1], g.i1node[2],
                                              g.i2node[2], -1);
    LAUNCH_CHECK(s);
    dev_rinvert(s, d.mr, nv);
    launch_scalar_bc(s, d.mr, g.nm, P.bc1, P.bc2, g.i1bc, g.i2bc);
    halo_exchange(s, &d.mr, 1);  // material_resample.f90:20
    dev_rinvert(s, d.vc, nv);
    {
        int bc[3] = {4, 4, 4}, a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = g.i1bc[i] - 1; a2[i] = g.i2bc[i]; }
        launch_scalar_bc(s, d.gam, g.nm, bc, bc, a1, a2);
    }
    k_scale<<<gfor(nv), 256, 0, s.stream>>>(d.s2, d.gam, g.dt, nv); LAUNCH_CHECK(s);
    k_average<<<gfor(nv), 256, 0, s.stream>>>(g, d.gam, d.s2, g.i1node[0], g.i2node[0], g.i1node[1], g.i2node[1], g.i1node[2],
                                              g.i2node[2], -1);
    LAUNCH_CHECK(s);
    dev_set_halo(s, vol(s, d.gam), 0.f, g.i1bc, g.i2bc);
    launch_scalar_bc(s, d.gam, g.nm, P.bc1, P.bc2, g.i1bc, g.i2bc);
    halo_exchange(s, &d.gam, 1);  // material_resample.f90:34
    {
        int a2[3];
        for (int i = 0; i < 3; i++) a2[i] = g.i2bc[i] - 1;
        dev_set_halo(s, vol(s, d.yy), 0.f, g.i1bc, a2);
    }
    if (g.ifn) { k_zero_plane<<<gfor(nv), 256, 0, s.stream>>>(g, d.yy, g.ifn - 1, g.irup); LAUNCH_CHECK(s); }
    for (int i = 0; i < 3; i++) {
        dev_fill(s, d.v[i], nv, 0.f); dev_fill(s, d.u[i], nv, 0.f); dev_fill(s, d.w1n[i], nv, 0.f);
        dev_fill(s, d.sd[i], nv, 0.f); dev_fill(s, d.so[i], nv, 0.f);
    }
    dev_fill(s, d.s1, nv, 0.f);
    dev_fill(s, d.s2, nv, 0.f);
}

// Mesh class of the step kernels: rectilinear (every real cell's brackets
// equal the reference cell's, bit for bit), terrain (x = x(j), y = y(k) and
// the z-free direction's brackets constant) or general.
static void rect_check(Solver& s) {
    Geom& g = s.g;
    s.rect = false;
    s.geom = GEOM_GENERAL;
    int jc[3], jn[3];
    for (int a = 0; a < 3; a++) {
        if (g.i2cell[a] - g.i1cell[a] < 2) return;  // too small to have interior references
        jc[a] = g.i1cell[a];
        jn[a] = g.i1node[a] + 1;
        if (g.ifn == a + 1) {
            while (jc[a] == g.irup) jc[a]++;
            while (jn[a] - 1 == g.irup || jn[a] == g.irup) jn[a]++;
            if (jc[a] > g.i2cell[a] || jn[a] > g.i2node[a] - 1) return;
        }
    }
    float* ref = (float*)s.d.red + kRedRef;
    k_ref_brackets<<<1, 1, 0, s.stream>>>(g, s.d.x[0], s.d.x[1], s.d.x[2], jc[0], jc[1], jc[2], jn[0], jn[1], jn[2], ref);
    LAUNCH_CHECK(s);
    unsigned* bad = (unsigned*)s.d.red + kRedBad;
    SORD_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), s.stream));
    k_rect_check<<<gfor(g.nv), 256, 0, s.stream>>>(g, s.d.x[0], s.d.x[1], s.d.x[2], ref, bad);
    LAUNCH_CHECK(s);
    unsigned hb = 0;
    float hr[48];
    SORD_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s.stream));
    SORD_CUDA(cudaMemcpyAsync(hr, ref, sizeof(float) * 48, cudaMemcpyDeviceToHost, s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    for (int a = 0; a < 3; a++)
        for (int t = 0; t < 8; t++) { s.br.bnc[a][t] = hr[8 * a + t]; s.br.bcn[a][t] = hr[24 + 8 * a + t]; }
    if (hb == 0) {
        s.rect = true;
        s.geom = GEOM_RECT;
        return;
    }
    if ((hb & (4u | 32u)) == 0) {
        // direction 3 (x-y brackets) constant: test x = x(j), y = y(k)
        alloc(s, &s.d.x1d, g.nm[0]);
        alloc(s, &s.d.y1d, g.nm[1]);
        k_line<<<div_up(g.nm[0], 128), 128, 0, s.stream>>>(s.d.x[0], s.d.x1d, g.nm[0], 1, g.idx(1, g.i1core[1], g.i1core[2]));
        LAUNCH_CHECK(s);
        k_line<<<div_up(g.nm[1], 128), 128, 0, s.stream>>>(s.d.x[1], s.d.y1d, g.nm[1], g.sy, g.idx(g.i1core[0], 1, g.i1core[2]));
        LAUNCH_CHECK(s);
        SORD_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), s.stream));
        k_terrain_check<<<gfor(g.nv), 256, 0, s.stream>>>(g, s.d.x[0], s.d.x[1], s.d.x1d, s.d.y1d, bad);
        LAUNCH_CHECK(s);
        SORD_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
        if (hb == 0) s.geom = GEOM_TERRAIN;
    }
}

void fault_init(Solver& s);

void setup_all(Solver& s) {
    // SORD_SETUP_TIMES=1: wait for the device after each phase and print the
    // phases' wall times (ms) to stderr, for finding where setup goes
    const char* env = getenv("SORD_SETUP_TIMES");
    const bool timed = env && env[0] == '1';
    static const char* names[9] = {"dimensions", "allocate", "grid", "material", "pml", "finite_source", "fault",
                                   "resample", "mesh_class"};
    void (*phase[9])(Solver&) = {setup_dimensions, allocate_arrays, init_grid, init_material, init_pml,
                                 init_finite_source, fault_init, resample_material, rect_check};
    double ms[9];
    for (int i = 0; i < 9; i++) {
        const long long t0 = s.clock_us();
        phase[i](s);
        if (timed) SORD_CUDA(cudaStreamSynchronize(s.stream));
        ms[i] = 1e-3 * (double)(s.clock_us() - t0);
    }
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    if (timed) {
        fprintf(stderr, "{\"setup_ms\": {");
        for (int i = 0; i < 9; i++) fprintf(stderr, "%s\"%s\": %.3f", i ? ", " : "", names[i], ms[i]);
        fprintf(stderr, "}}\n");
    }
}

}  // namespace sordgpu

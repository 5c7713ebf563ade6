// Double-node fault: initialisation (dynamic_rupture.f90:7-238,
// surf_normals.f90:53-128), slip bookkeeping of step_time
// (time_integration.f90:15-23, 67-113) and the rupture step
// (dynamic_rupture.f90:243-384).  One thread per fault-plane node; the
// plane arrays have the block's extents with 1 along the fault normal.
// Energy and moment sums are accumulated in FP64 in a fixed order.
#include <cmath>
#include <cstdio>

#include "sord.cuh"

namespace sordgpu {

#define LCHK(s) do { (s).launches++; SORD_CUDA(cudaGetLastError()); } while (0)

struct Plane {
    int n[3];       // plane extents (1 along the normal)
    int ax;         // normal axis 0..2
    int irup;       // minus side index (local, 1-based)
    long long np;
    long long off;  // volume index step from the minus to the plus side
};

__device__ __forceinline__ void plane_pos(const Plane& P, long long q, int p[3]) {
    p[0] = (int)(q % P.n[0]) + 1;
    p[1] = (int)((q / P.n[0]) % P.n[1]) + 1;
    p[2] = (int)(q / ((long long)P.n[0] * P.n[1])) + 1;
}
__device__ __forceinline__ long long vol_minus(const Geom& g, const Plane& P, const int p[3]) {
    int c[3] = {p[0], p[1], p[2]};
    c[P.ax] = P.irup;
    return g.idx(c[0], c[1], c[2]);
}
__device__ __forceinline__ bool plane_core(const Geom& g, const Plane& P, const int p[3]) {
    for (int d = 0; d < 3; d++)
        if (P.n[d] > 1 && (p[d] < g.i1core[d] || p[d] > g.i2core[d])) return false;
    return true;
}
__device__ __forceinline__ float fmin_(float a, float b) { return b < a ? b : a; }  // std::min(a, b)
__device__ __forceinline__ float fmax_(float a, float b) { return a < b ? b : a; }  // std::max(a, b)

#define FA(a) (F + (long long)(a) * P.np)

// node_normals (surf_normals.f90:53-128) on the fault plane from node coordinates
__global__ void k_normals(Geom g, Plane P, const float* x0, const float* x1, const float* x2, float* F) {
    const float* X[3] = {x0, x1, x2};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        bool in = plane_core(g, P, p);
        for (int a = 0; a < 3; a++) {
            float r = 0.f;
            if (in) {
                const float* B = X[(a + 1) % 3];
                const float* C = X[(a + 2) % 3];
                long long c0 = vol_minus(g, P, p);
                // the three cases of surf_normals.f90 use the cyclic in-plane pair
                int ua = (P.ax + 1) % 3, wa = (P.ax + 2) % 3;
                long long su = ua == 0 ? 1 : ua == 1 ? g.sy : g.sz;
                long long sw = wa == 0 ? 1 : wa == 1 ? g.sy : g.sz;
#define XB(du, dw) B[c0 + (du) * su + (dw) * sw]
#define XC(du, dw) C[c0 + (du) * su + (dw) * sw]
                r = g.h * (XB(1, 0) * (XC(0, 1) + XC(1, 1) - XC(0, -1) - XC(1, -1)) +
                           XB(-1, 0) * (XC(0, -1) + XC(-1, -1) - XC(0, 1) - XC(-1, 1)) +
                           XB(0, 1) * (XC(-1, 0) + XC(-1, 1) - XC(1, 0) - XC(1, 1)) +
                           XB(0, -1) * (XC(1, 0) + XC(1, -1) - XC(-1, 0) - XC(-1, -1)) +
                           XB(1, 1) * (XC(0, 1) - XC(1, 0)) + XB(-1, -1) * (XC(0, -1) - XC(-1, 0)) +
                           XB(-1, 1) * (XC(-1, 0) - XC(0, 1)) + XB(1, -1) * (XC(1, 0) - XC(0, -1)));
#undef XB
#undef XC
            }
            FA(F_NHAT + a)[q] = r;
        }
    }
}

// area, unit normal (dynamic_rupture.f90:121-130)
__global__ void k_fault_area(Plane P, float* F, float sgn) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        float n1 = FA(F_NHAT)[q], n2 = FA(F_NHAT + 1)[q], n3 = FA(F_NHAT + 2)[q];
        float s = sqrtf(n1 * n1 + n2 * n2 + n3 * n3);
        float a = sgn > 0.f ? s : -s;
        FA(F_AREA)[q] = a;
        float f = a != 0.f ? 1.0f / a : a;
        FA(F_F1)[q] = f;
        FA(F_NHAT)[q] = n1 * f; FA(F_NHAT + 1)[q] = n2 * f; FA(F_NHAT + 2)[q] = n3 * f;
    }
}

// resolved pre-traction (dynamic_rupture.f90:137-173)
__global__ void k_fault_t0(Plane P, float* F, float sv0, float sv1, float sv2) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        float n[3] = {FA(F_NHAT)[q], FA(F_NHAT + 1)[q], FA(F_NHAT + 2)[q]};
        float t1[3] = {FA(F_T1)[q], FA(F_T1 + 1)[q], FA(F_T1 + 2)[q]};
        float t2[3] = {FA(F_T2)[q], FA(F_T2 + 1)[q], FA(F_T2 + 2)[q]};
        float t3[3] = {FA(F_T3)[q], FA(F_T3 + 1)[q], FA(F_T3 + 2)[q]};
        float t0[3];
        for (int i = 0; i < 3; i++) {
            int j = (i + 1) % 3, k = (i + 2) % 3;
            t0[i] = t1[i] * n[i] + t2[j] * n[k] + t2[k] * n[j];
        }
        float a[3] = {n[1] * sv2 - n[2] * sv1, n[2] * sv0 - n[0] * sv2, n[0] * sv1 - n[1] * sv0};
        float f = sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (f != 0.f) f = 1.0f / f;
        for (int i = 0; i < 3; i++) a[i] = a[i] * f;
        float b[3] = {a[1] * n[2] - a[2] * n[1], a[2] * n[0] - a[0] * n[2], a[0] * n[1] - a[1] * n[0]};
        f = sqrtf(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        if (f != 0.f) f = 1.0f / f;
        for (int i = 0; i < 3; i++) b[i] = b[i] * f;
        for (int i = 0; i < 3; i++) t0[i] = t0[i] + t3[0] * b[i] + t3[1] * a[i] + t3[2] * n[i];
        for (int i = 0; i < 3; i++) {
            FA(F_T0 + i)[q] = t0[i];
            FA(F_T2 + i)[q] = a[i];
            FA(F_T1 + i)[q] = b[i];
        }
        FA(F_F1)[q] = f;
    }
}

// hypocentral radius from node coordinates (dynamic_rupture.f90:176-203)
__global__ void k_rhypo(Geom g, Plane P, const float* x0, const float* x1, const float* x2, float* F, float h0, float h1, float h2) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        long long c = vol_minus(g, P, p);
        float a = x0[c] - h0, b = x1[c] - h1, d = x2[c] - h2;
        FA(F_T2)[q] = a; FA(F_T2 + 1)[q] = b; FA(F_T2 + 2)[q] = d;
        FA(F_RHYPO)[q] = sqrtf(a * a + b * b + d * d);
    }
}

// lamf, muf: moduli at the fault plane, inverted (dynamic_rupture.f90:206-212)
__global__ void k_fault_moduli(Geom g, Plane P, const float* lam, const float* mu, float* F) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        long long c = vol_minus(g, P, p);
        float a = lam[c], b = mu[c];
        FA(F_LAMF)[q] = a != 0.f ? 1.0f / a : a;
        FA(F_MUF)[q] = b != 0.f ? 1.0f / b : b;
    }
}
// dst(2:n-1) = 0.5 * (src(2:n-1) + src(1:n-2)) along plane axis d (dynamic_rupture.f90:216-221)
__global__ void k_plane_avg(Plane P, float* dst, const float* src, int d, int last) {
    long long st = d == 0 ? 1 : d == 1 ? P.n[0] : (long long)P.n[0] * P.n[1];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        if (p[d] >= 2 && p[d] <= last) dst[q] = 0.5f * (src[q] + src[q - st]);
        else dst[q] = src[q];
    }
}
__global__ void k_pcopy(float* d, const float* s, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) d[q] = s[q];
}
__global__ void k_pinv(float* d, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        float v = d[q];
        if (v != 0.f) d[q] = 1.0f / v;
    }
}
__global__ void k_pfill(float* d, long long n, float v) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) d[q] = v;
}

// ------------------------------------------------------------ step_time
// previous slip rate: t2 = v+ - v-, f2 = |t2| (time_integration.f90:15-23)
__global__ void k_fault_pre(Geom g, Plane P, const float* v0, const float* v1, const float* v2, float* F) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        long long c = vol_minus(g, P, p), c2 = c + P.off;
        float a = v0[c2] - v0[c], b = v1[c2] - v1[c], d = v2[c2] - v2[c];
        FA(F_T2)[q] = a; FA(F_T2 + 1)[q] = b; FA(F_T2 + 2)[q] = d;
        FA(F_F2)[q] = sqrtf(a * a + b * b + d * d);
    }
}

// slip rate, path length, peak rate, rupture / arrest time, slip
// (time_integration.f90:67-93)
__global__ void k_fault_post(Geom g, Plane P, const float* v0, const float* v1, const float* v2, const float* u0,
                             const float* u1, const float* u2, float* F, float tm, float dt, float svtol) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        long long c = vol_minus(g, P, p), c2 = c + P.off;
        float a = v0[c2] - v0[c], b = v1[c2] - v1[c], d = v2[c2] - v2[c];
        FA(F_T1)[q] = a; FA(F_T1 + 1)[q] = b; FA(F_T1 + 2)[q] = d;
        float f1 = sqrtf(a * a + b * b + d * d);
        FA(F_F1)[q] = f1;
        FA(F_SL)[q] = FA(F_SL)[q] + dt * f1;
        FA(F_PSV)[q] = fmax_(FA(F_PSV)[q], f1);
        if (svtol > 0.f) {
            float f2 = FA(F_F2)[q];
            if (f1 >= svtol && FA(F_TRUP)[q] > 1e8f) FA(F_TRUP)[q] = tm - dt * (0.5f + (svtol - f1) / (f2 - f1));
            if (f1 >= svtol) FA(F_TARR)[q] = 1e9f;
            if (f1 < svtol && f2 >= svtol) FA(F_TARR)[q] = tm - dt * (0.5f + (svtol - f1) / (f2 - f1));
        }
        a = u0[c2] - u0[c]; b = u1[c2] - u1[c]; d = u2[c2] - u2[c];
        FA(F_T2)[q] = a; FA(F_T2 + 1)[q] = b; FA(F_T2 + 2)[q] = d;
        FA(F_F2)[q] = sqrtf(a * a + b * b + d * d);
    }
}

// ------------------------------------------------------------ rupture
struct RuptArgs {
    Geom g;
    Plane P;
    const float *v[3], *u[3], *mr;
    float* w[3];
    float* F;
    float dt, tm, rcrit, vrup, trelax;
    int it, faultopening;
};

// trial traction, slip-weakening friction, nucleation, force update
// (dynamic_rupture.f90:268-334) at fault node q (volume nodes c1, c2);
// returns the new traction t1
__device__ __forceinline__ void rupture_node(const RuptArgs& A, long long q, long long c1, long long c2, float (&t1)[3]) {
    const Plane& P = A.P;
    float* F = A.F;
    {
        const float dt = A.dt;
        float m1 = A.mr[c1], m2 = A.mr[c2];
        float area = FA(F_AREA)[q];
        float f1 = dt * dt * area * (m1 + m2);
        if (f1 != 0.f) f1 = 1.0f / f1;
        float n[3] = {FA(F_NHAT)[q], FA(F_NHAT + 1)[q], FA(F_NHAT + 2)[q]};
        float t0[3], t2[3], t3[3];
        for (int i = 0; i < 3; i++) {
            t0[i] = FA(F_T0 + i)[q];
            t1[i] = t0[i] + f1 * dt * (A.v[i][c2] - A.v[i][c1] + A.w[i][c2] * m2 * dt - A.w[i][c1] * m1 * dt);
            t2[i] = t1[i] + f1 * (A.u[i][c2] - A.u[i][c1]);
        }
        float tn = t1[0] * n[0] + t1[1] * n[1] + t1[2] * n[2];
        for (int i = 0; i < 3; i++) t3[i] = t1[i] - tn * n[i];
        float ts = sqrtf(t3[0] * t3[0] + t3[1] * t3[1] + t3[2] * t3[2]);
        float f2 = FA(F_F2)[q];
        if (A.it > 1) {
            tn = t2[0] * n[0] + t2[1] * n[1] + t2[2] * n[2];
            if (A.faultopening == 1) tn = fmin_(0.f, tn);
            for (int i = 0; i < 3; i++) t2[i] = A.v[i][c2] - A.v[i][c1];
            f2 = t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2];
            float mud = FA(F_MUD)[q], sl = FA(F_SL)[q], dcv = FA(F_DC)[q];
            f1 = mud;
            if (sl < dcv) f1 = f1 + (1.0f - sl / dcv) * (FA(F_MUS)[q] - mud);
            f1 = -fmin_(0.f, tn) * f1 + FA(F_CO)[q];
            if (A.rcrit > 0.f && A.vrup > 0.f) {
                float rh = FA(F_RHYPO)[q];
                float g2 = 1.0f;
                if (A.trelax > 0.f) g2 = fmin_((A.tm - rh / A.vrup) / A.trelax, 1.0f);
                g2 = (1.0f - g2) * ts + g2 * (-tn * mud + FA(F_CO)[q]);
                f2 = g2;
                if (rh < fmin_(A.rcrit, A.tm * A.vrup) && f2 < f1) f1 = f2;
            }
            f2 = 1.0f;
            if (ts > f1) f2 = f1 / ts;
            for (int i = 0; i < 3; i++) t3[i] = f2 * t3[i];
            ts = fmin_(ts, f1);
            for (int i = 0; i < 3; i++) t1[i] = t3[i] + tn * n[i];
        }
        for (int i = 0; i < 3; i++) {
            float g = area * (t1[i] - t0[i]);
            f2 = g;
            A.w[i][c1] = A.w[i][c1] + g;
            A.w[i][c2] = A.w[i][c2] - g;
        }
        for (int i = 0; i < 3; i++) { FA(F_T1 + i)[q] = t1[i]; FA(F_T2 + i)[q] = t2[i]; FA(F_T3 + i)[q] = t3[i]; }
        FA(F_TN)[q] = tn;
        FA(F_TS)[q] = ts;
        FA(F_F1)[q] = f1;
        FA(F_F2)[q] = f2;
    }
}
__global__ void k_rupture(RuptArgs A) {
    const Plane& P = A.P;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        const long long c1 = vol_minus(A.g, P, p), c2 = c1 + P.off;
        float t1[3];
        rupture_node(A, q, c1, c2, t1);
    }
}

// energies and moment per node (dynamic_rupture.f90:354-368) into FP64 block partials
__global__ void k_fault_energy(Geom g, Plane P, const float* v0, const float* v1, const float* v2, const float* u0,
                               const float* u1, const float* u2, const float* F, double* part) {
    double e0 = 0, e1 = 0, e2 = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        if (!plane_core(g, P, p)) continue;
        long long c = vol_minus(g, P, p), c2 = c + P.off;
        float area = FA(F_AREA)[q];
        float t1[3] = {FA(F_T1)[q], FA(F_T1 + 1)[q], FA(F_T1 + 2)[q]};
        float t0[3] = {FA(F_T0)[q], FA(F_T0 + 1)[q], FA(F_T0 + 2)[q]};
        float dv[3] = {v0[c2] - v0[c], v1[c2] - v1[c], v2[c2] - v2[c]};
        float du[3] = {u0[c2] - u0[c], u1[c2] - u1[c], u2[c2] - u2[c]};
        e0 += (double)((t1[0] * dv[0] + t1[1] * dv[1] + t1[2] * dv[2]) * area);
        e1 += (double)(((t0[0] + t1[0]) * du[0] + (t0[1] + t1[1]) * du[1] + (t0[2] + t1[2]) * du[2]) * area);
        e2 += (double)(FA(F_MUF)[q] * area * sqrtf(du[0] * du[0] + du[1] * du[1] + du[2] * du[2]));
    }
    __shared__ double s[3][256];
    s[0][threadIdx.x] = e0; s[1][threadIdx.x] = e1; s[2][threadIdx.x] = e2;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k)
            for (int i = 0; i < 3; i++) s[i][threadIdx.x] += s[i][threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int i = 0; i < 3; i++) part[3 * blockIdx.x + i] = s[i][0];
}
// sum partials in block order: efric += dt*sum, estrain = 0.5*sum, moment = sum
__global__ void k_fault_energy_fin(const double* part, int nb, double* acc, double dt) {
    if (threadIdx.x || blockIdx.x) return;
    double a = 0, b = 0, c = 0;
    for (int i = 0; i < nb; i++) { a += part[3 * i]; b += part[3 * i + 1]; c += part[3 * i + 2]; }
    acc[0] = acc[0] + dt * a;
    acc[1] = 0.5 * b;
    acc[2] = c;
}

// slip acceleration (dynamic_rupture.f90:371-376)
__global__ void k_slip_accel(Geom g, Plane P, const float* w0, const float* w1, const float* w2, const float* mr, float* F) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        long long c = vol_minus(g, P, p), c2 = c + P.off;
        float m1 = mr[c], m2 = mr[c2];
        float a = w0[c2] * m2 - w0[c] * m1, b = w1[c2] * m2 - w1[c] * m1, d = w2[c2] * m2 - w2[c] * m1;
        FA(F_T2)[q] = a; FA(F_T2 + 1)[q] = b; FA(F_T2 + 2)[q] = d;
        FA(F_F2)[q] = sqrtf(a * a + b * b + d * d);
    }
}

// ------------------------------------------------------------ fused step
// With the fused volume kernel, the two fault planes are finished here: the
// volume kernel leaves their force in w and their v, u unchanged.

__device__ __forceinline__ bool node_box(const Geom& g, long long c) {
    const int j = (int)(c % g.sy) + 1, k = (int)((c / g.sy) % g.nm[1]) + 1, l = (int)(c / g.sz) + 1;
    return j >= g.i1node[0] && j <= g.i2node[0] && k >= g.i1node[1] && k <= g.i2node[1] && l >= g.i1node[2] &&
           l <= g.i2node[2];
}
__device__ __forceinline__ bool node_core(const Geom& g, long long c) {
    const int j = (int)(c % g.sy) + 1, k = (int)((c / g.sy) % g.nm[1]) + 1, l = (int)(c / g.sz) + 1;
    return j >= g.i1core[0] && j <= g.i2core[0] && k >= g.i1core[1] && k <= g.i2core[1] && l >= g.i1core[2] &&
           l <= g.i2core[2];
}
__device__ __forceinline__ void block_max3(unsigned* dst, float v) {
    unsigned b = __float_as_uint(v);
    if (v != v) b = 0x7fc00000u;
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    __shared__ unsigned s[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) s[warp] = b;
    __syncthreads();
    if (warp == 0) {
        b = lane < nw ? s[lane] : 0u;
        for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
        if (lane == 0 && b) atomicMax(dst, b);
    }
}

// Rupture of step n after the fused volume kernel: trial traction and
// friction (rupture_node), the energy and moment partials of k_fault_energy,
// the slip acceleration of k_slip_accel and the mass division of both fault
// nodes (acceleration.f90:235-238) with their share of max |a|.
__global__ void k_rupture_fused(RuptArgs A, double* part, int stats, unsigned* red) {
    const Plane& P = A.P;
    const Geom& g = A.g;
    float* F = A.F;
    double e0 = 0, e1 = 0, e2 = 0;
    float am = 0.f;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        const long long c1 = vol_minus(g, P, p), c2 = c1 + P.off;
        float t1[3];
        rupture_node(A, q, c1, c2, t1);
        if (plane_core(g, P, p)) {
            const float area = FA(F_AREA)[q];
            const float t0[3] = {FA(F_T0)[q], FA(F_T0 + 1)[q], FA(F_T0 + 2)[q]};
            const float dv[3] = {A.v[0][c2] - A.v[0][c1], A.v[1][c2] - A.v[1][c1], A.v[2][c2] - A.v[2][c1]};
            const float du[3] = {A.u[0][c2] - A.u[0][c1], A.u[1][c2] - A.u[1][c1], A.u[2][c2] - A.u[2][c1]};
            e0 += (double)((t1[0] * dv[0] + t1[1] * dv[1] + t1[2] * dv[2]) * area);
            e1 += (double)(((t0[0] + t1[0]) * du[0] + (t0[1] + t1[1]) * du[1] + (t0[2] + t1[2]) * du[2]) * area);
            e2 += (double)(FA(F_MUF)[q] * area * sqrtf(du[0] * du[0] + du[1] * du[1] + du[2] * du[2]));
        }
        const float m1 = A.mr[c1], m2 = A.mr[c2];
        float a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = A.w[i][c1] * m1; a2[i] = A.w[i][c2] * m2; }
        const float sa = a2[0] - a1[0], sb = a2[1] - a1[1], sd = a2[2] - a1[2];
        FA(F_T2)[q] = sa; FA(F_T2 + 1)[q] = sb; FA(F_T2 + 2)[q] = sd;
        FA(F_F2)[q] = sqrtf(sa * sa + sb * sb + sd * sd);
        if (node_box(g, c1)) {
            for (int i = 0; i < 3; i++) A.w[i][c1] = a1[i];
            if (stats && node_core(g, c1)) {
                const float n = a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2];
                am = (n != n || n > am) ? n : am;
            }
        }
        if (node_box(g, c2)) {
            for (int i = 0; i < 3; i++) A.w[i][c2] = a2[i];
            if (stats && node_core(g, c2)) {
                const float n = a2[0] * a2[0] + a2[1] * a2[1] + a2[2] * a2[2];
                am = (n != n || n > am) ? n : am;
            }
        }
    }
    __shared__ double s[3][256];
    s[0][threadIdx.x] = e0; s[1][threadIdx.x] = e1; s[2][threadIdx.x] = e2;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k)
            for (int i = 0; i < 3; i++) s[i][threadIdx.x] += s[i][threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int i = 0; i < 3; i++) part[3 * blockIdx.x + i] = s[i][0];
    if (stats) block_max3(red + 0, am);
}

// Start of step n+1 for the two fault planes when the fused kernel of step
// n folded the leapfrog update: the previous slip rate of k_fault_pre, the
// update of both fault nodes (time_integration.f90:32-35) and the slip
// bookkeeping of k_fault_post.
__global__ void k_fault_fold(Geom g, Plane P, float* v0, float* v1, float* v2, float* u0, float* u1, float* u2,
                             const float* w0, const float* w1, const float* w2, float* F, float tm, float dt, float svtol) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.np; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        plane_pos(P, q, p);
        const long long c = vol_minus(g, P, p), c2 = c + P.off;
        float a = v0[c2] - v0[c], b = v1[c2] - v1[c], d = v2[c2] - v2[c];
        FA(F_T2)[q] = a; FA(F_T2 + 1)[q] = b; FA(F_T2 + 2)[q] = d;
        FA(F_F2)[q] = sqrtf(a * a + b * b + d * d);
        for (long long cc : {c, c2}) {
            if (!node_box(g, cc)) continue;
            float x;
            x = v0[cc] + dt * w0[cc]; v0[cc] = x; u0[cc] = u0[cc] + dt * x;
            x = v1[cc] + dt * w1[cc]; v1[cc] = x; u1[cc] = u1[cc] + dt * x;
            x = v2[cc] + dt * w2[cc]; v2[cc] = x; u2[cc] = u2[cc] + dt * x;
        }
        a = v0[c2] - v0[c]; b = v1[c2] - v1[c]; d = v2[c2] - v2[c];
        FA(F_T1)[q] = a; FA(F_T1 + 1)[q] = b; FA(F_T1 + 2)[q] = d;
        float f1 = sqrtf(a * a + b * b + d * d);
        FA(F_F1)[q] = f1;
        FA(F_SL)[q] = FA(F_SL)[q] + dt * f1;
        FA(F_PSV)[q] = fmax_(FA(F_PSV)[q], f1);
        if (svtol > 0.f) {
            float f2 = FA(F_F2)[q];
            if (f1 >= svtol && FA(F_TRUP)[q] > 1e8f) FA(F_TRUP)[q] = tm - dt * (0.5f + (svtol - f1) / (f2 - f1));
            if (f1 >= svtol) FA(F_TARR)[q] = 1e9f;
            if (f1 < svtol && f2 >= svtol) FA(F_TARR)[q] = tm - dt * (0.5f + (svtol - f1) / (f2 - f1));
        }
        a = u0[c2] - u0[c]; b = u1[c2] - u1[c]; d = u2[c2] - u2[c];
        FA(F_T2)[q] = a; FA(F_T2 + 1)[q] = b; FA(F_T2 + 2)[q] = d;
        FA(F_F2)[q] = sqrtf(a * a + b * b + d * d);
    }
}

// ------------------------------------------------------------ host
static unsigned gp(long long n) {
    long long b = (n + 255) / 256;
    if (b > 1024) b = 1024;
    return (unsigned)(b < 1 ? 1 : b);
}
static Plane plane_of(Solver& s) {
    Plane P;
    for (int i = 0; i < 3; i++) P.n[i] = s.fn3[i];
    P.ax = s.g.ifn - 1;
    P.irup = s.g.irup;
    P.np = s.d.np;
    P.off = P.ax == 0 ? 1 : P.ax == 1 ? s.g.sy : s.g.sz;
    return P;
}
static FieldView pv(Solver& s, int a) {
    FieldView f;
    f.p = s.fa(a);
    for (int i = 0; i < 3; i++) f.n[i] = s.fn3[i];
    return f;
}
static void core_box(Solver& s, int* a1, int* a2) {
    for (int i = 0; i < 3; i++) { a1[i] = s.g.i1core[i]; a2[i] = s.g.i2core[i]; }
    a1[s.g.ifn - 1] = 1;
    a2[s.g.ifn - 1] = 1;
}
static double* energy_acc(Solver& s) { return (double*)s.d.red + kRedEnergy; }

void fault_init(Solver& s) {
    Geom& g = s.g;
    Params& Pm = s.prm;
    if (Pm.faultnormal == "no") return;
    if (g.ifn == 0) return;
    for (int i = 0; i < 3; i++) s.fn3[i] = g.nm[i];
    s.fn3[g.ifn - 1] = 1;
    s.d.np = (long long)s.fn3[0] * s.fn3[1] * s.fn3[2];
    SORD_CUDA(dev_malloc(s, (void**)&s.d.fp, sizeof(float) * (size_t)(F_COUNT * s.d.np)));
    SORD_CUDA(cudaMemsetAsync(s.d.fp, 0, sizeof(float) * (size_t)(F_COUNT * s.d.np), s.stream));
    SORD_CUDA(cudaMemsetAsync(energy_acc(s), 0, sizeof(double) * 3, s.stream));
    Plane P = plane_of(s);
    float* F = s.d.fp;
    field_io(s, "<>", "mus", pv(s, F_MUS));
    field_io(s, "<>", "mud", pv(s, F_MUD));
    field_io(s, "<>", "dc", pv(s, F_DC));
    field_io(s, "<>", "co", pv(s, F_CO));
    field_io(s, "<>", "sxx", pv(s, F_T1));
    field_io(s, "<>", "syy", pv(s, F_T1 + 1));
    field_io(s, "<>", "szz", pv(s, F_T1 + 2));
    field_io(s, "<>", "syz", pv(s, F_T2));
    field_io(s, "<>", "szx", pv(s, F_T2 + 1));
    field_io(s, "<>", "sxy", pv(s, F_T2 + 2));
    field_io(s, "<>", "ts", pv(s, F_T3));
    field_io(s, "<>", "td", pv(s, F_T3 + 1));
    field_io(s, "<>", "tn", pv(s, F_T3 + 2));
    {
        int a1[3] = {1, 1, 1};
        float rr = dev_reduce_max(s, pv(s, F_T3 + 2), a1, s.fn3);
        if (rr > 0.f) fprintf(stderr, "Warning: positive normal traction: %g\n", (double)rr);
    }
    {
        int a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = g.i1pml[i] + 1; a2[i] = g.i2pml[i] - 1; }
        dev_set_halo(s, pv(s, F_CO), 1e20f, a1, a2);
    }
    k_normals<<<gp(P.np), 256, 0, s.stream>>>(g, P, s.d.x[0], s.d.x[1], s.d.x[2], F); LCHK(s);
    k_fault_area<<<gp(P.np), 256, 0, s.stream>>>(P, F, Pm.faultnormal[0] == '+' ? 1.f : -1.f); LCHK(s);
    field_io(s, ">", "nsx", pv(s, F_NHAT));
    field_io(s, ">", "nsy", pv(s, F_NHAT + 1));
    field_io(s, ">", "nsz", pv(s, F_NHAT + 2));
    k_fault_t0<<<gp(P.np), 256, 0, s.stream>>>(P, F, Pm.slipvector[0], Pm.slipvector[1], Pm.slipvector[2]); LCHK(s);
    if (Pm.rcrit > 0.f && Pm.vrup > 0.f) {
        float xh[3] = {0.f, 0.f, 0.f}, xi[3];
        int i1[3];
        for (int i = 0; i < 3; i++) { xi[i] = Pm.hypocenter[i] - (float)g.nnoff[i] + 1.0f; i1[i] = (int)std::floor(xi[i]); }
        if (i1[0] >= 1 && i1[0] < g.nm[0] && i1[1] >= 1 && i1[1] < g.nm[1] && i1[2] >= 1 && i1[2] < g.nm[2]) {
            for (int l = i1[2]; l <= i1[2] + 1; l++)
                for (int k = i1[1]; k <= i1[1] + 1; k++)
                    for (int j = i1[0]; j <= i1[0] + 1; j++) {
                        float w = (1.0f - std::fabs(xi[0] - (float)j)) * (1.0f - std::fabs(xi[1] - (float)k)) * (1.0f - std::fabs(xi[2] - (float)l));
                        for (int i = 0; i < 3; i++) {
                            float xv;
                            SORD_CUDA(cudaMemcpyAsync(&xv, s.d.x[i] + g.idx(j, k, l), sizeof(float), cudaMemcpyDeviceToHost, s.stream));
                            SORD_CUDA(cudaStreamSynchronize(s.stream));
                            xh[i] = xh[i] + w * xv;
                        }
                    }
        }
        k_rhypo<<<gp(P.np), 256, 0, s.stream>>>(g, P, s.d.x[0], s.d.x[1], s.d.x[2], F, xh[0], xh[1], xh[2]); LCHK(s);
    }
    k_fault_moduli<<<gp(P.np), 256, 0, s.stream>>>(g, P, s.d.lam, s.d.mu, F); LCHK(s);
    for (int arr : {F_LAMF, F_MUF}) {
        for (int d = 0; d < 3; d++) {
            if (d == g.ifn - 1) continue;
            k_pcopy<<<gp(P.np), 256, 0, s.stream>>>(s.fa(F_F2), s.fa(arr), P.np); LCHK(s);
            k_plane_avg<<<gp(P.np), 256, 0, s.stream>>>(P, s.fa(arr), s.fa(F_F2), d, g.nm[d] - 1); LCHK(s);
        }
    }
    k_pinv<<<gp(P.np), 256, 0, s.stream>>>(s.fa(F_MUF), P.np); LCHK(s);
    k_pfill<<<gp(P.np), 256, 0, s.stream>>>(s.fa(F_PSV), P.np, 0.f); LCHK(s);
    k_pfill<<<gp(P.np), 256, 0, s.stream>>>(s.fa(F_TRUP), P.np, 1e9f); LCHK(s);
    k_pfill<<<gp(P.np), 256, 0, s.stream>>>(s.fa(F_TARR), P.np, 0.f); LCHK(s);
    s.efric = 0;
}

void fault_time_pre(Solver& s) {
    Plane P = plane_of(s);
    k_fault_pre<<<gp(P.np), 256, 0, s.stream>>>(s.g, P, s.d.v[0], s.d.v[1], s.d.v[2], s.d.fp); LCHK(s);
}

static void fault_post_outputs(Solver& s);

void fault_time_post(Solver& s) {
    Plane P = plane_of(s);
    k_fault_post<<<gp(P.np), 256, 0, s.stream>>>(s.g, P, s.d.v[0], s.d.v[1], s.d.v[2], s.d.u[0], s.d.u[1], s.d.u[2], s.d.fp,
                                                 s.tm, s.g.dt, s.prm.svtol);
    LCHK(s);
    fault_post_outputs(s);
}

// outputs and statistics of the slip bookkeeping (time_integration.f90:94-113)
static void fault_post_outputs(Solver& s) {
    field_io(s, ">", "svx", pv(s, F_T1));
    field_io(s, ">", "svy", pv(s, F_T1 + 1));
    field_io(s, ">", "svz", pv(s, F_T1 + 2));
    field_io(s, ">", "svm", pv(s, F_F1));
    field_io(s, ">", "psv", pv(s, F_PSV));
    field_io(s, ">", "sux", pv(s, F_T2));
    field_io(s, ">", "suy", pv(s, F_T2 + 1));
    field_io(s, ">", "suz", pv(s, F_T2 + 2));
    field_io(s, ">", "sum", pv(s, F_F2));
    field_io(s, ">", "sl", pv(s, F_SL));
    field_io(s, ">", "trup", pv(s, F_TRUP));
    field_io(s, ">", "tarr", pv(s, F_TARR));
    if (s.it % s.prm.itstats == 0) {
        int a1[3], a2[3], o[3] = {1, 1, 1};
        core_box(s, a1, a2);
        s.svmax = std::max(-1.0f, dev_reduce_max(s, pv(s, F_F1), a1, a2));
        s.sumax = std::max(-1.0f, dev_reduce_max(s, pv(s, F_F2), a1, a2));
        s.slmax = dev_reduce_max(s, pv(s, F_SL), o, s.fn3);
        s.tarrmax = std::max(-1.0f, dev_reduce_max(s, pv(s, F_TARR), a1, a2));
    }
}

static RuptArgs rupt_args(Solver& s) {
    Params& Pm = s.prm;
    RuptArgs A;
    A.g = s.g;
    A.P = plane_of(s);
    for (int i = 0; i < 3; i++) { A.v[i] = s.d.v[i]; A.u[i] = s.d.u[i]; A.w[i] = s.d.w1n[i]; }
    A.mr = s.d.mr;
    A.F = s.d.fp;
    A.dt = s.g.dt;
    A.tm = s.tm;
    A.rcrit = Pm.rcrit;
    A.vrup = Pm.vrup;
    A.trelax = Pm.trelax;
    A.it = s.it;
    A.faultopening = Pm.faultopening;
    return A;
}

// outputs and statistics of the traction and friction (dynamic_rupture.f90:336-352)
static void rupture_outputs(Solver& s, bool st, const int* a1, const int* a2) {
    field_io(s, ">", "tx", pv(s, F_T1));
    field_io(s, ">", "ty", pv(s, F_T1 + 1));
    field_io(s, ">", "tz", pv(s, F_T1 + 2));
    field_io(s, ">", "tsx", pv(s, F_T3));
    field_io(s, ">", "tsy", pv(s, F_T3 + 1));
    field_io(s, ">", "tsz", pv(s, F_T3 + 2));
    field_io(s, ">", "tsm", pv(s, F_TS));
    field_io(s, ">", "tnm", pv(s, F_TN));
    field_io(s, ">", "fr", pv(s, F_F1));
    if (st) {
        s.tsmax = std::max(-1.0f, dev_reduce_max(s, pv(s, F_TS), a1, a2));
        s.tnmin = dev_reduce_min(s, pv(s, F_TN), a1, a2);
        s.tnmax = dev_reduce_max(s, pv(s, F_TN), a1, a2);
    }
}

// outputs of the slip acceleration and the energy statistics (dynamic_rupture.f90:371-384)
static void slip_accel_outputs(Solver& s, bool st, const int* a1, const int* a2) {
    field_io(s, ">", "sax", pv(s, F_T2));
    field_io(s, ">", "say", pv(s, F_T2 + 1));
    field_io(s, ">", "saz", pv(s, F_T2 + 2));
    field_io(s, ">", "sam", pv(s, F_F2));
    if (st) {
        s.samax = std::max(-1.0f, dev_reduce_max(s, pv(s, F_F2), a1, a2));
        double e[3];
        SORD_CUDA(cudaMemcpyAsync(e, energy_acc(s), sizeof e, cudaMemcpyDeviceToHost, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
        s.efric = e[0]; s.estrain = e[1]; s.moment = e[2];
    }
}

void fault_rupture(Solver& s) {
    RuptArgs A = rupt_args(s);
    const Plane& P = A.P;
    Params& Pm = s.prm;
    k_rupture<<<gp(P.np), 256, 0, s.stream>>>(A); LCHK(s);
    launch_vector_bc(s, s.d.w1n, Pm.bc1, Pm.bc2, s.g.i1bc, s.g.i2bc);
    const bool st = s.it % s.prm.itstats == 0;
    int a1[3], a2[3];
    core_box(s, a1, a2);
    rupture_outputs(s, st, a1, a2);
    double* part = (double*)s.d.red + kRedPart;
    unsigned nb = gp(P.np);
    k_fault_energy<<<nb, 256, 0, s.stream>>>(s.g, P, s.d.v[0], s.d.v[1], s.d.v[2], s.d.u[0], s.d.u[1], s.d.u[2], s.d.fp, part); LCHK(s);
    k_fault_energy_fin<<<1, 32, 0, s.stream>>>(part, (int)nb, energy_acc(s), (double)s.g.dt); LCHK(s);
    k_slip_accel<<<gp(P.np), 256, 0, s.stream>>>(s.g, P, s.d.w1n[0], s.d.w1n[1], s.d.w1n[2], s.d.mr, s.d.fp); LCHK(s);
    slip_accel_outputs(s, st, a1, a2);
}

// The fault half of a fused step, after the fused volume kernel (whose
// boundary conditions are no-ops, so vector_bc is skipped): rupture, energy
// sums, slip acceleration and the mass division of the fault nodes in one
// kernel, then the same outputs and statistics as fault_rupture.
void fault_rupture_fused(Solver& s) {
    RuptArgs A = rupt_args(s);
    const Plane& P = A.P;
    const bool st = s.it % s.prm.itstats == 0;
    double* part = (double*)s.d.red + kRedPart;
    unsigned nb = gp(P.np);
    k_rupture_fused<<<nb, 256, 0, s.stream>>>(A, part, st ? 1 : 0, (unsigned*)s.d.red); LCHK(s);
    k_fault_energy_fin<<<1, 32, 0, s.stream>>>(part, (int)nb, energy_acc(s), (double)s.g.dt); LCHK(s);
    int a1[3], a2[3];
    core_box(s, a1, a2);
    rupture_outputs(s, st, a1, a2);
    slip_accel_outputs(s, st, a1, a2);
}

// Start of a step after a folded fused step: previous slip rate, leapfrog
// update of the fault nodes and slip bookkeeping in one kernel, then the
// outputs of fault_time_post.
void fault_fold(Solver& s) {
    Plane P = plane_of(s);
    k_fault_fold<<<gp(P.np), 256, 0, s.stream>>>(s.g, P, s.d.v[0], s.d.v[1], s.d.v[2], s.d.u[0], s.d.u[1], s.d.u[2],
                                                 s.d.w1n[0], s.d.w1n[1], s.d.w1n[2], s.d.fp, s.tm, s.g.dt, s.prm.svtol);
    LCHK(s);
    fault_post_outputs(s);
}

}  // namespace sordgpu

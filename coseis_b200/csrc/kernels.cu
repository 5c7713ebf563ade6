// Per-step kernels of the SORD time loop (sord/sord.f90:39-47).
//
//   k_time    step_time volume part   time_integration.f90:25-41
//   k_stress  step_stress             stress.f90:133-365 (strain, PML g
//                                     memory, potency, Hooke, moment, 1/V)
//   k_hooke / k_vscale                the same two stages, split out when a
//                                     field-I/O hook sits between them
//   k_accel   step_accel              acceleration.f90:19-211 (divergence,
//                                     PML p memory, hourglass) and, when no
//                                     hook intervenes, :240-262 (f*mr, |a|)
//   k_mass    acceleration.f90:240-251
//   BC / injection helpers            boundary_cond.f90, field_io '.' ops
#include "inject.cuh"
#include "sord.cuh"
#include "stencil.cuh"

namespace sordgpu {

// ------------------------------------------------------------ reductions
// Maxima of non-negative FP32 values compare like their bit patterns, and
// NaN (0x7fc00000) sorts above +Inf, so a NaN anywhere wins the maximum,
// which is what the NaN/Inf check of statistics.f90:52-60 needs.
__device__ __forceinline__ void block_max_to(unsigned* dst, float v) {
    unsigned b = __float_as_uint(v);
    if (v != v) b = 0x7fc00000u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    __shared__ unsigned sm[32];
    int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
    int warp = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
    int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    if (lane == 0) sm[warp] = b;
    __syncthreads();
    if (warp == 0) {
        b = lane < nw ? sm[lane] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
        if (lane == 0 && b) atomicMax(dst, b);
    }
}

__device__ __forceinline__ bool in_core(const Geom& g, int j, int k, int l) {
    return j >= g.i1core[0] && j <= g.i2core[0] && k >= g.i1core[1] && k <= g.i2core[1] && l >= g.i1core[2] &&
           l <= g.i2core[2];
}

// ------------------------------------------------------------ k_time
// v = v + dt*a; u = u + dt*v; w1 = u + gam*v over the whole block, halo
// included (time_integration.f90:27-41); optional |v|^2, |u|^2 maxima over
// the core (time_integration.f90:47-64, utilities.f90:120-139).
__global__ void k_time(Geom g, float* __restrict__ v0, float* __restrict__ v1, float* __restrict__ v2,
                       float* __restrict__ u0, float* __restrict__ u1, float* __restrict__ u2,
                       float* __restrict__ w0, float* __restrict__ w1, float* __restrict__ w2,
                       const float* __restrict__ gam, int stats, unsigned* red) {
    float vm = 0.f, um = 0.f;
    const float dt = g.dt;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        float G = gam[q];
        float a, b, c;
        float vv[3], uu[3];
        a = v0[q] + dt * w0[q]; b = u0[q] + dt * a; v0[q] = a; u0[q] = b; w0[q] = b + G * a; vv[0] = a; uu[0] = b;
        a = v1[q] + dt * w1[q]; b = u1[q] + dt * a; v1[q] = a; u1[q] = b; w1[q] = b + G * a; vv[1] = a; uu[1] = b;
        a = v2[q] + dt * w2[q]; b = u2[q] + dt * a; v2[q] = a; u2[q] = b; w2[q] = b + G * a; vv[2] = a; uu[2] = b;
        if (stats) {
            int j = (int)(q % g.sy) + 1;
            int k = (int)((q / g.sy) % g.nm[1]) + 1;
            int l = (int)(q / g.sz) + 1;
            if (in_core(g, j, k, l)) {
                c = vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2];
                vm = (c != c || c > vm) ? c : vm;
                c = uu[0] * uu[0] + uu[1] * uu[1] + uu[2] * uu[2];
                um = (c != c || c > um) ? c : um;
            }
        }
    }
    if (stats) {
        block_max_to(red + 1, vm);
        __syncthreads();
        block_max_to(red + 2, um);
    }
}

// ------------------------------------------------------------ k_stress
struct StressArgs {
    Geom g;
    Brackets br;
    const float* __restrict__ x[3];
    const float* __restrict__ w[3];  // u + gam*v at nodes
    const float* __restrict__ u[3];
    const float* __restrict__ v[3];
    const float* __restrict__ lam;
    const float* __restrict__ mu;
    const float* __restrict__ vc;
    const float* __restrict__ pmlc;  // dn1 dn2 dc1 dc2
    Slabs sl;
    float* sd[3];
    float* so[3];
    InjectList pot, mom;
    int hooke;  // 0: write strain only (hooks follow), 1: full stress
    int stats;
    unsigned* red;
};

// Linear index into a cell slab memory g1..g6 for cell (j,k,l), comp ic.
__device__ __forceinline__ long long slab_index(const Geom& g, int axis, int t, int ii, int j, int k, int l, int ic) {
    long long e0 = axis == 0 ? t : g.nm[0], e1 = axis == 1 ? t : g.nm[1], e2 = axis == 2 ? t : g.nm[2];
    long long a0 = axis == 0 ? ii : j - 1, a1 = axis == 1 ? ii : k - 1, a2 = axis == 2 ? ii : l - 1;
    return a0 + e0 * (a1 + e1 * a2) + (long long)ic * e0 * e1 * e2;
}

template <bool RECT>
__global__ void __launch_bounds__(256) k_stress(StressArgs A) {
    const Geom& g = A.g;
    int j = g.i1cell[0] + blockIdx.x * blockDim.x + threadIdx.x;
    int k = g.i1cell[1] + blockIdx.y * blockDim.y + threadIdx.y;
    int l = g.i1cell[2] + blockIdx.z * blockDim.z + threadIdx.z;
    float wn = 0.f;
    __shared__ Inject lpot[kLocalInject], lmom[kLocalInject];
    __shared__ int lcnt[2];
    {
        const int bj = g.i1cell[0] + blockIdx.x * blockDim.x, bk = g.i1cell[1] + blockIdx.y * blockDim.y,
                  bl = g.i1cell[2] + blockIdx.z * blockDim.z;
        gather_inject(A.pot, lpot, &lcnt[0], g, bj, bj + blockDim.x - 1, bk, bk + blockDim.y - 1, bl, bl + blockDim.z - 1);
        gather_inject(A.mom, lmom, &lcnt[1], g, bj, bj + blockDim.x - 1, bk, bk + blockDim.y - 1, bl, bl + blockDim.z - 1);
        __syncthreads();
    }
    bool active = j <= g.i2cell[0] && k <= g.i2cell[1] && l <= g.i2cell[2];
    if (active) {
        const long long q = g.idx(j, k, l);
        // region of this cell: stress.f90:141-248
        bool nearS[3], farS[3], anyS = false;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            int c = d == 0 ? j : d == 1 ? k : l;
            nearS[d] = c <= g.i1pml[d];
            farS[d] = c >= g.i2pml[d] - 1;
            anyS = anyS || nearS[d] || farS[d];
        }
        long long cq[8];
#pragma unroll
        for (int n = 0; n < 8; n++) cq[n] = q + (n & 1) + ((n >> 1) & 1) * g.sy + ((n >> 2) & 1) * g.sz;
        float B[3][8];
        if (RECT) {
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int t = 0; t < 8; t++) B[a][t] = A.br.bnc[a][t];
        } else {
            float X[3][8];
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int n = 0; n < 8; n++) X[c][n] = A.x[c][cq[n]];
#pragma unroll
            for (int a = 0; a < 3; a++) brackets_nc(X, a, B[a]);
        }
        float ed[3], eo[3];
        const float h = g.h;
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            float W[8], U[8], V[8];
            if (anyS) {
#pragma unroll
                for (int t = 0; t < 8; t++) { U[t] = A.u[ic][cq[term_corner(t)]]; V[t] = A.v[ic][cq[term_corner(t)]]; }
            } else {
#pragma unroll
                for (int t = 0; t < 8; t++) W[t] = A.w[ic][cq[term_corner(t)]];
            }
#pragma unroll
            for (int iid = 0; iid < 3; iid++) {
                const int id = (ic + iid + 1) % 3;
                float s;
                if (nearS[id] || farS[id]) {
                    // damped direction: g' = v_i,j (stress.f90:159-248)
                    const float raw = stencil8(V, B[id], h);
                    s = raw;
                    const int c = id == 0 ? j : id == 1 ? k : l;
                    if (nearS[id]) {
                        int p = c + g.nnoff[id];
                        int ii = c - g.i1cell[id];
                        float* G = A.sl.g[id] + slab_index(g, id, A.sl.tg[id], ii, j, k, l, ic);
                        s = A.pmlc[3 * g.npml + p - 1] * raw + A.pmlc[2 * g.npml + p - 1] * *G;
                        *G = s;
                    }
                    if (farS[id]) {
                        int p = g.nn[id] - c - g.nnoff[id];
                        int ii = g.i2cell[id] - c;
                        float* G = A.sl.g[3 + id] + slab_index(g, id, A.sl.tg[3 + id], ii, j, k, l, ic);
                        s = A.pmlc[3 * g.npml + p - 1] * raw + A.pmlc[2 * g.npml + p - 1] * *G;
                        *G = s;
                    }
                } else if (anyS) {
                    s = stencil8(U, B[id], h);  // non-damped PML direction: g = u_i,j
                } else {
                    s = stencil8(W, B[id], h);  // elastic: g = (u + gam*v)_i,j
                }
                // strain assembly (stress.f90:251-282)
                if (ic == id) ed[ic] = s;
                else if (ic < id) eo[3 - ic - id] = 0.5f * s;
                else eo[3 - ic - id] = eo[3 - ic - id] + 0.5f * s;
            }
        }
        // potency ops / finite source (stress.f90:288-296)
        apply_inject(lpot, lcnt[0], A.pot, q, ed, eo);
        if (A.hooke) {
            // Hooke's law (stress.f90:310-330)
            const float lm = A.lam[q], m2 = 2.0f * A.mu[q];
            const float s1 = lm * (ed[0] + ed[1] + ed[2]);
#pragma unroll
            for (int i = 0; i < 3; i++) { ed[i] = m2 * ed[i] + s1; eo[i] = m2 * eo[i]; }
            apply_inject(lmom, lcnt[1], A.mom, q, ed, eo);
            // stress = moment / volume (stress.f90:344-355)
            const float r = A.vc[q];
#pragma unroll
            for (int i = 0; i < 3; i++) { ed[i] = ed[i] * r; eo[i] = eo[i] * r; }
            if (A.stats && in_core(g, j, k, l))
                wn = (ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]) + 2.0f * (eo[0] * eo[0] + eo[1] * eo[1] + eo[2] * eo[2]);
        }
#pragma unroll
        for (int i = 0; i < 3; i++) { A.sd[i][q] = ed[i]; A.so[i][q] = eo[i]; }
    }
    if (A.stats) block_max_to(A.red + 3, wn);
}

// Hooke's law and the volume scaling as separate passes over the whole block
// (halo included, like stress.f90:310-355) for steps with p**/m** hooks.
__global__ void k_hooke(Geom g, float* sd0, float* sd1, float* sd2, float* so0, float* so1, float* so2,
                        const float* __restrict__ lam, const float* __restrict__ mu) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        float s1 = lam[q] * (sd0[q] + sd1[q] + sd2[q]);
        float m = mu[q];
        sd0[q] = 2.0f * m * sd0[q] + s1; so0[q] = 2.0f * m * so0[q];
        sd1[q] = 2.0f * m * sd1[q] + s1; so1[q] = 2.0f * m * so1[q];
        sd2[q] = 2.0f * m * sd2[q] + s1; so2[q] = 2.0f * m * so2[q];
    }
}
__global__ void k_vscale(Geom g, float* sd0, float* sd1, float* sd2, float* so0, float* so1, float* so2,
                         const float* __restrict__ vc) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        float r = vc[q];
        sd0[q] = sd0[q] * r; so0[q] = so0[q] * r;
        sd1[q] = sd1[q] * r; so1[q] = so1[q] * r;
        sd2[q] = sd2[q] * r; so2[q] = so2[q] * r;
    }
}

// ------------------------------------------------------------ k_accel
// Tile of TX*TY*TZ nodes; shared memory holds the (TX+1)(TY+1)(TZ+1) cells
// around it (stress, yy, hourglass cell values) and the (TX+2)(TY+2)(TZ+2)
// nodes those cells touch (u, v for the hourglass, x for curvilinear
// brackets).
constexpr int TX = 32, TY = 4, TZ = 4;
constexpr int CX = TX + 1, CY = TY + 1, CZ = TZ + 1, NCELL = CX * CY * CZ;
constexpr int NX = TX + 2, NY = TY + 2, NZ = TZ + 2, NNODE = NX * NY * NZ;
constexpr int NT_ACC = TX * TY * TZ;

struct AccelArgs {
    Geom g;
    Brackets br;
    const float* __restrict__ x[3];
    const float* __restrict__ u[3];
    const float* __restrict__ v[3];
    const float* __restrict__ sd[3];
    const float* __restrict__ so[3];
    const float* __restrict__ yy;
    const float* __restrict__ mr;
    const float* __restrict__ pmlc;
    Slabs sl;
    float* f[3];  // w1n: force (mass = 0) or acceleration (mass = 1)
    float hg1, dh2;
    int hourglass;   // any(hourglass > 0)
    int hgvisc;      // hourglass(2) > 0 .and. npml > 0
    int mass;
    int stats;
    InjectList force;  // force point sources applied before the mass division
    unsigned* red;
};

template <bool RECT>
__global__ void __launch_bounds__(NT_ACC) k_accel(AccelArgs A) {
    extern __shared__ float smem[];
    float* sS = smem;                       // 6 * NCELL stress
    float* sY = sS + 6 * NCELL;             // yy
    float* sHE = sY + NCELL;                // hourglass cell value, elastic form
    float* sHP = sHE + NCELL;               // hourglass cell value, PML viscous form
    float* sW = sHP + NCELL;                // 3 * NNODE: hg1*u + dt*hg2*v
    float* sV = sW + 3 * NNODE;             // 3 * NNODE: v
    float* sX = sV + 3 * NNODE;             // 3 * NNODE: x (curvilinear only)
    const Geom& g = A.g;
    const int tid = threadIdx.x + TX * (threadIdx.y + TY * threadIdx.z);
    const int j0 = g.i1node[0] + blockIdx.x * TX, k0 = g.i1node[1] + blockIdx.y * TY, l0 = g.i1node[2] + blockIdx.z * TZ;
    // cells (j0-1 .. j0+TX-1) etc; nodes (j0-1 .. j0+TX)
    for (int c = tid; c < NCELL; c += NT_ACC) {
        int cj = c % CX, ck = (c / CX) % CY, cl = c / (CX * CY);
        int j = j0 - 1 + cj, k = k0 - 1 + ck, l = l0 - 1 + cl;
        bool ok = j <= g.nm[0] && k <= g.nm[1] && l <= g.nm[2];
        long long q = ok ? g.idx(j, k, l) : 0;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            sS[i * NCELL + c] = ok ? A.sd[i][q] : 0.f;
            sS[(3 + i) * NCELL + c] = ok ? A.so[i][q] : 0.f;
        }
        sY[c] = ok ? A.yy[q] : 0.f;
    }
    const bool needNodes = A.hourglass || !RECT;
    if (needNodes) {
        for (int n = tid; n < NNODE; n += NT_ACC) {
            int nj = n % NX, nk = (n / NX) % NY, nl = n / (NX * NY);
            int j = j0 - 1 + nj, k = k0 - 1 + nk, l = l0 - 1 + nl;
            bool ok = j <= g.nm[0] && k <= g.nm[1] && l <= g.nm[2];
            long long q = ok ? g.idx(j, k, l) : 0;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                float uu = ok ? A.u[i][q] : 0.f, vv = ok ? A.v[i][q] : 0.f;
                sW[i * NNODE + n] = A.hg1 * uu + A.dh2 * vv;
                sV[i * NNODE + n] = vv;
                if (!RECT) sX[i * NNODE + n] = ok ? A.x[i][q] : 0.f;
            }
        }
    }
    __syncthreads();

    const int tj = threadIdx.x, tk = threadIdx.y, tl = threadIdx.z;
    const int j = j0 + tj, k = k0 + tk, l = l0 + tl;
    const bool active = j <= g.i2node[0] && k <= g.i2node[1] && l <= g.i2node[2];
    // cell of term t around node (j,k,l): offsets (-1 or 0) per axis
    const int ct[8] = {0, 1, 0, 1, 0, 1, 0, 1};
    const int kt[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    const int lt[8] = {0, 0, 1, 1, 0, 0, 1, 1};
    float f[3] = {0.f, 0.f, 0.f};
    if (active) {
        // divergence f_i = w_ij,j (acceleration.f90:22-130)
        float B[3][8];
        if (RECT) {
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int t = 0; t < 8; t++) B[a][t] = A.br.bcn[a][t];
        } else {
            auto X = [&](int c, int m) -> float {
                int dj = m % 3 - 1, dk = (m / 3) % 3 - 1, dl = m / 9 - 1;
                return sX[c * NNODE + (tj + 1 + dj) + NX * ((tk + 1 + dk) + NY * (tl + 1 + dl))];
            };
#pragma unroll
            for (int a = 0; a < 3; a++) brackets_cn(X, a, B[a]);
        }
        int cidx[8];
#pragma unroll
        for (int t = 0; t < 8; t++) cidx[t] = (tj + ct[t]) + CX * ((tk + kt[t]) + CY * (tl + lt[t]));
        const float h = g.h;
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
#pragma unroll
            for (int iid = 0; iid < 3; iid++) {
                const int id = (ic + iid) % 3;
                const int comp = ic == id ? ic : 3 + (3 - ic - id);
                float F[8];
#pragma unroll
                for (int t = 0; t < 8; t++) F[t] = sS[comp * NCELL + cidx[t]];
                float s = stencil8(F, B[id], h);
                // PML p memory, damped direction id (acceleration.f90:37-104)
                const int c = id == 0 ? j : id == 1 ? k : l;
                if (c <= g.i1pml[id]) {
                    int p = c + g.nnoff[id];
                    int ii = c - g.i1node[id];
                    float* P = A.sl.p[id] + slab_index(g, id, A.sl.tp[id], ii, j, k, l, ic);
                    s = A.pmlc[g.npml + p - 1] * s + A.pmlc[p - 1] * *P;
                    *P = *P + g.dt * s;
                }
                if (c >= g.i2pml[id]) {
                    int p = g.nn[id] - c - g.nnoff[id] + 1;
                    int ii = g.i2node[id] - c;
                    float* P = A.sl.p[3 + id] + slab_index(g, id, A.sl.tp[3 + id], ii, j, k, l, ic);
                    s = A.pmlc[g.npml + p - 1] * s + A.pmlc[p - 1] * *P;
                    *P = *P + g.dt * s;
                }
                f[ic] = iid == 0 ? s : f[ic] + s;
            }
        }
    }
    if (A.hourglass) {
        // hourglass control, viscous only in the PML (acceleration.f90:132-211)
        bool ne = true;
        ne = ne && j >= g.i1pml[0] + 1 && j <= g.i2pml[0] - 1;
        ne = ne && k >= g.i1pml[1] + 1 && k <= g.i2pml[1] - 1;
        ne = ne && l >= g.i1pml[2] + 1 && l <= g.i2pml[2] - 1;
        for (int iq = 0; iq < 4; iq++) {
            for (int ic = 0; ic < 3; ic++) {
                for (int c = tid; c < NCELL; c += NT_ACC) {
                    int cj = c % CX, ck = (c / CX) % CY, cl = c / (CX * CY);
                    int J = j0 - 1 + cj, K = k0 - 1 + ck, L = l0 - 1 + cl;
                    bool valid = J >= g.i1cell[0] && J <= g.i2cell[0] && K >= g.i1cell[1] && K <= g.i2cell[1] &&
                                 L >= g.i1cell[2] && L <= g.i2cell[2];
                    bool inE = valid && J >= g.i1pml[0] && J <= g.i2pml[0] - 1 && K >= g.i1pml[1] &&
                               K <= g.i2pml[1] - 1 && L >= g.i1pml[2] && L <= g.i2pml[2] - 1;
                    bool inP = valid && (J <= g.i1pml[0] || J >= g.i2pml[0] - 1 || K <= g.i1pml[1] ||
                                         K >= g.i2pml[1] - 1 || L <= g.i1pml[2] || L >= g.i2pml[2] - 1);
                    float he = 0.f, hp = 0.f;
                    if (inE || (inP && A.hgvisc)) {
                        float Wc[8], Vc[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            int hc = hg_corner(t);
                            int n = (cj + (hc & 1)) + NX * ((ck + ((hc >> 1) & 1)) + NY * (cl + (hc >> 2)));
                            Wc[t] = sW[ic * NNODE + n];
                            Vc[t] = sV[ic * NNODE + n];
                        }
                        if (inE) he = hg_sum(Wc, iq) * sY[c];
                        if (inP && A.hgvisc) hp = A.dh2 * sY[c] * hg_sum(Vc, iq);
                    }
                    sHE[c] = he;
                    sHP[c] = hp;
                }
                __syncthreads();
                if (active) {
                    float s2 = 0.f;
                    if (ne || A.hgvisc) {
                        const float* H = ne ? sHE : sHP;
                        float Hc[8];
#pragma unroll
                        for (int t = 0; t < 8; t++)
                            Hc[t] = H[(tj + 1 - (hg_corner(t) & 1)) + CX * ((tk + 1 - ((hg_corner(t) >> 1) & 1)) + CY * (tl + 1 - (hg_corner(t) >> 2)))];
                        s2 = hg_sum(Hc, iq);
                    }
                    f[ic] = f[ic] - s2;
                }
                __syncthreads();
            }
        }
    }
    float an = 0.f;
    if (active) {
        const long long q = g.idx(j, k, l);
        for (int e = 0; e < A.force.n; e++)
            if (A.force.e[e].idx == q) {
                int c = A.force.e[e].comp;
                f[c] = f[c] + A.force.e[e].inc;
            }
        if (A.mass) {
            const float m = A.mr[q];
#pragma unroll
            for (int i = 0; i < 3; i++) f[i] = f[i] * m;
            if (A.stats && in_core(g, j, k, l)) an = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
        }
#pragma unroll
        for (int i = 0; i < 3; i++) A.f[i][q] = f[i];
    }
    if (A.stats && A.mass) block_max_to(A.red + 0, an);
}

// a = f * mr over the whole block (acceleration.f90:240-251) and |a|^2 max
__global__ void k_mass(Geom g, float* f0, float* f1, float* f2, const float* __restrict__ mr, int stats, unsigned* red) {
    float am = 0.f;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        float m = mr[q];
        float a = f0[q] * m, b = f1[q] * m, c = f2[q] * m;
        f0[q] = a; f1[q] = b; f2[q] = c;
        if (stats) {
            int j = (int)(q % g.sy) + 1;
            int k = (int)((q / g.sy) % g.nm[1]) + 1;
            int l = (int)(q / g.sz) + 1;
            if (in_core(g, j, k, l)) {
                float n = a * a + b * b + c * c;
                am = (n != n || n > am) ? n : am;
            }
        }
    }
    if (stats) block_max_to(red + 0, am);
}

// ------------------------------------------------------------ plane ops
// One boundary-condition plane operation on up to three component arrays:
// f[c](plane p of axis d) = sign[c] * f[c](plane ps)  (mode 1) or 0 (mode 0),
// for the components in `mask`; the other two axes span the whole block.
__global__ void k_plane(Geom g, int n0, int n1, int n2, float* f0, float* f1, float* f2, int d, int p, int ps, int mode,
                        int mask, float s0, float s1, float s2) {
    int nn_[3] = {n0, n1, n2};
    int ea = d == 0 ? 1 : 0, eb = d == 2 ? 1 : 2;
    long long n = (long long)nn_[ea] * nn_[eb];
    long long sy = n0, sz = (long long)n0 * n1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int ia = (int)(t % nn_[ea]), ib = (int)(t / nn_[ea]);
        int pos[3], src[3];
        pos[d] = p - 1; src[d] = ps - 1;
        pos[ea] = src[ea] = ia;
        pos[eb] = src[eb] = ib;
        long long qd = pos[0] + sy * pos[1] + sz * pos[2];
        long long qs = src[0] + sy * src[1] + sz * src[2];
        float* F[3] = {f0, f1, f2};
        float S[3] = {s0, s1, s2};
#pragma unroll
        for (int c = 0; c < 3; c++)
            if ((mask >> c) & 1 && F[c]) F[c][qd] = mode ? S[c] * F[c][qs] : 0.f;
    }
}

// Point injections f(idx) = f(idx) + inc in list order (one thread keeps the
// order of repeated indices).
__global__ void k_inject(float* f0, float* f1, float* f2, float* f3, float* f4, float* f5, const Inject* e, int n) {
    if (threadIdx.x || blockIdx.x) return;
    float* F[6] = {f0, f1, f2, f3, f4, f5};
    for (int i = 0; i < n; i++) {
        float* p = F[e[i].comp] + e[i].idx;
        *p = *p + e[i].inc;
    }
}

// ------------------------------------------------------------ launchers
static unsigned grid_1d(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

void launch_time_update(Solver& s, bool stats) {
    Device& d = s.d;
    cudaEvent_t e0 = nullptr;
    s.prof_begin(KC_TIME, &e0);
    k_time<<<grid_1d(s.g.nv), 256, 0, s.stream>>>(s.g, d.v[0], d.v[1], d.v[2], d.u[0], d.u[1], d.u[2], d.w1n[0], d.w1n[1],
                                                  d.w1n[2], d.gam, stats ? 1 : 0, (unsigned*)d.red);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
    s.prof_end(KC_TIME, e0);
}

void launch_stress(Solver& s, const InjectList& pot, const InjectList& mom, bool hooke) {
    Device& d = s.d;
    StressArgs A;
    A.g = s.g;
    A.br = s.br;
    for (int i = 0; i < 3; i++) {
        A.x[i] = d.x[i]; A.w[i] = d.w1n[i]; A.u[i] = d.u[i]; A.v[i] = d.v[i];
        A.sd[i] = d.sd[i]; A.so[i] = d.so[i];
    }
    A.lam = d.lam; A.mu = d.mu; A.vc = d.vc; A.pmlc = d.pmlc; A.sl = d.slabs;
    A.pot = pot; A.mom = mom;
    A.hooke = hooke ? 1 : 0;
    A.stats = (hooke && s.it % s.prm.itstats == 0) ? 1 : 0;
    A.red = (unsigned*)d.red;
    dim3 b(32, 4, 2);
    int n0 = s.g.i2cell[0] - s.g.i1cell[0] + 1, n1 = s.g.i2cell[1] - s.g.i1cell[1] + 1, n2 = s.g.i2cell[2] - s.g.i1cell[2] + 1;
    if (n0 < 1 || n1 < 1 || n2 < 1) return;
    dim3 gr(div_up(n0, b.x), div_up(n1, b.y), div_up(n2, b.z));
    cudaEvent_t e0 = nullptr;
    s.prof_begin(KC_STRESS, &e0);
    if (s.rect) k_stress<true><<<gr, b, 0, s.stream>>>(A);
    else k_stress<false><<<gr, b, 0, s.stream>>>(A);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
    s.prof_end(KC_STRESS, e0);
}

void launch_hooke(Solver& s) {
    Device& d = s.d;
    k_hooke<<<grid_1d(s.g.nv), 256, 0, s.stream>>>(s.g, d.sd[0], d.sd[1], d.sd[2], d.so[0], d.so[1], d.so[2], d.lam, d.mu);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

void launch_volume_scale(Solver& s) {
    Device& d = s.d;
    k_vscale<<<grid_1d(s.g.nv), 256, 0, s.stream>>>(s.g, d.sd[0], d.sd[1], d.sd[2], d.so[0], d.so[1], d.so[2], d.vc);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

static size_t accel_smem(bool rect) {
    return sizeof(float) * (size_t)(6 * NCELL + 4 * NCELL + 6 * NNODE + (rect ? 0 : 3 * NNODE));
}

void launch_accel(Solver& s, bool mass, bool stats, const InjectList& force) {
    Device& d = s.d;
    AccelArgs A;
    A.g = s.g;
    A.br = s.br;
    for (int i = 0; i < 3; i++) {
        A.x[i] = d.x[i]; A.u[i] = d.u[i]; A.v[i] = d.v[i]; A.sd[i] = d.sd[i]; A.so[i] = d.so[i]; A.f[i] = d.w1n[i];
    }
    A.yy = d.yy; A.mr = d.mr; A.pmlc = d.pmlc; A.sl = d.slabs;
    A.hg1 = s.prm.hourglass[0];
    A.dh2 = s.g.dt * s.prm.hourglass[1];
    A.hourglass = (s.prm.hourglass[0] > 0.f || s.prm.hourglass[1] > 0.f) ? 1 : 0;
    A.hgvisc = (s.prm.hourglass[1] > 0.f && s.g.npml > 0) ? 1 : 0;
    A.mass = mass ? 1 : 0;
    A.stats = stats ? 1 : 0;
    A.force = force;
    A.red = (unsigned*)d.red;
    int n0 = s.g.i2node[0] - s.g.i1node[0] + 1, n1 = s.g.i2node[1] - s.g.i1node[1] + 1, n2 = s.g.i2node[2] - s.g.i1node[2] + 1;
    dim3 b(TX, TY, TZ);
    dim3 gr(div_up(n0, TX), div_up(n1, TY), div_up(n2, TZ));
    size_t sm = accel_smem(s.rect);
    cudaEvent_t e0 = nullptr;
    s.prof_begin(KC_ACCEL, &e0);
    if (s.rect) {
        smem_limit((const void*)k_accel<true>, (int)accel_smem(true));
        k_accel<true><<<gr, b, sm, s.stream>>>(A);
    } else {
        smem_limit((const void*)k_accel<false>, (int)accel_smem(false));
        k_accel<false><<<gr, b, sm, s.stream>>>(A);
    }
    s.launches++;
    SORD_CUDA(cudaGetLastError());
    s.prof_end(KC_ACCEL, e0);
}

void launch_mass(Solver& s, bool stats) {
    Device& d = s.d;
    cudaEvent_t e0 = nullptr;
    s.prof_begin(KC_MASS, &e0);
    k_mass<<<grid_1d(s.g.nv), 256, 0, s.stream>>>(s.g, d.w1n[0], d.w1n[1], d.w1n[2], d.mr, stats ? 1 : 0, (unsigned*)d.red);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
    s.prof_end(KC_MASS, e0);
}

static void plane(Solver& s, const int* fn, float* f0, float* f1, float* f2, int d, int p, int ps, int mode, int mask,
                  const float* sg) {
    long long n = (long long)(d == 0 ? fn[1] * (long long)fn[2] : d == 1 ? fn[0] * (long long)fn[2] : fn[0] * (long long)fn[1]);
    k_plane<<<grid_1d(n), 256, 0, s.stream>>>(s.g, fn[0], fn[1], fn[2], f0, f1, f2, d, p, ps, mode, mask,
                                              sg ? sg[0] : 0.f, sg ? sg[1] : 0.f, sg ? sg[2] : 0.f);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

// vector_bc (boundary_cond.f90:30-115) on a node vector field over the block.
void launch_vector_bc(Solver& s, float* const f[3], const int* bc1, const int* bc2, const int* i1, const int* i2) {
    const int* nm = s.g.nm;
    int b1[3], b2[3];
    for (int i = 0; i < 3; i++) {
        b1[i] = bc1[i] % 10; b2[i] = bc2[i] % 10;
        if (nm[i] == 1 || i1[i] < 1 || i1[i] > nm[i]) b1[i] = 99;
        if (nm[i] == 1 || i2[i] < 1 || i2[i] > nm[i]) b2[i] = 99;
    }
    const int* a[2] = {i1, i2};
    int* bb[2] = {b1, b2};
    for (int side = 0; side < 2; side++)
        for (int d = 0; d < 3; d++)
            if (bb[side][d] == -1) plane(s, nm, f[0], f[1], f[2], d, a[side][d], 0, 0, (7 & ~(1 << d)), nullptr);
    for (int side = 0; side < 2; side++)
        for (int d = 0; d < 3; d++)
            if (bb[side][d] == 1) plane(s, nm, f[0], f[1], f[2], d, a[side][d], 0, 0, 1 << d, nullptr);
    for (int side = 0; side < 2; side++)
        for (int d = 0; d < 3; d++)
            if (bb[side][d] == 3) plane(s, nm, f[0], f[1], f[2], d, a[side][d], 0, 0, 7, nullptr);
    for (int i = 0; i < 3; i++) {
        if (i1[i] >= nm[i]) b1[i] = 99;
        if (i2[i] <= 1) b2[i] = 99;
    }
    const float one[3] = {1.f, 1.f, 1.f};
    for (int d = 0; d < 3; d++)
        if (b1[d] == 4) plane(s, nm, f[0], f[1], f[2], d, i1[d], i1[d] + 1, 1, 7, one);
    for (int d = 0; d < 3; d++)
        if (b2[d] == 4) plane(s, nm, f[0], f[1], f[2], d, i2[d], i2[d] - 1, 1, 7, one);
    for (int d = 0; d < 3; d++) {
        if (std::abs(b1[d]) == 2) {
            float sg = bc1[d] >= 0 ? 1.f : -1.f;
            float S[3] = {sg, sg, sg};
            S[d] = -sg;
            plane(s, nm, f[0], f[1], f[2], d, i1[d], i1[d] + 1, 1, 7, S);
        }
    }
    for (int d = 0; d < 3; d++) {
        if (std::abs(b2[d]) == 2) {
            float sg = bc2[d] >= 0 ? 1.f : -1.f;
            float S[3] = {sg, sg, sg};
            S[d] = -sg;
            plane(s, nm, f[0], f[1], f[2], d, i2[d], i2[d] - 1, 1, 7, S);
        }
    }
}

// scalar_bc (boundary_cond.f90:7-27) on a field of extents fn.
void launch_scalar_bc(Solver& s, float* f, const int* fn, const int* bc1, const int* bc2, const int* i1, const int* i2) {
    int b1[3], b2[3];
    for (int i = 0; i < 3; i++) {
        b1[i] = std::abs(bc1[i] % 10); b2[i] = std::abs(bc2[i] % 10);
        if (b1[i] == 4) b1[i] = 2;
        if (b2[i] == 4) b2[i] = 2;
        if (fn[i] == 1 || i1[i] < 1 || i1[i] >= fn[i]) b1[i] = 99;
        if (fn[i] == 1 || i2[i] <= 1 || i2[i] > fn[i]) b2[i] = 99;
    }
    const float one[3] = {1.f, 1.f, 1.f};
    for (int d = 0; d < 3; d++)
        if (b1[d] == 2) plane(s, fn, f, nullptr, nullptr, d, i1[d], i1[d] + 1, 1, 1, one);
    for (int d = 0; d < 3; d++)
        if (b2[d] == 2) plane(s, fn, f, nullptr, nullptr, d, i2[d], i2[d] - 1, 1, 1, one);
}

void launch_inject(Solver& s, float* const f[6], const InjectList& l) {
    if (l.n <= 0) return;
    k_inject<<<1, 32, 0, s.stream>>>(f[0], f[1], f[2], f[3], f[4], f[5], l.e, l.n);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

}  // namespace sordgpu

// Discrete adjoint of the SORD time loop for gradients of a receiver misfit
// (no counterpart in the reference, which has no derivatives).
//
// The forward step n (sord/sord.f90:39-47 without field-I/O hooks) is, for
// the supported class (rectilinear mesh, no PML, no fault, free or other
// no-op boundary conditions):
//
//   v_n = v_{n-1} + dt a_{n-1},  u_n = u_{n-1} + dt v_n        (time_integration.f90:27-41)
//   w = u_n + g v_n,  G_ij = Dnc_j(w_i)                          (stress.f90:133-282)
//   sigma = vc (2 mu e + lam tr(e) I + M(t_n) weights)           (stress.f90:310-355)
//   f_i = Dcn_j(sigma_ij) - sum_q Hcn_q(yy Hnc_q(hg1 u + dt hg2 v)_i)   (acceleration.f90:22-211)
//   a_n = mr f                                                   (acceleration.f90:240-251)
//
// with receivers sampling v_n (or u_n) after the update.  The adjoint runs
// the transposed operators backwards in time: given (ubar, vbar) of step
// n + 1, abar_n = dt (vbar + dt ubar), fbar = mr abar, sigmabar = Dcn^T fbar,
// then the transposed Hooke law, Dnc^T and the hourglass pair Hnc/Hcn (each
// the transpose of the other), accumulating per cell dL/dlam, dL/dmu, dL/dyy
// and per node dL/dmr, plus dL/d(moment value) of every '.' moment op.
//
// Memory: the forward stores (u, v, a) every `seg` steps; the backward pass
// recomputes each segment from its checkpoint into a segment buffer and runs
// the adjoint steps of the segment from it (uniform checkpointing:
// 1 forward + 1 recomputation + the adjoint).  With seg = 1 every state is
// kept and nothing is recomputed; segment 0 picks that when all states fit
// in half of the free device memory, else segments of about sqrt(nt).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sord.cuh"
#include "timefn.h"
#include "stencil.cuh"

namespace sordgpu {

struct RecvEntry {
    long long idx;  // node index
    int comp;       // 0..2
    int disp;       // 1: u receiver, 0: v receiver
    float r;        // trilinear weight
    int off;        // first sample in the trace array
    int it1, dit, ns;
};
struct MomEntry {
    long long idx;  // cell index
    int comp;       // 0..5 (xx yy zz yz zx xy)
    int slot;       // moment op number
    float w;        // d(injected value)/d(op value)
};

struct AdjointState {
    int seg = 0;
    int nck = 0;               // checkpoints stored
    std::vector<float*> ckpt;  // (u, v, a) at steps 0, seg, 2 seg, ...; 9 nv floats each
    float* segbuf[2] = {};     // two segment buffers of seg states (9 nv floats each)
    float* ub[2][3] = {};      // adjoint state, double-buffered
    float* vb[2][3] = {};
    float *glam = nullptr, *gmu = nullptr, *gyy = nullptr, *gmr = nullptr;
    RecvEntry* recv = nullptr;
    int nrecv = 0;
    float* trace = nullptr;
    MomEntry* mom = nullptr;
    double* gmom = nullptr;     // per moment op: value, delay, position x y z (5 slots each)
    std::vector<double> gsrc;   // delay and position gradients of the last backward pass
    std::vector<int> recv_ops;  // op indices of '.>' receivers, recorded before the forward run
    std::vector<int> mom_ops;   // op indices of '.' moment ops
};

// ------------------------------------------------------------ kernels
struct AdjArgs {
    Geom g;
    Brackets br;
    Brackets brh;                     // br scaled by h
    const float *u[3], *v[3], *a[3];  // forward state of step n
    const float *ubi[3], *vbi[3];     // adjoint state of step n + 1
    float *ubo[3], *vbo[3];           // adjoint state of step n
    const float *lam, *mu, *yy, *vc, *mr, *gam;
    float *glam, *gmu, *gyy, *gmr;
    float hg1, dh2, dt;
    int hourglass;
    int nbx, segl;                    // tiles along j, node planes per block
};

__device__ __forceinline__ bool in_nodes(const Geom& g, int j, int k, int l) {
    return j >= g.i1node[0] && j <= g.i2node[0] && k >= g.i1node[1] && k <= g.i2node[1] && l >= g.i1node[2] &&
           l <= g.i2node[2];
}
__device__ __forceinline__ bool in_cells(const Geom& g, int j, int k, int l) {
    return j >= g.i1cell[0] && j <= g.i2cell[0] && k >= g.i1cell[1] && k <= g.i2cell[1] && l >= g.i1cell[2] &&
           l <= g.i2cell[2];
}
// fbar = mr dt (vbar + dt ubar) of node q, zero off the force nodes
__device__ __forceinline__ float fbar(const AdjArgs& A, long long q, bool act, int i) {
    return act ? A.mr[q] * (A.dt * (A.vbi[i][q] + A.dt * A.ubi[i][q])) : 0.f;
}

// One adjoint step over a tile column, streaming along l like the forward
// step kernel: a block of 32 x 8 threads owns node columns j0..j0+30 x
// k0..k0+6 (outputs) and computes the cells j0-1..j0+30 x k0-1..k0+6 they
// touch.  The raw node values of a plane (forward u, v, a, g, mr and the
// adjoint ubar, vbar of step n + 1) are copied into a three-slot shared ring
// with cp.async two planes ahead; cell planes (Gbar of the transposed
// strain, yy sbar of the hourglass) sit in a two-slot ring.  Cell gradients
// are written by the block that owns the cell (tx, ty >= 1), node gradients
// and the adjoint state by the owner of the node; the adjoint state is
// double-buffered (in: step n + 1, out: step n) because neighbouring blocks
// read the in-state of their halo nodes.  The transposed operators use fused
// multiply-adds with the brackets scaled by h: the gradients are those of
// the reference-order forward step to FP32 rounding.
constexpr int AJ = 32, AK = 8, ANJ = AJ + 1, ANK = AK + 1, ANP = ANJ * ANK, ANC = AJ * AK;
constexpr int ARF = 17, ACF = 18;  // raw floats per node, cell floats
// raw node fields
enum { RU = 0, RV = 3, RUB = 6, RVB = 9, RA = 12, RG = 15, RM = 16 };
constexpr size_t kAdjSmem = sizeof(float) * (3 * ARF * ANP + 2 * ACF * ANC);

__global__ void __launch_bounds__(AJ * AK, 2) k_adj_step(AdjArgs A) {
    extern __shared__ float sm[];
    float* sR = sm;                     // [slot][field][node]
    float* sC = sm + 3 * ARF * ANP;     // [slot][field][cell]
    const Geom& g = A.g;
    const float dt = A.dt;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + AJ * ty;
    const int bx = blockIdx.x % A.nbx, by = blockIdx.x / A.nbx;
    const int j0 = g.i1node[0] + bx * (AJ - 1), k0 = g.i1node[1] + by * (AK - 1);
    const int L0 = g.i1node[2] + blockIdx.y * A.segl, L1 = min(L0 + A.segl - 1, g.i2node[2]);
    const int J = j0 - 1 + tx, K = k0 - 1 + ty;  // this thread's cell column

    auto issue = [&](int p) {
        float* d = sR + (p % 3) * (ARF * ANP);
        for (int n = tid; n < ANP; n += AJ * AK) {
            const int j = j0 - 1 + n % ANJ, k = k0 - 1 + n / ANJ;
            if (j <= g.nm[0] && k <= g.nm[1] && p >= 1 && p <= g.nm[2]) {
                const long long q = g.idx(j, k, p);
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    cp_async4(d + (RU + i) * ANP + n, A.u[i] + q);
                    cp_async4(d + (RV + i) * ANP + n, A.v[i] + q);
                    cp_async4(d + (RUB + i) * ANP + n, A.ubi[i] + q);
                    cp_async4(d + (RVB + i) * ANP + n, A.vbi[i] + q);
                    cp_async4(d + (RA + i) * ANP + n, A.a[i] + q);
                }
                cp_async4(d + RG * ANP + n, A.gam + q);
                cp_async4(d + RM * ANP + n, A.mr + q);
            } else {
#pragma unroll
                for (int f = 0; f < ARF; f++) d[f * ANP + n] = 0.f;
            }
        }
        cp_async_commit();
    };

    auto cells = [&](int l, bool own) {
        float* o = sC + (l & 1) * (ACF * ANC) + tid;
        if (!in_cells(g, J, K, l)) {
#pragma unroll
            for (int f = 0; f < ACF; f++) o[f * ANC] = 0.f;
            return;
        }
        const long long q = g.idx(J, K, l);
        const float r = A.vc[q], lm = A.lam[q], m2 = 2.0f * A.mu[q], yc = A.yy[q];
        const float* r0 = sR + (l % 3) * (ARF * ANP);
        const float* r1 = sR + ((l + 1) % 3) * (ARF * ANP);
        // corner values by corner id dj + 2 dk + 4 dl: w = u + g v,
        // hg1 u + dt hg2 v, fbar = mr dt (vbar + dt ubar) on force nodes
        float cw[3][8], ch[3][8], cf[3][8];
#pragma unroll
        for (int n = 0; n < 8; n++) {
            const int dj = n & 1, dk = (n >> 1) & 1, dl = n >> 2;
            const float* b = (dl ? r1 : r0) + (tx + dj) + ANJ * (ty + dk);
            const bool act = in_nodes(g, J + dj, K + dk, l + dl);
            const float gm = b[RG * ANP], mm = b[RM * ANP];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const float uu = b[(RU + i) * ANP], vv = b[(RV + i) * ANP];
                cw[i][n] = fmaf(gm, vv, uu);
                ch[i][n] = fmaf(A.dh2, vv, A.hg1 * uu);
                cf[i][n] = act ? mm * (dt * fmaf(dt, b[(RUB + i) * ANP], b[(RVB + i) * ANP])) : 0.f;
            }
        }
        // forward strain (stress.f90:251-282)
        float G[3][3];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            float W[8];
#pragma unroll
            for (int t = 0; t < 8; t++) W[t] = cw[ic][term_corner(t)];
#pragma unroll
            for (int id = 0; id < 3; id++) G[ic][id] = dot8(W, A.brh.bnc[id]);
        }
        float ed[3], eo[3];
#pragma unroll
        for (int i = 0; i < 3; i++) ed[i] = G[i][i];
        eo[0] = 0.5f * G[1][2] + 0.5f * G[2][1];
        eo[1] = 0.5f * G[0][2] + 0.5f * G[2][0];
        eo[2] = 0.5f * G[0][1] + 0.5f * G[1][0];
        // sigmabar = vc Dcn^T fbar: the node of diff_cn term t is at cell corner (1-ct, 1-kt, 1-lt)
        float F[3][8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int ct = t & 1, lt = (t >> 1) & 1, kt = (t >> 2) & 1;
            const int n = (1 - ct) + 2 * (1 - kt) + 4 * (1 - lt);
#pragma unroll
            for (int i = 0; i < 3; i++) F[i][t] = cf[i][n];
        }
        float sd[3], so[3];
#pragma unroll
        for (int i = 0; i < 3; i++) sd[i] = dot8(F[i], A.brh.bcn[i]) * r;
        so[0] = (dot8(F[1], A.brh.bcn[2]) + dot8(F[2], A.brh.bcn[1])) * r;
        so[1] = (dot8(F[0], A.brh.bcn[2]) + dot8(F[2], A.brh.bcn[0])) * r;
        so[2] = (dot8(F[0], A.brh.bcn[1]) + dot8(F[1], A.brh.bcn[0])) * r;
        // Hooke's law transposed
        const float tr = ed[0] + ed[1] + ed[2], st = sd[0] + sd[1] + sd[2];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            o[i * ANC] = m2 * sd[i] + lm * st;         // Gbar_ii
            o[(3 + i) * ANC] = 0.5f * (m2 * so[i]);    // Gbar_jk = Gbar_kj
        }
        float gy = 0.f;
        if (A.hourglass) {
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                float Hc[8], Fc[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int n = hg_corner(t);
                    Hc[t] = ch[ic][n];
                    Fc[t] = cf[ic][n];
                }
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    const float sb = -hg_sum(Fc, iq);
                    gy = gy + sb * hg_sum(Hc, iq);
                    o[(6 + 3 * iq + ic) * ANC] = yc * sb;
                }
            }
        } else {
#pragma unroll
            for (int f = 6; f < ACF; f++) o[f * ANC] = 0.f;
        }
        if (own && tx >= 1 && ty >= 1) {
            A.glam[q] = A.glam[q] + st * tr;
            A.gmu[q] = A.gmu[q] + 2.0f * (sd[0] * ed[0] + sd[1] * ed[1] + sd[2] * ed[2]) +
                       2.0f * (so[0] * eo[0] + so[1] * eo[1] + so[2] * eo[2]);
            if (A.hourglass) A.gyy[q] = A.gyy[q] + gy;
        }
    };

    auto nodes = [&](int l) {
        const int jn = j0 + tx, kn = k0 + ty;
        if (tx >= AJ - 1 || ty >= AK - 1 || jn > g.i2node[0] || kn > g.i2node[1]) return;
        const float* c0 = sC + ((l - 1) & 1) * (ACF * ANC);  // cell plane l - 1
        const float* c1 = sC + (l & 1) * (ACF * ANC);        // cell plane l
        // cells at minus the corner offsets: smem cell (tx + 1 - dj, ty + 1 - dk)
        float wb[3] = {0.f, 0.f, 0.f}, hb[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int n = term_corner(t);
            const float* b = ((n >> 2) ? c0 : c1) + (tx + 1 - (n & 1)) + AJ * (ty + 1 - ((n >> 1) & 1));
            float Gb[6];
#pragma unroll
            for (int m = 0; m < 6; m++) Gb[m] = b[m * ANC];
#pragma unroll
            for (int ic = 0; ic < 3; ic++)
#pragma unroll
                for (int id = 0; id < 3; id++) {
                    const int comp = ic == id ? ic : 3 + (3 - ic - id);
                    wb[ic] = fmaf(A.brh.bnc[id][t], Gb[comp], wb[ic]);
                }
        }
        if (A.hourglass) {
#pragma unroll
            for (int ic = 0; ic < 3; ic++)
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    float S[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        const int n = hg_corner(t);
                        S[t] = (((n >> 2) ? c0 : c1) + (tx + 1 - (n & 1)) + AJ * (ty + 1 - ((n >> 1) & 1)))[(6 + 3 * iq + ic) * ANC];
                    }
                    hb[ic] = hb[ic] + hg_sum(S, iq);
                }
        }
        const float* b = sR + (l % 3) * (ARF * ANP) + (tx + 1) + ANJ * (ty + 1);
        const long long q = g.idx(jn, kn, l);
        const float m = b[RM * ANP], gm = b[RG * ANP];
        float gmr = 0.f;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float ub = b[(RUB + i) * ANP];
            const float vt = b[(RVB + i) * ANP] + dt * ub;
            const float ab = dt * vt;
            if (m != 0.f) gmr = gmr + (b[(RA + i) * ANP] / m) * ab;
            A.ubo[i][q] = ub + wb[i] + A.hg1 * hb[i];
            A.vbo[i][q] = vt + gm * wb[i] + A.dh2 * hb[i];
        }
        A.gmr[q] = A.gmr[q] + gmr;
    };

    issue(L0 - 1);
    issue(L0);
    cp_async_wait_all();
    __syncthreads();
    issue(L0 + 1);
    cells(L0 - 1, false);
#pragma unroll 1
    for (int l = L0; l <= L1; l++) {
        cp_async_wait_all();
        __syncthreads();  // raw plane l+1 landed; cell plane l-1 and nodes(l-1) complete
        if (l + 1 <= L1) issue(l + 2);
        cells(l, true);
        __syncthreads();  // cell plane l complete
        nodes(l);
    }
    cp_async_wait_all();
}

// dL/d(moment op value) at the source cells of step n: vc * (Dcn^T fbar)
// of the injected component times d(injection)/d(value).
__global__ void k_adj_moment(AdjArgs A, const MomEntry* e, int n, double* gmom) {
    const Geom& g = A.g;
    const float h = g.h;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const MomEntry E = e[i];
        float F[3][8];
        for (int t = 0; t < 8; t++) {
            const int ct = t & 1, lt = (t >> 1) & 1, kt = (t >> 2) & 1;
            const long long nd = E.idx + (1 - ct) + (1 - kt) * g.sy + (1 - lt) * g.sz;
            const int j = (int)(nd % g.sy) + 1, k = (int)((nd / g.sy) % g.nm[1]) + 1, l = (int)(nd / g.sz) + 1;
            const bool act = in_nodes(g, j, k, l);
            for (int c = 0; c < 3; c++) F[c][t] = fbar(A, nd, act, c);
        }
        float s;
        if (E.comp < 3) s = stencil8(F[E.comp], A.br.bcn[E.comp], h);
        else {
            const int a = E.comp == 5 ? 0 : E.comp == 4 ? 0 : 1, b = E.comp == 5 ? 1 : 2;
            s = stencil8(F[a], A.br.bcn[b], h) + stencil8(F[b], A.br.bcn[a], h);
        }
        atomicAdd(gmom + E.slot, (double)(s * A.vc[E.idx] * E.w));
    }
}

// Receiver misfit sources of step n: ubar/vbar += weight * dL/d(sample).
struct Ptr3 {
    float* p[3];
};
__global__ void k_adj_recv(const RecvEntry* e, int n, int it, const float* trace, Ptr3 ub, Ptr3 vb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const RecvEntry E = e[i];
        if (it < E.it1 || (it - E.it1) % E.dit != 0) continue;
        const int sidx = (it - E.it1) / E.dit;
        if (sidx >= E.ns) continue;
        float* dst = E.disp ? ub.p[E.comp] : vb.p[E.comp];
        atomicAdd(dst + E.idx, E.r * trace[E.off + sidx]);
    }
}

// Leapfrog update of time_integration.f90:32-35 from state p (u, v, a; 9 nv
// floats) into state q, whose a is then written by the fused step.
__global__ void k_adj_advance(const float* __restrict__ p, float* __restrict__ q, long long nv, float dt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float a = p[(3 + c) * nv + i] + dt * p[(6 + c) * nv + i];
            q[(3 + c) * nv + i] = a;
            q[c * nv + i] = p[c * nv + i] + dt * a;
        }
}

// ------------------------------------------------------------ host

void adjoint_free(Solver& s) {
    AdjointState* A = s.adj;
    if (!A) return;
    for (float* p : A->ckpt) dev_free(s, p);
    dev_free(s, A->segbuf[0]);
    dev_free(s, A->segbuf[1]);
    for (int b = 0; b < 2; b++)
        for (int i = 0; i < 3; i++) { dev_free(s, A->ub[b][i]); dev_free(s, A->vb[b][i]); }
    dev_free(s, A->glam); dev_free(s, A->gmu); dev_free(s, A->gyy); dev_free(s, A->gmr);
    dev_free(s, A->recv); dev_free(s, A->trace); dev_free(s, A->mom); dev_free(s, A->gmom);
    delete A;
    s.adj = nullptr;
}

static float* dalloc(Solver& s, size_t n) {
    void* p = nullptr;
    if (dev_malloc(s, &p, sizeof(float) * std::max<size_t>(n, 1)) != cudaSuccess) {
        cudaGetLastError();
        throw SordError(SORD_E_NOMEM, "adjoint: cannot allocate device memory");
    }
    SORD_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * std::max<size_t>(n, 1), s.stream));
    return (float*)p;
}

// The class of runs whose adjoint is built here.
void adjoint_check(Solver& s) {
    const Params& P = s.prm;
    if (s.geom != GEOM_RECT) throw SordError(SORD_E_PARAM, "adjoint: rectilinear meshes only");
    if (s.g.ifn != 0) throw SordError(SORD_E_PARAM, "adjoint: no fault");
    for (int i = 0; i < 3; i++)
        if (P.bc1[i] == 10 || P.bc2[i] == 10) throw SordError(SORD_E_PARAM, "adjoint: no PML");
    for (int n = 1; n <= s.nt; n++)
        if (!s.fusable(n)) throw SordError(SORD_E_PARAM, "adjoint: every step must be a plain step (no field-I/O hooks other than outputs and '.' moment/potency ops, no-op boundary conditions)");
    if (P.nsource != 0) throw SordError(SORD_E_PARAM, "adjoint: finite source files are not supported");
}

// (u, v, a) of the solver into one state record of 9 nv floats, one kernel
struct State9 {
    const float* p[9];
};
__global__ void k_adj_save(State9 src, float* __restrict__ dst, long long nv) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 9; c++) dst[c * nv + i] = src.p[c][i];
}
static void save_state(Solver& s, float* dst) {
    const long long nv = s.g.nv;
    State9 src;
    for (int i = 0; i < 3; i++) { src.p[i] = s.d.u[i]; src.p[3 + i] = s.d.v[i]; src.p[6 + i] = s.d.w1n[i]; }
    k_adj_save<<<(unsigned)std::max(1LL, std::min((nv + 255) / 256, 148LL * 16)), 256, 0, s.stream>>>(src, dst, nv);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

int adjoint_segment(Solver& s, int seg) {
    if (seg > 0) return std::max(1, std::min(seg, std::max(s.nt, 1)));
    size_t fr = 0, tot = 0;
    SORD_CUDA(cudaMemGetInfo(&fr, &tot));
    const double all = 36.0 * (double)s.g.nv * (double)(s.nt + 1);
    if (all < 0.5 * (double)fr) return 1;
    return std::max(1, (int)std::ceil(std::sqrt((double)std::max(s.nt, 1))));
}

void adjoint_begin(Solver& s, int seg) {
    if (s.it != 0) throw SordError(SORD_E_STATE, "adjoint: the forward run must start at step 0");
    adjoint_check(s);
    adjoint_free(s);
    AdjointState* A = new AdjointState();
    s.adj = A;
    A->seg = seg;
    for (size_t i = 0; i < s.ops.size(); i++) {
        const IoOp& io = s.ops[i];
        const std::string& f = io.field;
        if (io.op == ".>" && (f == "vx" || f == "vy" || f == "vz" || f == "ux" || f == "uy" || f == "uz"))
            A->recv_ops.push_back((int)i);
        if (io.op == "." && f.size() == 3 && f[0] == 'm') A->mom_ops.push_back((int)i);
    }
    const size_t nv = (size_t)s.g.nv;
    // seg = 1: the states after every step, the last included
    const int nseg = A->seg == 1 ? s.nt + 1 : (s.nt + A->seg - 1) / A->seg;
    for (int k = 0; k < std::max(nseg, 1); k++) A->ckpt.push_back(dalloc(s, 9 * nv));
    A->nck = 1;
    save_state(s, A->ckpt[0]);
    SORD_CUDA(cudaStreamSynchronize(s.stream));
}

// After each forward segment: the state at the end of step s.it.
void adjoint_checkpoint(Solver& s) {
    AdjointState* A = s.adj;
    if (!A || (s.it >= s.nt && A->seg != 1) || A->nck >= (int)A->ckpt.size()) return;
    save_state(s, A->ckpt[A->nck++]);
}

void bare_step(Solver& s, int n, bool update, bool fold);
void moment_entries(Solver& s, int opi, std::vector<Inject>& out);
int probe_of_op(const Solver& s, size_t opi, long long* idx, float* r);

void adjoint_backward(Solver& s, int nrec, const char* const* files, const float* const* dtrace, const int* ntrace,
                      float* glam, float* gmu, float* gyy, float* gmr, double* gmom, int nmom) {
    AdjointState* A = s.adj;
    if (!A) throw SordError(SORD_E_STATE, "adjoint: no forward run recorded");
    if (s.it != s.nt) throw SordError(SORD_E_STATE, "adjoint: the forward run is not complete");
    if (nmom != (int)A->mom_ops.size())
        throw SordError(SORD_E_PARAM, "adjoint: expected " + std::to_string(A->mom_ops.size()) + " moment gradients");
    const Geom& g = s.g;
    const size_t nv = (size_t)g.nv;
    // receivers: map each file to its op and probe
    std::vector<RecvEntry> rec;
    std::vector<float> tr;
    for (int i = 0; i < nrec; i++) {
        int opi = -1;
        for (int o : A->recv_ops)
            if (s.ops[o].fname == files[i]) opi = o;
        if (opi < 0) throw SordError(SORD_E_PARAM, std::string("adjoint: no velocity/displacement receiver writes ") + files[i]);
        const IoOp& io = s.ops[opi];
        long long idx[8];
        float r[8];
        const int np = probe_of_op(s, (size_t)opi, idx, r);
        const int comp = io.field[1] - 'x';
        const int disp = io.field[0] == 'u';
        const int off = (int)tr.size();
        tr.insert(tr.end(), dtrace[i], dtrace[i] + ntrace[i]);
        for (int t = 0; t < np; t++)
            rec.push_back(RecvEntry{idx[t], comp, disp, r[t], off, io.ii[3][0], io.ii[3][2], ntrace[i]});
    }
    if (!A->ub[0][0]) {
        for (int b = 0; b < 2; b++)
            for (int i = 0; i < 3; i++) { A->ub[b][i] = dalloc(s, nv); A->vb[b][i] = dalloc(s, nv); }
        A->glam = dalloc(s, nv); A->gmu = dalloc(s, nv); A->gyy = dalloc(s, nv); A->gmr = dalloc(s, nv);
        if (A->seg > 1)
            for (int b = 0; b < 2; b++) A->segbuf[b] = dalloc(s, (size_t)A->seg * 9 * nv);
    } else {
        for (int b = 0; b < 2; b++)
            for (int i = 0; i < 3; i++) {
                SORD_CUDA(cudaMemsetAsync(A->ub[b][i], 0, sizeof(float) * nv, s.stream));
                SORD_CUDA(cudaMemsetAsync(A->vb[b][i], 0, sizeof(float) * nv, s.stream));
            }
        for (float* p : {A->glam, A->gmu, A->gyy, A->gmr}) SORD_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * nv, s.stream));
    }
    dev_free(s, A->recv); dev_free(s, A->trace); dev_free(s, A->gmom); dev_free(s, A->mom);
    A->recv = nullptr; A->trace = nullptr; A->gmom = nullptr; A->mom = nullptr;
    A->nrecv = (int)rec.size();
    if (!rec.empty()) {
        SORD_CUDA(dev_malloc(s, (void**)&A->recv, sizeof(RecvEntry) * rec.size()));
        SORD_CUDA(cudaMemcpyAsync(A->recv, rec.data(), sizeof(RecvEntry) * rec.size(), cudaMemcpyHostToDevice, s.stream));
    }
    A->trace = dalloc(s, tr.size());
    if (!tr.empty()) SORD_CUDA(cudaMemcpyAsync(A->trace, tr.data(), sizeof(float) * tr.size(), cudaMemcpyHostToDevice, s.stream));
    // gradient slots: nmom values, then per op its delay and its x y z position
    const int nslot = 5 * std::max(nmom, 1);
    SORD_CUDA(dev_malloc(s, (void**)&A->gmom, sizeof(double) * nslot));
    SORD_CUDA(cudaMemsetAsync(A->gmom, 0, sizeof(double) * nslot, s.stream));
    // moment-source entries of every step, uploaded once: me[moff[n] .. moff[n+1]).
    // An injection is val tf(t - t0) r(x1); d/d val = tf r, d/d t0 = -val tf' r,
    // d/d x1 = val tf dr/dx1 (per metre: divided by the spacing).
    std::vector<MomEntry> me;
    std::vector<int> moff(s.nt + 2, 0);
    for (int n = 1; n <= s.nt; n++) {
        moff[n] = (int)me.size();
        s.it = n;
        s.tm = s.prm.tm0 + g.dt * (float)(n - 1);
        for (size_t m = 0; m < A->mom_ops.size(); m++) {
            IoOp& io = s.ops[A->mom_ops[m]];
            std::vector<Inject> e;
            moment_entries(s, A->mom_ops[m], e);
            if (e.empty()) continue;
            for (const Inject& x : e)
                if (io.val != 0.f) me.push_back(MomEntry{x.idx, x.comp, (int)m, x.inc / io.val});
            std::vector<PointWeight> pw;
            FieldView cells{s.d.sd[0], {g.nm[0], g.nm[1], g.nm[2]}};
            point_weights(s, io, cells, pw);
            const double tf = host_time_function(io.fname, s.tm, g.dt, io.tau);
            const double rate = host_time_function_rate(io.fname, (double)s.tm, (double)io.tau);
            for (const PointWeight& w : pw) {
                const int comp = e[0].comp;
                me.push_back(MomEntry{w.idx, comp, nmom + (int)m, (float)(-(double)io.val * rate * w.r)});
                for (int d = 0; d < 3; d++)
                    me.push_back(MomEntry{w.idx, comp, 2 * nmom + 3 * (int)m + d,
                                          (float)((double)io.val * tf * w.dr[d] / (double)s.prm.delta[d])});
            }
        }
    }
    moff[s.nt + 1] = (int)me.size();
    SORD_CUDA(dev_malloc(s, (void**)&A->mom, sizeof(MomEntry) * std::max<size_t>(me.size(), 1)));
    if (!me.empty())
        SORD_CUDA(cudaMemcpyAsync(A->mom, me.data(), sizeof(MomEntry) * me.size(), cudaMemcpyHostToDevice, s.stream));

    AdjArgs K;
    K.g = g;
    K.br = s.br;
    for (int a = 0; a < 3; a++)
        for (int t = 0; t < 8; t++) {
            K.brh.bnc[a][t] = s.g.h * s.br.bnc[a][t];
            K.brh.bcn[a][t] = s.g.h * s.br.bcn[a][t];
        }
    K.lam = s.d.lam; K.mu = s.d.mu; K.yy = s.d.yy; K.vc = s.d.vc; K.mr = s.d.mr; K.gam = s.d.gam;
    K.glam = A->glam; K.gmu = A->gmu; K.gyy = A->gyy; K.gmr = A->gmr;
    K.hg1 = s.prm.hourglass[0];
    K.dh2 = g.dt * s.prm.hourglass[1];
    K.dt = g.dt;
    K.hourglass = (s.prm.hourglass[0] > 0.f || s.prm.hourglass[1] > 0.f) ? 1 : 0;
    // tiles over the force nodes; planes split so that each SM gets a few blocks
    int sms = 148;
    SORD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device));
    K.nbx = (g.i2node[0] - g.i1node[0] + AJ - 1) / (AJ - 1);
    const int nby = (g.i2node[1] - g.i1node[1] + AK - 1) / (AK - 1);
    const int planes = g.i2node[2] - g.i1node[2] + 1;
    const int nsg = std::max(1, std::min((4 * sms + K.nbx * nby - 1) / (K.nbx * nby), planes / 8));
    K.segl = (planes + nsg - 1) / nsg;
    const dim3 agrid((unsigned)(K.nbx * nby), (unsigned)((planes + K.segl - 1) / K.segl));
    smem_limit((const void*)k_adj_step, (int)kAdjSmem);
    int cur = 0;  // buffer holding the adjoint state of step n + 1
    // the solver's own state arrays: recomputation points u, v, w1n into the
    // segment buffer; this guard puts them back on every exit
    struct Live {
        Solver& s;
        float* p[15];
        explicit Live(Solver& s_) : s(s_) {
            for (int i = 0; i < 3; i++) {
                p[i] = s.d.u[i]; p[3 + i] = s.d.v[i]; p[6 + i] = s.d.w1n[i]; p[9 + i] = s.d.ub[i]; p[12 + i] = s.d.vb[i];
            }
        }
        void restore() {
            for (int i = 0; i < 3; i++) {
                s.d.u[i] = p[i]; s.d.v[i] = p[3 + i]; s.d.w1n[i] = p[6 + i]; s.d.ub[i] = p[9 + i]; s.d.vb[i] = p[12 + i];
            }
        }
        ~Live() { restore(); }
    } live(s);
    // device time of the backward pass (sord_last_step_ms), set-up and
    // allocations excluded
    SORD_CUDA(cudaEventRecord(s.ev0, s.stream));

    const int seg = A->seg;
    const int nseg = (s.nt + seg - 1) / seg;
    if (A->nck < (seg == 1 ? s.nt + 1 : nseg)) throw SordError(SORD_E_STATE, "adjoint: missing checkpoints");
    // The adjoint steps run on their own stream, so that the recomputation of
    // segment k - 1 (on the solver's stream, into the other segment buffer)
    // overlaps the adjoint pass over segment k.
    struct Streams {
        cudaStream_t as = nullptr;
        cudaEvent_t ev[5] = {};  // rec_done[2], adj_done[2], start
        ~Streams() {
            for (auto e : ev) if (e) cudaEventDestroy(e);
            if (as) cudaStreamDestroy(as);
        }
    } S;
    SORD_CUDA(cudaStreamCreateWithFlags(&S.as, cudaStreamNonBlocking));
    for (auto& e : S.ev) SORD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaEvent_t* rec_done = S.ev;
    cudaEvent_t* adj_done = S.ev + 2;
    SORD_CUDA(cudaEventRecord(S.ev[4], s.stream));
    SORD_CUDA(cudaStreamWaitEvent(S.as, S.ev[4], 0));
    auto recompute = [&](int k) {
        const int n0 = k * seg, n1 = std::min(s.nt, n0 + seg);
        float* base = A->segbuf[k & 1];
        // the buffer was last read by the adjoint pass over segment k + 2
        SORD_CUDA(cudaStreamWaitEvent(s.stream, adj_done[k & 1], 0));
        // from the checkpoint straight into the segment buffer: the leapfrog
        // update of the first step reads the checkpoint, then each fused step
        // runs on state n in place and writes u, v of step n + 1 into the
        // next state (the folded update)
        k_adj_advance<<<std::max(1LL, std::min((long long)(nv + 255) / 256, 148LL * 16)), 256, 0, s.stream>>>(
            A->ckpt[k], base, (long long)nv, g.dt);
        s.launches++;
        for (int n = n0 + 1; n <= n1; n++) {
            float* st = base + (size_t)(n - n0 - 1) * 9 * nv;
            const bool fold = n < n1;
            for (int i = 0; i < 3; i++) {
                s.d.u[i] = st + i * nv; s.d.v[i] = st + (3 + i) * nv; s.d.w1n[i] = st + (6 + i) * nv;
                if (fold) { s.d.ub[i] = st + (9 + i) * nv; s.d.vb[i] = st + (12 + i) * nv; }
            }
            bare_step(s, n, false, fold);
        }
        live.restore();
        SORD_CUDA(cudaEventRecord(rec_done[k & 1], s.stream));
    };
    if (seg > 1) recompute(nseg - 1);
    for (int k = nseg - 1; k >= 0; k--) {
        const int n0 = k * seg, n1 = std::min(s.nt, n0 + seg);
        if (seg > 1) {
            if (k > 0) recompute(k - 1);
            SORD_CUDA(cudaStreamWaitEvent(S.as, rec_done[k & 1], 0));
        }
        for (int n = n1; n >= n0 + 1; n--) {
            const float* st = seg > 1 ? A->segbuf[k & 1] + (size_t)(n - n0 - 1) * 9 * nv : A->ckpt[n];
            for (int i = 0; i < 3; i++) {
                K.u[i] = st + i * nv; K.v[i] = st + (3 + i) * nv; K.a[i] = st + (6 + i) * nv;
                K.ubi[i] = A->ub[cur][i]; K.vbi[i] = A->vb[cur][i];
                K.ubo[i] = A->ub[1 - cur][i]; K.vbo[i] = A->vb[1 - cur][i];
            }
            // moment sources of step n
            const int nme = moff[n + 1] - moff[n];
            if (nme > 0) k_adj_moment<<<1, 128, 0, S.as>>>(K, A->mom + moff[n], nme, A->gmom);
            k_adj_step<<<agrid, dim3(AJ, AK), kAdjSmem, S.as>>>(K);
            cur = 1 - cur;
            if (A->nrecv) {
                Ptr3 pu{{A->ub[cur][0], A->ub[cur][1], A->ub[cur][2]}}, pv{{A->vb[cur][0], A->vb[cur][1], A->vb[cur][2]}};
                k_adj_recv<<<std::max(1, (A->nrecv + 255) / 256), 256, 0, S.as>>>(A->recv, A->nrecv, n, A->trace, pu, pv);
            }
            s.launches += 1 + (nme > 0 ? 1 : 0) + (A->nrecv ? 1 : 0);
            SORD_CUDA(cudaGetLastError());
        }
        SORD_CUDA(cudaEventRecord(adj_done[k & 1], S.as));
    }
    // join the adjoint stream back into the solver's
    SORD_CUDA(cudaEventRecord(S.ev[4], S.as));
    SORD_CUDA(cudaStreamWaitEvent(s.stream, S.ev[4], 0));
    s.it = s.nt;
    SORD_CUDA(cudaEventRecord(s.ev1, s.stream));
    SORD_CUDA(cudaEventSynchronize(s.ev1));
    float ms = 0;
    SORD_CUDA(cudaEventElapsedTime(&ms, s.ev0, s.ev1));
    s.last_step_ms = ms;
    // gradients of the real cells and nodes, global order (j fastest)
    std::vector<float> buf(nv);
    auto out = [&](const float* d, float* host, bool cell) {
        if (!host) return;
        SORD_CUDA(cudaMemcpyAsync(buf.data(), d, sizeof(float) * nv, cudaMemcpyDeviceToHost, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
        const int e0 = s.g.nn[0] - (cell ? 1 : 0), e1 = s.g.nn[1] - (cell ? 1 : 0), e2 = s.g.nn[2] - (cell ? 1 : 0);
        size_t o = 0;
        for (int l = 1; l <= e2; l++)
            for (int k = 1; k <= e1; k++)
                for (int j = 1; j <= e0; j++) host[o++] = buf[g.idx(j - g.nnoff[0], k - g.nnoff[1], l - g.nnoff[2])];
    };
    out(A->glam, glam, true);
    out(A->gmu, gmu, true);
    out(A->gyy, gyy, true);
    out(A->gmr, gmr, false);
    A->gsrc.assign(5 * (size_t)std::max(nmom, 1), 0.0);
    SORD_CUDA(cudaMemcpyAsync(A->gsrc.data(), A->gmom, sizeof(double) * A->gsrc.size(), cudaMemcpyDeviceToHost,
                              s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    if (gmom && nmom > 0) std::copy(A->gsrc.begin(), A->gsrc.begin() + nmom, gmom);
    A->gsrc.erase(A->gsrc.begin(), A->gsrc.begin() + std::max(nmom, 1));
}

// Delay (t0) and position gradients of each '.' moment op from the last
// backward pass: gx[3 m + d] = dL/d(position d of op m) per metre, gt[m] =
// dL/d(delay of op m's time function) per second.
void adjoint_source_gradients(Solver& s, double* gx, double* gt, int nmom) {
    AdjointState* A = s.adj;
    if (!A || A->gsrc.empty()) throw SordError(SORD_E_STATE, "adjoint: no backward pass recorded");
    if (nmom != (int)A->mom_ops.size())
        throw SordError(SORD_E_PARAM, "adjoint: expected " + std::to_string(A->mom_ops.size()) + " moment ops");
    for (int m = 0; m < nmom; m++) {
        if (gt) gt[m] = A->gsrc[m];
        for (int d = 0; d < 3; d++)
            if (gx) gx[3 * m + d] = A->gsrc[nmom + 3 * m + d];
    }
}

}  // namespace sordgpu

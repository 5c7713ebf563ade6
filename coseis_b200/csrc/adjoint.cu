// Discrete adjoint of the SORD time loop for gradients of a receiver misfit
// (no counterpart in the reference, which has no derivatives).
//
// The forward step n (sord/sord.f90:39-47 without field-I/O hooks) is, for
// the supported class (rectilinear mesh, no fault, free, PML or other no-op
// boundary conditions), away from the PML bands:
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
// Runs without PML take one fused kernel per adjoint step (k_adj_step); runs
// with PML take a cell pass and a node pass (k_adjp_cells, k_adjp_nodes) that
// add the transposed PML recursions (see there).
//
// Memory: the forward stores (u, v, a), with PML also the cell and node
// memories, every `seg` steps; the backward pass
// recomputes each segment from its checkpoint into a segment buffer and runs
// the adjoint steps of the segment from it (uniform checkpointing:
// 1 forward + 1 recomputation + the adjoint).  With seg = 1 every state is
// kept and nothing is recomputed; segment 0 picks that when all states fit
// in half of the free device memory, else segments of about sqrt(nt).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
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
    // A state record: (u, v, a) in 9 nv floats, then with PML the cell and
    // node memories of the step (g slabs at gofs, p slabs at pofs).
    size_t rsz = 0;
    size_t gofs[6] = {}, pofs[6] = {}, gsz[6] = {}, psz[6] = {};
    bool pml = false;
    std::vector<float*> ckpt;  // records at steps 0, seg, 2 seg, ...
    float* segbuf[2] = {};     // two segment buffers of seg records
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
    // binomial schedule: snaps records hold S_0 and the states the
    // recursion keeps, one more the state the forward run ends with;
    // recpos[r] = the step whose state record r holds (-1 free)
    int snaps = 0;
    bool spent = false;         // the backward pass has run
    std::vector<int> recpos;
    std::vector<int> stops;     // forward: steps after which a state is kept
    float* work[3] = {};        // recomputation records
    float* gbar[6] = {};        // PML: adjoint cell and node memories
    float* pbar[6] = {};
    float* cs = nullptr;        // PML: CS_COUNT cell volumes of the cell pass
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
    // the nodes this kernel updates (and the cells, by lower corner, whose
    // gradients it accumulates): all force nodes, or with PML the box whose
    // 8 cells and their corners lie outside every PML band
    int box1[3], box2[3];
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
    const int j0 = A.box1[0] + bx * (AJ - 1), k0 = A.box1[1] + by * (AK - 1);
    const int L0 = A.box1[2] + blockIdx.y * A.segl, L1 = min(L0 + A.segl - 1, A.box2[2]);
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
        if (own && tx >= 1 && ty >= 1 && J <= A.box2[0] && K <= A.box2[1]) {
            A.glam[q] = A.glam[q] + st * tr;
            A.gmu[q] = A.gmu[q] + 2.0f * (sd[0] * ed[0] + sd[1] * ed[1] + sd[2] * ed[2]) +
                       2.0f * (so[0] * eo[0] + so[1] * eo[1] + so[2] * eo[2]);
            if (A.hourglass) A.gyy[q] = A.gyy[q] + gy;
        }
    };

    auto nodes = [&](int l) {
        const int jn = j0 + tx, kn = k0 + ty;
        if (tx >= AJ - 1 || ty >= AK - 1 || jn > A.box2[0] || kn > A.box2[1]) return;
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

// ------------------------------------------------ the adjoint step with PML
//
// With PML faces the step carries two more linear recursions
// (sord/stress.f90:42-131, sord/acceleration.f90:37-104): in the cell band of
// direction id the strain term G_ic,id is g = dc2 Dnc_id(v_ic) + dc1 g (the
// cell memory), in the other bands of the cell u replaces w = u + gam v, and
// in the node band of id the divergence term F = Dcn_id(sigma_ic,id) becomes
// F' = dn2 F + dn1 p with p = p + dt F' (the node memory).  The hourglass
// force is the stiffness-plus-viscous form on nodes [i1pml+1, i2pml-1] and
// the viscous form dt hg2 yy Hnc(v) on the band nodes
// (sord/acceleration.f90:132-211).  The adjoint carries gbar and pbar, the
// adjoints of the two memories, backwards with the state.  It runs as two
// passes per step: a cell pass (one thread per cell) that forms sigmabar from
// the corners' force adjoints, transposes Hooke's law, advances gbar and
// writes the cell's routed strain adjoints and hourglass values to a scratch
// volume, and a node pass (one thread per node) that gathers them from the 8
// cells into ubar, vbar and advances pbar.  Cells and nodes each have one
// owner, so gbar and pbar are updated in place.  The nodes two or more
// inside every band (box1..box2: their cells and the cells' corners carry
// no PML term) are left to k_adj_step, which runs restricted to that box;
// the passes skip them, and the cells that k_adj_step owns keep their
// gradients from it.
enum {
    CS_Y = 0,     // 9: routed strain adjoint of pair (ic, id) at 3 ic + id
    CS_HE = 9,    // 12: yy sbar of the stiffness-plus-viscous hourglass (3 iq + ic)
    CS_HV = 21,   // 12: dt hg2 yy sbar of the viscous (PML) hourglass
    CS_SIG = 33,  // 6: vc sigmabar (xx yy zz yz zx xy) for the moment gradients
    CS_COUNT = 39
};

struct AdjPmlArgs {
    Geom g;
    Brackets brh;                     // brackets scaled by h
    const float *u[3], *v[3], *a[3];  // forward state of step n
    const float* gf[6];               // forward cell memories after step n
    const float *ubi[3], *vbi[3];     // adjoint state of step n + 1
    float *ubo[3], *vbo[3];           // adjoint state of step n
    float* gbar[6];                   // adjoint cell memories (in place)
    float* pbar[6];                   // adjoint node memories (in place)
    int tg[6], tp[6];                 // slab thicknesses
    const float *lam, *mu, *yy, *vc, *mr, *gam, *pmlc;
    float *glam, *gmu, *gyy, *gmr;
    float* cs;                        // CS_COUNT cell volumes
    float hg1, dh2, dt;
    int hourglass, hgvisc;
    int box1[3], box2[3];             // the nodes k_adj_step updates (see AdjArgs)
};
__device__ __forceinline__ bool node_in_box(const int* b1, const int* b2, int j, int k, int l) {
    return j >= b1[0] && j <= b2[0] && k >= b1[1] && k <= b2[1] && l >= b1[2] && l <= b2[2];
}

// Slab element of cell or node (j, k, l), component ic: the slab of axis
// `axis` has thickness t along it and ii counts from the face
// (sord/boundary_pml.f90:40-80 layout).
__device__ __forceinline__ long long adj_slab(const Geom& g, int axis, int t, int ii, int j, int k, int l, int ic) {
    const long long e0 = axis == 0 ? t : g.nm[0], e1 = axis == 1 ? t : g.nm[1], e2 = axis == 2 ? t : g.nm[2];
    const long long a0 = axis == 0 ? ii : j - 1, a1 = axis == 1 ? ii : k - 1, a2 = axis == 2 ? ii : l - 1;
    return a0 + e0 * (a1 + e1 * a2) + (long long)ic * e0 * e1 * e2;
}
// Band of a cell along d: 1 near (slab d), 2 far (slab 3 + d), 0 none;
// `ii` the slab layer, `p` the 1-based damping profile index.
__device__ __forceinline__ int cell_band(const Geom& g, int d, int c, int& ii, int& p) {
    if (c <= g.i1pml[d]) { ii = c - g.i1cell[d]; p = c + g.nnoff[d]; return 1; }
    if (c >= g.i2pml[d] - 1) { ii = g.i2cell[d] - c; p = g.nn[d] - c - g.nnoff[d]; return 2; }
    return 0;
}
__device__ __forceinline__ int node_band(const Geom& g, int d, int c, int& ii, int& p) {
    if (c <= g.i1pml[d]) { ii = c - g.i1node[d]; p = c + g.nnoff[d]; return 1; }
    if (c >= g.i2pml[d]) { ii = g.i2node[d] - c; p = g.nn[d] - c - g.nnoff[d] + 1; return 2; }
    return 0;
}
// node of the stiffness-plus-viscous hourglass
__device__ __forceinline__ bool hg_inner(const Geom& g, int j, int k, int l) {
    return j >= g.i1pml[0] + 1 && j <= g.i2pml[0] - 1 && k >= g.i1pml[1] + 1 && k <= g.i2pml[1] - 1 &&
           l >= g.i1pml[2] + 1 && l <= g.i2pml[2] - 1;
}
__device__ __forceinline__ float adj_fbar(const AdjPmlArgs& A, long long q, int i) {
    return A.mr[q] * (A.dt * fmaf(A.dt, A.ubi[i][q], A.vbi[i][q]));
}

__global__ void __launch_bounds__(128) k_adjp_cells(AdjPmlArgs A) {
    const Geom& g = A.g;
    const int J = g.i1cell[0] + blockIdx.x * blockDim.x + threadIdx.x;
    const int K = g.i1cell[1] + blockIdx.y * blockDim.y + threadIdx.y;
    const int L = g.i1cell[2] + blockIdx.z * blockDim.z + threadIdx.z;
    if (J > g.i2cell[0] || K > g.i2cell[1] || L > g.i2cell[2]) return;
    // cells whose 8 corners k_adj_step updates are its alone; of the others
    // this pass writes the scratch values, and the gradients of those that
    // k_adj_step does not own (by lower corner)
    if (node_in_box(A.box1, A.box2, J, K, L) && node_in_box(A.box1, A.box2, J + 1, K + 1, L + 1)) return;
    const bool grad = !node_in_box(A.box1, A.box2, J, K, L);
    const long long q = g.idx(J, K, L);
    const long long nv = g.nv;
    const float dt = A.dt, r = A.vc[q], lm = A.lam[q], m2 = 2.0f * A.mu[q], yc = A.yy[q];
    int cb[3], cii[3], cp[3];
    cb[0] = cell_band(g, 0, J, cii[0], cp[0]);
    cb[1] = cell_band(g, 1, K, cii[1], cp[1]);
    cb[2] = cell_band(g, 2, L, cii[2], cp[2]);
    const bool anyb = cb[0] || cb[1] || cb[2];
    // corner force adjoints: fb per component (0 off the force nodes); Fb per
    // pair (ic, id), which passes the node memory of the band of id
    float fb[3][8];
    bool inner[8];
    float sd[3] = {0.f, 0.f, 0.f}, so[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
    for (int n = 0; n < 8; n++) {
        const int j = J + (n & 1), k = K + ((n >> 1) & 1), l = L + (n >> 2);
        const bool act = in_nodes(g, j, k, l);
        const long long qn = g.idx(j, k, l);
        inner[n] = hg_inner(g, j, k, l);
        float Fb[3][3];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            fb[ic][n] = act ? adj_fbar(A, qn, ic) : 0.f;
#pragma unroll
            for (int id = 0; id < 3; id++) Fb[ic][id] = fb[ic][n];
        }
        if (act) {
#pragma unroll
            for (int id = 0; id < 3; id++) {
                int ii, p;
                const int b = node_band(g, id, id == 0 ? j : id == 1 ? k : l, ii, p);
                if (!b) continue;
                const int sidx = b == 1 ? id : 3 + id;
                const float dn2 = A.pmlc[g.npml + p - 1];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    const float pb = A.pbar[sidx][adj_slab(g, id, A.tp[sidx], ii, j, k, l, ic)];
                    Fb[ic][id] = dn2 * fmaf(dt, pb, fb[ic][n]);
                }
            }
        }
        // the diff_cn term t whose node is this corner: t = ct + 2 lt + 4 kt
        // with corner (1 - ct, 1 - kt, 1 - lt)
        const int ct = 1 - (n & 1), kt = 1 - ((n >> 1) & 1), lt = 1 - (n >> 2);
        const int t = ct + 2 * lt + 4 * kt;
#pragma unroll
        for (int i = 0; i < 3; i++) sd[i] = fmaf(Fb[i][i], A.brh.bcn[i][t], sd[i]);
        so[0] = fmaf(Fb[1][2], A.brh.bcn[2][t], fmaf(Fb[2][1], A.brh.bcn[1][t], so[0]));
        so[1] = fmaf(Fb[0][2], A.brh.bcn[2][t], fmaf(Fb[2][0], A.brh.bcn[0][t], so[1]));
        so[2] = fmaf(Fb[0][1], A.brh.bcn[1][t], fmaf(Fb[1][0], A.brh.bcn[0][t], so[2]));
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        sd[i] = sd[i] * r;
        so[i] = so[i] * r;
        A.cs[(CS_SIG + i) * nv + q] = sd[i];
        A.cs[(CS_SIG + 3 + i) * nv + q] = so[i];
    }
    // Hooke's law transposed: Gbar_ii, and Gbar_jk = Gbar_kj
    const float st = sd[0] + sd[1] + sd[2];
    float Gd[3], Go[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        Gd[i] = m2 * sd[i] + lm * st;
        Go[i] = 0.5f * (m2 * so[i]);
    }
    // forward strain by region, routed adjoints, cell memories
    float ed[3], eo[3] = {0.f, 0.f, 0.f};
    long long cq[8];
#pragma unroll
    for (int n = 0; n < 8; n++) cq[n] = q + (n & 1) + ((n >> 1) & 1) * g.sy + (n >> 2) * g.sz;
#pragma unroll 1
    for (int ic = 0; ic < 3; ic++) {
        float U[8], W[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const long long qn = cq[term_corner(t)];
            U[t] = A.u[ic][qn];
            W[t] = fmaf(A.gam[qn], A.v[ic][qn], U[t]);
        }
#pragma unroll
        for (int id = 0; id < 3; id++) {
            float G, X = ic == id ? Gd[ic] : Go[3 - ic - id];
            if (cb[id]) {
                const int sidx = cb[id] == 1 ? id : 3 + id;
                const long long e = adj_slab(g, id, A.tg[sidx], cii[id], J, K, L, ic);
                G = A.gf[sidx][e];
                const float xt = X + A.gbar[sidx][e];
                A.gbar[sidx][e] = A.pmlc[2 * g.npml + cp[id] - 1] * xt;
                X = A.pmlc[3 * g.npml + cp[id] - 1] * xt;
            } else {
                G = dot8(anyb ? U : W, A.brh.bnc[id]);
            }
            A.cs[(CS_Y + 3 * ic + id) * nv + q] = X;
            if (ic == id) ed[ic] = G;
            else eo[3 - ic - id] = eo[3 - ic - id] + 0.5f * G;
        }
    }
    if (grad) {
        A.glam[q] = A.glam[q] + st * (ed[0] + ed[1] + ed[2]);
        A.gmu[q] = A.gmu[q] + 2.0f * (sd[0] * ed[0] + sd[1] * ed[1] + sd[2] * ed[2]) +
                   2.0f * (so[0] * eo[0] + so[1] * eo[1] + so[2] * eo[2]);
    }
    if (!A.hourglass) return;
    const bool inE = J >= g.i1pml[0] && J <= g.i2pml[0] - 1 && K >= g.i1pml[1] && K <= g.i2pml[1] - 1 &&
                     L >= g.i1pml[2] && L <= g.i2pml[2] - 1;
    const bool inV = anyb && A.hgvisc;
    float gy = 0.f;
#pragma unroll 1
    for (int ic = 0; ic < 3; ic++) {
        float Fe[8], Fv[8], Hc[8], Vc[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int n = hg_corner(t);
            const long long qn = cq[n];
            Fe[t] = inner[n] ? fb[ic][n] : 0.f;
            Fv[t] = inner[n] ? 0.f : fb[ic][n];
            Vc[t] = A.v[ic][qn];
            Hc[t] = fmaf(A.dh2, Vc[t], A.hg1 * A.u[ic][qn]);
        }
#pragma unroll
        for (int iq = 0; iq < 4; iq++) {
            const float se = inE ? -hg_sum(Fe, iq) : 0.f;
            const float sv = inV ? -hg_sum(Fv, iq) : 0.f;
            gy = gy + se * hg_sum(Hc, iq) + sv * (A.dh2 * hg_sum(Vc, iq));
            A.cs[(CS_HE + 3 * iq + ic) * nv + q] = yc * se;
            A.cs[(CS_HV + 3 * iq + ic) * nv + q] = A.dh2 * (yc * sv);
        }
    }
    if (grad) A.gyy[q] = A.gyy[q] + gy;
}

__global__ void __launch_bounds__(128) k_adjp_nodes(AdjPmlArgs A) {
    const Geom& g = A.g;
    const int j = g.i1node[0] + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = g.i1node[1] + blockIdx.y * blockDim.y + threadIdx.y;
    const int l = g.i1node[2] + blockIdx.z * blockDim.z + threadIdx.z;
    if (j > g.i2node[0] || k > g.i2node[1] || l > g.i2node[2]) return;
    if (node_in_box(A.box1, A.box2, j, k, l)) return;  // k_adj_step's node
    const long long q = g.idx(j, k, l);
    const long long nv = g.nv;
    const float dt = A.dt;
    // strain adjoints of the 8 cells: cell = node - corner of term t
    float wb[3] = {0.f, 0.f, 0.f}, ux[3] = {0.f, 0.f, 0.f}, vx[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
    for (int t = 0; t < 8; t++) {
        const int n = term_corner(t);
        const int J = j - (n & 1), K = k - ((n >> 1) & 1), L = l - (n >> 2);
        if (!in_cells(g, J, K, L)) continue;
        const long long qc = g.idx(J, K, L);
        int cb[3], ii, p;
        cb[0] = cell_band(g, 0, J, ii, p);
        cb[1] = cell_band(g, 1, K, ii, p);
        cb[2] = cell_band(g, 2, L, ii, p);
        const bool anyb = cb[0] || cb[1] || cb[2];
#pragma unroll
        for (int ic = 0; ic < 3; ic++)
#pragma unroll
            for (int id = 0; id < 3; id++) {
                const float c = A.brh.bnc[id][t] * A.cs[(CS_Y + 3 * ic + id) * nv + qc];
                if (cb[id]) vx[ic] = vx[ic] + c;
                else if (anyb) ux[ic] = ux[ic] + c;
                else wb[ic] = wb[ic] + c;
            }
    }
    float he[3] = {0.f, 0.f, 0.f}, hv[3] = {0.f, 0.f, 0.f};
    if (A.hourglass) {
        long long qc[8];
        bool ok[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int n = hg_corner(t);
            const int J = j - (n & 1), K = k - ((n >> 1) & 1), L = l - (n >> 2);
            ok[t] = in_cells(g, J, K, L);
            qc[t] = ok[t] ? g.idx(J, K, L) : 0;
        }
#pragma unroll 1
        for (int ic = 0; ic < 3; ic++)
#pragma unroll 1
            for (int iq = 0; iq < 4; iq++) {
                float Se[8], Sv[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    Se[t] = ok[t] ? A.cs[(CS_HE + 3 * iq + ic) * nv + qc[t]] : 0.f;
                    Sv[t] = ok[t] ? A.cs[(CS_HV + 3 * iq + ic) * nv + qc[t]] : 0.f;
                }
                he[ic] = he[ic] + hg_sum(Se, iq);
                hv[ic] = hv[ic] + hg_sum(Sv, iq);
            }
    }
    const float m = A.mr[q], gm = A.gam[q];
    float gmr = 0.f, fb[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float ub = A.ubi[i][q], vb = A.vbi[i][q];
        fb[i] = adj_fbar(A, q, i);
        const float vt = vb + dt * ub;
        const float ab = dt * vt;
        if (m != 0.f) gmr = gmr + (A.a[i][q] / m) * ab;
        A.ubo[i][q] = ub + wb[i] + ux[i] + A.hg1 * he[i];
        A.vbo[i][q] = vt + gm * wb[i] + vx[i] + A.dh2 * he[i] + hv[i];
    }
    A.gmr[q] = A.gmr[q] + gmr;
    // node memories: pbar(n) = pbar(n+1) + dn1 (fbar + dt pbar(n+1))
#pragma unroll
    for (int id = 0; id < 3; id++) {
        int ii, p;
        const int b = node_band(g, id, id == 0 ? j : id == 1 ? k : l, ii, p);
        if (!b) continue;
        const int sidx = b == 1 ? id : 3 + id;
        const float dn1 = A.pmlc[p - 1];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            float* P = A.pbar[sidx] + adj_slab(g, id, A.tp[sidx], ii, j, k, l, ic);
            const float pb = *P;
            *P = pb + dn1 * fmaf(dt, pb, fb[ic]);
        }
    }
}

// dL/d(moment op value) with PML: the cell pass left vc sigmabar per cell.
// A cell (by linear index) whose 8 corners all lie in the node box [b1, b2].
__device__ __forceinline__ bool cell_in_box(const Geom& g, long long idx, const int* b1, const int* b2) {
    const int j = (int)(idx % g.sy) + 1, k = (int)((idx / g.sy) % g.nm[1]) + 1, l = (int)(idx / g.sz) + 1;
    return j >= b1[0] && j + 1 <= b2[0] && k >= b1[1] && k + 1 <= b2[1] && l >= b1[2] && l + 1 <= b2[2];
}
// The entries whose cell has a corner outside the box of the fused kernel
// (k_adj_moment takes the others).
__global__ void k_adjp_moment(AdjArgs K, const float* __restrict__ sig, const MomEntry* e, int n, double* gmom) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const MomEntry E = e[i];
        if (cell_in_box(K.g, E.idx, K.box1, K.box2)) continue;
        atomicAdd(gmom + E.slot, (double)(sig[E.comp * K.g.nv + E.idx] * E.w));
    }
}

// dL/d(moment op value) at the source cells of step n: vc * (Dcn^T fbar)
// of the injected component times d(injection)/d(value).
__global__ void k_adj_moment(AdjArgs A, const MomEntry* e, int n, double* gmom) {
    const Geom& g = A.g;
    const float h = g.h;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const MomEntry E = e[i];
        if (!cell_in_box(g, E.idx, A.box1, A.box2)) continue;
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
    for (int i = 0; i < 6; i++) { dev_free(s, A->gbar[i]); dev_free(s, A->pbar[i]); }
    dev_free(s, A->cs);
    for (float* w : A->work) dev_free(s, w);
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
    // PML: the bands of opposite faces must not meet (each cell and node
    // has at most one memory per axis)
    for (int i = 0; i < 3; i++)
        if (s.g.npml > 0 && s.g.i2pml[i] - s.g.i1pml[i] < 2)
            throw SordError(SORD_E_PARAM, "adjoint: the PML bands of opposite faces overlap");
    for (int n = 1; n <= s.nt; n++)
        if (!s.fusable(n)) throw SordError(SORD_E_PARAM, "adjoint: every step must be a plain step (no field-I/O hooks other than outputs and '.' moment/potency ops, no-op boundary conditions)");
    if (P.nsource != 0) throw SordError(SORD_E_PARAM, "adjoint: finite source files are not supported");
}

// The solver's PML cell and node memories into a state record (save) or
// back from one (restore), one copy per slab.
static void pml_memories(Solver& s, float* rec, bool save) {
    AdjointState* A = s.adj;
    for (int i = 0; i < 6; i++) {
        if (A->gsz[i]) {
            float* r = rec + A->gofs[i];
            SORD_CUDA(cudaMemcpyAsync(save ? r : s.d.slabs.g[i], save ? s.d.slabs.g[i] : r, sizeof(float) * A->gsz[i],
                                      cudaMemcpyDeviceToDevice, s.stream));
        }
        if (A->psz[i]) {
            float* r = rec + A->pofs[i];
            SORD_CUDA(cudaMemcpyAsync(save ? r : s.d.slabs.p[i], save ? s.d.slabs.p[i] : r, sizeof(float) * A->psz[i],
                                      cudaMemcpyDeviceToDevice, s.stream));
        }
    }
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
    pml_memories(s, dst, true);
}

int adjoint_segment(Solver& s, int seg) {
    if (seg > 0) return std::max(1, std::min(seg, std::max(s.nt, 1)));
    size_t fr = 0, tot = 0;
    SORD_CUDA(cudaMemGetInfo(&fr, &tot));
    // one record: (u, v, a) and the PML memories
    double rec = 9.0 * (double)s.g.nv;
    for (int i = 0; i < 6; i++)
        rec += 3.0 * (double)(s.g.nv / s.g.nm[i % 3]) * (double)(s.d.slabs.tg[i] + s.d.slabs.tp[i]);
    const double all = 4.0 * rec * (double)(s.nt + 1);
    if (all < 0.5 * (double)fr) return 1;
    return std::max(1, (int)std::ceil(std::sqrt((double)std::max(s.nt, 1))));
}

// Binomial checkpointing (Griewank's revolve schedule, restated): to run the
// adjoint steps hi .. lo + 1 when the states S_lo and S_hi are kept and c
// more records are free, keep S_m at
//   m - lo = max(1, min(beta(s, r - 1), l - beta(s - 1, r - 1))),
// l = hi - lo, s = c + 1, r the least with beta(s, r) = C(s + r, s) >= l,
// reverse (m, hi] with c - 1 free records, release S_hi and reverse (lo, m]
// with c.  That split is optimal for this recursion; it recomputes
// r l - beta(s + 1, r - 1) forward steps (the first chain of splits is the
// forward run itself).
static long long beta(long long s, long long r, long long cap) {
    long long b = 1;
    for (long long i = 1; i <= r; i++) {
        b = b * (s + i) / i;
        if (b > cap) return cap + 1;
    }
    return b;
}
int binomial_split(int l, int s) {
    int r = 0;
    while (beta(s, r, l) < l) r++;
    const long long m = std::min(beta(s, r - 1, l), (long long)l - beta(s - 1, r - 1, l));
    return (int)std::max(1LL, std::min(m, (long long)l - 1));
}
// forward steps the binomial recursion takes to reverse l steps with s
// snapshots (its first chain of splits, which the forward run keeps,
// included)
long long binomial_cost(int l, int s) {
    if (l <= 1) return 0;
    // one snapshot: every state is recomputed from the first
    if (s <= 1) return (long long)l * (l - 1) / 2;
    int r = 0;
    while (beta(s, r, l) < l) r++;
    return (long long)r * l - beta(s + 1, r - 1, (long long)r * l);
}

void adjoint_begin(Solver& s, int seg, int snaps) {
    if (s.it != 0) throw SordError(SORD_E_STATE, "adjoint: the forward run must start at step 0");
    adjoint_check(s);
    adjoint_free(s);
    AdjointState* A = new AdjointState();
    s.adj = A;
    // more snapshots than steps keep every state already
    if (snaps > 0) snaps = std::min(snaps, std::max(s.nt, 1));
    A->seg = snaps > 0 ? 0 : seg;
    A->snaps = snaps;
    for (size_t i = 0; i < s.ops.size(); i++) {
        const IoOp& io = s.ops[i];
        const std::string& f = io.field;
        if (io.op == ".>" && (f == "vx" || f == "vy" || f == "vz" || f == "ux" || f == "uy" || f == "uz"))
            A->recv_ops.push_back((int)i);
        if (io.op == "." && f.size() == 3 && f[0] == 'm') A->mom_ops.push_back((int)i);
    }
    const size_t nv = (size_t)s.g.nv;
    // seg = 1: the states after every step, the last included
    const int nseg = A->seg == 1 ? s.nt + 1 : A->seg > 1 ? (s.nt + A->seg - 1) / A->seg : 0;
    // record layout: the PML memories follow (u, v, a)
    size_t o = 9 * nv;
    for (int i = 0; i < 6; i++) {
        const size_t other = (size_t)(s.g.nv / s.g.nm[i % 3]);
        A->gsz[i] = other * (size_t)s.d.slabs.tg[i] * 3;
        A->psz[i] = other * (size_t)s.d.slabs.tp[i] * 3;
        A->gofs[i] = o; o += A->gsz[i];
        A->pofs[i] = o; o += A->psz[i];
        if (A->gsz[i] || A->psz[i]) A->pml = true;
    }
    A->rsz = o;
    if (snaps > 0) {
        // the first chain of splits, which the forward run keeps, and its end
        int lo = 0;
        for (int c = snaps - 1; c >= 1 && s.nt - lo >= 2; c--) {
            lo += binomial_split(s.nt - lo, c + 1);
            A->stops.push_back(lo);
        }
        A->stops.push_back(s.nt);
        for (int k = 0; k <= snaps; k++) A->ckpt.push_back(dalloc(s, A->rsz));
        A->recpos.assign(snaps + 1, -1);
        A->recpos[0] = 0;
    } else {
        for (int k = 0; k < std::max(nseg, 1); k++) A->ckpt.push_back(dalloc(s, A->rsz));
        if (A->seg == 1)
            for (int n = 1; n <= s.nt; n++) A->stops.push_back(n);
        else
            for (int n = A->seg; n < s.nt + A->seg; n += A->seg) A->stops.push_back(std::min(n, s.nt));
    }
    A->nck = 1;
    save_state(s, A->ckpt[0]);
    SORD_CUDA(cudaStreamSynchronize(s.stream));
}

const std::vector<int>& adjoint_stops(Solver& s) { return s.adj->stops; }

// After each forward segment: the state at the end of step s.it.
void adjoint_checkpoint(Solver& s) {
    AdjointState* A = s.adj;
    if (!A) return;
    if (A->snaps > 0) {
        for (size_t r = 0; r < A->recpos.size(); r++)
            if (A->recpos[r] < 0) {
                A->recpos[r] = s.it;
                save_state(s, A->ckpt[r]);
                A->nck++;
                return;
            }
        throw SordError(SORD_E_STATE, "adjoint: no free checkpoint record");
    }
    if ((s.it >= s.nt && A->seg != 1) || A->nck >= (int)A->ckpt.size()) return;
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
        if (A->pml) {
            for (int i = 0; i < 6; i++) {
                A->gbar[i] = dalloc(s, A->gsz[i]);
                A->pbar[i] = dalloc(s, A->psz[i]);
            }
            A->cs = dalloc(s, (size_t)CS_COUNT * nv);
        }
        if (A->seg > 1)
            for (int b = 0; b < 2; b++) A->segbuf[b] = dalloc(s, (size_t)A->seg * A->rsz);
    } else {
        for (int b = 0; b < 2; b++)
            for (int i = 0; i < 3; i++) {
                SORD_CUDA(cudaMemsetAsync(A->ub[b][i], 0, sizeof(float) * nv, s.stream));
                SORD_CUDA(cudaMemsetAsync(A->vb[b][i], 0, sizeof(float) * nv, s.stream));
            }
        for (float* p : {A->glam, A->gmu, A->gyy, A->gmr}) SORD_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * nv, s.stream));
        if (A->pml)
            for (int i = 0; i < 6; i++) {
                if (A->gsz[i]) SORD_CUDA(cudaMemsetAsync(A->gbar[i], 0, sizeof(float) * A->gsz[i], s.stream));
                if (A->psz[i]) SORD_CUDA(cudaMemsetAsync(A->pbar[i], 0, sizeof(float) * A->psz[i], s.stream));
            }
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
    // the nodes of the fused kernel: all force nodes, or with PML those two
    // nodes or more inside every band (their cells and the cells' corners
    // carry no PML term); the two-pass kernels take the rest
    bool fused_box = true;
    for (int d = 0; d < 3; d++) {
        K.box1[d] = g.i1node[d];
        K.box2[d] = g.i2node[d];
        if (A->pml) {
            if (g.i1pml[d] >= g.i1node[d]) K.box1[d] = g.i1pml[d] + 2;
            if (g.i2pml[d] <= g.i2node[d]) K.box2[d] = g.i2pml[d] - 2;
        }
        if (K.box1[d] > K.box2[d]) fused_box = false;
    }
    if (!fused_box)
        for (int d = 0; d < 3; d++) { K.box1[d] = 1; K.box2[d] = 0; }
    K.nbx = std::max(1, (K.box2[0] - K.box1[0] + AJ - 1) / (AJ - 1));
    const int nby = std::max(1, (K.box2[1] - K.box1[1] + AK - 1) / (AK - 1));
    const int planes = std::max(1, K.box2[2] - K.box1[2] + 1);
    const int nsg = std::max(1, std::min((4 * sms + K.nbx * nby - 1) / (K.nbx * nby), planes / 8));
    K.segl = (planes + nsg - 1) / nsg;
    const dim3 agrid((unsigned)(K.nbx * nby), (unsigned)((planes + K.segl - 1) / K.segl));
    smem_limit((const void*)k_adj_step, (int)kAdjSmem);
    // PML runs: the two-pass step over cells and nodes
    AdjPmlArgs KP{};
    KP.g = g;
    KP.brh = K.brh;
    for (int i = 0; i < 6; i++) {
        KP.gbar[i] = A->gbar[i]; KP.pbar[i] = A->pbar[i];
        KP.tg[i] = s.d.slabs.tg[i]; KP.tp[i] = s.d.slabs.tp[i];
    }
    KP.lam = s.d.lam; KP.mu = s.d.mu; KP.yy = s.d.yy; KP.vc = s.d.vc; KP.mr = s.d.mr; KP.gam = s.d.gam;
    KP.pmlc = s.d.pmlc;
    KP.glam = A->glam; KP.gmu = A->gmu; KP.gyy = A->gyy; KP.gmr = A->gmr;
    KP.cs = A->cs;
    KP.hg1 = K.hg1; KP.dh2 = K.dh2; KP.dt = K.dt;
    KP.hourglass = K.hourglass;
    KP.hgvisc = (s.prm.hourglass[1] > 0.f && g.npml > 0) ? 1 : 0;
    for (int d = 0; d < 3; d++) { KP.box1[d] = K.box1[d]; KP.box2[d] = K.box2[d]; }
    const dim3 pblock(32, 4, 1);
    auto pgrid = [&](const int* i1, const int* i2) {
        return dim3((unsigned)((i2[0] - i1[0] + 32) / 32), (unsigned)((i2[1] - i1[1] + 4) / 4), (unsigned)(i2[2] - i1[2] + 1));
    };
    const dim3 pcgrid = pgrid(g.i1cell, g.i2cell), pngrid = pgrid(g.i1node, g.i2node);
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
    const int nseg = seg > 0 ? (s.nt + seg - 1) / seg : 0;
    if (A->snaps == 0 && A->nck < (seg == 1 ? s.nt + 1 : nseg))
        throw SordError(SORD_E_STATE, "adjoint: missing checkpoints");
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
    // adjoint step n on the forward state record st, on stream `as`
    auto adjoint_step = [&](int n, const float* st, cudaStream_t as) {
        for (int i = 0; i < 3; i++) {
            K.u[i] = st + i * nv; K.v[i] = st + (3 + i) * nv; K.a[i] = st + (6 + i) * nv;
            K.ubi[i] = A->ub[cur][i]; K.vbi[i] = A->vb[cur][i];
            K.ubo[i] = A->ub[1 - cur][i]; K.vbo[i] = A->vb[1 - cur][i];
        }
        // moment sources of step n
        const int nme = moff[n + 1] - moff[n];
        if (A->pml) {
            for (int i = 0; i < 3; i++) {
                KP.u[i] = K.u[i]; KP.v[i] = K.v[i]; KP.a[i] = K.a[i];
                KP.ubi[i] = K.ubi[i]; KP.vbi[i] = K.vbi[i]; KP.ubo[i] = K.ubo[i]; KP.vbo[i] = K.vbo[i];
            }
            for (int i = 0; i < 6; i++) KP.gf[i] = st + A->gofs[i];
            // the fused kernel on the nodes away from the PML, the two
            // passes on the rest (they write disjoint nodes and cells)
            if (fused_box) {
                if (nme > 0) k_adj_moment<<<1, 128, 0, as>>>(K, A->mom + moff[n], nme, A->gmom);
                k_adj_step<<<agrid, dim3(AJ, AK), kAdjSmem, as>>>(K);
                s.launches += 1 + (nme > 0 ? 1 : 0);
            }
            k_adjp_cells<<<pcgrid, pblock, 0, as>>>(KP);
            if (nme > 0) k_adjp_moment<<<1, 128, 0, as>>>(K, A->cs + (size_t)CS_SIG * nv, A->mom + moff[n], nme, A->gmom);
            k_adjp_nodes<<<pngrid, pblock, 0, as>>>(KP);
            s.launches++;
        } else {
            if (nme > 0) k_adj_moment<<<1, 128, 0, as>>>(K, A->mom + moff[n], nme, A->gmom);
            k_adj_step<<<agrid, dim3(AJ, AK), kAdjSmem, as>>>(K);
        }
        cur = 1 - cur;
        if (A->nrecv) {
            Ptr3 pu{{A->ub[cur][0], A->ub[cur][1], A->ub[cur][2]}}, pv{{A->vb[cur][0], A->vb[cur][1], A->vb[cur][2]}};
            k_adj_recv<<<std::max(1, (A->nrecv + 255) / 256), 256, 0, as>>>(A->recv, A->nrecv, n, A->trace, pu, pv);
        }
        s.launches += 1 + (nme > 0 ? 1 : 0) + (A->nrecv ? 1 : 0);
        SORD_CUDA(cudaGetLastError());
    };
    // recompute S_n from the record `from` of step lo into `dst`: a chain of
    // folded steps through two work records, the last one landing in dst
    auto advance_to = [&](float* from, int lo, int n, float* dst) {
        auto rec = [&](int k) { return k == n ? dst : A->work[(n - k) & 1]; };
        k_adj_advance<<<std::max(1LL, std::min((long long)(nv + 255) / 256, 148LL * 16)), 256, 0, s.stream>>>(
            from, rec(lo + 1), (long long)nv, g.dt);
        s.launches++;
        if (A->pml) pml_memories(s, from, false);
        for (int k = lo + 1; k <= n; k++) {
            float* st = rec(k);
            const bool fold = k < n;
            for (int i = 0; i < 3; i++) {
                s.d.u[i] = st + i * nv; s.d.v[i] = st + (3 + i) * nv; s.d.w1n[i] = st + (6 + i) * nv;
                if (fold) { s.d.ub[i] = rec(k + 1) + i * nv; s.d.vb[i] = rec(k + 1) + (3 + i) * nv; }
            }
            bare_step(s, k, false, fold);
        }
        if (A->pml) pml_memories(s, dst, true);
        live.restore();
    };
    if (A->snaps > 0) {
        // binomial schedule, everything on the solver's stream
        for (int w = 0; w < 3; w++)
            if (!A->work[w]) A->work[w] = dalloc(s, A->rsz);
        auto rec_of = [&](int pos) {
            for (size_t r = 0; r < A->recpos.size(); r++)
                if (A->recpos[r] == pos) return (int)r;
            return -1;
        };
        auto take = [&](int pos) {
            for (size_t r = 0; r < A->recpos.size(); r++)
                if (A->recpos[r] < 0) { A->recpos[r] = pos; return (int)r; }
            throw SordError(SORD_E_STATE, "adjoint: no free checkpoint record");
        };
        // the adjoint steps hi, hi - 1, ..., lo + 1, with S_lo in record rlo,
        // S_hi in record rhi and c more records free; record rhi is
        // released once step hi has run, rlo stays with the caller
        std::function<void(int, int, int, int, int)> rev = [&](int lo, int hi, int c, int rlo, int rhi) {
            if (hi - lo == 1) {
                adjoint_step(hi, A->ckpt[rhi], s.stream);
                A->recpos[rhi] = -1;
                return;
            }
            if (c == 0) {
                adjoint_step(hi, A->ckpt[rhi], s.stream);
                A->recpos[rhi] = -1;
                for (int n = hi - 1; n > lo; n--) {
                    advance_to(A->ckpt[rlo], lo, n, A->work[2]);
                    adjoint_step(n, A->work[2], s.stream);
                }
                return;
            }
            const int m = lo + binomial_split(hi - lo, c + 1);
            int rm = rec_of(m);  // the forward run keeps the first chain
            if (rm < 0) {
                rm = take(m);
                advance_to(A->ckpt[rlo], lo, m, A->ckpt[rm]);
            }
            rev(m, hi, c - 1, rm, rhi);
            rev(lo, m, c, rlo, rm);
        };
        // the records are reused as the recursion goes: one backward pass
        // per forward run
        if (A->spent) throw SordError(SORD_E_STATE, "adjoint: binomial checkpointing allows one backward pass per forward run");
        A->spent = true;
        const int rend = rec_of(s.nt);
        if (rend < 0 || A->recpos[0] != 0) throw SordError(SORD_E_STATE, "adjoint: missing checkpoints");
        if (s.nt > 0) rev(0, s.nt, A->snaps - 1, 0, rend);
    } else {
        auto recompute = [&](int k) {
            const int n0 = k * seg, n1 = std::min(s.nt, n0 + seg);
            float* base = A->segbuf[k & 1];
            // the buffer was last read by the adjoint pass over segment k + 2
            SORD_CUDA(cudaStreamWaitEvent(s.stream, adj_done[k & 1], 0));
            // from the checkpoint straight into the segment buffer: the
            // leapfrog update of the first step reads the checkpoint, then
            // each fused step runs on state n in place and writes u, v of
            // step n + 1 into the next state (the folded update)
            k_adj_advance<<<std::max(1LL, std::min((long long)(nv + 255) / 256, 148LL * 16)), 256, 0, s.stream>>>(
                A->ckpt[k], base, (long long)nv, g.dt);
            s.launches++;
            // the PML memories of the checkpoint into the solver's slabs; each
            // recomputed step's memories into its record
            if (A->pml) pml_memories(s, A->ckpt[k], false);
            for (int n = n0 + 1; n <= n1; n++) {
                float* st = base + (size_t)(n - n0 - 1) * A->rsz;
                const bool fold = n < n1;
                for (int i = 0; i < 3; i++) {
                    s.d.u[i] = st + i * nv; s.d.v[i] = st + (3 + i) * nv; s.d.w1n[i] = st + (6 + i) * nv;
                    if (fold) { s.d.ub[i] = st + A->rsz + i * nv; s.d.vb[i] = st + A->rsz + (3 + i) * nv; }
                }
                bare_step(s, n, false, fold);
                if (A->pml) pml_memories(s, st, true);
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
            for (int n = n1; n >= n0 + 1; n--)
                adjoint_step(n, seg > 1 ? A->segbuf[k & 1] + (size_t)(n - n0 - 1) * A->rsz : A->ckpt[n], S.as);
            SORD_CUDA(cudaEventRecord(adj_done[k & 1], S.as));
        }
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

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
    float* segbuf = nullptr;   // seg states of 9 nv floats
    float* ub[3] = {};
    float* vb[3] = {};
    float* fb[3] = {};
    float* cs = nullptr;       // 18 nv cell values
    float *glam = nullptr, *gmu = nullptr, *gyy = nullptr, *gmr = nullptr;
    RecvEntry* recv = nullptr;
    int nrecv = 0;
    float* trace = nullptr;
    MomEntry* mom = nullptr;
    double* gmom = nullptr;
    int nmomslot = 0;
    std::vector<int> recv_ops;  // op indices of '.>' receivers, recorded before the forward run
    std::vector<int> mom_ops;   // op indices of '.' moment ops
};

// ------------------------------------------------------------ kernels
struct AdjArgs {
    Geom g;
    Brackets br;
    const float *u[3], *v[3], *a[3];  // forward state of step n
    float *ub[3], *vb[3], *fb[3];
    float* cs;
    const float *lam, *mu, *yy, *vc, *mr, *gam;
    float *glam, *gmu, *gyy, *gmr;
    float hg1, dh2;
    int hourglass;
};

__device__ __forceinline__ void node_jkl(const Geom& g, long long q, int& j, int& k, int& l) {
    j = (int)(q % g.sy) + 1;
    k = (int)((q / g.sy) % g.nm[1]) + 1;
    l = (int)(q / g.sz) + 1;
}
__device__ __forceinline__ bool in_nodes(const Geom& g, int j, int k, int l) {
    return j >= g.i1node[0] && j <= g.i2node[0] && k >= g.i1node[1] && k <= g.i2node[1] && l >= g.i1node[2] &&
           l <= g.i2node[2];
}
__device__ __forceinline__ bool in_cells(const Geom& g, int j, int k, int l) {
    return j >= g.i1cell[0] && j <= g.i2cell[0] && k >= g.i1cell[1] && k <= g.i2cell[1] && l >= g.i1cell[2] &&
           l <= g.i2cell[2];
}

// abar = dt (vbar + dt ubar); vbar <- vbar + dt ubar; fbar = mr abar on the
// force nodes; dL/dmr += f . abar with f = a / mr.
__global__ void k_adj_mass(AdjArgs A, float dt) {
    const Geom& g = A.g;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int j, k, l;
        node_jkl(g, q, j, k, l);
        const bool act = in_nodes(g, j, k, l);
        const float m = A.mr[q];
        float gm = 0.f;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float vt = A.vb[i][q] + dt * A.ub[i][q];
            A.vb[i][q] = vt;
            const float ab = dt * vt;
            A.fb[i][q] = act ? m * ab : 0.f;
            if (act && m != 0.f) gm = gm + (A.a[i][q] / m) * ab;
        }
        if (act) A.gmr[q] = A.gmr[q] + gm;
    }
}

// Cell pass: forward strain of step n, sigmabar = vc Dcn^T fbar, the
// transposed Hooke law, hourglass cell adjoints; per-cell gradients.
// cs[0..2] = Gbar_ii, cs[3..5] = Gbar of the off-diagonal pairs (yz zx xy),
// cs[6 + 3 q + i] = yy * sbar_q,i.
__global__ void k_adj_cells(AdjArgs A) {
    const Geom& g = A.g;
    const float h = g.h;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nv; q += (long long)gridDim.x * blockDim.x) {
        int j, k, l;
        node_jkl(g, q, j, k, l);
        if (!in_cells(g, j, k, l)) continue;
        long long cq[8];
#pragma unroll
        for (int n = 0; n < 8; n++) cq[n] = q + (n & 1) + ((n >> 1) & 1) * g.sy + ((n >> 2) & 1) * g.sz;
        // corner values, by corner id dj + 2 dk + 4 dl
        float cu[3][8], cv[3][8], cf[3][8], cg[8];
#pragma unroll
        for (int n = 0; n < 8; n++) {
            cg[n] = __ldg(A.gam + cq[n]);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                cu[i][n] = __ldg(A.u[i] + cq[n]);
                cv[i][n] = __ldg(A.v[i] + cq[n]);
                cf[i][n] = __ldg(A.fb[i] + cq[n]);
            }
        }
        // forward strain (stress.f90:251-282), w = u + g v at the corners
        float G[3][3];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            float W[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int n = term_corner(t);
                W[t] = cu[ic][n] + cg[n] * cv[ic][n];
            }
#pragma unroll
            for (int id = 0; id < 3; id++) G[ic][id] = stencil8(W, A.br.bnc[id], h);
        }
        float ed[3], eo[3];
#pragma unroll
        for (int i = 0; i < 3; i++) ed[i] = G[i][i];
        eo[0] = 0.5f * G[1][2] + 0.5f * G[2][1];
        eo[1] = 0.5f * G[0][2] + 0.5f * G[2][0];
        eo[2] = 0.5f * G[0][1] + 0.5f * G[1][0];
        // sigmabar = Dcn^T fbar: node of diff_cn term t is c + (1-ct, 1-kt, 1-lt)
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
        for (int i = 0; i < 3; i++) sd[i] = stencil8(F[i], A.br.bcn[i], h);
        so[0] = stencil8(F[1], A.br.bcn[2], h) + stencil8(F[2], A.br.bcn[1], h);
        so[1] = stencil8(F[0], A.br.bcn[2], h) + stencil8(F[2], A.br.bcn[0], h);
        so[2] = stencil8(F[0], A.br.bcn[1], h) + stencil8(F[1], A.br.bcn[0], h);
        const float r = A.vc[q];
#pragma unroll
        for (int i = 0; i < 3; i++) { sd[i] = sd[i] * r; so[i] = so[i] * r; }
        // Hooke's law transposed; dL/dlam, dL/dmu
        const float lm = A.lam[q], m2 = 2.0f * A.mu[q];
        const float tr = ed[0] + ed[1] + ed[2], st = sd[0] + sd[1] + sd[2];
        A.glam[q] = A.glam[q] + st * tr;
        A.gmu[q] = A.gmu[q] + 2.0f * (sd[0] * ed[0] + sd[1] * ed[1] + sd[2] * ed[2]) +
                   2.0f * (so[0] * eo[0] + so[1] * eo[1] + so[2] * eo[2]);
        float* cs = A.cs;
        const long long nv = g.nv;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            cs[i * nv + q] = m2 * sd[i] + lm * st;  // Gbar_ii
            cs[(3 + i) * nv + q] = 0.5f * (m2 * so[i]);  // Gbar_ij = Gbar_ji
        }
        if (A.hourglass) {
            const float yc = A.yy[q];
            float gy = 0.f;
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                float Hc[8], Fc[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int n = hg_corner(t);
                    Hc[t] = A.hg1 * cu[ic][n] + A.dh2 * cv[ic][n];
                    Fc[t] = cf[ic][n];
                }
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    const float sb = -hg_sum(Fc, iq);
                    gy = gy + sb * hg_sum(Hc, iq);
                    cs[(6 + 3 * iq + ic) * nv + q] = yc * sb;
                }
            }
            A.gyy[q] = A.gyy[q] + gy;
        }
    }
}

// Node pass: wbar = Dnc^T Gbar, hbar = sum_q Hcn_q(yy sbar_q);
// ubar += wbar + hg1 hbar, vbar += g wbar + dt hg2 hbar.
__global__ void k_adj_nodes(AdjArgs A) {
    const Geom& g = A.g;
    const float h = g.h;
    const long long nv = g.nv;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv; q += (long long)gridDim.x * blockDim.x) {
        int j, k, l;
        node_jkl(g, q, j, k, l);
        float wb[3] = {0.f, 0.f, 0.f}, hb[3] = {0.f, 0.f, 0.f};
        const float* __restrict__ cs = A.cs;
        // cells at minus the corner offsets, by corner id dj + 2 dk + 4 dl
        bool ok[8];
        long long cc[8];
#pragma unroll
        for (int n = 0; n < 8; n++) {
            const int dj = n & 1, dk = (n >> 1) & 1, dl = n >> 2;
            ok[n] = in_cells(g, j - dj, k - dk, l - dl);
            cc[n] = q - dj - dk * g.sy - dl * g.sz;
        }
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int n = term_corner(t);
            if (!ok[n]) continue;
            float Gb[6];
#pragma unroll
            for (int m = 0; m < 6; m++) Gb[m] = __ldg(cs + m * nv + cc[n]);
#pragma unroll
            for (int ic = 0; ic < 3; ic++)
#pragma unroll
                for (int id = 0; id < 3; id++) {
                    const int comp = ic == id ? ic : 3 + (3 - ic - id);
                    wb[ic] = wb[ic] + h * A.br.bnc[id][t] * Gb[comp];
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
                        S[t] = ok[n] ? __ldg(cs + (6 + 3 * iq + ic) * nv + cc[n]) : 0.f;
                    }
                    hb[ic] = hb[ic] + hg_sum(S, iq);
                }
        }
        const float gm = A.gam[q];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            A.ub[i][q] = A.ub[i][q] + wb[i] + A.hg1 * hb[i];
            A.vb[i][q] = A.vb[i][q] + gm * wb[i] + A.dh2 * hb[i];
        }
    }
}

// dL/d(moment op value) at the source cells of step n: vc * (Dcn^T fbar)
// of the injected component times d(injection)/d(value).
__global__ void k_adj_moment(Geom g, Brackets br, const MomEntry* e, int n, float* const* fb, const float* vc,
                             double* gmom) {
    const float h = g.h;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const MomEntry E = e[i];
        float F[3][8];
        for (int t = 0; t < 8; t++) {
            const int ct = t & 1, lt = (t >> 1) & 1, kt = (t >> 2) & 1;
            const long long nd = E.idx + (1 - ct) + (1 - kt) * g.sy + (1 - lt) * g.sz;
            for (int c = 0; c < 3; c++) F[c][t] = fb[c][nd];
        }
        float s;
        if (E.comp < 3) s = stencil8(F[E.comp], br.bcn[E.comp], h);
        else {
            const int a = E.comp == 3 ? 1 : E.comp == 4 ? 0 : 0, b = E.comp == 3 ? 2 : E.comp == 4 ? 2 : 1;
            s = stencil8(F[a], br.bcn[b], h) + stencil8(F[b], br.bcn[a], h);
        }
        atomicAdd(gmom + E.slot, (double)(s * vc[E.idx] * E.w));
    }
}

// Receiver misfit sources of step n: ubar/vbar += weight * dL/d(sample).
__global__ void k_adj_recv(const RecvEntry* e, int n, int it, const float* trace, float* const* ub, float* const* vb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const RecvEntry E = e[i];
        if (it < E.it1 || (it - E.it1) % E.dit != 0) continue;
        const int sidx = (it - E.it1) / E.dit;
        if (sidx >= E.ns) continue;
        float* dst = E.disp ? ub[E.comp] : vb[E.comp];
        atomicAdd(dst + E.idx, E.r * trace[E.off + sidx]);
    }
}

// ------------------------------------------------------------ host
static unsigned gsz(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)std::max(1LL, std::min(b, 148LL * 16));
}

void adjoint_free(Solver& s) {
    AdjointState* A = s.adj;
    if (!A) return;
    for (float* p : A->ckpt) dev_free(s, p);
    dev_free(s, A->segbuf);
    for (int i = 0; i < 3; i++) { dev_free(s, A->ub[i]); dev_free(s, A->vb[i]); dev_free(s, A->fb[i]); }
    dev_free(s, A->cs);
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

static void save_state(Solver& s, float* dst) {
    const size_t nv = (size_t)s.g.nv, b = sizeof(float) * nv;
    for (int i = 0; i < 3; i++) {
        SORD_CUDA(cudaMemcpyAsync(dst + (0 + i) * nv, s.d.u[i], b, cudaMemcpyDeviceToDevice, s.stream));
        SORD_CUDA(cudaMemcpyAsync(dst + (3 + i) * nv, s.d.v[i], b, cudaMemcpyDeviceToDevice, s.stream));
        SORD_CUDA(cudaMemcpyAsync(dst + (6 + i) * nv, s.d.w1n[i], b, cudaMemcpyDeviceToDevice, s.stream));
    }
}
static void load_state(Solver& s, const float* src) {
    const size_t nv = (size_t)s.g.nv, b = sizeof(float) * nv;
    for (int i = 0; i < 3; i++) {
        SORD_CUDA(cudaMemcpyAsync(s.d.u[i], src + (0 + i) * nv, b, cudaMemcpyDeviceToDevice, s.stream));
        SORD_CUDA(cudaMemcpyAsync(s.d.v[i], src + (3 + i) * nv, b, cudaMemcpyDeviceToDevice, s.stream));
        SORD_CUDA(cudaMemcpyAsync(s.d.w1n[i], src + (6 + i) * nv, b, cudaMemcpyDeviceToDevice, s.stream));
    }
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

void bare_step(Solver& s, int n);
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
    if (!A->ub[0]) {
        for (int i = 0; i < 3; i++) { A->ub[i] = dalloc(s, nv); A->vb[i] = dalloc(s, nv); A->fb[i] = dalloc(s, nv); }
        A->cs = dalloc(s, 18 * nv);
        A->glam = dalloc(s, nv); A->gmu = dalloc(s, nv); A->gyy = dalloc(s, nv); A->gmr = dalloc(s, nv);
        if (A->seg > 1) A->segbuf = dalloc(s, (size_t)A->seg * 9 * nv);
    } else {
        for (int i = 0; i < 3; i++) {
            SORD_CUDA(cudaMemsetAsync(A->ub[i], 0, sizeof(float) * nv, s.stream));
            SORD_CUDA(cudaMemsetAsync(A->vb[i], 0, sizeof(float) * nv, s.stream));
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
    SORD_CUDA(dev_malloc(s, (void**)&A->gmom, sizeof(double) * std::max(nmom, 1)));
    SORD_CUDA(cudaMemsetAsync(A->gmom, 0, sizeof(double) * std::max(nmom, 1), s.stream));
    const int cap = 4096;
    SORD_CUDA(dev_malloc(s, (void**)&A->mom, sizeof(MomEntry) * cap));
    std::vector<MomEntry> me;
    MomEntry* hmom = (MomEntry*)pinned_get(sizeof(MomEntry) * cap);
    cudaEvent_t mev = nullptr;
    SORD_CUDA(cudaEventCreateWithFlags(&mev, cudaEventDisableTiming));
    SORD_CUDA(cudaEventRecord(mev, s.stream));

    AdjArgs K;
    K.g = g;
    K.br = s.br;
    for (int i = 0; i < 3; i++) { K.ub[i] = A->ub[i]; K.vb[i] = A->vb[i]; K.fb[i] = A->fb[i]; }
    K.cs = A->cs;
    K.lam = s.d.lam; K.mu = s.d.mu; K.yy = s.d.yy; K.vc = s.d.vc; K.mr = s.d.mr; K.gam = s.d.gam;
    K.glam = A->glam; K.gmu = A->gmu; K.gyy = A->gyy; K.gmr = A->gmr;
    K.hg1 = s.prm.hourglass[0];
    K.dh2 = g.dt * s.prm.hourglass[1];
    K.hourglass = (s.prm.hourglass[0] > 0.f || s.prm.hourglass[1] > 0.f) ? 1 : 0;
    float** dfb = nullptr;  // device copies of the three fbar / ubar / vbar pointers
    SORD_CUDA(dev_malloc(s, (void**)&dfb, sizeof(float*) * 9));
    float* hp[9] = {A->fb[0], A->fb[1], A->fb[2], A->ub[0], A->ub[1], A->ub[2], A->vb[0], A->vb[1], A->vb[2]};
    SORD_CUDA(cudaMemcpyAsync(dfb, hp, sizeof hp, cudaMemcpyHostToDevice, s.stream));

    const int seg = A->seg;
    const int nseg = (s.nt + seg - 1) / seg;
    if (A->nck < (seg == 1 ? s.nt + 1 : nseg)) throw SordError(SORD_E_STATE, "adjoint: missing checkpoints");
    const unsigned gb = gsz((long long)nv);
    for (int k = nseg - 1; k >= 0; k--) {
        const int n0 = k * seg, n1 = std::min(s.nt, n0 + seg);
        if (seg > 1) {
            load_state(s, A->ckpt[k]);
            for (int n = n0 + 1; n <= n1; n++) {
                bare_step(s, n);
                save_state(s, A->segbuf + (size_t)(n - n0 - 1) * 9 * nv);
            }
        }
        for (int n = n1; n >= n0 + 1; n--) {
            const float* st = seg > 1 ? A->segbuf + (size_t)(n - n0 - 1) * 9 * nv : A->ckpt[n];
            for (int i = 0; i < 3; i++) { K.u[i] = st + i * nv; K.v[i] = st + (3 + i) * nv; K.a[i] = st + (6 + i) * nv; }
            k_adj_mass<<<gb, 256, 0, s.stream>>>(K, g.dt);
            k_adj_cells<<<gb, 256, 0, s.stream>>>(K);
            // moment sources of step n
            me.clear();
            s.it = n;
            s.tm = s.prm.tm0 + g.dt * (float)(n - 1);
            for (size_t m = 0; m < A->mom_ops.size(); m++) {
                const IoOp& io = s.ops[A->mom_ops[m]];
                std::vector<Inject> e;
                moment_entries(s, A->mom_ops[m], e);
                for (const Inject& x : e)
                    if (io.val != 0.f) me.push_back(MomEntry{x.idx, x.comp, (int)m, x.inc / io.val});
            }
            if (!me.empty()) {
                if ((int)me.size() > cap) throw SordError(SORD_E_PARAM, "adjoint: too many moment injections in one step");
                SORD_CUDA(cudaEventSynchronize(mev));
                std::memcpy(hmom, me.data(), sizeof(MomEntry) * me.size());
                SORD_CUDA(cudaMemcpyAsync(A->mom, hmom, sizeof(MomEntry) * me.size(), cudaMemcpyHostToDevice, s.stream));
                SORD_CUDA(cudaEventRecord(mev, s.stream));
                k_adj_moment<<<1, 128, 0, s.stream>>>(g, s.br, A->mom, (int)me.size(), dfb, s.d.vc, A->gmom);
            }
            k_adj_nodes<<<gb, 256, 0, s.stream>>>(K);
            if (A->nrecv)
                k_adj_recv<<<std::max(1, (A->nrecv + 255) / 256), 256, 0, s.stream>>>(A->recv, A->nrecv, n, A->trace, dfb + 3, dfb + 6);
            s.launches += 3 + (me.empty() ? 0 : 1) + (A->nrecv ? 1 : 0);
            SORD_CUDA(cudaGetLastError());
        }
    }
    s.it = s.nt;
    SORD_CUDA(cudaEventSynchronize(mev));
    cudaEventDestroy(mev);
    pinned_put(hmom);
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
    if (gmom && nmom > 0) {
        SORD_CUDA(cudaMemcpyAsync(gmom, A->gmom, sizeof(double) * nmom, cudaMemcpyDeviceToHost, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
    }
    dev_free(s, dfb);
    SORD_CUDA(cudaStreamSynchronize(s.stream));
}

}  // namespace sordgpu

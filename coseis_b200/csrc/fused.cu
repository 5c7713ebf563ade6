// Fused step kernel: one pass over the mesh computes a whole time step of
// sord/sord.f90:42-44 for steps whose field-I/O hooks allow it:
//
//   cell phase   strain (9 support-operator gradients, PML g memory),
//                potency / moment point injections, Hooke's law, 1/V
//                (stress.f90:133-355) and the elastic hourglass cell values
//                yy * hourglass_nc(hg1 u + dt hg2 v) (acceleration.f90:136-163)
//   node phase   divergence (diff_cn) with PML p memory, hourglass_cn,
//                viscous-only hourglass in the PML, force injections,
//                a = f * mr, and the leapfrog update of the NEXT step
//                v' = v + dt a, u' = u + dt v' (time_integration.f90:27-41)
//
// Each block owns a 31 x 7 column of output nodes (32 x 8 cells including
// the -1 halo) and streams along l: node planes sit in a 3-plane shared
// ring (u, v, gam, coordinates), cell planes in a 2-plane ring (stress,
// hourglass values, divergence brackets), and plane l+3 is prefetched into
// registers while planes l-1..l+1 are being used.  Cells on tile borders are
// computed by both neighbours (from identical inputs, so identically); the
// owner writes the PML g memory, which is double-buffered like v and u so
// no block reads a value another block has already advanced.
//
// Support-operator brackets: rectilinear meshes use the per-direction
// constants verified at setup; terrain meshes (x = x(j), y = y(k)) compute
// the two z-dependent directions per cell from 1-D x, y and the z plane;
// general meshes compute all three.  Each cell's brackets are evaluated
// once and shared by the cell's gradient and its eight corner nodes'
// divergence (stencil.cuh: cell_cn_brackets).
#include "inject.cuh"
#include "sord.cuh"
#include "stencil.cuh"

namespace sordgpu {

constexpr int FJ = 32, FK = 8;                // cell tile = threads
constexpr int FNJ = FJ + 1, FNK = FK + 1;     // node region of a plane
constexpr int FOJ = FJ - 1, FOK = FK - 1;     // output nodes of a tile
constexpr int NPL = FNJ * FNK;                // 297 nodes per plane
constexpr int NCL = FJ * FK;                  // 256 cells per plane
constexpr int NTH = FJ * FK;

template <int GEOM>
struct Lay {
    static constexpr int NCOORD = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 1 : 3;
    static constexpr int PRE = 7 + NCOORD;    // prefetched: u(3) v(3) gam coords
    static constexpr int NODEF = 9 + NCOORD;  // shared: u(3) v(3) w = u + gam v (3) coords
    static constexpr int CO = 9;              // first coordinate field
    static constexpr int NDIR = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 2 : 3;
    static constexpr int CELLF = 6 + 12 + 8 * NDIR;  // stress, hourglass, divergence brackets
    static constexpr size_t bytes = sizeof(float) * (size_t)(3 * NPL * NODEF + 2 * NCL * CELLF);
};

__device__ __forceinline__ void bmax(unsigned* dst, float v) {
    unsigned b = __float_as_uint(v);
    if (v != v) b = 0x7fc00000u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    __shared__ unsigned s[32];
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = t & 31, warp = t >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
    __syncthreads();
    if (lane == 0) s[warp] = b;
    __syncthreads();
    if (warp == 0) {
        b = lane < nw ? s[lane] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
        if (lane == 0 && b) atomicMax(dst, b);
    }
}
__device__ __forceinline__ float fmaxn(float m, float c) { return (c != c || c > m) ? c : m; }

__device__ __forceinline__ long long slab_idx(const Geom& g, int axis, int t, int ii, int j, int k, int l, int ic) {
    long long e0 = axis == 0 ? t : g.nm[0], e1 = axis == 1 ? t : g.nm[1], e2 = axis == 2 ? t : g.nm[2];
    long long a0 = axis == 0 ? ii : j - 1, a1 = axis == 1 ? ii : k - 1, a2 = axis == 2 ? ii : l - 1;
    return a0 + e0 * (a1 + e1 * a2) + (long long)ic * e0 * e1 * e2;
}

template <int GEOM>
__global__ void __launch_bounds__(NTH, GEOM == GEOM_GENERAL ? 1 : 2) k_step(StepArgs A) {
    using L = Lay<GEOM>;
    extern __shared__ float sm[];
    float* sN = sm;                          // [3 slots][NODEF][NPL]
    float* sC = sm + 3 * L::NODEF * NPL;     // [2 slots][CELLF][NCL]
#define NODE(slot, f, i) sN[((slot) * L::NODEF + (f)) * NPL + (i)]
#define CELL(slot, f, i) sC[((slot) * L::CELLF + (f)) * NCL + (i)]
    const Geom& g = A.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + FJ * ty;
    const int j0 = g.i1node[0] + blockIdx.x * FOJ, k0 = g.i1node[1] + blockIdx.y * FOK;
    const int L0 = g.i1node[2] + blockIdx.z * A.segl;
    const int L1 = min(L0 + A.segl - 1, g.i2node[2]);
    const int J = j0 - 1 + tx, K = k0 - 1 + ty;      // this thread's cell column
    const int jn = j0 + tx, kn = k0 + ty;            // this thread's node column
    const bool outcol = tx < FOJ && ty < FOK && jn <= g.i2node[0] && kn <= g.i2node[1];
    const bool cellcol = J >= g.i1cell[0] && J <= g.i2cell[0] && K >= g.i1cell[1] && K <= g.i2cell[1];
    const bool owncol = J >= j0 && K >= k0;
    const float h = g.h, dt = g.dt;
    float st_a = 0.f, st_v = 0.f, st_u = 0.f, st_w = 0.f;

    // point injections that fall inside this block (cells / nodes it computes)
    __shared__ Inject lpot[kLocalInject], lmom[kLocalInject], lfrc[kLocalInject];
    __shared__ int lcnt[3];
    gather_inject(A.pot, lpot, &lcnt[0], g, j0 - 1, j0 + FOJ - 1, k0 - 1, k0 + FOK - 1, L0 - 1, L1);
    gather_inject(A.mom, lmom, &lcnt[1], g, j0 - 1, j0 + FOJ - 1, k0 - 1, k0 + FOK - 1, L0 - 1, L1);
    gather_inject(A.force, lfrc, &lcnt[2], g, j0, j0 + FOJ - 1, k0, k0 + FOK - 1, L0, L1);
    __syncthreads();
    const int npot = lcnt[0], nmom = lcnt[1], nfrc = lcnt[2];

    // ---------------------------------------------------------------- loads
    float pre[2][L::PRE];
    auto fetch = [&](int l) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH;
            const int nj = n % FNJ, nk = n / FNJ;
            const int j = j0 - 1 + nj, k = k0 - 1 + nk;
            const bool ok = n < NPL && j <= g.nm[0] && k <= g.nm[1] && l >= 1 && l <= g.nm[2];
            const long long q = ok ? g.idx(j, k, l) : 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                pre[r][c] = ok ? A.uin[c][q] : 0.f;
                pre[r][3 + c] = ok ? A.vin[c][q] : 0.f;
            }
            pre[r][6] = ok ? A.gam[q] : 0.f;
            if (GEOM == GEOM_TERRAIN) pre[r][7] = ok ? A.x[2][q] : 0.f;
            if (GEOM == GEOM_GENERAL)
#pragma unroll
                for (int c = 0; c < 3; c++) pre[r][7 + c] = ok ? A.x[c][q] : 0.f;
        }
    };
    auto store = [&](int slot) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH;
            if (n < NPL) {
#pragma unroll
                for (int f = 0; f < 6; f++) NODE(slot, f, n) = pre[r][f];
                // w1 = u + gam * v (time_integration.f90:36)
#pragma unroll
                for (int c = 0; c < 3; c++) NODE(slot, 6 + c, n) = pre[r][c] + pre[r][6] * pre[r][3 + c];
#pragma unroll
                for (int f = 0; f < L::NCOORD; f++) NODE(slot, L::CO + f, n) = pre[r][7 + f];
            }
        }
    };

    // per-plane statics of this thread's cell (lam, mu, 1/V, yy) and node
    // (mass ratio), loaded one plane ahead of their use
    float cur[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    auto stat_load = [&](int l, float* o) {
        const bool cv = cellcol && l >= g.i1cell[2] && l <= g.i2cell[2];
        const long long qc = cv ? g.idx(J, K, l) : 0;
        o[0] = cv ? A.lam[qc] : 0.f;
        o[1] = cv ? A.mu[qc] : 0.f;
        o[2] = cv ? A.vc[qc] : 0.f;
        o[3] = cv ? A.yy[qc] : 0.f;
        const bool nv = outcol && l >= g.i1node[2] && l <= g.i2node[2];
        o[4] = nv ? A.mr[g.idx(jn, kn, l)] : 0.f;
    };

    // ---------------------------------------------------------------- cell phase
    auto cells = [&](int l) {
        const int cs = l & 1;
        const bool valid = cellcol && l >= g.i1cell[2] && l <= g.i2cell[2];
        float ed[3] = {0.f, 0.f, 0.f}, eo[3] = {0.f, 0.f, 0.f};
        float he[12];
#pragma unroll
        for (int i = 0; i < 12; i++) he[i] = 0.f;
        float cnb[L::NDIR > 0 ? L::NDIR : 1][8];
        if (valid) {
            const long long q = g.idx(J, K, l);
            const int s0 = l % 3, s1 = (l + 1) % 3;
            int ni[8], ns[8];
#pragma unroll
            for (int n = 0; n < 8; n++) {
                ni[n] = (tx + (n & 1)) + FNJ * (ty + ((n >> 1) & 1));
                ns[n] = (n >> 2) ? s1 : s0;
            }
            float B[3][8];
            if (GEOM == GEOM_RECT) {
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int t = 0; t < 8; t++) B[a][t] = A.br.bnc[a][t];
            } else {
                float X[3][8];
                if (GEOM == GEOM_TERRAIN) {
                    const float xa = A.x1d[J - 1], xb = A.x1d[J], ya = A.y1d[K - 1], yb = A.y1d[K];
#pragma unroll
                    for (int n = 0; n < 8; n++) {
                        X[0][n] = (n & 1) ? xb : xa;
                        X[1][n] = ((n >> 1) & 1) ? yb : ya;
                        X[2][n] = NODE(ns[n], L::CO, ni[n]);
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 3; c++)
#pragma unroll
                        for (int n = 0; n < 8; n++) X[c][n] = NODE(ns[n], L::CO + c, ni[n]);
                }
#pragma unroll
                for (int a = 0; a < L::NDIR; a++) {
                    brackets_nc(X, a, B[a]);
                    cell_cn_brackets(X, a, B[a], cnb[a]);
                }
                if (GEOM == GEOM_TERRAIN)
#pragma unroll
                    for (int t = 0; t < 8; t++) B[2][t] = A.br.bnc[2][t];
            }
            // region of the cell (stress.f90:141-248)
            bool nearS[3], farS[3], anyS = false;
            const int cc[3] = {J, K, l};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                nearS[d] = cc[d] <= g.i1pml[d];
                farS[d] = cc[d] >= g.i2pml[d] - 1;
                anyS = anyS || nearS[d] || farS[d];
            }
            const bool own = owncol && l >= L0;
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                float W[8], U[8], V[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int n = term_corner(t);
                    const float uu = NODE(ns[n], ic, ni[n]), vv = NODE(ns[n], 3 + ic, ni[n]);
                    U[t] = uu;
                    V[t] = vv;
                    W[t] = NODE(ns[n], 6 + ic, ni[n]);
                }
#pragma unroll
                for (int iid = 0; iid < 3; iid++) {
                    const int id = (ic + iid + 1) % 3;
                    float s;
                    if (nearS[id] || farS[id]) {
                        const float raw = stencil8(V, B[id], h);
                        s = raw;
                        const int c = cc[id];
                        if (nearS[id]) {
                            const int p = c + g.nnoff[id];
                            const long long gi = slab_idx(g, id, A.sl.tg[id], c - g.i1cell[id], J, K, l, ic);
                            s = A.pmlc[3 * g.npml + p - 1] * raw + A.pmlc[2 * g.npml + p - 1] * A.sl.g[id][gi];
                            if (own) A.gout[id][gi] = s;
                        }
                        if (farS[id]) {
                            const int p = g.nn[id] - c - g.nnoff[id];
                            const long long gi = slab_idx(g, id, A.sl.tg[3 + id], g.i2cell[id] - c, J, K, l, ic);
                            s = A.pmlc[3 * g.npml + p - 1] * raw + A.pmlc[2 * g.npml + p - 1] * A.sl.g[3 + id][gi];
                            if (own) A.gout[3 + id][gi] = s;
                        }
                    } else if (anyS) {
                        s = stencil8(U, B[id], h);
                    } else {
                        s = stencil8(W, B[id], h);
                    }
                    if (ic == id) ed[ic] = s;
                    else if (ic < id) eo[3 - ic - id] = 0.5f * s;
                    else eo[3 - ic - id] = eo[3 - ic - id] + 0.5f * s;
                }
            }
            apply_inject(lpot, npot, A.pot, q, ed, eo);
            {
                const float lm = cur[0], m2 = 2.0f * cur[1];
                const float s1 = lm * (ed[0] + ed[1] + ed[2]);
#pragma unroll
                for (int i = 0; i < 3; i++) { ed[i] = m2 * ed[i] + s1; eo[i] = m2 * eo[i]; }
            }
            apply_inject(lmom, nmom, A.mom, q, ed, eo);
            {
                const float r = cur[2];
#pragma unroll
                for (int i = 0; i < 3; i++) { ed[i] = ed[i] * r; eo[i] = eo[i] * r; }
            }
            if (A.stats && own)
                st_w = fmaxn(st_w, (ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]) + 2.0f * (eo[0] * eo[0] + eo[1] * eo[1] + eo[2] * eo[2]));
            // elastic hourglass cell values (acceleration.f90:141-156)
            if (A.hourglass) {
                bool inE = true;
#pragma unroll
                for (int d = 0; d < 3; d++) inE = inE && cc[d] >= g.i1pml[d] && cc[d] <= g.i2pml[d] - 1;
                if (inE) {
                    const float y = cur[3];
#pragma unroll
                    for (int ic = 0; ic < 3; ic++) {
                        float W2[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            const int n = hg_corner(t);
                            W2[t] = A.hg1 * NODE(ns[n], ic, ni[n]) + A.dh2 * NODE(ns[n], 3 + ic, ni[n]);
                        }
#pragma unroll
                        for (int iq = 0; iq < 4; iq++) he[3 * iq + ic] = hg_sum(W2, iq) * y;
                    }
                }
            }
        } else {
#pragma unroll
            for (int a = 0; a < L::NDIR; a++)
#pragma unroll
                for (int t = 0; t < 8; t++) cnb[a][t] = 0.f;
        }
#pragma unroll
        for (int i = 0; i < 3; i++) { CELL(cs, i, tid) = ed[i]; CELL(cs, 3 + i, tid) = eo[i]; }
#pragma unroll
        for (int i = 0; i < 12; i++) CELL(cs, 6 + i, tid) = he[i];
#pragma unroll
        for (int a = 0; a < L::NDIR; a++)
#pragma unroll
            for (int t = 0; t < 8; t++) CELL(cs, 18 + 8 * a + t, tid) = cnb[a][t];
    };

    // ---------------------------------------------------------------- node phase
    auto nodes = [&](int l) {
        if (!outcol) return;
        const long long q = g.idx(jn, kn, l);
        const int sn = l % 3;
        const int ni0 = (tx + 1) + FNJ * (ty + 1);
        // cells of diff_cn term t: (j-1|j, k-1|k, l-1|l)
        int ci[8], cs[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int oj = (t & 1) ? 0 : -1, ok = (t >> 2) ? 0 : -1, ol = ((t >> 1) & 1) ? 0 : -1;
            ci[t] = (tx + 1 + oj) + FJ * (ty + 1 + ok);
            cs[t] = (l + ol) & 1;
        }
        float f[3];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
#pragma unroll
            for (int iid = 0; iid < 3; iid++) {
                const int id = (ic + iid) % 3;
                const int comp = ic == id ? ic : 3 + (3 - ic - id);
                float F[8], B[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    F[t] = CELL(cs[t], comp, ci[t]);
                    if (GEOM == GEOM_RECT || (GEOM == GEOM_TERRAIN && id == 2)) B[t] = A.br.bcn[id][t];
                    else B[t] = CELL(cs[t], 18 + 8 * id + t, ci[t]);
                }
                float s = stencil8(F, B, h);
                const int c = id == 0 ? jn : id == 1 ? kn : l;
                if (c <= g.i1pml[id]) {
                    const int p = c + g.nnoff[id];
                    float* P = A.sl.p[id] + slab_idx(g, id, A.sl.tp[id], c - g.i1node[id], jn, kn, l, ic);
                    s = A.pmlc[g.npml + p - 1] * s + A.pmlc[p - 1] * *P;
                    *P = *P + dt * s;
                }
                if (c >= g.i2pml[id]) {
                    const int p = g.nn[id] - c - g.nnoff[id] + 1;
                    float* P = A.sl.p[3 + id] + slab_idx(g, id, A.sl.tp[3 + id], g.i2node[id] - c, jn, kn, l, ic);
                    s = A.pmlc[g.npml + p - 1] * s + A.pmlc[p - 1] * *P;
                    *P = *P + dt * s;
                }
                f[ic] = iid == 0 ? s : f[ic] + s;
            }
        }
        if (A.hourglass) {
            const int cn_[3] = {jn, kn, l};
            bool ne = true;
#pragma unroll
            for (int d = 0; d < 3; d++) ne = ne && cn_[d] >= g.i1pml[d] + 1 && cn_[d] <= g.i2pml[d] - 1;
            if (ne) {
                int hi[8], hs[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int o = hg_corner(t);
                    hi[t] = (tx + 1 - (o & 1)) + FJ * (ty + 1 - ((o >> 1) & 1));
                    hs[t] = (l - (o >> 2)) & 1;
                }
#pragma unroll
                for (int iq = 0; iq < 4; iq++)
#pragma unroll
                    for (int ic = 0; ic < 3; ic++) {
                        float H[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) H[t] = CELL(hs[t], 6 + 3 * iq + ic, hi[t]);
                        f[ic] = f[ic] - hg_sum(H, iq);
                    }
            } else if (A.hgvisc) {
                // viscous-only hourglass in the PML, cell values formed here from
                // the node ring (acceleration.f90:164-199)
                float yc[8];
                bool okc[8];
                int cb[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int o = hg_corner(t);
                    const int Jc = jn - (o & 1), Kc = kn - ((o >> 1) & 1), Lc = l - (o >> 2);
                    const bool real = Jc >= g.i1cell[0] && Jc <= g.i2cell[0] && Kc >= g.i1cell[1] && Kc <= g.i2cell[1] &&
                                      Lc >= g.i1cell[2] && Lc <= g.i2cell[2];
                    const bool slab = Jc <= g.i1pml[0] || Jc >= g.i2pml[0] - 1 || Kc <= g.i1pml[1] || Kc >= g.i2pml[1] - 1 ||
                                      Lc <= g.i1pml[2] || Lc >= g.i2pml[2] - 1;
                    okc[t] = real && slab;
                    yc[t] = okc[t] ? A.dh2 * A.yy[g.idx(Jc, Kc, Lc)] : 0.f;
                    cb[t] = o;
                }
                // each component's four modes share the cell corner loads; the
                // updates of f[ic] keep the reference's mode order
#pragma unroll 1
                for (int ic = 0; ic < 3; ic++) {
                    float Hq[4][8];
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        if (okc[t]) {
                            const int o = cb[t];
                            float Vc[8];
#pragma unroll
                            for (int m = 0; m < 8; m++) {
                                const int n = hg_corner(m);
                                const int dj = (n & 1) - (o & 1), dk = ((n >> 1) & 1) - ((o >> 1) & 1), dl = (n >> 2) - (o >> 2);
                                Vc[m] = NODE((l + dl + 3) % 3, 3 + ic, (tx + 1 + dj) + FNJ * (ty + 1 + dk));
                            }
#pragma unroll
                            for (int iq = 0; iq < 4; iq++) Hq[iq][t] = yc[t] * hg_sum(Vc, iq);
                        } else {
#pragma unroll
                            for (int iq = 0; iq < 4; iq++) Hq[iq][t] = 0.f;
                        }
                    }
                    float fi = f[0];
                    if (ic == 1) fi = f[1];
                    if (ic == 2) fi = f[2];
#pragma unroll
                    for (int iq = 0; iq < 4; iq++) fi = fi - hg_sum(Hq[iq], iq);
                    if (ic == 0) f[0] = fi;
                    if (ic == 1) f[1] = fi;
                    if (ic == 2) f[2] = fi;
                }
            }
        }
        {
            const Inject* E = nfrc >= 0 ? lfrc : A.force.e;
            const int n = nfrc >= 0 ? nfrc : A.force.n;
            for (int e = 0; e < n; e++)
                if (E[e].idx == q) {
                    const int c = E[e].comp;
                    f[c] = f[c] + E[e].inc;
                }
        }
        const float m = cur[4];
#pragma unroll
        for (int i = 0; i < 3; i++) f[i] = f[i] * m;
        const float v0 = NODE(sn, 3, ni0), v1 = NODE(sn, 4, ni0), v2 = NODE(sn, 5, ni0);
        const float u0 = NODE(sn, 0, ni0), u1 = NODE(sn, 1, ni0), u2 = NODE(sn, 2, ni0);
        if (A.stats) {
            st_a = fmaxn(st_a, f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
            st_v = fmaxn(st_v, v0 * v0 + v1 * v1 + v2 * v2);
            st_u = fmaxn(st_u, u0 * u0 + u1 * u1 + u2 * u2);
        }
        if (A.aout[0])
#pragma unroll
            for (int i = 0; i < 3; i++) A.aout[i][q] = f[i];
        if (A.fold) {
            // leapfrog update of the next step (time_integration.f90:32-35)
            float a, b;
            a = v0 + dt * f[0]; b = u0 + dt * a; A.vout[0][q] = a; A.uout[0][q] = b;
            a = v1 + dt * f[1]; b = u1 + dt * a; A.vout[1][q] = a; A.uout[1][q] = b;
            a = v2 + dt * f[2]; b = u2 + dt * a; A.vout[2][q] = a; A.uout[2][q] = b;
        }
    };

    // ---------------------------------------------------------------- stream
    fetch(L0 - 1);
    store((L0 - 1) % 3);
    fetch(L0);
    store(L0 % 3);
    fetch(L0 + 1);
    store((L0 + 1) % 3);
    stat_load(L0 - 1, cur);
    __syncthreads();
    cells(L0 - 1);
    stat_load(L0, cur);
    fetch(L0 + 2);
    for (int l = L0; l <= L1; l++) {
        __syncthreads();
        cells(l);
        float nxt[5];
        stat_load(l + 1, nxt);
        __syncthreads();
        nodes(l);
        __syncthreads();
        store((l + 2) % 3);
        fetch(l + 3);
#pragma unroll
        for (int i = 0; i < 5; i++) cur[i] = nxt[i];
    }
    if (A.stats) {
        bmax(A.red + 0, st_a);
        bmax(A.red + 1, st_v);
        bmax(A.red + 2, st_u);
        bmax(A.red + 3, st_w);
    }
#undef NODE
#undef CELL
}

template <int GEOM>
static void launch_geom(Solver& s, const StepArgs& A, dim3 grid) {
    static bool set = false;
    if (!set) {
        SORD_CUDA(cudaFuncSetAttribute(k_step<GEOM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay<GEOM>::bytes));
        set = true;
    }
    k_step<GEOM><<<grid, dim3(FJ, FK), Lay<GEOM>::bytes, s.stream>>>(A);
}

void launch_fused(Solver& s, const InjectList& pot, const InjectList& mom, const InjectList& force, bool fold, bool write_a,
                  bool stats) {
    Device& d = s.d;
    StepArgs A;
    A.g = s.g;
    A.br = s.br;
    A.x1d = d.x1d;
    A.y1d = d.y1d;
    for (int i = 0; i < 3; i++) {
        A.x[i] = d.x[i];
        A.vin[i] = d.v[i];
        A.uin[i] = d.u[i];
        A.vout[i] = d.vb[i];
        A.uout[i] = d.ub[i];
        A.aout[i] = (write_a || !fold) ? d.w1n[i] : nullptr;
    }
    A.gam = d.gam; A.mr = d.mr; A.lam = d.lam; A.mu = d.mu; A.vc = d.vc; A.yy = d.yy;
    A.pmlc = d.pmlc;
    A.sl = d.slabs;
    for (int i = 0; i < 6; i++) A.gout[i] = d.gb[i];
    A.pot = pot; A.mom = mom; A.force = force;
    A.hg1 = s.prm.hourglass[0];
    A.dh2 = s.g.dt * s.prm.hourglass[1];
    A.hourglass = (s.prm.hourglass[0] > 0.f || s.prm.hourglass[1] > 0.f) ? 1 : 0;
    A.hgvisc = (s.prm.hourglass[1] > 0.f && s.g.npml > 0) ? 1 : 0;
    A.fold = fold ? 1 : 0;
    A.stats = stats ? 1 : 0;
    A.red = (unsigned*)d.red;
    const Geom& g = s.g;
    int nj = g.i2node[0] - g.i1node[0] + 1, nk = g.i2node[1] - g.i1node[1] + 1, nl = g.i2node[2] - g.i1node[2] + 1;
    unsigned bx = div_up(nj, FOJ), by = div_up(nk, FOK);
    long long bxy = (long long)bx * by;
    int nseg = (int)std::min<long long>(std::max<long long>(1, (4LL * 148 + bxy - 1) / bxy), std::max(1, nl / 8));
    A.segl = (nl + nseg - 1) / nseg;
    nseg = (nl + A.segl - 1) / A.segl;
    dim3 grid(bx, by, nseg);
    cudaEvent_t e0 = nullptr;
    s.prof_begin(KC_FUSED, &e0);
    if (s.geom == GEOM_RECT) launch_geom<GEOM_RECT>(s, A, grid);
    else if (s.geom == GEOM_TERRAIN) launch_geom<GEOM_TERRAIN>(s, A, grid);
    else launch_geom<GEOM_GENERAL>(s, A, grid);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
    s.prof_end(KC_FUSED, e0);
    if (fold) {
        for (int i = 0; i < 3; i++) {
            std::swap(d.v[i], d.vb[i]);
            std::swap(d.u[i], d.ub[i]);
        }
    }
    for (int i = 0; i < 6; i++) std::swap(d.slabs.g[i], d.gb[i]);
}

}  // namespace sordgpu

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
// the -1 halo) and streams along l.  Node planes are staged raw (u, v, gam,
// coordinates) by cp.async into shared memory one plane ahead, then turned
// into a 3-plane ring of the per-node values the cells need: w = u + gam v,
// the hourglass input hg1 u + dt hg2 v, and the coordinates.  Cell planes
// (stress, hourglass values, divergence brackets) sit in a 2-plane ring.
// Two barriers per plane.  Cells on tile borders are computed by both
// neighbours (from identical inputs, so identically); the owner writes the
// PML g memory, which is double-buffered like v and u so no block reads a
// value another block has already advanced.
//
// Planes of blocks whose whole tile lies outside the PML, with no point
// source in the block, run a fast path with the PML, boundary and injection
// branches compiled out; the arithmetic of both paths is the same, so a
// cell computed by either is bit-identical.
//
// Support-operator brackets: rectilinear meshes use the per-direction
// constants verified at setup; terrain meshes (x = x(j), y = y(k)) compute
// the two z-dependent directions per cell from 1-D x, y and the z plane;
// general meshes compute all three.  Each cell's brackets are evaluated
// once and shared by the cell's gradient and its eight corner nodes'
// divergence (stencil.cuh: cell_cn_brackets).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "inject.cuh"
#include "pair.cuh"
#include "sord.cuh"
#include "stencil.cuh"

// SORD_FAST_PAIRED selects packed f32x2 evaluation (pair.cuh) of the
// interior kernel's independent stencils; 0 evaluates them one at a time.
// Both give bit-identical results.
#ifndef SORD_FAST_PAIRED
#define SORD_FAST_PAIRED 0
#endif

namespace sordgpu {

constexpr bool kPaired = SORD_FAST_PAIRED != 0;
constexpr int FJ = 32, FK = 8;                // cell tile = threads
constexpr int FNJ = FJ + 1, FNK = FK + 1;     // node region of a plane
constexpr int FOJ = FJ - 1, FOK = FK - 1;     // output nodes of a tile
constexpr int NPL = FNJ * FNK;                // 297 nodes per plane
constexpr int NCL = FJ * FK;                  // 256 cells per plane
constexpr int NTH = FJ * FK;

// Shared-memory layout.  Node planes: float4 groups per node,
//   group 0 = (w_x, w_y, w_z, coordinate 0), group 1 = (h_x, h_y, h_z,
//   coordinate 1), group 2 = (coordinate 2, -, -, -) on general meshes,
// with w = u + gam v and h = hg1 u + dt hg2 v; terrain meshes store z as
// coordinate 0, general meshes x, y, z.  Cell planes: float4 groups per cell,
//   0: s_xx s_yy s_zz s_yz   1: s_zx s_xy hA0   2: hA1 hA2   3: hA3 hB0 hB1
//   4: hB2 hB3 - -   5..8: (b0, b1) divergence brackets of terms 2g, 2g+1
//   9, 10: b2 of terms 0..7 (general meshes)
// where hA_iq = hourglass values of mode iq for components (x, y) and
// hB_iq the z component, so every packed pair is an aligned float2.
template <int GEOM>
struct Lay {
    static constexpr int NCOORD = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 1 : 3;
    static constexpr int RAWF = 7 + NCOORD;                   // staged plane: u(3) v(3) gam coords
    static constexpr int RAWSZ = (RAWF * NPL + 3) & ~3;        // floats, float4-aligned end
    static constexpr int NGN = GEOM == GEOM_GENERAL ? 3 : 2;  // float4 groups per node
    static constexpr int NDIR = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 2 : 3;
    static constexpr int NGC = GEOM == GEOM_RECT ? 5 : GEOM == GEOM_TERRAIN ? 9 : 11;  // float4 groups per cell
    static constexpr size_t bytes = sizeof(float) * (size_t)RAWSZ + sizeof(float4) * (size_t)(3 * NPL * NGN + 2 * NCL * NGC);
    // fast arithmetic: one cell plane (each node plane reads only the cells
    // above it); groups: (e11 e22 e33 e23), (e31 e12) as float2, then per
    // reading node column q: its hourglass sums for the node above and
    // below, and its divergence brackets (NQ groups)
    // (terrain: 2 groups per q, the lower-cell brackets of all q in 2 float2 groups)
    static constexpr int NQ = NDIR == 3 ? 3 : 2;
    static constexpr int NGCF = 2 + 4 * NQ + (NDIR == 2 ? 2 : 0);
    // the interior kernel in fast arithmetic stores, per reading node column
    // q, that node's whole force terms from the cell: (fu_x, fu_y, fu_z,
    // fl_x) as float4 group q and (fl_y, fl_z) as float2 in groups 4-5
    static constexpr int NGCR = 6;
    // ... and on rectilinear and terrain meshes copies each node plane
    // straight into the ring as raw (u, gam), (v, z) groups: no staging plane
    static constexpr bool RAWRING = GEOM != GEOM_GENERAL;
    static constexpr size_t bytes_fm = sizeof(float) * (size_t)(RAWRING ? 0 : RAWSZ) +
                                       sizeof(float4) * (size_t)(3 * NPL * NGN + NCL * NGCR);
};
// scalar field numbers of the node and cell groups
__host__ __device__ constexpr int nf_co(int c) { return c == 0 ? 3 : c == 1 ? 7 : 8; }
__host__ __device__ constexpr int cf_hg(int iq, int ic) { return ic < 2 ? 6 + 2 * iq + ic : 14 + iq; }
__host__ __device__ constexpr int cf_br(int a, int t) { return a < 2 ? 20 + 2 * t + a : 36 + t; }

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

// Mass, statistics, acceleration output and the folded leapfrog update of
// node q = (jn, kn, l) with force f (acceleration.f90:235-238,
// time_integration.f90:32-35).  A node on either plane of a double-node
// fault keeps its force: the rupture step adds the fault traction to it,
// divides by the mass and, when the step is folded, advances its v and u;
// the fold copies its v and u into the new buffers.
template <bool FM = false>
__device__ __forceinline__ void finish_node(const StepArgs& A, long long q, int jn, int kn, int l, float (&f)[3],
                                            float m, const float (&uv)[6], float dt, float& st_a, float& st_v,
                                            float& st_u) {
    const int fc = A.fax == 0 ? jn : A.fax == 1 ? kn : l;
    const bool fnode = A.fax >= 0 && (unsigned)(fc - A.firup) <= 1u;
    const float u0 = uv[0], u1 = uv[1], u2 = uv[2], v0 = uv[3], v1 = uv[4], v2 = uv[5];
    if (fnode) {
#pragma unroll
        for (int i = 0; i < 3; i++) A.fout[i][q] = f[i];
        if (A.stats) {
            st_v = fmaxn(st_v, v0 * v0 + v1 * v1 + v2 * v2);
            st_u = fmaxn(st_u, u0 * u0 + u1 * u1 + u2 * u2);
        }
        if (A.fold) {
            A.vout[0][q] = v0; A.uout[0][q] = u0;
            A.vout[1][q] = v1; A.uout[1][q] = u1;
            A.vout[2][q] = v2; A.uout[2][q] = u2;
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < 3; i++) f[i] = f[i] * m;
    if (A.stats) {
        st_a = fmaxn(st_a, f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        st_v = fmaxn(st_v, v0 * v0 + v1 * v1 + v2 * v2);
        st_u = fmaxn(st_u, u0 * u0 + u1 * u1 + u2 * u2);
    }
    if (A.aout[0])
#pragma unroll
        for (int i = 0; i < 3; i++) A.aout[i][q] = f[i];
    if (A.fold) {
        float a, b;
        if (FM) {
            a = fmaf(dt, f[0], v0); b = fmaf(dt, a, u0); A.vout[0][q] = a; A.uout[0][q] = b;
            a = fmaf(dt, f[1], v1); b = fmaf(dt, a, u1); A.vout[1][q] = a; A.uout[1][q] = b;
            a = fmaf(dt, f[2], v2); b = fmaf(dt, a, u2); A.vout[2][q] = a; A.uout[2][q] = b;
        } else {
            a = v0 + dt * f[0]; b = u0 + dt * a; A.vout[0][q] = a; A.uout[0][q] = b;
            a = v1 + dt * f[1]; b = u1 + dt * a; A.vout[1][q] = a; A.uout[1][q] = b;
            a = v2 + dt * f[2]; b = u2 + dt * a; A.vout[2][q] = a; A.uout[2][q] = b;
        }
    }
}

__device__ __forceinline__ long long slab_idx(const Geom& g, int axis, int t, int ii, int j, int k, int l, int ic) {
    long long e0 = axis == 0 ? t : g.nm[0], e1 = axis == 1 ? t : g.nm[1], e2 = axis == 2 ? t : g.nm[2];
    long long a0 = axis == 0 ? ii : j - 1, a1 = axis == 1 ? ii : k - 1, a2 = axis == 2 ? ii : l - 1;
    return a0 + e0 * (a1 + e1 * a2) + (long long)ic * e0 * e1 * e2;
}

// 4-byte asynchronous global -> shared copy (no register staging).

// Shared-memory layout of the PML-shell kernel: plain per-field planes
// (node ring: w(3), hourglass input(3), coordinates; cell ring: stress(6),
// hourglass(12), divergence brackets(8 per direction)).
template <int GEOM, int NPLS, int NCLS>
struct LayS {
    static constexpr int NCOORD = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 1 : 3;
    static constexpr int RAWF = 7 + NCOORD;   // staged plane: u(3) v(3) gam coords
    static constexpr int NODEF = 6 + NCOORD;  // ring: w = u + gam v (3), hg1 u + dt hg2 v (3), coords
    static constexpr int HG = 3;              // first hourglass-input field
    static constexpr int CO = 6;              // first coordinate field
    static constexpr int NDIR = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 2 : 3;
    static constexpr int CELLF = 6 + 12 + 8 * NDIR;  // stress, hourglass, divergence brackets
    static constexpr size_t bytes = sizeof(float) * (size_t)(NPLS * RAWF + 3 * NPLS * NODEF + 2 * NCLS * CELLF);
};


// PML-shell kernel: 16 x 16 threads per block, each block the node box of
// one work item of A.items (j0, k0, last j, last k, first and last plane,
// at most 15 x 15 nodes), with every PML, boundary and point-source term of
// the step.
constexpr int SJ = 16, SK = 16;  // shell tile (cells = threads)
// FM: the fast arithmetic of k_interior for the support-operator sums.
template <int GEOM, bool FM>
__global__ void __launch_bounds__(SJ * SK, GEOM == GEOM_GENERAL ? 1 : 2) k_shell(StepArgs A) {
    constexpr int FJ = SJ, FK = SK, FNJ = FJ + 1, FNK = FK + 1, FOJ = FJ - 1, FOK = FK - 1;
    constexpr int NPL = FNJ * FNK, NCL = FJ * FK, NTH = FJ * FK;
    (void)FNK;
    constexpr bool FASTK = false;
    using L = LayS<GEOM, NPL, NCL>;
    extern __shared__ float sm[];
    float* sR = sm;                          // [RAWF][NPL] staged plane
    float* sN = sR + L::RAWF * NPL;          // [3 slots][NODEF][NPL]
    float* sC = sN + 3 * L::NODEF * NPL;     // [2 slots][CELLF][NCL]
#define RAW(f, i) sR[(f) * NPL + (i)]
#define NODE(slot, f, i) sN[((slot) * L::NODEF + (f)) * NPL + (i)]
#define CELL(slot, f, i) sC[((slot) * L::CELLF + (f)) * NCL + (i)]
    const Geom& g = A.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + FJ * ty;
    const int* it = A.items + 6 * blockIdx.x;
    const int j0 = it[0], k0 = it[1], jm = it[2], km = it[3], L0 = it[4], L1 = it[5];
    const int J = j0 - 1 + tx, K = k0 - 1 + ty;      // this thread's cell column
    const int jn = j0 + tx, kn = k0 + ty;            // this thread's node column
    const bool outcol = tx < FOJ && ty < FOK && jn <= jm && kn <= km;
    const bool cellcol = J >= g.i1cell[0] && J <= g.i2cell[0] && K >= g.i1cell[1] && K <= g.i2cell[1];
    // the cell of node column (J, K) belongs to the block that owns that node
    const bool owncol = J >= j0 && J <= jm && K >= k0 && K <= km;
    const float h = g.h, dt = g.dt;
    float st_a = 0.f, st_v = 0.f, st_u = 0.f, st_w = 0.f;
    // terrain meshes: this thread's cell column's x (j, j+1) and y (k, k+1)
    float txa = 0.f, txb = 0.f, tya = 0.f, tyb = 0.f;
    if (GEOM == GEOM_TERRAIN && cellcol) {
        txa = A.x1d[J - 1];
        txb = A.x1d[J];
        tya = A.y1d[K - 1];
        tyb = A.y1d[K];
    }
    const float hdx = h * (txb - txa), hdy = h * (tyb - tya);

    // point injections that fall inside this block (cells / nodes it computes)
    __shared__ Inject lpot[kLocalInject], lmom[kLocalInject], lfrc[kLocalInject];
    __shared__ int lcnt[3];
    // A fast-kernel block whose (j, k) box holds a point source of this step
    // leaves that column to the general kernel (the host lists it there).
    const int gl1 = FASTK ? 0 : L0 - 1, gl2 = FASTK ? g.nm[2] + 1 : L1;
    gather_inject(A.pot, lpot, &lcnt[0], g, j0 - 1, j0 + FOJ - 1, k0 - 1, k0 + FOK - 1, gl1, gl2);
    gather_inject(A.mom, lmom, &lcnt[1], g, j0 - 1, j0 + FOJ - 1, k0 - 1, k0 + FOK - 1, gl1, gl2);
    gather_inject(A.force, lfrc, &lcnt[2], g, j0, j0 + FOJ - 1, k0, k0 + FOK - 1, FASTK ? gl1 : L0, gl2);
    __syncthreads();
    const int npot = lcnt[0], nmom = lcnt[1], nfrc = lcnt[2];
    if (FASTK && (npot != 0 || nmom != 0 || nfrc != 0)) return;

    // ---------------------------------------------------------------- loads
    // stage node plane l (u, v, gam, coordinates) into sR asynchronously
    auto fetch = [&](int l) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH;
            if (n < NPL) {
                const int nj = n % FNJ, nk = n / FNJ;
                const int j = j0 - 1 + nj, k = k0 - 1 + nk;
                const bool ok = j <= g.nm[0] && k <= g.nm[1] && l >= 1 && l <= g.nm[2];
                if (ok) {
                    const long long q = g.idx(j, k, l);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        cp_async4(&RAW(c, n), A.uin[c] + q);
                        cp_async4(&RAW(3 + c, n), A.vin[c] + q);
                    }
                    cp_async4(&RAW(6, n), A.gam + q);
                    if (GEOM == GEOM_TERRAIN) cp_async4(&RAW(7, n), A.x[2] + q);
                    if (GEOM == GEOM_GENERAL)
#pragma unroll
                        for (int c = 0; c < 3; c++) cp_async4(&RAW(7 + c, n), A.x[c] + q);
                } else {
#pragma unroll
                    for (int f = 0; f < L::RAWF; f++) RAW(f, n) = 0.f;
                }
            }
        }
        cp_async_commit();
    };
    // staged plane -> ring slot: w1 = u + gam * v (time_integration.f90:36)
    // and the hourglass input hg1 u + dt hg2 v (acceleration.f90:141)
    auto store = [&](int slot) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH;
            if (n < NPL) {
                const float gm = RAW(6, n);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float u = RAW(c, n), v = RAW(3 + c, n);
                    NODE(slot, c, n) = FM ? fmaf(gm, v, u) : u + gm * v;
                    NODE(slot, L::HG + c, n) = FM ? fmaf(A.dh2, v, A.hg1 * u) : A.hg1 * u + A.dh2 * v;
                }
#pragma unroll
                for (int f = 0; f < L::NCOORD; f++) NODE(slot, L::CO + f, n) = RAW(7 + f, n);
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
    // this thread's node u, v (for the update and statistics), one plane ahead
    float uv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    auto uv_load = [&](int l, float* o) {
        const bool nv = outcol && l >= g.i1node[2] && l <= g.i2node[2];
        const long long q = nv ? g.idx(jn, kn, l) : 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            o[c] = nv ? A.uin[c][q] : 0.f;
            o[3 + c] = nv ? A.vin[c][q] : 0.f;
        }
    };

    // ---------------------------------------------------------------- cell phase
    auto cells = [&](int l, auto fast_tag) {
        constexpr bool F = decltype(fast_tag)::value;
        const int cs = l & 1;
        const bool valid = F || (cellcol && l >= g.i1cell[2] && l <= g.i2cell[2]);
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
                    for (int t = 0; t < 8; t++) B[a][t] = FM ? A.brh.bnc[a][t] : A.br.bnc[a][t];
            } else if constexpr (FM) {
                // brackets scaled by h; divergence brackets = negated gradient brackets
                float X[3][8];
#pragma unroll
                for (int n = 0; n < 8; n++)
#pragma unroll
                    for (int c = 0; c < L::NCOORD; c++) X[3 - L::NCOORD + c][n] = NODE(ns[n], L::CO + c, ni[n]);
                if (GEOM == GEOM_TERRAIN) {
                    terrain_brackets_0(hdy, X[2], B[0]);
                    terrain_brackets_1(hdx, X[2], B[1]);
#pragma unroll
                    for (int t = 0; t < 8; t++) B[2][t] = A.brh.bnc[2][t];
                } else {
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        brackets_nc(X, a, B[a]);
#pragma unroll
                        for (int t = 0; t < 8; t++) B[a][t] = h * B[a][t];
                    }
                }
#pragma unroll
                for (int a = 0; a < L::NDIR; a++)
#pragma unroll
                    for (int t = 0; t < 8; t++) cnb[a][t] = -B[a][cn_of_nc(t)];
            } else {
                float X[3][8];
                if (GEOM == GEOM_TERRAIN) {
                    const float xa = txa, xb = txb, ya = tya, yb = tyb;
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
            // a cell plane below the first node plane is a halo of a partitioned run;
            // the part takes it (the PML g memory of that halo cell advances here)
            const bool own = owncol && (l >= L0 || l < g.i1node[2]);
            if constexpr (F) {
                // strain of an interior cell: gradients of w = u + gam v
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    float W[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        const int n = term_corner(t);
                        W[t] = NODE(ns[n], ic, ni[n]);
                    }
#pragma unroll
                    for (int iid = 0; iid < 3; iid++) {
                        const int id = (ic + iid + 1) % 3;
                        const float s = stencil8(W, B[id], h);
                        if (ic == id) ed[ic] = s;
                        else if (ic < id) eo[3 - ic - id] = 0.5f * s;
                        else eo[3 - ic - id] = eo[3 - ic - id] + 0.5f * s;
                    }
                }
            } else {
                // region of the cell (stress.f90:141-248)
                bool nearS[3], farS[3], anyS = false;
                const int cc[3] = {J, K, l};
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    nearS[d] = cc[d] <= g.i1pml[d];
                    farS[d] = cc[d] >= g.i2pml[d] - 1;
                    anyS = anyS || nearS[d] || farS[d];
                }
                // PML cells that are not elastic-hourglass cells carry the
                // viscous hourglass values dt hg2 yy hourglass_nc(v) in the
                // hourglass slots (acceleration.f90:164-183)
                bool inEc = true;
#pragma unroll
                for (int d = 0; d < 3; d++) inEc = inEc && cc[d] >= g.i1pml[d] && cc[d] <= g.i2pml[d] - 1;
                const bool visc = A.hourglass && A.hgvisc && anyS && !inEc;
                const float yv = A.dh2 * cur[3];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    float W[8], U[8], V[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        const int n = term_corner(t);
                        W[t] = NODE(ns[n], ic, ni[n]);
                        U[t] = 0.f;
                        V[t] = 0.f;
                    }
                    if (anyS) {
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            const int n = term_corner(t);
                            const long long qn = g.idx(J + (n & 1), K + ((n >> 1) & 1), l + (n >> 2));
                            U[t] = A.uin[ic][qn];
                            V[t] = A.vin[ic][qn];
                        }
                    }
                    if (visc) {
                        float Vc[8], Vh[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) Vc[term_corner(t)] = V[t];
#pragma unroll
                        for (int t = 0; t < 8; t++) Vh[t] = Vc[hg_corner(t)];
#pragma unroll
                        for (int iq = 0; iq < 4; iq++) he[3 * iq + ic] = yv * hg_sum(Vh, iq);
                    }
#pragma unroll
                    for (int iid = 0; iid < 3; iid++) {
                        const int id = (ic + iid + 1) % 3;
                        float s;
                        if (nearS[id] || farS[id]) {
                            const float raw = FM ? dot8(V, B[id]) : stencil8(V, B[id], h);
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
                            s = FM ? dot8(U, B[id]) : stencil8(U, B[id], h);
                        } else {
                            s = FM ? dot8(W, B[id]) : stencil8(W, B[id], h);
                        }
                        if (ic == id) ed[ic] = s;
                        else if (ic < id) eo[3 - ic - id] = 0.5f * s;
                        else eo[3 - ic - id] = eo[3 - ic - id] + 0.5f * s;
                    }
                }
                apply_inject(lpot, npot, A.pot, q, ed, eo);
            }
            {
                const float lm = cur[0], m2 = 2.0f * cur[1];
                const float s1v = lm * (ed[0] + ed[1] + ed[2]);
#pragma unroll
                for (int i = 0; i < 3; i++) { ed[i] = m2 * ed[i] + s1v; eo[i] = m2 * eo[i]; }
            }
            if constexpr (!F) apply_inject(lmom, nmom, A.mom, q, ed, eo);
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
                if constexpr (!F) {
                    const int cc[3] = {J, K, l};
#pragma unroll
                    for (int d = 0; d < 3; d++) inE = inE && cc[d] >= g.i1pml[d] && cc[d] <= g.i2pml[d] - 1;
                }
                if (inE) {
                    const float y = cur[3];
#pragma unroll
                    for (int ic = 0; ic < 3; ic++) {
                        float W2[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            const int n = hg_corner(t);
                            W2[t] = NODE(ns[n], L::HG + ic, ni[n]);
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
    auto nodes = [&](int l, auto fast_tag) {
        constexpr bool F = decltype(fast_tag)::value;
        if (!outcol) return;
        const long long q = g.idx(jn, kn, l);
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
                float Fv[8], B[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    Fv[t] = CELL(cs[t], comp, ci[t]);
                    if (GEOM == GEOM_RECT || (GEOM == GEOM_TERRAIN && id == 2)) B[t] = FM ? A.brh.bcn[id][t] : A.br.bcn[id][t];
                    else B[t] = CELL(cs[t], 18 + 8 * id + t, ci[t]);
                }
                float s = FM ? dot8(Fv, B) : stencil8(Fv, B, h);
                if constexpr (!F) {
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
                }
                f[ic] = iid == 0 ? s : f[ic] + s;
            }
        }
        if (A.hourglass) {
            bool ne = true;
            if constexpr (!F) {
                const int cn_[3] = {jn, kn, l};
#pragma unroll
                for (int d = 0; d < 3; d++) ne = ne && cn_[d] >= g.i1pml[d] + 1 && cn_[d] <= g.i2pml[d] - 1;
            }
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
            } else if constexpr (!F) {
                if (A.hgvisc) {
                    // viscous-only hourglass in the PML (acceleration.f90:164-199):
                    // every cell of a PML node is a PML cell; pure PML cells
                    // hold their viscous values in the hourglass slots, cells
                    // that are also elastic-hourglass cells (the layer next to
                    // the elastic region) are evaluated here from v
                    int hi[8], hs[8], kind[8];
                    float yc[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        const int o = hg_corner(t);
                        hi[t] = (tx + 1 - (o & 1)) + FJ * (ty + 1 - ((o >> 1) & 1));
                        hs[t] = (l - (o >> 2)) & 1;
                        const int Jc = jn - (o & 1), Kc = kn - ((o >> 1) & 1), Lc = l - (o >> 2);
                        const bool real = Jc >= g.i1cell[0] && Jc <= g.i2cell[0] && Kc >= g.i1cell[1] &&
                                          Kc <= g.i2cell[1] && Lc >= g.i1cell[2] && Lc <= g.i2cell[2];
                        const bool slab = Jc <= g.i1pml[0] || Jc >= g.i2pml[0] - 1 || Kc <= g.i1pml[1] ||
                                          Kc >= g.i2pml[1] - 1 || Lc <= g.i1pml[2] || Lc >= g.i2pml[2] - 1;
                        const bool inEc = Jc >= g.i1pml[0] && Jc <= g.i2pml[0] - 1 && Kc >= g.i1pml[1] &&
                                          Kc <= g.i2pml[1] - 1 && Lc >= g.i1pml[2] && Lc <= g.i2pml[2] - 1;
                        kind[t] = !(real && slab) ? 0 : inEc ? 2 : 1;
                        yc[t] = kind[t] == 2 ? A.dh2 * A.yy[g.idx(Jc, Kc, Lc)] : 0.f;
                    }
#pragma unroll 1
                    for (int ic = 0; ic < 3; ic++) {
                        float Hq[4][8];
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            if (kind[t] == 1) {
#pragma unroll
                                for (int iq = 0; iq < 4; iq++) Hq[iq][t] = CELL(hs[t], 6 + 3 * iq + ic, hi[t]);
                            } else if (kind[t] == 2) {
                                const int o = hg_corner(t);
                                float Vc[8];
#pragma unroll
                                for (int m = 0; m < 8; m++) {
                                    const int n = hg_corner(m);
                                    const int dj = (n & 1) - (o & 1), dk = ((n >> 1) & 1) - ((o >> 1) & 1),
                                              dl = (n >> 2) - (o >> 2);
                                    Vc[m] = A.vin[ic][g.idx(jn + dj, kn + dk, l + dl)];
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
        }
        if constexpr (!F) {
            const Inject* E = nfrc >= 0 ? lfrc : A.force.e;
            const int n = nfrc >= 0 ? nfrc : A.force.n;
            for (int e = 0; e < n; e++)
                if (E[e].idx == q) {
                    const int c = E[e].comp;
                    const float inc = E[e].inc;
                    if (c == 0) f[0] = f[0] + inc;
                    else if (c == 1) f[1] = f[1] + inc;
                    else f[2] = f[2] + inc;
                }
        }
        finish_node<FM>(A, q, jn, kn, l, f, cur[4], uv, dt, st_a, st_v, st_u);
    };

    // ---------------------------------------------------------------- stream
    // ring: planes L0-1, L0, L0+1; staged: L0+2 in flight
#pragma unroll 1
    for (int p = -1; p <= 1; p++) {
        fetch(L0 + p);
        cp_async_wait_all();
        __syncthreads();
        store((L0 + p + 3) % 3);
        __syncthreads();
    }
    fetch(L0 + 2);
    stat_load(L0 - 1, cur);
    uv_load(L0, uv);
    cells(L0 - 1, std::false_type{});
    stat_load(L0, cur);
#pragma unroll 1
    for (int l = L0; l <= L1; l++) {
        cells(l, std::false_type{});
        float nxt[5], nuv[6];
        stat_load(l + 1, nxt);
        cp_async_wait_all();
        __syncthreads();  // cell plane l complete, staged plane l+2 landed
        store((l + 2) % 3);
        nodes(l, std::false_type{});
        uv_load(l + 1, nuv);
        __syncthreads();  // ring slot l+2 complete, staging and cell slot l-1 free
        fetch(l + 3);
#pragma unroll
        for (int i = 0; i < 5; i++) cur[i] = nxt[i];
#pragma unroll
        for (int i = 0; i < 6; i++) uv[i] = nuv[i];
    }
    cp_async_wait_all();
    if (A.stats) {
        bmax(A.red + 0, st_a);
        bmax(A.red + 1, st_v);
        bmax(A.red + 2, st_u);
        bmax(A.red + 3, st_w);
    }
#undef RAW
#undef NODE
#undef CELL
}

// Zero one cell of the fast-arithmetic cell plane (layout of Lay: NGCF
// groups of ncl float4) in the pattern the cell phase writes it: group 1
// and, with two bracket directions, the lower-bracket groups hold float2
// values at index tid, which a float4 store at tid would miss (and would
// clear two other cells' values instead).
template <int NDIR, int NQ>
__device__ __forceinline__ void zero_cell_fm(float4* sC, int tid, int ncl) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    sC[tid] = z;
    reinterpret_cast<float2*>(sC + ncl)[tid] = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float4* cq = sC + (2 + NQ * q) * ncl + tid;
        cq[0] = z;
        cq[ncl] = z;
        if (NDIR == 3) cq[2 * ncl] = z;
        if (NDIR == 2) reinterpret_cast<float2*>(sC + (2 + 4 * NQ) * ncl)[q * ncl + tid] = make_float2(0.f, 0.f);
    }
}

// Zero one cell of the interior kernel's fast-arithmetic cell plane (Lay:
// NGCR groups: four float4 groups, then four float2 arrays).
__device__ __forceinline__ void zero_cell_fr(float4* sC, int tid, int ncl) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        sC[q * ncl + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<float2*>(sC + 4 * ncl)[q * ncl + tid] = make_float2(0.f, 0.f);
    }
}

// Interior kernel: tiles of 31 x 7 nodes from (A.jf, A.kf), planes A.lf0..A.lf1,
// strictly inside the non-PML region, with no PML or boundary terms.
// FM (fast arithmetic): fused multiply-adds, brackets scaled by h once per
// cell, divergence brackets taken as the negated gradient brackets and, on
// terrain meshes, the closed-form brackets of stencil.cuh; equal to the
// reference-order kernel in exact arithmetic, not bit for bit.
template <int GEOM, bool FASTK, bool FM>
__global__ void __launch_bounds__(NTH, GEOM == GEOM_GENERAL ? 1 : 2) k_interior(StepArgs A) {
    using L = Lay<GEOM>;
    constexpr int NGN = L::NGN, NGC = L::NGC, NDIR = L::NDIR;
    extern __shared__ float4 sm4[];
    // fast arithmetic on rectilinear and terrain meshes: the ring holds the
    // raw (u, gam) and (v, z) of each node, copied in by cp.async, and a
    // cell forms w and the hourglass input of its corners from them
    constexpr bool RR = FM && L::RAWRING;
    float* sR = reinterpret_cast<float*>(sm4);  // [RAWF][NPL] staged plane
    float4* sN = sm4 + (RR ? 0 : L::RAWSZ / 4);  // [3 slots][NGN][NPL]
    float4* sC = sN + 3 * NGN * NPL;            // [2 slots][NGC][NCL]; fast arithmetic [NGCF][NCL]
    constexpr int NQ = L::NQ, NGCF = L::NGCF;
#define RAW(f, i) sR[(f) * NPL + (i)]
    const Geom& g = A.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + FJ * ty;
    const int L0 = A.lf0 + blockIdx.z * A.segl;
    const int L1 = min(L0 + A.segl - 1, A.lf1);
    const int j0 = A.jf + blockIdx.x * FOJ, k0 = A.kf + blockIdx.y * FOK;
    const int J = j0 - 1 + tx, K = k0 - 1 + ty;      // this thread's cell column
    const int jn = j0 + tx, kn = k0 + ty;            // this thread's node column
    // the last tile of each row may be partial: its cells past (jend, kend)
    // are computed but feed no output node
    const bool outcol = tx < FOJ && ty < FOK && jn <= A.jend && kn <= A.kend;
    const bool cellcol = J >= g.i1cell[0] && J <= g.i2cell[0] && K >= g.i1cell[1] && K <= g.i2cell[1];
    const bool owncol = J >= j0 && J <= A.jend && K >= k0 && K <= A.kend;
    const float h = g.h, dt = g.dt;
    const unsigned long long nz = f2_pack(A.negzero, A.negzero);  // (-0.0, -0.0) from the host (pair.cuh)
    float st_a = 0.f, st_v = 0.f, st_u = 0.f, st_w = 0.f;
    // terrain meshes: this thread's cell column's x (j, j+1) and y (k, k+1)
    float txa = 0.f, txb = 0.f, tya = 0.f, tyb = 0.f;
    if (GEOM == GEOM_TERRAIN && cellcol) {
        txa = A.x1d[J - 1];
        txb = A.x1d[J];
        tya = A.y1d[K - 1];
        tyb = A.y1d[K];
    }
    // fast arithmetic on terrain meshes: the bracket spacings times h
    const float hdx = h * (txb - txa), hdy = h * (tyb - tya);

    // point injections that fall inside this block (cells / nodes it computes)
    __shared__ Inject lpot[kLocalInject], lmom[kLocalInject], lfrc[kLocalInject];
    __shared__ int lcnt[3];
    // A fast-kernel block whose (j, k) box holds a point source of this step
    // leaves that column to the general kernel (the host lists it there).
    const int gl1 = FASTK ? 0 : L0 - 1, gl2 = FASTK ? g.nm[2] + 1 : L1;
    gather_inject(A.pot, lpot, &lcnt[0], g, j0 - 1, j0 + FOJ - 1, k0 - 1, k0 + FOK - 1, gl1, gl2);
    gather_inject(A.mom, lmom, &lcnt[1], g, j0 - 1, j0 + FOJ - 1, k0 - 1, k0 + FOK - 1, gl1, gl2);
    gather_inject(A.force, lfrc, &lcnt[2], g, j0, j0 + FOJ - 1, k0, k0 + FOK - 1, FASTK ? gl1 : L0, gl2);
    __syncthreads();
    const int npot = lcnt[0], nmom = lcnt[1], nfrc = lcnt[2];
    if (FASTK && (npot != 0 || nmom != 0 || nfrc != 0)) return;

    // ---------------------------------------------------------------- loads
    // stage node plane l (u, v, gam, coordinates) into sR asynchronously
    auto fetch = [&](int l) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH;
            if (n < NPL) {
                const int nj = n % FNJ, nk = n / FNJ;
                const int j = j0 - 1 + nj, k = k0 - 1 + nk;
                const bool ok = j <= g.nm[0] && k <= g.nm[1] && l >= 1 && l <= g.nm[2];
                if (RR) {
                    // ring slot of plane l: group 0 (u, gam), group 1 (v, z)
                    float* d0 = reinterpret_cast<float*>(sN + (l % 3) * (NGN * NPL) + n);
                    float* d1 = reinterpret_cast<float*>(sN + (l % 3) * (NGN * NPL) + NPL + n);
                    if (ok) {
                        const long long q = g.idx(j, k, l);
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            cp_async4(d0 + c, A.uin[c] + q);
                            cp_async4(d1 + c, A.vin[c] + q);
                        }
                        cp_async4(d0 + 3, A.gam + q);
                        if (GEOM == GEOM_TERRAIN) cp_async4(d1 + 3, A.x[2] + q);
                        else d1[3] = 0.f;
                    } else {
#pragma unroll
                        for (int c = 0; c < 4; c++) { d0[c] = 0.f; d1[c] = 0.f; }
                    }
                } else if (ok) {
                    const long long q = g.idx(j, k, l);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        cp_async4(&RAW(c, n), A.uin[c] + q);
                        cp_async4(&RAW(3 + c, n), A.vin[c] + q);
                    }
                    cp_async4(&RAW(6, n), A.gam + q);
                    if (GEOM == GEOM_TERRAIN) cp_async4(&RAW(7, n), A.x[2] + q);
                    if (GEOM == GEOM_GENERAL)
#pragma unroll
                        for (int c = 0; c < 3; c++) cp_async4(&RAW(7 + c, n), A.x[c] + q);
                } else {
#pragma unroll
                    for (int f = 0; f < L::RAWF; f++) RAW(f, n) = 0.f;
                }
            }
        }
        cp_async_commit();
    };
    // staged plane -> ring slot: w1 = u + gam * v (time_integration.f90:36)
    // and the hourglass input hg1 u + dt hg2 v (acceleration.f90:141)
    auto store = [&](int slot) {
        float4* dst = sN + slot * (NGN * NPL);
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH;
            if (n < NPL) {
                const float gm = RAW(6, n);
                float w[3], hh[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float u = RAW(c, n), v = RAW(3 + c, n);
                    w[c] = FM ? fmaf(gm, v, u) : u + gm * v;
                    hh[c] = FM ? fmaf(A.dh2, v, A.hg1 * u) : A.hg1 * u + A.dh2 * v;
                }
                const float c0 = L::NCOORD > 0 ? RAW(7, n) : 0.f;
                const float c1 = L::NCOORD > 1 ? RAW(8, n) : 0.f;
                dst[n] = make_float4(w[0], w[1], w[2], c0);
                dst[NPL + n] = make_float4(hh[0], hh[1], hh[2], c1);
                if (NGN > 2) dst[2 * NPL + n] = make_float4(L::NCOORD > 2 ? RAW(9, n) : 0.f, 0.f, 0.f, 0.f);
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
    // this thread's node u, v (for the update and statistics), one plane ahead
    float uv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    auto uv_load = [&](int l, float* o) {
        const bool nv = outcol && l >= g.i1node[2] && l <= g.i2node[2];
        const long long q = nv ? g.idx(jn, kn, l) : 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            o[c] = nv ? A.uin[c][q] : 0.f;
            o[3 + c] = nv ? A.vin[c][q] : 0.f;
        }
    };

    // one cell's results into cell slot cs (layout of Lay)
#define WRITE_CELL(cs, ed, eo, he, cnb)                                                                   \
    do {                                                                                                   \
        float4* cw_ = sC + (cs) * (NGC * NCL) + tid;                                                       \
        cw_[0] = make_float4(ed[0], ed[1], ed[2], eo[0]);                                                  \
        cw_[NCL] = make_float4(eo[1], eo[2], he[0], he[1]);                                                \
        cw_[2 * NCL] = make_float4(he[3], he[4], he[6], he[7]);                                            \
        cw_[3 * NCL] = make_float4(he[9], he[10], he[2], he[5]);                                           \
        cw_[4 * NCL] = make_float4(he[8], he[11], 0.f, 0.f);                                               \
        if (NDIR >= 2)                                                                                     \
            _Pragma("unroll") for (int q2 = 0; q2 < 4; q2++) cw_[(5 + q2) * NCL] =                         \
                make_float4(cnb[0][2 * q2], cnb[1][2 * q2], cnb[0][2 * q2 + 1], cnb[1][2 * q2 + 1]);        \
        if (NDIR == 3) {                                                                                   \
            cw_[9 * NCL] = make_float4(cnb[NDIR - 1][0], cnb[NDIR - 1][1], cnb[NDIR - 1][2], cnb[NDIR - 1][3]); \
            cw_[10 * NCL] = make_float4(cnb[NDIR - 1][4], cnb[NDIR - 1][5], cnb[NDIR - 1][6], cnb[NDIR - 1][7]); \
        }                                                                                                  \
    } while (0)

    // ---------------------------------------------------------------- cell phase
    constexpr bool CARRY = FM && GEOM != GEOM_GENERAL;
    float4 ca[4], cb[4];  // plane l+1 corners of the last cell computed, for plane l+1's cell
    // fast arithmetic: the terms of this thread's own cell for its own node
    // column (reader q = 0) stay in registers for the node phase
    float ownu[3] = {0.f, 0.f, 0.f}, ownl[3] = {0.f, 0.f, 0.f};
    int carry_l = -1000;  // the plane of that cell
    auto cells = [&](int l, auto fast_tag) {
        constexpr bool F = decltype(fast_tag)::value;
        const int cs = FM ? 0 : l & 1;
        const bool valid = (F || cellcol) && l >= g.i1cell[2] && l <= g.i2cell[2];
        if (!valid) {
            if constexpr (FM) {
                zero_cell_fr(sC, tid, NCL);
#pragma unroll
                for (int i = 0; i < 3; i++) { ownu[i] = 0.f; ownl[i] = 0.f; }
            } else {
                float4* cw = sC + cs * (NGC * NCL) + tid;
#pragma unroll
                for (int i = 0; i < NGC; i++) cw[i * NCL] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            return;
        }
        const long long q = g.idx(J, K, l);
        // corner values by corner id n = dj + 2 dk + 4 dl (node planes l, l+1);
        // fast arithmetic keeps the plane l+1 corners for the next plane's cell
        float Wc[3][8], Hc[3][8], X0[8], X1[8], X2[8];
        {
            const float4* p0 = sN + (l % 3) * (NGN * NPL) + (tx + FNJ * ty);
            const float4* p1 = sN + ((l + 1) % 3) * (NGN * NPL) + (tx + FNJ * ty);
            const bool reuse = CARRY && carry_l == l - 1;
#pragma unroll
            for (int n = 0; n < 8; n++) {
                const float4* p = ((n >> 2) ? p1 : p0) + (n & 1) + FNJ * ((n >> 1) & 1);
                float4 a, b;
                if (CARRY && n < 4 && reuse) {
                    a = ca[n];
                    b = cb[n];
                } else {
                    a = p[0];
                    b = p[NPL];
                    if constexpr (RR) {
                        // raw (u, gam), (v, z) -> (w, z), (hourglass input, 0):
                        // w1 = u + gam * v (time_integration.f90:36) and
                        // hg1 u + dt hg2 v (acceleration.f90:141)
                        const float4 u = a, v = b;
                        a = make_float4(fmaf(u.w, v.x, u.x), fmaf(u.w, v.y, u.y), fmaf(u.w, v.z, u.z), v.w);
                        b = make_float4(fmaf(A.dh2, v.x, A.hg1 * u.x), fmaf(A.dh2, v.y, A.hg1 * u.y),
                                        fmaf(A.dh2, v.z, A.hg1 * u.z), 0.f);
                    }
                }
                if (CARRY && n >= 4) {
                    ca[n - 4] = a;
                    cb[n - 4] = b;
                }
                Wc[0][n] = a.x; Wc[1][n] = a.y; Wc[2][n] = a.z;
                Hc[0][n] = b.x; Hc[1][n] = b.y; Hc[2][n] = b.z;
                if (GEOM == GEOM_TERRAIN) {
                    X0[n] = (n & 1) ? txb : txa;
                    X1[n] = ((n >> 1) & 1) ? tyb : tya;
                    X2[n] = a.w;
                } else if (GEOM == GEOM_GENERAL) {
                    X0[n] = a.w;
                    X1[n] = b.w;
                    X2[n] = p[2 * NPL].x;
                }
            }
            if (CARRY) carry_l = l;
        }
        // support-operator brackets; directions 0 and 1 in the two lanes
        float B[3][8];
        float cnb[NDIR > 0 ? NDIR : 1][8];
        if constexpr (FM) {
            // brackets scaled by h; divergence brackets = negated gradient brackets
            if (GEOM == GEOM_RECT) {
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int t = 0; t < 8; t++) B[a][t] = A.brh.bnc[a][t];
            } else if (GEOM == GEOM_TERRAIN) {
                terrain_brackets_0(hdy, X2, B[0]);
                terrain_brackets_1(hdx, X2, B[1]);
#pragma unroll
                for (int t = 0; t < 8; t++) B[2][t] = A.brh.bnc[2][t];
            } else {
                brackets_nc_g<float>(X1, X2, B[0]);
                brackets_nc_g<float>(X2, X0, B[1]);
                brackets_nc_g<float>(X0, X1, B[2]);
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int t = 0; t < 8; t++) B[a][t] = h * B[a][t];
            }
#pragma unroll
            for (int a = 0; a < NDIR; a++)
#pragma unroll
                for (int t = 0; t < 8; t++) cnb[a][t] = -B[a][cn_of_nc(t)];
        } else if (GEOM == GEOM_RECT) {
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int t = 0; t < 8; t++) B[a][t] = A.br.bnc[a][t];
        } else if (kPaired) {
            F2 PB[8], PC[8], P[8], PN[8];
#pragma unroll
            for (int n = 0; n < 8; n++) {
                PB[n] = f2(X1[n], X2[n], nz);
                PC[n] = f2(X2[n], X0[n], nz);
            }
            brackets_nc_g<F2>(PB, PC, P);
            cell_cn_brackets_g<F2>(PB, PC, P, PN, f2(0.0f, nz));
#pragma unroll
            for (int t = 0; t < 8; t++) {
                B[0][t] = P[t].x();
                B[1][t] = P[t].y();
                cnb[0][t] = PN[t].x();
                cnb[1][t] = PN[t].y();
            }
            if (GEOM == GEOM_TERRAIN) {
#pragma unroll
                for (int t = 0; t < 8; t++) B[2][t] = A.br.bnc[2][t];
            } else {
                brackets_nc_g<float>(X0, X1, B[2]);
                cell_cn_brackets_g<float>(X0, X1, B[2], cnb[NDIR - 1], 0.0f);
            }
        } else {
            brackets_nc_g<float>(X1, X2, B[0]);
            cell_cn_brackets_g<float>(X1, X2, B[0], cnb[0], 0.0f);
            brackets_nc_g<float>(X2, X0, B[1]);
            cell_cn_brackets_g<float>(X2, X0, B[1], cnb[1], 0.0f);
            if (GEOM == GEOM_TERRAIN) {
#pragma unroll
                for (int t = 0; t < 8; t++) B[2][t] = A.br.bnc[2][t];
            } else {
                brackets_nc_g<float>(X0, X1, B[2]);
                cell_cn_brackets_g<float>(X0, X1, B[2], cnb[NDIR - 1], 0.0f);
            }
        }
        float ed[3], eo[3], he[12];
#pragma unroll
        for (int i = 0; i < 12; i++) he[i] = 0.f;
        const bool own = owncol && l >= L0;
        if constexpr (F && FM) {
            // gradients; the off-diagonal pairs are summed here and halved
            // with the modulus below
            float sg[3][3];
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                float W[8];
#pragma unroll
                for (int t = 0; t < 8; t++) W[t] = Wc[ic][term_corner(t)];
#pragma unroll
                for (int id = 0; id < 3; id++) sg[ic][id] = dot8(W, B[id]);
            }
#pragma unroll
            for (int i = 0; i < 3; i++) ed[i] = sg[i][i];
            eo[0] = sg[1][2] + sg[2][1];
            eo[1] = sg[0][2] + sg[2][0];
            eo[2] = sg[0][1] + sg[1][0];
        } else if constexpr (F && !kPaired) {
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                float W[8];
#pragma unroll
                for (int t = 0; t < 8; t++) W[t] = Wc[ic][term_corner(t)];
#pragma unroll
                for (int iid = 0; iid < 3; iid++) {
                    const int id = (ic + iid + 1) % 3;
                    const float s = stencil8(W, B[id], h);
                    if (ic == id) ed[ic] = s;
                    else if (ic < id) eo[3 - ic - id] = 0.5f * s;
                    else eo[3 - ic - id] = eo[3 - ic - id] + 0.5f * s;
                }
            }
        } else if constexpr (F) {
            // strain of an interior cell: s[ic][id] = stencil8(w_ic, B[id]);
            // (ic0, ic1) paired per iid, ic2's first two directions paired
            const F2 h2 = f2(h, nz);
            float sg[3][3];
            F2 W01[8];
            float W2v[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int n = term_corner(t);
                W01[t] = f2(Wc[0][n], Wc[1][n], nz);
                W2v[t] = Wc[2][n];
            }
#pragma unroll
            for (int iid = 0; iid < 3; iid++) {
                const int ia = (0 + iid + 1) % 3, ib = (1 + iid + 1) % 3;
                F2 Bp[8];
#pragma unroll
                for (int t = 0; t < 8; t++) Bp[t] = f2(B[ia][t], B[ib][t], nz);
                const F2 r = stencil8<F2>(W01, Bp, h2);
                sg[0][ia] = r.x();
                sg[1][ib] = r.y();
            }
            {
                F2 W22[8], Bp[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    W22[t] = f2(W2v[t], nz);
                    Bp[t] = f2(B[0][t], B[1][t], nz);
                }
                const F2 r = stencil8<F2>(W22, Bp, h2);
                sg[2][0] = r.x();
                sg[2][1] = r.y();
                sg[2][2] = stencil8<float>(W2v, B[2], h);
            }
#pragma unroll
            for (int i = 0; i < 3; i++) ed[i] = sg[i][i];
            eo[0] = 0.5f * sg[1][2] + 0.5f * sg[2][1];
            eo[1] = 0.5f * sg[0][2] + 0.5f * sg[2][0];
            eo[2] = 0.5f * sg[0][1] + 0.5f * sg[1][0];
        } else {
            // region of the cell (stress.f90:141-248)
            bool nearS[3], farS[3], anyS = false;
            const int cc[3] = {J, K, l};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                nearS[d] = cc[d] <= g.i1pml[d];
                farS[d] = cc[d] >= g.i2pml[d] - 1;
                anyS = anyS || nearS[d] || farS[d];
            }
            // PML cells that are not elastic-hourglass cells carry the viscous
            // hourglass values dt hg2 yy hourglass_nc(v) in the hourglass
            // slots (acceleration.f90:164-183)
            bool inEc = true;
#pragma unroll
            for (int d = 0; d < 3; d++) inEc = inEc && cc[d] >= g.i1pml[d] && cc[d] <= g.i2pml[d] - 1;
            const bool visc = A.hourglass && A.hgvisc && anyS && !inEc;
            const float yv = A.dh2 * cur[3];
#pragma unroll
            for (int i = 0; i < 3; i++) { ed[i] = 0.f; eo[i] = 0.f; }
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                float W[8], U[8], V[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    W[t] = Wc[ic][term_corner(t)];
                    U[t] = 0.f;
                    V[t] = 0.f;
                }
                if (anyS) {
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        const int n = term_corner(t);
                        const long long qn = g.idx(J + (n & 1), K + ((n >> 1) & 1), l + (n >> 2));
                        U[t] = A.uin[ic][qn];
                        V[t] = A.vin[ic][qn];
                    }
                }
                if (visc) {
                    float Vc[8], Vh[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) Vc[term_corner(t)] = V[t];
#pragma unroll
                    for (int t = 0; t < 8; t++) Vh[t] = Vc[hg_corner(t)];
#pragma unroll
                    for (int iq = 0; iq < 4; iq++) he[3 * iq + ic] = yv * hg_sum(Vh, iq);
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
        }
        if constexpr (FM) {
            // (2 mu e + lam tr e) / V; the off-diagonal sums carry the 1/2
            const float r = cur[2], mur = cur[1] * r, m2r = mur + mur;
            const float s1r = (cur[0] * r) * (ed[0] + ed[1] + ed[2]);
#pragma unroll
            for (int i = 0; i < 3; i++) { ed[i] = fmaf(m2r, ed[i], s1r); eo[i] = mur * eo[i]; }
        } else {
            {
                const float lm = cur[0], m2 = 2.0f * cur[1];
                const float s1v = lm * (ed[0] + ed[1] + ed[2]);
#pragma unroll
                for (int i = 0; i < 3; i++) { ed[i] = m2 * ed[i] + s1v; eo[i] = m2 * eo[i]; }
            }
            if constexpr (!F) apply_inject(lmom, nmom, A.mom, q, ed, eo);
            {
                const float r = cur[2];
#pragma unroll
                for (int i = 0; i < 3; i++) { ed[i] = ed[i] * r; eo[i] = eo[i] * r; }
            }
        }
        if (A.stats && own)
            st_w = fmaxn(st_w, (ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]) + 2.0f * (eo[0] * eo[0] + eo[1] * eo[1] + eo[2] * eo[2]));
        // elastic hourglass cell values (acceleration.f90:141-156)
        if (A.hourglass) {
            bool inE = true;
            if constexpr (!F) {
                const int cc[3] = {J, K, l};
#pragma unroll
                for (int d = 0; d < 3; d++) inE = inE && cc[d] >= g.i1pml[d] && cc[d] <= g.i2pml[d] - 1;
            }
            if (FM && inE) {
                // the four mode sums by butterflies (stencil.cuh: hg_modes)
                const float y = cur[3];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    float m[4];
                    hg_modes<float>(Hc[ic], m);
#pragma unroll
                    for (int iq = 0; iq < 4; iq++) he[3 * iq + ic] = m[iq] * y;
                }
            } else if (inE && (!F || !kPaired)) {
                const float y = cur[3];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    float W2[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) W2[t] = Hc[ic][hg_corner(t)];
#pragma unroll
                    for (int iq = 0; iq < 4; iq++) he[3 * iq + ic] = hg_sum(W2, iq) * y;
                }
            } else if (inE) {
                const float y = cur[3];
                F2 H01[8];
                float H2v[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int n = hg_corner(t);
                    H01[t] = f2(Hc[0][n], Hc[1][n], nz);
                    H2v[t] = Hc[2][n];
                }
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    const F2 r = hg_sum<F2>(H01, iq) * f2(y, nz);
                    he[3 * iq] = r.x();
                    he[3 * iq + 1] = r.y();
                    he[3 * iq + 2] = hg_sum<float>(H2v, iq) * y;
                }
            }
        }
        if constexpr (FM) {
            // fast layout: for each node column q = cj + 2 ck that reads this
            // cell, the cell's whole terms of that column's force at node
            // plane l (fu, the node above the cell) and l + 1 (fl, the node
            // below it): the hourglass_cn sums (the signs of hourglass_cn
            // terms hg_term(7 - p) at cell position p, stencil.cuh:
            // hg_reader) plus the divergence of the cell's stress with that
            // node's diff_cn brackets
            const float S[6] = {ed[0], ed[1], ed[2], eo[0], eo[1], eo[2]};
            float hr[3][4];
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                const float m[4] = {he[ic], he[3 + ic], he[6 + ic], he[9 + ic]};
                hg_readers_pre<float>(m, hr[ic]);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int cj = q & 1, ck = q >> 1;
                const int tu = cj + 2 + 4 * ck, tl = cj + 4 * ck;
                float Bu[3], Bl[3];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    Bu[a] = a < NDIR ? cnb[a < NDIR ? a : 0][tu] : A.brh.bcn[a][tu];
                    Bl[a] = a < NDIR ? cnb[a < NDIR ? a : 0][tl] : A.brh.bcn[a][tl];
                }
                float fu[3], fl[3];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) hg_reader<float>(hr[ic], q, fu[ic], fl[ic]);
#pragma unroll
                for (int ic = 0; ic < 3; ic++)
#pragma unroll
                    for (int iid = 0; iid < 3; iid++) {
                        const int id = (ic + iid) % 3, comp = ic == id ? ic : 3 + (3 - ic - id);
                        fu[ic] = fmaf(S[comp], Bu[id], fu[ic]);
                        fl[ic] = fmaf(S[comp], Bl[id], fl[ic]);
                    }
                if (q == 0) {
#pragma unroll
                    for (int i = 0; i < 3; i++) { ownu[i] = fu[i]; ownl[i] = fl[i]; }
                    continue;
                }
                sC[q * NCL + tid] = make_float4(fu[0], fu[1], fu[2], fl[0]);
                reinterpret_cast<float2*>(sC + 4 * NCL)[q * NCL + tid] = make_float2(fl[1], fl[2]);
            }
        } else {
            WRITE_CELL(cs, ed, eo, he, cnb);
        }
    };

    // ---------------------------------------------------------------- node phase
    // The eight cells of node (jn, kn, l) are cell positions p = cj + 2 ck + 4 cl
    // at (J + cj, K + ck, l - 1 + cl); diff_cn term t sits at position
    // pt(t), hourglass_cn term t at position ph(t).
    // (reference order only; fast arithmetic uses nodes_fm below)
    auto nodes = [&](int l, auto fast_tag) {
        constexpr bool F = decltype(fast_tag)::value;
        if (!outcol) return;
        const long long q = g.idx(jn, kn, l);
        const float4* c0 = sC + ((l - 1) & 1) * (NGC * NCL) + tid;  // cell plane l-1
        const float4* c1 = sC + (l & 1) * (NGC * NCL) + tid;        // cell plane l
        auto cpos = [&](int p) { return ((p >> 2) ? c1 : c0) + (p & 1) + FJ * ((p >> 1) & 1); };
        auto pt = [](int t) { return (t & 1) + 2 * (t >> 2) + 4 * ((t >> 1) & 1); };
        auto ph = [](int t) {
            const int o = hg_corner(t);
            return (1 - (o & 1)) + 2 * (1 - ((o >> 1) & 1)) + 4 * (1 - (o >> 2));
        };
        // stress (6) and divergence brackets by diff_cn term
        float S[6][8], Bc[3][8], HA0[2][8];  // HA0: mode-0 (x, y) hourglass values by diff_cn term
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const float4* cp = cpos(pt(t));
            const float4 a = cp[0], b = cp[NCL];
            S[0][t] = a.x; S[1][t] = a.y; S[2][t] = a.z; S[3][t] = a.w; S[4][t] = b.x; S[5][t] = b.y;
            HA0[0][t] = b.z;
            HA0[1][t] = b.w;
            if (NDIR >= 2) {
                const float2 bb = reinterpret_cast<const float2*>(cp + (5 + t / 2) * NCL)[t % 2];
                Bc[0][t] = bb.x;
                Bc[1][t] = bb.y;
            }
            if (NDIR == 3) Bc[2][t] = reinterpret_cast<const float*>(cp + (9 + t / 4) * NCL)[t % 4];
            if (GEOM == GEOM_RECT)
#pragma unroll
                for (int id = 0; id < 3; id++) Bc[id][t] = A.br.bcn[id][t];
            if (GEOM == GEOM_TERRAIN) Bc[2][t] = A.br.bcn[2][t];
        }
        float f[3];
        if constexpr (F && !kPaired) {
#pragma unroll
            for (int ic = 0; ic < 3; ic++)
#pragma unroll
                for (int iid = 0; iid < 3; iid++) {
                    const int id = (ic + iid) % 3;
                    const int comp = ic == id ? ic : 3 + (3 - ic - id);
                    const float s = stencil8(S[comp], Bc[id], h);
                    f[ic] = iid == 0 ? s : f[ic] + s;
                }
        } else if constexpr (F) {
            // f[ic] = sum over iid of stencil8(sigma(ic, id), Bc[id]), id = (ic + iid) % 3;
            // (ic0, ic1) paired per iid, ic2's first two terms paired
            const F2 h2 = f2(h, nz);
            F2 f01;
#pragma unroll
            for (int iid = 0; iid < 3; iid++) {
                const int ia = iid, ib = (1 + iid) % 3;
                const int ca = 0 == ia ? 0 : 3 + (3 - 0 - ia), cb = 1 == ib ? 1 : 3 + (3 - 1 - ib);
                F2 Fp[8], Bp[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    Fp[t] = f2(S[ca][t], S[cb][t], nz);
                    Bp[t] = f2(Bc[ia][t], Bc[ib][t], nz);
                }
                const F2 r = stencil8<F2>(Fp, Bp, h2);
                f01 = iid == 0 ? r : f01 + r;
            }
            F2 Fp[8], Bp[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                Fp[t] = f2(S[2][t], S[4][t], nz);
                Bp[t] = f2(Bc[2][t], Bc[0][t], nz);
            }
            const F2 r = stencil8<F2>(Fp, Bp, h2);
            f[2] = r.x() + r.y();
            f[2] = f[2] + stencil8<float>(S[3], Bc[1], h);
            f[0] = f01.x();
            f[1] = f01.y();
        } else {
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
#pragma unroll
                for (int iid = 0; iid < 3; iid++) {
                    const int id = (ic + iid) % 3;
                    const int comp = ic == id ? ic : 3 + (3 - ic - id);
                    float s = stencil8(S[comp], Bc[id], h);
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
        }
        if (A.hourglass) {
            bool ne = true;
            if constexpr (!F) {
                const int cn_[3] = {jn, kn, l};
#pragma unroll
                for (int d = 0; d < 3; d++) ne = ne && cn_[d] >= g.i1pml[d] + 1 && cn_[d] <= g.i2pml[d] - 1;
            }
            // hourglass values of mode iq by hourglass_cn term: (x, y) pair and z
#define HVALS(iq, hA, hB)                                                      \
    _Pragma("unroll") for (int t = 0; t < 8; t++) {                            \
        const float4* cp_ = cpos(ph(t));                                       \
        if ((iq) == 0) {                                                       \
            const float4 b_ = cp_[NCL];                                        \
            hA[t] = f2(b_.z, b_.w, nz);                                        \
            hB[t] = cp_[3 * NCL].z;                                            \
        } else if ((iq) == 1) {                                                \
            const float4 b_ = cp_[2 * NCL];                                    \
            hA[t] = f2(b_.x, b_.y, nz);                                        \
            hB[t] = cp_[3 * NCL].w;                                            \
        } else if ((iq) == 2) {                                                \
            const float4 b_ = cp_[2 * NCL];                                    \
            hA[t] = f2(b_.z, b_.w, nz);                                        \
            hB[t] = cp_[4 * NCL].x;                                            \
        } else {                                                               \
            const float4 b_ = cp_[3 * NCL];                                    \
            hA[t] = f2(b_.x, b_.y, nz);                                        \
            hB[t] = cp_[4 * NCL].y;                                            \
        }                                                                      \
    }
            if (ne && F && !kPaired) {
                // each cell's hourglass groups once, as 128 / 64-bit loads:
                // g1.zw = mode 0 (x, y), g2 = modes 1, 2 (x, y), g3 = mode 3
                // (x, y), z of modes 0, 1, g4 = z of modes 2, 3
                float H[4][3][8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int p = ph(t);
                    // diff_cn term at the same cell position
                    const int tp = (p & 1) + 4 * ((p >> 1) & 1) + 2 * (p >> 2);
                    const float4* cp_ = cpos(p);
                    const float4 g2 = cp_[2 * NCL], g3 = cp_[3 * NCL];
                    const float2 g4 = reinterpret_cast<const float2*>(cp_ + 4 * NCL)[0];
                    H[0][0][t] = HA0[0][tp]; H[0][1][t] = HA0[1][tp]; H[0][2][t] = g3.z;
                    H[1][0][t] = g2.x; H[1][1][t] = g2.y; H[1][2][t] = g3.w;
                    H[2][0][t] = g2.z; H[2][1][t] = g2.w; H[2][2][t] = g4.x;
                    H[3][0][t] = g3.x; H[3][1][t] = g3.y; H[3][2][t] = g4.y;
                }
#pragma unroll
                for (int iq = 0; iq < 4; iq++)
#pragma unroll
                    for (int ic = 0; ic < 3; ic++) f[ic] = f[ic] - hg_sum(H[iq][ic], iq);
            } else if (ne && (!F || !kPaired)) {
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    F2 hA[8];
                    float hB[8];
                    HVALS(iq, hA, hB);
                    float Hx[8], Hy[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) { Hx[t] = hA[t].x(); Hy[t] = hA[t].y(); }
                    f[0] = f[0] - hg_sum(Hx, iq);
                    f[1] = f[1] - hg_sum(Hy, iq);
                    f[2] = f[2] - hg_sum(hB, iq);
                }
            } else if (ne) {
                F2 f01 = f2(f[0], f[1], nz);
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    F2 hA[8];
                    float hB[8];
                    HVALS(iq, hA, hB);
                    f01 = f01 - hg_sum<F2>(hA, iq);
                    f[2] = f[2] - hg_sum<float>(hB, iq);
                }
                f[0] = f01.x();
                f[1] = f01.y();
            } else if constexpr (!F) {
                if (A.hgvisc) {
                    // viscous-only hourglass in the PML (acceleration.f90:164-199):
                    // every cell of a PML node is a PML cell; pure PML cells
                    // hold their viscous values in the hourglass slots, cells
                    // that are also elastic-hourglass cells (the layer next to
                    // the elastic region) are evaluated here from v
                    int kind[8];
                    float yc[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) {
                        const int o = hg_corner(t);
                        const int Jc = jn - (o & 1), Kc = kn - ((o >> 1) & 1), Lc = l - (o >> 2);
                        const bool real = Jc >= g.i1cell[0] && Jc <= g.i2cell[0] && Kc >= g.i1cell[1] &&
                                          Kc <= g.i2cell[1] && Lc >= g.i1cell[2] && Lc <= g.i2cell[2];
                        const bool slab = Jc <= g.i1pml[0] || Jc >= g.i2pml[0] - 1 || Kc <= g.i1pml[1] ||
                                          Kc >= g.i2pml[1] - 1 || Lc <= g.i1pml[2] || Lc >= g.i2pml[2] - 1;
                        const bool inEc = Jc >= g.i1pml[0] && Jc <= g.i2pml[0] - 1 && Kc >= g.i1pml[1] &&
                                          Kc <= g.i2pml[1] - 1 && Lc >= g.i1pml[2] && Lc <= g.i2pml[2] - 1;
                        kind[t] = !(real && slab) ? 0 : inEc ? 2 : 1;
                        yc[t] = kind[t] == 2 ? A.dh2 * A.yy[g.idx(Jc, Kc, Lc)] : 0.f;
                    }
#pragma unroll
                    for (int iq = 0; iq < 4; iq++) {
                        F2 hA[8];
                        float hB[8];
                        HVALS(iq, hA, hB);
                        float Hq[3][8];
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            Hq[0][t] = kind[t] == 1 ? hA[t].x() : 0.f;
                            Hq[1][t] = kind[t] == 1 ? hA[t].y() : 0.f;
                            Hq[2][t] = kind[t] == 1 ? hB[t] : 0.f;
                        }
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            if (kind[t] == 2) {
                                const int o = hg_corner(t);
#pragma unroll
                                for (int ic = 0; ic < 3; ic++) {
                                    float Vc[8];
#pragma unroll
                                    for (int m = 0; m < 8; m++) {
                                        const int n = hg_corner(m);
                                        const int dj = (n & 1) - (o & 1), dk = ((n >> 1) & 1) - ((o >> 1) & 1),
                                                  dl = (n >> 2) - (o >> 2);
                                        const float* vp = ic == 0 ? A.vin[0] : ic == 1 ? A.vin[1] : A.vin[2];
                                        Vc[m] = vp[g.idx(jn + dj, kn + dk, l + dl)];
                                    }
                                    const float hv = yc[t] * hg_sum(Vc, iq);
                                    if (ic == 0) Hq[0][t] = hv;
                                    else if (ic == 1) Hq[1][t] = hv;
                                    else Hq[2][t] = hv;
                                }
                            }
                        }
#pragma unroll
                        for (int ic = 0; ic < 3; ic++) f[ic] = f[ic] - hg_sum(Hq[ic], iq);
                    }
                }
            }
        }
        if constexpr (!F) {
            const Inject* E = nfrc >= 0 ? lfrc : A.force.e;
            const int n = nfrc >= 0 ? nfrc : A.force.n;
            for (int e = 0; e < n; e++)
                if (E[e].idx == q) {
                    const int c = E[e].comp;
                    const float inc = E[e].inc;
                    if (c == 0) f[0] = f[0] + inc;
                    else if (c == 1) f[1] = f[1] + inc;
                    else f[2] = f[2] + inc;
                }
        }
        finish_node<FM>(A, q, jn, kn, l, f, cur[4], uv, dt, st_a, st_v, st_u);
    };

    // ------------------------------------------------- node phase, fast arithmetic
    // Each cell plane is read once: at node plane l a thread takes the four
    // cells of plane l around its node column, adds their terms to node l
    // (cells above it) and keeps their terms for node l + 1 (cells below it)
    // in fc for the next plane.
    float fc[3] = {0.f, 0.f, 0.f};
    auto nodes_fm = [&](int l, bool finish) {
        if (!outcol) return;
        // the four cells of plane l around the node column: their terms for
        // node l (above them) and for node l + 1 (below), the latter carried
        // q = 0 is this thread's own cell, whose terms are in registers
        float fu[3] = {fc[0] + ownu[0], fc[1] + ownu[1], fc[2] + ownu[2]};
        float fl[3] = {ownl[0], ownl[1], ownl[2]};
#pragma unroll
        for (int q = 1; q < 4; q++) {
            const int ci = tid + (q & 1) + FJ * (q >> 1);  // the cell (J + cj, K + ck)
            const float4 a = sC[q * NCL + ci];
            const float2 b = reinterpret_cast<const float2*>(sC + 4 * NCL)[q * NCL + ci];
            fu[0] = fu[0] + a.x;
            fu[1] = fu[1] + a.y;
            fu[2] = fu[2] + a.z;
            fl[0] = fl[0] + a.w;
            fl[1] = fl[1] + b.x;
            fl[2] = fl[2] + b.y;
        }
#pragma unroll
        for (int i = 0; i < 3; i++) fc[i] = fl[i];
        if (!finish) return;
        if constexpr (RR) {
            // this node's raw u, v from ring slot l
            const float4* pn = sN + (l % 3) * (NGN * NPL) + (tx + 1) + FNJ * (ty + 1);
            const float4 a = pn[0], b = pn[NPL];
            const float uvl[6] = {a.x, a.y, a.z, b.x, b.y, b.z};
            finish_node<FM>(A, g.idx(jn, kn, l), jn, kn, l, fu, cur[4], uvl, dt, st_a, st_v, st_u);
        } else {
            finish_node<FM>(A, g.idx(jn, kn, l), jn, kn, l, fu, cur[4], uv, dt, st_a, st_v, st_u);
        }
    };

    // ---------------------------------------------------------------- stream
    // ring: planes L0-1, L0, L0+1; staged: L0+2 in flight
    constexpr std::integral_constant<bool, FASTK> path{};
    if constexpr (RR) {
        // raw ring: planes L0-1, L0, L0+1 straight into their slots; plane
        // l + 3 goes into slot l once cells(l) and nodes(l) are done with it
#pragma unroll 1
        for (int p = -1; p <= 1; p++) fetch(L0 + p);
        cp_async_wait_all();
        __syncthreads();
        stat_load(L0 - 1, cur);
        cells(L0 - 1, path);
        __syncthreads();  // cell plane L0-1 complete: its terms for node L0
        nodes_fm(L0 - 1, false);
        __syncthreads();  // one cell slot: read before cells(L0) overwrites it; slot L0-1 free
        fetch(L0 + 2);
        stat_load(L0, cur);
#pragma unroll 1
        for (int l = L0; l <= L1; l++) {
            cells(l, path);
            float nxt[5];
            stat_load(l + 1, nxt);
            cp_async_wait_all();
            __syncthreads();  // cell plane l complete, plane l+2 landed
            nodes_fm(l, true);
            __syncthreads();  // cell plane and ring slot l free
            fetch(l + 3);
#pragma unroll
            for (int i = 0; i < 5; i++) cur[i] = nxt[i];
        }
        cp_async_wait_all();
        if (A.stats) {
            bmax(A.red + 0, st_a);
            bmax(A.red + 1, st_v);
            bmax(A.red + 2, st_u);
            bmax(A.red + 3, st_w);
        }
        return;
    }
#pragma unroll 1
    for (int p = -1; p <= 1; p++) {
        fetch(L0 + p);
        cp_async_wait_all();
        __syncthreads();
        store((L0 + p + 3) % 3);
        __syncthreads();
    }
    fetch(L0 + 2);
    stat_load(L0 - 1, cur);
    uv_load(L0, uv);
    cells(L0 - 1, path);
    if constexpr (FM) {
        __syncthreads();  // cell plane L0-1 complete: its terms for node L0
        nodes_fm(L0 - 1, false);
        __syncthreads();  // one cell slot: read before cells(L0) overwrites it
    }
    stat_load(L0, cur);
#pragma unroll 1
    for (int l = L0; l <= L1; l++) {
        cells(l, path);
        float nxt[5], nuv[6];
        stat_load(l + 1, nxt);
        cp_async_wait_all();
        __syncthreads();  // cell plane l complete, staged plane l+2 landed
        store((l + 2) % 3);
        if constexpr (FM) nodes_fm(l, true);
        else nodes(l, path);
        uv_load(l + 1, nuv);
        __syncthreads();  // ring slot l+2 complete, staging and cell slot l-1 free
        fetch(l + 3);
#pragma unroll
        for (int i = 0; i < 5; i++) cur[i] = nxt[i];
#pragma unroll
        for (int i = 0; i < 6; i++) uv[i] = nuv[i];
    }
    cp_async_wait_all();
    if (A.stats) {
        bmax(A.red + 0, st_a);
        bmax(A.red + 1, st_v);
        bmax(A.red + 2, st_u);
        bmax(A.red + 3, st_w);
    }
#undef RAW
#undef WRITE_CELL
#undef HVALS
}

#include "slab.cuh"

// A region of shell items made by one push_box call: boxes of 15 x 15
// nodes from (j1, k1) and ipl planes from l1, l outermost, j innermost.
struct BoxRegion {
    int j1, k1, l1, j2, k2, l2, ipl, nbj, nbk, nbl, first;
};

// Work decomposition of a fused step, fixed by the mesh.  The interior
// rectangle holds the node columns (j, k) whose adjacent cells all lie
// strictly inside the non-PML region, jf..jend x kf..kend; it is tiled by
// 31 x 7 node tiles from (jf, kf) (the last tile of a row may be partial)
// and runs the interior kernel over the node planes lf0..lf1 whose cells are
// interior (or the halo plane of a free surface).  Everything else -- the
// PML faces at full depth, the PML planes of the interior rectangle, and in
// each step the interior tiles holding a point source -- is covered by
// masked 15 x 15 node boxes for the shell kernel.  Boxes and tiles partition
// the nodes, so every node, and every PML memory, is updated once.
struct FusedPlan {
    int jf = 0, jend = -1, kf = 0, kend = -1;   // interior rectangle (inclusive)
    int nbx = 0, nby = 0;                       // interior tiles
    int lf0 = 0, lf1 = -1;                      // interior node planes (inclusive)
    int segl = 0, nseg = 1;                     // interior planes per block, blocks per column
    int ipl = 16;                               // planes per item of a point-source tile
    std::vector<int> base;                      // shell items without point sources (6 ints each)
    std::vector<int> bmask;                     // per base item: k_slab class (0..3: MASK 1, 2, 4, 7)
    std::vector<BoxRegion> regions;             // how the base items were laid out
    std::vector<int> cur;                       // items of the last upload
    int* d_items = nullptr;
    int* h_items = nullptr;                     // pinned staging
    int cap = 0;                                // items
    cudaEvent_t done = nullptr;
    // the PML-shell kernel runs on a second stream, concurrently with the
    // interior kernel (they write disjoint nodes and read the same inputs)
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // each k_slab class on its own stream, forked from and joined back into
    // the stream of the shell launches, so that the classes' tails overlap
    cudaStream_t cst[4] = {};
    cudaEvent_t cfork = nullptr, cdone[4] = {};
};

void fused_free(Solver& s) {
    FusedPlan* P = s.fplan;
    if (!P) return;
    if (P->done) cudaEventDestroy(P->done);
    if (P->fork) cudaEventDestroy(P->fork);
    if (P->join) cudaEventDestroy(P->join);
    if (P->side) cudaStreamDestroy(P->side);
    if (P->cfork) cudaEventDestroy(P->cfork);
    for (int c = 0; c < 4; c++) {
        if (P->cdone[c]) cudaEventDestroy(P->cdone[c]);
        if (P->cst[c]) cudaStreamDestroy(P->cst[c]);
    }
    dev_free(s, P->d_items);
    pinned_put(P->h_items);
    delete P;
    s.fplan = nullptr;
}

// Planes per block.  Each block streams its column through the planes, so
// a small mesh is cut into shorter plane ranges until both kernels have
// about kWaveBlocks blocks per SM; a range starts with a prologue of about
// two planes, so it is kept at kMinPlanes planes or more.
static constexpr int kItemPlanes = 96;
static constexpr int kMinPlanes = 8;
static constexpr int kWaveBlocks = 4;
// planes per item of an interior tile holding a point source (k_shell): a
// few tile columns only, so short items spread them over the SMs
static constexpr int kSourcePlanes = 16;

// shell items covering node box [j1, j2] x [k1, k2] x [l1, l2]
static void push_box(std::vector<int>& v, int ipl, int j1, int j2, int k1, int k2, int l1, int l2,
                     std::vector<BoxRegion>* reg = nullptr) {
    if (j1 > j2 || k1 > k2 || l1 > l2) return;
    if (reg)
        reg->push_back({j1, k1, l1, j2, k2, l2, ipl, (j2 - j1) / (SJ - 1) + 1, (k2 - k1) / (SK - 1) + 1,
                        (l2 - l1) / ipl + 1, (int)v.size() / 6});
    for (int a = l1; a <= l2; a += ipl)
        for (int k = k1; k <= k2; k += SK - 1)
            for (int j = j1; j <= j2; j += SJ - 1) {
                const int it[6] = {j, k, std::min(j2, j + SJ - 2), std::min(k2, k + SK - 2), a,
                                   std::min(l2, a + ipl - 1)};
                v.insert(v.end(), it, it + 6);
            }
}

static FusedPlan& fused_plan(Solver& s) {
    if (s.fplan) return *s.fplan;
    FusedPlan* P = new FusedPlan();
    s.fplan = P;
    const Geom& g = s.g;
    // Node c along axis d is interior when it is outside the PML and each
    // adjacent cell is either a real cell outside the PML or a cell outside
    // the mesh (a boundary without PML, whose coefficients are zero: the
    // kernel then adds exactly zero for it, as the reference does).
    auto cin = [&](int d, int c) { return c > g.i1pml[d] && c < g.i2pml[d] - 1 && c >= g.i1cell[d] && c <= g.i2cell[d]; };
    auto cellok = [&](int d, int c) { return c < g.i1cell[d] || c > g.i2cell[d] || cin(d, c); };
    auto nodeok = [&](int d, int c) { return c >= g.i1pml[d] + 1 && c <= g.i2pml[d] - 1 && cellok(d, c - 1) && cellok(d, c); };
    auto range = [&](int d, int& a, int& b) {
        a = 0;
        b = -1;
        for (int c = g.i1node[d]; c <= g.i2node[d]; c++)
            if (nodeok(d, c)) {
                if (b < a) a = c;
                if (b == c - 1 || b < a) b = c;
            }
    };
    range(0, P->jf, P->jend);
    range(1, P->kf, P->kend);
    range(2, P->lf0, P->lf1);
    const bool inner = P->jend >= P->jf && P->kend >= P->kf && P->lf1 >= P->lf0;
    const int L1 = g.i1node[2], L2 = g.i2node[2];
    int sms = 148;
    SORD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device));
    const int want = kWaveBlocks * sms;
    // regions of the shell, cut where the PML of another axis begins so that
    // each is damped along as few axes as possible (its k_slab class)
    struct RegionBox {
        int lo[3], hi[3];
    };
    std::vector<RegionBox> rb;
    auto add = [&](int j1, int j2, int k1, int k2, int l1, int l2) {
        if (j1 <= j2 && k1 <= k2 && l1 <= l2) rb.push_back({{j1, k1, l1}, {j2, k2, l2}});
    };
    if (!inner) {
        add(g.i1node[0], g.i2node[0], g.i1node[1], g.i2node[1], L1, L2);
    } else {
        const int kr[3][2] = {{g.i1node[1], P->kf - 1}, {P->kf, P->kend}, {P->kend + 1, g.i2node[1]}};
        const int lr[3][2] = {{L1, P->lf0 - 1}, {P->lf0, P->lf1}, {P->lf1 + 1, L2}};
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                add(g.i1node[0], P->jf - 1, kr[a][0], kr[a][1], lr[b][0], lr[b][1]);
                add(P->jend + 1, g.i2node[0], kr[a][0], kr[a][1], lr[b][0], lr[b][1]);
            }
        for (int b = 0; b < 3; b++) {
            add(P->jf, P->jend, g.i1node[1], P->kf - 1, lr[b][0], lr[b][1]);
            add(P->jf, P->jend, P->kend + 1, g.i2node[1], lr[b][0], lr[b][1]);
        }
        add(P->jf, P->jend, P->kf, P->kend, L1, P->lf0 - 1);
        add(P->jf, P->jend, P->kf, P->kend, P->lf1 + 1, L2);
    }
    // k_slab class of a node box: axis d needs the PML terms when a real cell
    // the box computes (node range a..b -> cells a-1..b) or one of its real
    // nodes lies in a PML slab of d; one axis -> its own class, more -> all
    auto klass = [&](const int* lo, const int* hi) {
        int m = 0;
        for (int d = 0; d < 3; d++) {
            for (int c = std::max(lo[d] - 1, g.i1cell[d]); c <= std::min(hi[d], g.i2cell[d]); c++)
                if (c <= g.i1pml[d] || c >= g.i2pml[d] - 1) m |= 1 << d;
            for (int c = std::max(lo[d], g.i1node[d]); c <= std::min(hi[d], g.i2node[d]); c++)
                if (c <= g.i1pml[d] || c >= g.i2pml[d]) m |= 1 << d;
        }
        return m == 2 ? 1 : m == 4 ? 2 : (m == 0 || m == 1) ? 0 : 3;
    };
    // Planes per item, per class: each class is one launch (on its own
    // stream), so its items are cut as long as the launch still has about
    // kWaveBlocks blocks per SM, and no shorter than kMinPlanes (an item
    // starts with a prologue of about two planes).
    std::vector<int> rcls;
    for (const RegionBox& r : rb) rcls.push_back(klass(r.lo, r.hi));
    int iplc[4];
    for (int c = 0; c < 4; c++) {
        auto count = [&](int ipl) {
            long long n = 0;
            for (size_t i = 0; i < rb.size(); i++)
                if (rcls[i] == c)
                    n += (long long)((rb[i].hi[0] - rb[i].lo[0]) / (SJ - 1) + 1) * ((rb[i].hi[1] - rb[i].lo[1]) / (SK - 1) + 1) *
                         ((rb[i].hi[2] - rb[i].lo[2]) / ipl + 1);
            return n;
        };
        int ipl = kItemPlanes;
        while (ipl > kMinPlanes && count(ipl) < want) ipl = std::max(kMinPlanes, ipl * 2 / 3);
        iplc[c] = ipl;
    }
    P->regions.clear();
    for (size_t i = 0; i < rb.size(); i++)
        push_box(P->base, iplc[rcls[i]], rb[i].lo[0], rb[i].hi[0], rb[i].lo[1], rb[i].hi[1], rb[i].lo[2], rb[i].hi[2],
                 &P->regions);
    P->ipl = kSourcePlanes;
    for (size_t i = 0; i < P->base.size(); i += 6) {
        const int* b = &P->base[i];
        const int lo[3] = {b[0], b[1], b[4]}, hi[3] = {b[2], b[3], b[5]};
        P->bmask.push_back(klass(lo, hi));
    }
    if (!inner) {
        P->jend = P->jf - 1;
    } else {
        P->nbx = (int)div_up(P->jend - P->jf + 1, FOJ);
        P->nby = (int)div_up(P->kend - P->kf + 1, FOK);
        const int planes = P->lf1 - P->lf0 + 1, cols = P->nbx * P->nby;
        const int nseg = std::max(1, std::min((want + cols - 1) / cols, planes / kMinPlanes));
        P->segl = (planes + nseg - 1) / nseg;
        P->nseg = (planes + P->segl - 1) / P->segl;
    }
    P->cap = (int)P->base.size() / 6 + 16384;
    SORD_CUDA(dev_malloc(s, (void**)&P->d_items, sizeof(int) * 6 * P->cap));
    P->h_items = (int*)pinned_get(sizeof(int) * 6 * P->cap);
    SORD_CUDA(cudaEventCreateWithFlags(&P->done, cudaEventDisableTiming));
    SORD_CUDA(cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming));
    SORD_CUDA(cudaEventCreateWithFlags(&P->join, cudaEventDisableTiming));
    SORD_CUDA(cudaStreamCreateWithFlags(&P->side, cudaStreamNonBlocking));
    SORD_CUDA(cudaEventCreateWithFlags(&P->cfork, cudaEventDisableTiming));
    for (int c = 0; c < 4; c++) {
        SORD_CUDA(cudaEventCreateWithFlags(&P->cdone[c], cudaEventDisableTiming));
        SORD_CUDA(cudaStreamCreateWithFlags(&P->cst[c], cudaStreamNonBlocking));
    }
    return *P;
}

// Interior tiles whose (j, k) box holds a point source of this step; the
// boxes are those the interior kernel tests (cells j0-1..j0+30 for potency /
// moment entries, nodes j0..j0+30 for forces), so both sides agree.
static void source_tiles(const Solver& s, const FusedPlan& P, const std::vector<Inject>& e, bool cell,
                         std::vector<std::pair<int, int>>& out) {
    const Geom& g = s.g;
    for (const Inject& x : e) {
        const int j = (int)(x.idx % g.sy) + 1, k = (int)((x.idx / g.sy) % g.nm[1]) + 1;
        for (int bx = 0; bx < P.nbx; bx++) {
            const int j0 = P.jf + bx * FOJ;
            if (!(cell ? (j >= j0 - 1 && j <= j0 + FOJ - 1) : (j >= j0 && j <= j0 + FOJ - 1))) continue;
            for (int by = 0; by < P.nby; by++) {
                const int k0 = P.kf + by * FOK;
                if (cell ? (k >= k0 - 1 && k <= k0 + FOK - 1) : (k >= k0 && k <= k0 + FOK - 1)) out.push_back({bx, by});
            }
        }
    }
}

template <int GEOM, bool FASTK>
static void launch_mode(Solver& s, const StepArgs& A, dim3 grid, cudaStream_t st) {
    const size_t bytes = FASTK ? (s.arith ? Lay<GEOM>::bytes_fm : Lay<GEOM>::bytes)
                               : LayS<GEOM, (SJ + 1) * (SK + 1), SJ * SK>::bytes;
    if (FASTK && s.arith) {
        smem_limit((const void*)k_interior<GEOM, true, true>, (int)bytes);
        k_interior<GEOM, true, true><<<grid, dim3(FJ, FK), bytes, st>>>(A);
    } else if (FASTK) {
        smem_limit((const void*)k_interior<GEOM, true, false>, (int)bytes);
        k_interior<GEOM, true, false><<<grid, dim3(FJ, FK), bytes, st>>>(A);
    } else if (s.arith) {
        smem_limit((const void*)k_shell<GEOM, true>, (int)bytes);
        k_shell<GEOM, true><<<grid, dim3(SJ, SK), bytes, st>>>(A);
    } else {
        smem_limit((const void*)k_shell<GEOM, false>, (int)bytes);
        k_shell<GEOM, false><<<grid, dim3(SJ, SK), bytes, st>>>(A);
    }
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

template <int GEOM, int MASK>
static void launch_slab_m(Solver& s, const StepArgs& A, unsigned n, cudaStream_t st) {
    const size_t bytes = LaySl<GEOM>::bytes;
    smem_limit((const void*)k_slab<GEOM, MASK>, (int)bytes);
    k_slab<GEOM, MASK><<<dim3(n, 1, 1), dim3(SJ, SK), bytes, st>>>(A);
    s.launches++;
    SORD_CUDA(cudaGetLastError());
}

template <int GEOM>
static void launch_slab_g(Solver& s, const StepArgs& A, int cls, unsigned n, cudaStream_t st) {
    if (cls == 0) launch_slab_m<GEOM, 1>(s, A, n, st);
    else if (cls == 1) launch_slab_m<GEOM, 2>(s, A, n, st);
    else if (cls == 2) launch_slab_m<GEOM, 4>(s, A, n, st);
    else launch_slab_m<GEOM, 7>(s, A, n, st);
}

static void launch_slab(Solver& s, const StepArgs& A, int cls, unsigned n, cudaStream_t st) {
    if (s.geom == GEOM_RECT) launch_slab_g<GEOM_RECT>(s, A, cls, n, st);
    else if (s.geom == GEOM_TERRAIN) launch_slab_g<GEOM_TERRAIN>(s, A, cls, n, st);
    else launch_slab_g<GEOM_GENERAL>(s, A, cls, n, st);
}

template <bool FASTK>
static void launch_geom(Solver& s, const StepArgs& A, dim3 grid, cudaStream_t st) {
    if (s.geom == GEOM_RECT) launch_mode<GEOM_RECT, FASTK>(s, A, grid, st);
    else if (s.geom == GEOM_TERRAIN) launch_mode<GEOM_TERRAIN, FASTK>(s, A, grid, st);
    else launch_mode<GEOM_GENERAL, FASTK>(s, A, grid, st);
}

void launch_fused(Solver& s, const InjectList& pot, const InjectList& mom, const InjectList& force,
                  const std::vector<Inject>& hpot, const std::vector<Inject>& hmom, const std::vector<Inject>& hforce,
                  bool fold, bool write_a, bool stats) {
    Device& d = s.d;
    FusedPlan& P = fused_plan(s);
    StepArgs A;
    A.g = s.g;
    A.br = s.br;
    for (int a = 0; a < 3; a++)
        for (int t = 0; t < 8; t++) {
            A.brh.bnc[a][t] = s.g.h * s.br.bnc[a][t];
            A.brh.bcn[a][t] = s.g.h * s.br.bcn[a][t];
        }
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
    A.jf = P.jf;
    A.kf = P.kf;
    A.jend = P.jend;
    A.kend = P.kend;
    A.lf0 = P.lf0;
    A.lf1 = P.lf1;
    A.segl = P.segl;
    A.items = P.d_items;
    A.negzero = -0.0f;
    A.fax = s.g.ifn - 1;
    A.firup = s.g.irup;
    for (int i = 0; i < 3; i++) A.fout[i] = d.w1n[i];

    // shell items of this step: the fixed list, plus the interior planes of
    // the interior tiles holding a point source
    std::vector<std::pair<int, int>> src;
    if (P.nbx > 0) {
        source_tiles(s, P, hpot, true, src);
        source_tiles(s, P, hmom, true, src);
        source_tiles(s, P, hforce, false, src);
        std::sort(src.begin(), src.end());
        src.erase(std::unique(src.begin(), src.end()), src.end());
    }
    // In fast arithmetic the boxes without a point source go to k_slab, by
    // class; k_shell takes the rest (the boxes k_shell tests: cells
    // j0-1..j0+14 for potency / moment entries, nodes j0..j0+14 for forces).
    // Upload order: k_shell items, then the k_slab classes.
    const int nbase = (int)P.base.size() / 6;
    std::vector<char> hit(nbase, s.arith ? 0 : 1);
    if (s.arith) {
        // an entry at (j, k, l) reaches box (j0, k0, L0..L1) when
        // j0 - o <= j <= j0 + 14 (o = 1 for cells), likewise k, and
        // L0 - o <= l <= L1: at most two boxes per axis in each region
        auto mark = [&](const std::vector<Inject>& e, bool cell) {
            const int o = cell ? 1 : 0;
            auto span = [](int x, int x1, int step, int n, int lo, int hi, int& a, int& b) {
                // boxes i (origin x1 + step i) with origin + lo <= x <= origin + hi
                a = std::max(0, (int)std::ceil((double)(x - hi - x1) / step));
                b = std::min(n - 1, (int)std::floor((double)(x - lo - x1) / step));
            };
            for (const Inject& x : e) {
                const int j = (int)(x.idx % s.g.sy) + 1, k = (int)((x.idx / s.g.sy) % s.g.nm[1]) + 1;
                const int l = (int)(x.idx / s.g.sz) + 1;
                for (const BoxRegion& r : P.regions) {
                    int ja, jb, ka, kb, la, lb;
                    span(j, r.j1, SJ - 1, r.nbj, -o, SJ - 2, ja, jb);
                    span(k, r.k1, SK - 1, r.nbk, -o, SK - 2, ka, kb);
                    span(l, r.l1, r.ipl, r.nbl, -o, r.ipl - 1, la, lb);
                    for (int bl = la; bl <= lb; bl++)
                        for (int bk = ka; bk <= kb; bk++)
                            for (int bj = ja; bj <= jb; bj++) {
                                const int i = r.first + (bl * r.nbk + bk) * r.nbj + bj;
                                if (l <= P.base[6 * i + 5]) hit[i] = 1;
                            }
                }
            }
        };
        mark(hpot, true);
        mark(hmom, true);
        mark(hforce, false);
    }
    std::vector<int> items;
    for (int i = 0; i < nbase; i++)
        if (hit[i]) items.insert(items.end(), P.base.begin() + 6 * i, P.base.begin() + 6 * i + 6);
    for (auto& c : src) {
        const int j0 = P.jf + c.first * FOJ, k0 = P.kf + c.second * FOK;
        push_box(items, P.ipl, j0, std::min(P.jend, j0 + FOJ - 1), k0, std::min(P.kend, k0 + FOK - 1), P.lf0, P.lf1);
    }
    const int nshell = (int)items.size() / 6;
    int nslab[4] = {0, 0, 0, 0};
    for (int m = 0; m < 4; m++)
        for (int i = 0; i < nbase; i++)
            if (!hit[i] && P.bmask[i] == m) {
                items.insert(items.end(), P.base.begin() + 6 * i, P.base.begin() + 6 * i + 6);
                nslab[m]++;
            }
    const int nitems = (int)items.size() / 6;
    if (items != P.cur) {
        if (nitems > P.cap) throw SordError(SORD_E_PARAM, "too many point-source tiles in one step");
        SORD_CUDA(cudaEventSynchronize(P.done));
        std::memcpy(P.h_items, items.data(), sizeof(int) * items.size());
        SORD_CUDA(cudaMemcpyAsync(P.d_items, P.h_items, sizeof(int) * items.size(), cudaMemcpyHostToDevice, s.stream));
        SORD_CUDA(cudaEventRecord(P.done, s.stream));
        P.cur = items;
    }

    cudaEvent_t e0 = nullptr;
    s.prof_begin(KC_FUSED, &e0);
    const bool inner = P.nbx > 0 && P.nby > 0;
    const dim3 igrid(P.nbx, P.nby, P.nseg);
    // the shell launches: k_shell, then each k_slab class
    auto shell_launches = [&](cudaStream_t st) {
        if (nshell > 0) launch_geom<false>(s, A, dim3((unsigned)nshell, 1, 1), st);
        SORD_CUDA(cudaEventRecord(P.cfork, st));
        int off = nshell;
        for (int m = 0; m < 4; m++) {
            if (nslab[m] == 0) continue;
            StepArgs B = A;
            B.items = P.d_items + 6 * (size_t)off;
            SORD_CUDA(cudaStreamWaitEvent(P.cst[m], P.cfork, 0));
            launch_slab(s, B, m, (unsigned)nslab[m], P.cst[m]);
            SORD_CUDA(cudaEventRecord(P.cdone[m], P.cst[m]));
            SORD_CUDA(cudaStreamWaitEvent(st, P.cdone[m], 0));
            off += nslab[m];
        }
    };
    if (inner && nitems > 0) {
        SORD_CUDA(cudaEventRecord(P.fork, s.stream));
        SORD_CUDA(cudaStreamWaitEvent(P.side, P.fork, 0));
        shell_launches(P.side);
        launch_geom<true>(s, A, igrid, s.stream);
        SORD_CUDA(cudaEventRecord(P.join, P.side));
        SORD_CUDA(cudaStreamWaitEvent(s.stream, P.join, 0));
    } else if (inner) {
        launch_geom<true>(s, A, igrid, s.stream);
    } else if (nitems > 0) {
        shell_launches(s.stream);
    }
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

// PML-shell step kernel in fast arithmetic (included by fused.cu).
//
// k_slab does, on the node boxes of the PML shell, the same whole step as
// k_interior in fast arithmetic (fused multiply-adds, h-scaled brackets,
// divergence brackets as negated gradient brackets, one cell plane in
// shared memory read once per node plane, hourglass sums combined per
// reading node in the cell, the upper cell corners carried in registers),
// with the PML terms of the reference added:
//
//   cells  strain: the damped direction of a PML cell differentiates v and
//          advances the g memory (stress.f90:42-131), the other directions
//          of a PML cell differentiate u, a cell outside the PML
//          differentiates w = u + gam v (stress.f90:18-40); elastic hourglass
//          values yy hourglass_nc(hg1 u + dt hg2 v) on cells of the elastic
//          hourglass region, viscous ones dt hg2 yy hourglass_nc(v) on PML
//          cells (acceleration.f90:136-199); each reading node takes the
//          elastic values if it lies outside the PML, the viscous ones if it
//          lies inside (the layer of cells next to the elastic region holds
//          both)
//   nodes  the divergence of each damped direction of a PML node advances
//          the p memory (acceleration.f90:37-104) before it joins the force
//
// The node ring holds raw u, v and gam (w and the hourglass input are
// formed per cell corner).  MASK (bit d: axis d may be damped somewhere in
// the box) compiles in the PML terms of those axes; which cells and nodes
// are damped is decided per cell and node at run time, so a box may only
// be given a MASK that covers every damped axis in it.  Boxes holding a
// point source of the step are left to k_shell.
#pragma once

template <int GEOM>
struct LaySl {
    static constexpr int NPL = (SJ + 1) * (SK + 1);  // 289 nodes per plane
    static constexpr int NCL = SJ * SK;              // 256 cells per plane
    static constexpr int NCOORD = GEOM == GEOM_RECT ? 0 : GEOM == GEOM_TERRAIN ? 1 : 3;
    static constexpr int RAWF = 7 + NCOORD;                   // staged plane: u(3) v(3) gam coords
    static constexpr int RAWSZ = (RAWF * NPL + 3) & ~3;        // floats, float4-aligned end
    // node groups: (u, coordinate 0), (v, gam), general meshes (coordinates 1, 2)
    static constexpr int NGN = GEOM == GEOM_GENERAL ? 3 : 2;
    static constexpr int NDIR = Lay<GEOM>::NDIR, NQ = Lay<GEOM>::NQ, NGCF = Lay<GEOM>::NGCF;
    static constexpr size_t bytes = sizeof(float) * (size_t)RAWSZ + sizeof(float4) * (size_t)(3 * NPL * NGN + NCL * NGCF);
};

template <int GEOM, int MASK>
__global__ void __launch_bounds__(SJ * SK, GEOM == GEOM_GENERAL ? 1 : 2) k_slab(StepArgs A) {
    constexpr int TJ = SJ, TK = SK, TNJ = TJ + 1, TOJ = TJ - 1, TOK = TK - 1;
    using L = LaySl<GEOM>;
    constexpr int NPL_ = L::NPL, NCL_ = L::NCL, NTH_ = TJ * TK;
    constexpr int NGN = L::NGN, NDIR = L::NDIR, NQ = L::NQ, NGCF = L::NGCF;
    constexpr bool DJ = (MASK & 1) != 0, DK = (MASK & 2) != 0, DL = (MASK & 4) != 0;
    constexpr bool CARRY = GEOM != GEOM_GENERAL;
    extern __shared__ float4 sm4[];
    float* sR = reinterpret_cast<float*>(sm4);  // [RAWF][NPL] staged plane
    float4* sN = sm4 + L::RAWSZ / 4;            // [3 slots][NGN][NPL]
    float4* sC = sN + 3 * NGN * NPL_;           // [NGCF][NCL] one cell plane
#define RAWS(f, i) sR[(f) * NPL_ + (i)]
    const Geom& g = A.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TJ * ty;
    const int* it = A.items + 6 * blockIdx.x;
    const int j0 = it[0], k0 = it[1], jm = it[2], km = it[3], L0 = it[4], L1 = it[5];
    const int J = j0 - 1 + tx, K = k0 - 1 + ty;  // this thread's cell column
    const int jn = j0 + tx, kn = k0 + ty;        // this thread's node column
    const bool outcol = tx < TOJ && ty < TOK && jn <= jm && kn <= km;
    const bool cellcol = J >= g.i1cell[0] && J <= g.i2cell[0] && K >= g.i1cell[1] && K <= g.i2cell[1];
    const bool owncol = J >= j0 && J <= jm && K >= k0 && K <= km;
    const float dt = g.dt;
    float st_a = 0.f, st_v = 0.f, st_u = 0.f, st_w = 0.f;
    float txa = 0.f, txb = 0.f, tya = 0.f, tyb = 0.f;
    if (GEOM == GEOM_TERRAIN && cellcol) {
        txa = A.x1d[J - 1];
        txb = A.x1d[J];
        tya = A.y1d[K - 1];
        tyb = A.y1d[K];
    }
    const float hdx = g.h * (txb - txa), hdy = g.h * (tyb - tya);
    // PML slabs of this thread's cell column (near, far) and node column
    const bool cnj = DJ && J <= g.i1pml[0], cfj = DJ && J >= g.i2pml[0] - 1;
    const bool cnk = DK && K <= g.i1pml[1], cfk = DK && K >= g.i2pml[1] - 1;
    const bool ceJ = !DJ || (J >= g.i1pml[0] && J <= g.i2pml[0] - 1);
    const bool ceK = !DK || (K >= g.i1pml[1] && K <= g.i2pml[1] - 1);

    // ---------------------------------------------------------------- loads
    auto fetch = [&](int l) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH_;
            if (n < NPL_) {
                const int nj = n % TNJ, nk = n / TNJ;
                const int j = j0 - 1 + nj, k = k0 - 1 + nk;
                const bool ok = j <= g.nm[0] && k <= g.nm[1] && l >= 1 && l <= g.nm[2];
                if (ok) {
                    const long long q = g.idx(j, k, l);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        cp_async4(&RAWS(c, n), A.uin[c] + q);
                        cp_async4(&RAWS(3 + c, n), A.vin[c] + q);
                    }
                    cp_async4(&RAWS(6, n), A.gam + q);
                    if (GEOM == GEOM_TERRAIN) cp_async4(&RAWS(7, n), A.x[2] + q);
                    if (GEOM == GEOM_GENERAL)
#pragma unroll
                        for (int c = 0; c < 3; c++) cp_async4(&RAWS(7 + c, n), A.x[c] + q);
                } else {
#pragma unroll
                    for (int f = 0; f < L::RAWF; f++) RAWS(f, n) = 0.f;
                }
            }
        }
        cp_async_commit();
    };
    // staged plane -> ring slot: (u, coordinate 0), (v, gam) [, (coordinates 1, 2)]
    auto store = [&](int slot) {
        float4* dst = sN + slot * (NGN * NPL_);
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int n = tid + r * NTH_;
            if (n < NPL_) {
                const float c0 = L::NCOORD > 0 ? RAWS(7, n) : 0.f;
                dst[n] = make_float4(RAWS(0, n), RAWS(1, n), RAWS(2, n), c0);
                dst[NPL_ + n] = make_float4(RAWS(3, n), RAWS(4, n), RAWS(5, n), RAWS(6, n));
                if (NGN > 2) dst[2 * NPL_ + n] = make_float4(L::NCOORD > 2 ? RAWS(8, n) : 0.f, L::NCOORD > 2 ? RAWS(9, n) : 0.f, 0.f, 0.f);
            }
        }
    };
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
    float4 ca[4], cb[4];  // plane l+1 corners of the last cell computed
    int carry_l = -1000;
    auto cells = [&](int l) {
        const bool valid = cellcol && l >= g.i1cell[2] && l <= g.i2cell[2];
        if (!valid) {
            zero_cell_fm<NDIR, NQ>(sC, tid, NCL_);
            return;
        }
        // one damped axis (classes 1, 2, 4): this cell's g memory is loaded
        // first, so its latency passes under the corner loads and brackets
        constexpr bool PF = MASK == 1 || MASK == 2 || MASK == 4;
        constexpr int PD = MASK == 1 ? 0 : MASK == 2 ? 1 : 2;
        float gpre[3] = {0.f, 0.f, 0.f};
        if constexpr (PF) {
            const bool pn = PD == 0 ? cnj : PD == 1 ? cnk : (DL && l <= g.i1pml[2]);
            const bool pf = PD == 0 ? cfj : PD == 1 ? cfk : (DL && l >= g.i2pml[2] - 1);
            if (pn || pf) {
                const int c = PD == 0 ? J : PD == 1 ? K : l;
                const int sb = pn ? PD : 3 + PD;
#pragma unroll
                for (int ic = 0; ic < 3; ic++)
                    gpre[ic] = A.sl.g[sb][slab_idx(g, PD, A.sl.tg[sb], pn ? c - g.i1cell[PD] : g.i2cell[PD] - c, J, K, l, ic)];
            }
        }
        float Uc[3][8], Vc[3][8], Gc[8], X0[8], X1[8], X2[8];
        {
            const float4* p0 = sN + (l % 3) * (NGN * NPL_) + (tx + TNJ * ty);
            const float4* p1 = sN + ((l + 1) % 3) * (NGN * NPL_) + (tx + TNJ * ty);
            const bool reuse = CARRY && carry_l == l - 1;
#pragma unroll
            for (int n = 0; n < 8; n++) {
                const float4* p = ((n >> 2) ? p1 : p0) + (n & 1) + TNJ * ((n >> 1) & 1);
                float4 a, b;
                if (CARRY && n < 4 && reuse) {
                    a = ca[n];
                    b = cb[n];
                } else {
                    a = p[0];
                    b = p[NPL_];
                }
                if (CARRY && n >= 4) {
                    ca[n - 4] = a;
                    cb[n - 4] = b;
                }
                Uc[0][n] = a.x; Uc[1][n] = a.y; Uc[2][n] = a.z;
                Vc[0][n] = b.x; Vc[1][n] = b.y; Vc[2][n] = b.z;
                Gc[n] = b.w;
                if (GEOM == GEOM_TERRAIN) {
                    X0[n] = (n & 1) ? txb : txa;
                    X1[n] = ((n >> 1) & 1) ? tyb : tya;
                    X2[n] = a.w;
                } else if (GEOM == GEOM_GENERAL) {
                    const float4 c = p[2 * NPL_];
                    X0[n] = a.w;
                    X1[n] = c.x;
                    X2[n] = c.y;
                }
            }
            if (CARRY) carry_l = l;
        }
        // region of the cell (stress.f90:18-131, acceleration.f90:136-199)
        const bool cnl = DL && l <= g.i1pml[2], cfl = DL && l >= g.i2pml[2] - 1;
        const bool sj = cnj || cfj, sk = cnk || cfk, sl = cnl || cfl;
        const bool anyS = sj || sk || sl;
        const bool inEc = ceJ && ceK && (!DL || (l >= g.i1pml[2] && l <= g.i2pml[2] - 1));
        // a cell plane below the first node plane is a halo of a partitioned run;
        // the part takes it (the PML g memory of that halo cell advances here)
        const bool own = owncol && (l >= L0 || l < g.i1node[2]);
        // brackets scaled by h; divergence brackets = negated gradient brackets
        float B[3][8];
        float cnb[NDIR > 0 ? NDIR : 1][8];
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
                for (int t = 0; t < 8; t++) B[a][t] = g.h * B[a][t];
        }
#pragma unroll
        for (int a = 0; a < NDIR; a++)
#pragma unroll
            for (int t = 0; t < 8; t++) cnb[a][t] = -B[a][cn_of_nc(t)];
        // gradients: v along a damped direction (with the g memory), u along
        // the others in a PML cell, w = u + gam v outside the PML
        float sg[3][3];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            float W[8], V[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int n = term_corner(t);
                V[t] = Vc[ic][n];
                W[t] = anyS ? Uc[ic][n] : fmaf(Gc[n], Vc[ic][n], Uc[ic][n]);
            }
#pragma unroll
            for (int id = 0; id < 3; id++) {
                if ((MASK >> id) & 1) {
                    const bool dmp = id == 0 ? sj : id == 1 ? sk : sl;
                    float Z[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) Z[t] = dmp ? V[t] : W[t];
                    float s = dot8(Z, B[id]);
                    if (dmp) {
                        const bool nr = id == 0 ? cnj : id == 1 ? cnk : cnl;
                        const int c = id == 0 ? J : id == 1 ? K : l;
                        const int p = nr ? c + g.nnoff[id] : g.nn[id] - c - g.nnoff[id];
                        const int sb = nr ? id : 3 + id;
                        const long long gi = slab_idx(g, id, A.sl.tg[sb], nr ? c - g.i1cell[id] : g.i2cell[id] - c, J, K, l, ic);
                        const float gm = PF ? gpre[ic] : A.sl.g[sb][gi];
                        s = fmaf(A.pmlc[3 * g.npml + p - 1], s, A.pmlc[2 * g.npml + p - 1] * gm);
                        if (own) A.gout[sb][gi] = s;
                    }
                    sg[ic][id] = s;
                } else {
                    sg[ic][id] = dot8(W, B[id]);
                }
            }
        }
        float ed[3], eo[3];
#pragma unroll
        for (int i = 0; i < 3; i++) ed[i] = sg[i][i];
        eo[0] = sg[1][2] + sg[2][1];
        eo[1] = sg[0][2] + sg[2][0];
        eo[2] = sg[0][1] + sg[1][0];
        {
            // (2 mu e + lam tr e) / V; the off-diagonal sums carry the 1/2
            const float r = cur[2], mur = cur[1] * r, m2r = mur + mur;
            const float s1r = (cur[0] * r) * (ed[0] + ed[1] + ed[2]);
#pragma unroll
            for (int i = 0; i < 3; i++) { ed[i] = fmaf(m2r, ed[i], s1r); eo[i] = mur * eo[i]; }
        }
        if (A.stats && own)
            st_w = fmaxn(st_w, (ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]) + 2.0f * (eo[0] * eo[0] + eo[1] * eo[1] + eo[2] * eo[2]));
        // hourglass cell values: he for the readers of the cell's own kind,
        // hv (viscous) for the PML readers of a cell of both kinds
        float he[12], hv[12];
#pragma unroll
        for (int i = 0; i < 12; i++) { he[i] = 0.f; hv[i] = 0.f; }
        const bool dual = A.hourglass && inEc && anyS;
        if (A.hourglass) {
            const float y = cur[3], yv = A.dh2 * cur[3];
            const bool visc = A.hgvisc && anyS;
#pragma unroll
            for (int ic = 0; ic < 3; ic++) {
                // corner values (corner id order) and their four mode sums
                // by butterflies (stencil.cuh: hg_modes)
                float H[8], me[4], mv[4];
#pragma unroll
                for (int n = 0; n < 8; n++) H[n] = fmaf(A.dh2, Vc[ic][n], A.hg1 * Uc[ic][n]);
                hg_modes<float>(H, me);
                hg_modes<float>(Vc[ic], mv);
#pragma unroll
                for (int iq = 0; iq < 4; iq++) {
                    const float e = inEc ? me[iq] * y : 0.f;
                    const float v = visc ? yv * mv[iq] : 0.f;
                    he[3 * iq + ic] = inEc ? e : v;
                    hv[3 * iq + ic] = v;
                }
            }
        }
        // fast layout (Lay::NGCF): stress, then per reading node column q the
        // hourglass sums for the node above and below the cell and the
        // divergence brackets
        float4* cw = sC + tid;
        cw[0] = make_float4(ed[0], ed[1], ed[2], eo[0]);
        reinterpret_cast<float2*>(sC + NCL_)[tid] = make_float2(eo[1], eo[2]);
        // the reading columns' sums from four shared sums per component
        // (stencil.cuh: hg_readers_pre / hg_reader)
        float her[3][4], hvr[3][4];
#pragma unroll
        for (int ic = 0; ic < 3; ic++) {
            const float me[4] = {he[ic], he[3 + ic], he[6 + ic], he[9 + ic]};
            const float mv[4] = {hv[ic], hv[3 + ic], hv[6 + ic], hv[9 + ic]};
            hg_readers_pre<float>(me, her[ic]);
            hg_readers_pre<float>(mv, hvr[ic]);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float yu[3], yl[3];
#pragma unroll
            for (int ic = 0; ic < 3; ic++) hg_reader<float>(her[ic], q, yu[ic], yl[ic]);
            if (dual) {
                // readers of node column (J + 1 - cj, K + 1 - ck), planes l and l + 1
                const int rj = J + 1 - (q & 1), rk = K + 1 - (q >> 1);
                const bool pjk = (DJ && (rj <= g.i1pml[0] || rj >= g.i2pml[0])) ||
                                 (DK && (rk <= g.i1pml[1] || rk >= g.i2pml[1]));
                const bool pu = pjk || (DL && (l <= g.i1pml[2] || l >= g.i2pml[2]));
                const bool pl = pjk || (DL && (l + 1 <= g.i1pml[2] || l + 1 >= g.i2pml[2]));
                float vu[3], vl[3];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) hg_reader<float>(hvr[ic], q, vu[ic], vl[ic]);
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    yu[ic] = pu ? vu[ic] : yu[ic];
                    yl[ic] = pl ? vl[ic] : yl[ic];
                }
            }
            float4* cq = cw + (2 + NQ * q) * NCL_;
            cq[0] = make_float4(yu[0], yu[1], yu[2], yl[0]);
            if constexpr (NDIR == 3) {
                const int tu = (q & 1) + 2 + 4 * (q >> 1), tl = (q & 1) + 4 * (q >> 1);
                cq[NCL_] = make_float4(yl[1], yl[2], cnb[0][tu], cnb[1][tu]);
                cq[2 * NCL_] = make_float4(cnb[0][tl], cnb[1][tl], cnb[NDIR - 1][tu], cnb[NDIR - 1][tl]);
            } else if constexpr (NDIR == 2) {
                const int tu = (q & 1) + 2 + 4 * (q >> 1), tl = (q & 1) + 4 * (q >> 1);
                cq[NCL_] = make_float4(yl[1], yl[2], cnb[0][tu], cnb[1][tu]);
                reinterpret_cast<float2*>(sC + (2 + 4 * NQ) * NCL_)[q * NCL_ + tid] = make_float2(cnb[0][tl], cnb[1][tl]);
            } else {
                cq[NCL_] = make_float4(yl[1], yl[2], 0.f, 0.f);
            }
        }
    };

    // ---------------------------------------------------------------- node phase
    // fc: terms of the cells below node l + 1 carried from plane l; fcd:
    // their divergence along each damped axis, kept apart for the p memory
    float fc[3] = {0.f, 0.f, 0.f};
    float fcd[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    auto nodes_fm = [&](int l, bool finish) {
        if (!outcol) return;
        // one damped axis: this node's p memory is loaded first (see the
        // cell phase's g memory)
        constexpr bool PF = MASK == 1 || MASK == 2 || MASK == 4;
        constexpr int PD = MASK == 1 ? 0 : MASK == 2 ? 1 : 2;
        float ppre[3] = {0.f, 0.f, 0.f};
        if constexpr (PF) {
            const int c = PD == 0 ? jn : PD == 1 ? kn : l;
            const bool nr = c <= g.i1pml[PD], fr = c >= g.i2pml[PD];
            if (finish && (nr || fr)) {
                const int sb = nr ? PD : 3 + PD;
#pragma unroll
                for (int ic = 0; ic < 3; ic++)
                    ppre[ic] = A.sl.p[sb][slab_idx(g, PD, A.sl.tp[sb], nr ? c - g.i1node[PD] : g.i2node[PD] - c, jn, kn, l, ic)];
            }
        }
        float fu[3] = {fc[0], fc[1], fc[2]}, fl[3] = {0.f, 0.f, 0.f};
        float fud[3][3], fld[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int ic = 0; ic < 3; ic++) { fud[d][ic] = fcd[d][ic]; fld[d][ic] = 0.f; }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int cj = q & 1, ck = q >> 1;
            const int ci = tid + cj + TJ * ck;  // the cell (J + cj, K + ck)
            const float4 a = sC[ci];
            const float2 e = reinterpret_cast<const float2*>(sC + NCL_)[ci];
            const float S[6] = {a.x, a.y, a.z, a.w, e.x, e.y};
            const float4* cq = sC + (2 + NQ * q) * NCL_ + ci;
            const float4 y0 = cq[0], y1 = cq[NCL_];
            const int tu = cj + 2 + 4 * ck, tl = cj + 4 * ck;
            float Bu[3], Bl[3];
            if constexpr (NDIR == 3) {
                const float4 y2 = cq[2 * NCL_];
                Bu[0] = y1.z;
                Bu[1] = y1.w;
                Bl[0] = y2.x;
                Bl[1] = y2.y;
                Bu[2] = y2.z;
                Bl[2] = y2.w;
            } else if constexpr (NDIR == 2) {
                const float2 bl = reinterpret_cast<const float2*>(sC + (2 + 4 * NQ) * NCL_)[q * NCL_ + ci];
                Bu[0] = y1.z;
                Bu[1] = y1.w;
                Bl[0] = bl.x;
                Bl[1] = bl.y;
            }
#pragma unroll
            for (int id = NDIR; id < 3; id++) {
                Bu[id] = A.brh.bcn[id][tu];
                Bl[id] = A.brh.bcn[id][tl];
            }
#pragma unroll
            for (int ic = 0; ic < 3; ic++)
#pragma unroll
                for (int iid = 0; iid < 3; iid++) {
                    const int id = (ic + iid) % 3, comp = ic == id ? ic : 3 + (3 - ic - id);
                    if ((MASK >> id) & 1) {
                        fud[id][ic] = fmaf(S[comp], Bu[id], fud[id][ic]);
                        fld[id][ic] = fmaf(S[comp], Bl[id], fld[id][ic]);
                    } else {
                        fu[ic] = fmaf(S[comp], Bu[id], fu[ic]);
                        fl[ic] = fmaf(S[comp], Bl[id], fl[ic]);
                    }
                }
            if (A.hourglass) {
                fu[0] = fu[0] + y0.x;
                fu[1] = fu[1] + y0.y;
                fu[2] = fu[2] + y0.z;
                fl[0] = fl[0] + y0.w;
                fl[1] = fl[1] + y1.x;
                fl[2] = fl[2] + y1.y;
            }
        }
#pragma unroll
        for (int i = 0; i < 3; i++) fc[i] = fl[i];
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int ic = 0; ic < 3; ic++) fcd[d][ic] = fld[d][ic];
        if (!finish) return;
        // p memory of the damped directions (acceleration.f90:37-104)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (!((MASK >> d) & 1)) continue;
            const int c = d == 0 ? jn : d == 1 ? kn : l;
            const bool nr = c <= g.i1pml[d], fr = c >= g.i2pml[d];
            if (nr || fr) {
                const int p = nr ? c + g.nnoff[d] : g.nn[d] - c - g.nnoff[d] + 1;
                const int sb = nr ? d : 3 + d;
                const float dn1 = A.pmlc[p - 1], dn2 = A.pmlc[g.npml + p - 1];
#pragma unroll
                for (int ic = 0; ic < 3; ic++) {
                    float* P = A.sl.p[sb] + slab_idx(g, d, A.sl.tp[sb], nr ? c - g.i1node[d] : g.i2node[d] - c, jn, kn, l, ic);
                    const float pv = PF ? ppre[ic] : *P;
                    const float s = fmaf(dn2, fud[d][ic], dn1 * pv);
                    *P = fmaf(dt, s, pv);
                    fu[ic] = fu[ic] + s;
                }
            } else {
#pragma unroll
                for (int ic = 0; ic < 3; ic++) fu[ic] = fu[ic] + fud[d][ic];
            }
        }
        finish_node<true>(A, g.idx(jn, kn, l), jn, kn, l, fu, cur[4], uv, dt, st_a, st_v, st_u);
    };

    // ---------------------------------------------------------------- stream
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
    cells(L0 - 1);
    __syncthreads();  // cell plane L0-1 complete: its terms for node L0
    nodes_fm(L0 - 1, false);
    __syncthreads();  // one cell slot: read before cells(L0) overwrites it
    stat_load(L0, cur);
#pragma unroll 1
    for (int l = L0; l <= L1; l++) {
        cells(l);
        float nxt[5], nuv[6];
        stat_load(l + 1, nxt);
        cp_async_wait_all();
        __syncthreads();  // cell plane l complete, staged plane l+2 landed
        store((l + 2) % 3);
        nodes_fm(l, true);
        uv_load(l + 1, nuv);
        __syncthreads();  // ring slot l+2 complete, staging and the cell slot free
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
#undef RAWS
}

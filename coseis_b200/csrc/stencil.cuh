// Support-operator and hourglass stencils as device functions.
//
// Every expression keeps the operand order of the Fortran it restates; the
// library is compiled with -fmad=false so that each product and sum rounds
// separately, exactly like the reference's (and the oracle's) FP32 code.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define SORD_HD __host__ __device__ __forceinline__
#else
#define SORD_HD inline
#endif

namespace sordgpu {

// Cell corners in the term order of diff_nc (diff_nc_op.f90:19-70):
// (0,0,0) (1,0,0) (0,1,0) (1,1,0) (0,0,1) (1,0,1) (1,1,1) (0,1,1);
// corner id = dj + 2*dk + 4*dl.
SORD_HD int term_corner(int t) { return t < 6 ? t : 13 - t; }

// Brackets of diff_nc for one direction at one cell, from the two other
// coordinates xb, xc at the corners n = dj + 2*dk + 4*dl.  B[t] multiplies
// term t.  sord/diff_nc_op.f90:19-70.  T is float, or a pair type whose
// operators apply the same IEEE operation to two independent lanes.
template <class T>
SORD_HD void brackets_nc_g(const T* xb, const T* xc, T B[8]) {
#define XB(j, k, l) xb[(j) + 2 * (k) + 4 * (l)]
#define XC(j, k, l) xc[(j) + 2 * (k) + 4 * (l)]
    B[0] = (XB(0, 1, 1) - XB(1, 0, 0)) * (XC(0, 1, 0) - XC(0, 0, 1)) + XB(1, 0, 0) * (XC(1, 0, 1) - XC(1, 1, 0)) +
           (XB(1, 0, 1) - XB(0, 1, 0)) * (XC(0, 0, 1) - XC(1, 0, 0)) + XB(0, 1, 0) * (XC(1, 1, 0) - XC(0, 1, 1)) +
           (XB(1, 1, 0) - XB(0, 0, 1)) * (XC(1, 0, 0) - XC(0, 1, 0)) + XB(0, 0, 1) * (XC(0, 1, 1) - XC(1, 0, 1));
    B[1] = (XB(1, 1, 1) - XB(0, 0, 0)) * (XC(1, 0, 1) - XC(1, 1, 0)) + XB(0, 0, 0) * (XC(0, 1, 0) - XC(0, 0, 1)) +
           (XB(0, 1, 0) - XB(1, 0, 1)) * (XC(1, 1, 0) - XC(0, 0, 0)) + XB(1, 0, 1) * (XC(0, 0, 1) - XC(1, 1, 1)) +
           (XB(0, 0, 1) - XB(1, 1, 0)) * (XC(0, 0, 0) - XC(1, 0, 1)) + XB(1, 1, 0) * (XC(1, 1, 1) - XC(0, 1, 0));
    B[2] = (XB(1, 1, 1) - XB(0, 0, 0)) * (XC(1, 1, 0) - XC(0, 1, 1)) + XB(0, 0, 0) * (XC(0, 0, 1) - XC(1, 0, 0)) +
           (XB(1, 0, 0) - XB(0, 1, 1)) * (XC(0, 0, 0) - XC(1, 1, 0)) + XB(0, 1, 1) * (XC(1, 1, 1) - XC(0, 0, 1)) +
           (XB(0, 0, 1) - XB(1, 1, 0)) * (XC(0, 1, 1) - XC(0, 0, 0)) + XB(1, 1, 0) * (XC(1, 0, 0) - XC(1, 1, 1));
    B[3] = (XB(0, 0, 0) - XB(1, 1, 1)) * (XC(0, 1, 0) - XC(1, 0, 0)) + XB(1, 1, 1) * (XC(1, 0, 1) - XC(0, 1, 1)) +
           (XB(0, 1, 1) - XB(1, 0, 0)) * (XC(1, 1, 1) - XC(0, 1, 0)) + XB(1, 0, 0) * (XC(0, 0, 0) - XC(1, 0, 1)) +
           (XB(1, 0, 1) - XB(0, 1, 0)) * (XC(1, 0, 0) - XC(1, 1, 1)) + XB(0, 1, 0) * (XC(0, 1, 1) - XC(0, 0, 0));
    B[4] = (XB(1, 1, 1) - XB(0, 0, 0)) * (XC(0, 1, 1) - XC(1, 0, 1)) + XB(0, 0, 0) * (XC(1, 0, 0) - XC(0, 1, 0)) +
           (XB(1, 0, 0) - XB(0, 1, 1)) * (XC(1, 0, 1) - XC(0, 0, 0)) + XB(0, 1, 1) * (XC(0, 1, 0) - XC(1, 1, 1)) +
           (XB(0, 1, 0) - XB(1, 0, 1)) * (XC(0, 0, 0) - XC(0, 1, 1)) + XB(1, 0, 1) * (XC(1, 1, 1) - XC(1, 0, 0));
    B[5] = (XB(0, 0, 0) - XB(1, 1, 1)) * (XC(1, 0, 0) - XC(0, 0, 1)) + XB(1, 1, 1) * (XC(0, 1, 1) - XC(1, 1, 0)) +
           (XB(0, 1, 1) - XB(1, 0, 0)) * (XC(0, 0, 1) - XC(1, 1, 1)) + XB(1, 0, 0) * (XC(1, 1, 0) - XC(0, 0, 0)) +
           (XB(1, 1, 0) - XB(0, 0, 1)) * (XC(1, 1, 1) - XC(1, 0, 0)) + XB(0, 0, 1) * (XC(0, 0, 0) - XC(0, 1, 1));
    B[6] = (XB(1, 0, 0) - XB(0, 1, 1)) * (XC(1, 1, 0) - XC(1, 0, 1)) + XB(0, 1, 1) * (XC(0, 0, 1) - XC(0, 1, 0)) +
           (XB(0, 1, 0) - XB(1, 0, 1)) * (XC(0, 1, 1) - XC(1, 1, 0)) + XB(1, 0, 1) * (XC(1, 0, 0) - XC(0, 0, 1)) +
           (XB(0, 0, 1) - XB(1, 1, 0)) * (XC(1, 0, 1) - XC(0, 1, 1)) + XB(1, 1, 0) * (XC(0, 1, 0) - XC(1, 0, 0));
    B[7] = (XB(0, 0, 0) - XB(1, 1, 1)) * (XC(0, 0, 1) - XC(0, 1, 0)) + XB(1, 1, 1) * (XC(1, 1, 0) - XC(1, 0, 1)) +
           (XB(1, 0, 1) - XB(0, 1, 0)) * (XC(1, 1, 1) - XC(0, 0, 1)) + XB(0, 1, 0) * (XC(0, 0, 0) - XC(1, 1, 0)) +
           (XB(1, 1, 0) - XB(0, 0, 1)) * (XC(0, 1, 0) - XC(1, 1, 1)) + XB(0, 0, 1) * (XC(1, 0, 1) - XC(0, 0, 0));
#undef XB
#undef XC
}

// Direction a (0-based) with X[c][n] = coordinate c at corner n.
SORD_HD void brackets_nc(const float (*X)[8], int a, float B[8]) {
    brackets_nc_g<float>(X[(a + 1) % 3], X[(a + 2) % 3], B);
}

// Brackets of diff_cn for direction a at one node; X[c][m] is coordinate c
// at neighbour m = (dj+1) + 3*(dk+1) + 9*(dl+1), dj,dk,dl in -1..1.
// B[t] multiplies the cell of term t: (j-1,k-1,l-1) (j,k-1,l-1) (j-1,k-1,l)
// (j,k-1,l) (j-1,k,l-1) (j,k,l-1) (j-1,k,l) (j,k,l).  sord/diff_cn_op.f90:19-70.
template <class T, class XA>
SORD_HD void brackets_cn_g(const XA& xb, const XA& xc, T B[8]) {
#define XB(j, k, l) xb((j) + 1 + 3 * ((k) + 1) + 9 * ((l) + 1))
#define XC(j, k, l) xc((j) + 1 + 3 * ((k) + 1) + 9 * ((l) + 1))
    B[0] = (XB(-1, 0, 0) - XB(0, -1, -1)) * (XC(0, 0, -1) - XC(0, -1, 0)) + XB(-1, 0, 0) * (XC(-1, 0, -1) - XC(-1, -1, 0)) +
           (XB(0, -1, 0) - XB(-1, 0, -1)) * (XC(-1, 0, 0) - XC(0, 0, -1)) + XB(0, -1, 0) * (XC(-1, -1, 0) - XC(0, -1, -1)) +
           (XB(0, 0, -1) - XB(-1, -1, 0)) * (XC(0, -1, 0) - XC(-1, 0, 0)) + XB(0, 0, -1) * (XC(0, -1, -1) - XC(-1, 0, -1));
    B[1] = (XB(1, 0, 0) - XB(0, -1, -1)) * (XC(0, -1, 0) - XC(0, 0, -1)) + XB(1, 0, 0) * (XC(1, -1, 0) - XC(1, 0, -1)) +
           (XB(0, -1, 0) - XB(1, 0, -1)) * (XC(0, 0, -1) - XC(1, 0, 0)) + XB(0, -1, 0) * (XC(0, -1, -1) - XC(1, -1, 0)) +
           (XB(0, 0, -1) - XB(1, -1, 0)) * (XC(1, 0, 0) - XC(0, -1, 0)) + XB(0, 0, -1) * (XC(1, 0, -1) - XC(0, -1, -1));
    B[2] = (XB(0, 0, 1) - XB(-1, -1, 0)) * (XC(-1, 0, 0) - XC(0, -1, 0)) + XB(0, 0, 1) * (XC(-1, 0, 1) - XC(0, -1, 1)) +
           (XB(-1, 0, 0) - XB(0, -1, 1)) * (XC(0, -1, 0) - XC(0, 0, 1)) + XB(-1, 0, 0) * (XC(-1, -1, 0) - XC(-1, 0, 1)) +
           (XB(0, -1, 0) - XB(-1, 0, 1)) * (XC(0, 0, 1) - XC(-1, 0, 0)) + XB(0, -1, 0) * (XC(0, -1, 1) - XC(-1, -1, 0));
    B[3] = (XB(0, -1, 0) - XB(1, 0, 1)) * (XC(1, 0, 0) - XC(0, 0, 1)) + XB(0, -1, 0) * (XC(1, -1, 0) - XC(0, -1, 1)) +
           (XB(0, 0, 1) - XB(1, -1, 0)) * (XC(0, -1, 0) - XC(1, 0, 0)) + XB(0, 0, 1) * (XC(0, -1, 1) - XC(1, 0, 1)) +
           (XB(1, 0, 0) - XB(0, -1, 1)) * (XC(0, 0, 1) - XC(0, -1, 0)) + XB(1, 0, 0) * (XC(1, 0, 1) - XC(1, -1, 0));
    B[4] = (XB(0, 1, 0) - XB(-1, 0, -1)) * (XC(0, 0, -1) - XC(-1, 0, 0)) + XB(0, 1, 0) * (XC(0, 1, -1) - XC(-1, 1, 0)) +
           (XB(0, 0, -1) - XB(-1, 1, 0)) * (XC(-1, 0, 0) - XC(0, 1, 0)) + XB(0, 0, -1) * (XC(-1, 0, -1) - XC(0, 1, -1)) +
           (XB(-1, 0, 0) - XB(0, 1, -1)) * (XC(0, 1, 0) - XC(0, 0, -1)) + XB(-1, 0, 0) * (XC(-1, 1, 0) - XC(-1, 0, -1));
    B[5] = (XB(0, 0, -1) - XB(1, 1, 0)) * (XC(0, 1, 0) - XC(1, 0, 0)) + XB(0, 0, -1) * (XC(0, 1, -1) - XC(1, 0, -1)) +
           (XB(1, 0, 0) - XB(0, 1, -1)) * (XC(0, 0, -1) - XC(0, 1, 0)) + XB(1, 0, 0) * (XC(1, 0, -1) - XC(1, 1, 0)) +
           (XB(0, 1, 0) - XB(1, 0, -1)) * (XC(1, 0, 0) - XC(0, 0, -1)) + XB(0, 1, 0) * (XC(1, 1, 0) - XC(0, 1, -1));
    B[6] = (XB(-1, 0, 0) - XB(0, 1, 1)) * (XC(0, 0, 1) - XC(0, 1, 0)) + XB(-1, 0, 0) * (XC(-1, 0, 1) - XC(-1, 1, 0)) +
           (XB(0, 1, 0) - XB(-1, 0, 1)) * (XC(-1, 0, 0) - XC(0, 0, 1)) + XB(0, 1, 0) * (XC(-1, 1, 0) - XC(0, 1, 1)) +
           (XB(0, 0, 1) - XB(-1, 1, 0)) * (XC(0, 1, 0) - XC(-1, 0, 0)) + XB(0, 0, 1) * (XC(0, 1, 1) - XC(-1, 0, 1));
    B[7] = (XB(1, 0, 0) - XB(0, 1, 1)) * (XC(0, 1, 0) - XC(0, 0, 1)) + XB(1, 0, 0) * (XC(1, 1, 0) - XC(1, 0, 1)) +
           (XB(0, 1, 0) - XB(1, 0, 1)) * (XC(0, 0, 1) - XC(1, 0, 0)) + XB(0, 1, 0) * (XC(0, 1, 1) - XC(1, 1, 0)) +
           (XB(0, 0, 1) - XB(1, 1, 0)) * (XC(1, 0, 0) - XC(0, 1, 0)) + XB(0, 0, 1) * (XC(1, 0, 1) - XC(0, 1, 1));
#undef XB
#undef XC
}

template <class XA>
struct CoordOf {
    const XA& X;
    int c;
    SORD_HD float operator()(int m) const { return X(c, m); }
};
template <class XA>
SORD_HD void brackets_cn(const XA& X, int a, float B[8]) {
    CoordOf<XA> xb{X, (a + 1) % 3}, xc{X, (a + 2) % 3};
    brackets_cn_g<float>(xb, xc, B);
}

// Weighted 8-term sum  d = h*F0*B0; d = d + h*Ft*Bt  (diff_nc / diff_cn).
template <class T>
SORD_HD T stencil8(const T F[8], const T B[8], T h) {
    T d = h * F[0] * B[0];
#pragma unroll
    for (int t = 1; t < 8; t++) d = d + h * F[t] * B[t];
    return d;
}

// Hourglass sign patterns (hourglass_op.f90): the 8 terms of hourglass_nc
// are the corners 000 111 011 100 101 010 110 001 (offsets dj dk dl), those
// of hourglass_cn the cells at minus the same offsets.  hg_corner(t) is the
// corner id of term t; hg_neg(iq, t) is 1 where term t is subtracted.
SORD_HD int hg_corner(int t) { return (int)((0x43251670u >> (4 * t)) & 0xFu); }
// the inverse: the hourglass term whose corner is c
SORD_HD int hg_term(int c) { return (int)((0x12476530u >> (4 * c)) & 0xFu); }
SORD_HD int hg_neg(int iq, int t) { return (int)(((0xAA3CCCF0u >> (8 * iq)) >> t) & 1u); }

template <class T>
SORD_HD T hg_sum(const T A[8], int iq) {
    T r = A[0];
#pragma unroll
    for (int t = 1; t < 8; t++) r = hg_neg(iq, t) ? r - A[t] : r + A[t];
    return r;
}

// Divergence brackets of one cell as seen from each of its corners: cn[t] is
// the diff_cn bracket (direction a) that the node at corner o(t) applies to
// this cell, o(t) being the corner for which the cell is that node's term t
// (diff_cn term t sits at cell offsets (j-1|j, k-1|k, l-1|l) from the node).
// Terms 0, 3, 4 and 7 of diff_cn are the negations of diff_nc terms 6, 2, 5
// and 0 (same operand order); they are formed as 0 - x, which also gives the
// +0 that the diff_cn sum gives when the bracket cancels exactly (pinned
// bitwise by tests/stencil_identity.cpp); terms 1, 2, 5, 6 differ in operand
// order and are evaluated with the diff_cn expression.  X[c][n]: cell corner
// coordinates.
template <class T>
SORD_HD void cell_cn_brackets_g(const T* xb, const T* xc, const T nc[8], T cn[8], T zero) {
    cn[0] = zero - nc[6];
    cn[3] = zero - nc[2];
    cn[4] = zero - nc[5];
    cn[7] = zero - nc[0];
    // node-relative accessors for the four remaining terms; the node sits at
    // cell corner o = (oj, ok, ol) and neighbour d maps to corner o + d.
    struct Acc {
        const T* x;
        int o;
        SORD_HD T operator()(int m) const {
            int dj = m % 3 - 1, dk = (m / 3) % 3 - 1, dl = m / 9 - 1;
            int oj = o & 1, ok = (o >> 1) & 1, ol = (o >> 2) & 1;
            return x[(oj + dj) + 2 * (ok + dk) + 4 * (ol + dl)];
        }
    };
    T B[8];
    {  // term 1: cell (j, k-1, l-1) -> node at corner (0,1,1)
        Acc b{xb, 6}, c{xc, 6};
        brackets_cn_g<T>(b, c, B);
        cn[1] = B[1];
    }
    {  // term 2: cell (j-1, k-1, l) -> node at corner (1,1,0)
        Acc b{xb, 3}, c{xc, 3};
        brackets_cn_g<T>(b, c, B);
        cn[2] = B[2];
    }
    {  // term 5: cell (j, k, l-1) -> node at corner (0,0,1)
        Acc b{xb, 4}, c{xc, 4};
        brackets_cn_g<T>(b, c, B);
        cn[5] = B[5];
    }
    {  // term 6: cell (j-1, k, l) -> node at corner (1,0,0)
        Acc b{xb, 1}, c{xc, 1};
        brackets_cn_g<T>(b, c, B);
        cn[6] = B[6];
    }
}
SORD_HD void cell_cn_brackets(const float (*X)[8], int a, const float nc[8], float cn[8]) {
    cell_cn_brackets_g<float>(X[(a + 1) % 3], X[(a + 2) % 3], nc, cn, 0.0f);
}

// ---------------------------------------------------------------------------
// Fast arithmetic: the same operators with fused multiply-adds and fewer
// operations, equal to the reference's values in exact arithmetic (not bit
// for bit; the rounding differs).
//
// In exact arithmetic every divergence bracket of a cell is the negated
// gradient bracket of the same cell and corner: cn[t] = -nc[cn_of_nc(t)]
// (the support operators are adjoint, diff_cn_op.f90 / diff_nc_op.f90).
SORD_HD int cn_of_nc(int t) { return (int)((0x01452376u >> (4 * t)) & 0xFu); }

// On a terrain mesh x depends on j only and y on k only, so the diff_nc
// brackets (diff_nc_op.f90:19-70) of the two z-dependent directions reduce
// to one spacing times small integer combinations of the corner z values
// (corner n = dj + 2 dk + 4 dl).  Direction 0 (xb = y, xc = z), s = dy:
//   B0 = s (2 (z1 - z4) + (z3 - z6)), B2 = s ((z1 - z4) + 2 (z3 - z6)),
//   B1 = s (2 (z5 - z0) + (z7 - z2)), B3 = s ((z5 - z0) + 2 (z7 - z2)),
//   B4 = -B1, B5 = -B0, B6 = -B2, B7 = -B3.
// Direction 1 (xb = z, xc = x), s = dx:
//   B0 = s (2 (z2 - z4) + (z3 - z5)), B1 = s ((z2 - z4) + 2 (z3 - z5)),
//   B2 = s (2 (z6 - z0) + (z7 - z1)), B3 = s ((z6 - z0) + 2 (z7 - z1)),
//   B4 = -B2, B5 = -B3, B6 = -B1, B7 = -B0.
// s carries any common factor (the kernels pass h dy and h dx).
SORD_HD void terrain_brackets_0(float s, const float z[8], float B[8]) {
    const float a = z[1] - z[4], b = z[3] - z[6], c = z[5] - z[0], d = z[7] - z[2];
    B[0] = s * fmaf(2.0f, a, b);
    B[1] = s * fmaf(2.0f, c, d);
    B[2] = s * fmaf(2.0f, b, a);
    B[3] = s * fmaf(2.0f, d, c);
    B[4] = -B[1];
    B[5] = -B[0];
    B[6] = -B[2];
    B[7] = -B[3];
}
SORD_HD void terrain_brackets_1(float s, const float z[8], float B[8]) {
    const float a = z[2] - z[4], b = z[3] - z[5], c = z[6] - z[0], d = z[7] - z[1];
    B[0] = s * fmaf(2.0f, a, b);
    B[1] = s * fmaf(2.0f, b, a);
    B[2] = s * fmaf(2.0f, c, d);
    B[3] = s * fmaf(2.0f, d, c);
    B[4] = -B[2];
    B[5] = -B[3];
    B[6] = -B[1];
    B[7] = -B[0];
}

// Hourglass by butterflies.  With x = (-1)^dj, y = (-1)^dk, z = (-1)^dl at
// corner n = dj + 2 dk + 4 dl, the four hourglass modes of hourglass_op.f90
// (hg_sum over the term order) are the sign patterns y z, x z, x y and
// x y z.  hg_modes forms all four from the corner values by a pruned
// Walsh-Hadamard transform: pair sums and differences along x, then along
// y, then along z (18 additions instead of 28).
template <class T>
SORD_HD void hg_modes(const T X[8], T m[4]) {
    T Sy[2], Dx[2], Dxy[2];
#pragma unroll
    for (int dl = 0; dl < 2; dl++) {
        const T* P = X + 4 * dl;
        const T s0 = P[0] + P[1], s1 = P[2] + P[3], d0 = P[0] - P[1], d1 = P[2] - P[3];
        Sy[dl] = s0 - s1;
        Dx[dl] = d0 + d1;
        Dxy[dl] = d0 - d1;
    }
    m[0] = Sy[0] - Sy[1];
    m[1] = Dx[0] - Dx[1];
    m[2] = Dxy[0] + Dxy[1];
    m[3] = Dxy[0] - Dxy[1];
}
// The hourglass_cn sums of one cell for the node column q = cj + 2 ck that
// reads it (the node above the cell: yu, below it: yl), from the cell's four
// mode values m: the signed sums over the modes of the cell's term for that
// node (hg_neg(iq, hg_term(7 - p)) at cell position p), which are
// -(z (y m0 + x m1) + x y (m2 + z m3)) with x = 2 cj - 1, y = 2 ck - 1,
// z = +1 (yu) or -1 (yl).  hg_readers_pre forms the four shared sums once
// (a, b, pp, pm), hg_reader the two values of column q from them.
template <class T>
SORD_HD void hg_readers_pre(const T m[4], T r[4]) {
    r[0] = m[0] + m[1];
    r[1] = m[0] - m[1];
    r[2] = m[2] + m[3];
    r[3] = m[2] - m[3];
}
template <class T>
SORD_HD void hg_reader(const T r[4], int q, T& yu, T& yl) {
    const T a = r[0], b = r[1], pp = r[2], pm = r[3];
    if (q == 0) { yu = a - pp; yl = -a - pm; }
    else if (q == 1) { yu = b + pp; yl = pm - b; }
    else if (q == 2) { yu = pp - b; yl = b + pm; }
    else { yu = -a - pp; yl = a - pm; }
}

// F . B with fused multiply-adds (B already scaled by h).
SORD_HD float dot8(const float F[8], const float B[8]) {
    float d = F[0] * B[0];
#pragma unroll
    for (int t = 1; t < 8; t++) d = fmaf(F[t], B[t], d);
    return d;
}

}  // namespace sordgpu

// Support-operator and hourglass stencils as device functions.
//
// Every expression keeps the operand order of the Fortran it restates; the
// library is compiled with -fmad=false so that each product and sum rounds
// separately, exactly like the reference's (and the oracle's) FP32 code.
#pragma once

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

// Brackets of diff_nc for direction a (0-based) at one cell; X[c][n] is
// coordinate c at corner n = dj + 2*dk + 4*dl.  B[t] multiplies term t.
// sord/diff_nc_op.f90:19-70.
SORD_HD void brackets_nc(const float (*X)[8], int a, float B[8]) {
    const float* xb = X[(a + 1) % 3];
    const float* xc = X[(a + 2) % 3];
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

// Brackets of diff_cn for direction a at one node; X[c][m] is coordinate c
// at neighbour m = (dj+1) + 3*(dk+1) + 9*(dl+1), dj,dk,dl in -1..1.
// B[t] multiplies the cell of term t: (j-1,k-1,l-1) (j,k-1,l-1) (j-1,k-1,l)
// (j,k-1,l) (j-1,k,l-1) (j,k,l-1) (j-1,k,l) (j,k,l).  sord/diff_cn_op.f90:19-70.
template <class XA>
SORD_HD void brackets_cn(const XA& X, int a, float B[8]) {
    int b = (a + 1) % 3, c = (a + 2) % 3;
#define XB(j, k, l) X(b, (j) + 1 + 3 * ((k) + 1) + 9 * ((l) + 1))
#define XC(j, k, l) X(c, (j) + 1 + 3 * ((k) + 1) + 9 * ((l) + 1))
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

// Weighted 8-term sum  d = h*F0*B0; d = d + h*Ft*Bt  (diff_nc / diff_cn).
SORD_HD float stencil8(const float F[8], const float B[8], float h) {
    float d = h * F[0] * B[0];
#pragma unroll
    for (int t = 1; t < 8; t++) d = d + h * F[t] * B[t];
    return d;
}

// Hourglass sign patterns (hourglass_op.f90): the 8 terms of hourglass_nc
// are the corners 000 111 011 100 101 010 110 001 (offsets dj dk dl), those
// of hourglass_cn the cells at minus the same offsets.  hg_corner(t) is the
// corner id of term t; hg_neg(iq, t) is 1 where term t is subtracted.
SORD_HD int hg_corner(int t) { return (int)((0x43251670u >> (4 * t)) & 0xFu); }
SORD_HD int hg_neg(int iq, int t) { return (int)(((0xAA3CCCF0u >> (8 * iq)) >> t) & 1u); }

SORD_HD float hg_sum(const float A[8], int iq) {
    float r = A[0];
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
SORD_HD void cell_cn_brackets(const float (*X)[8], int a, const float nc[8], float cn[8]) {
    cn[0] = 0.0f - nc[6];
    cn[3] = 0.0f - nc[2];
    cn[4] = 0.0f - nc[5];
    cn[7] = 0.0f - nc[0];
    // node-relative accessors for the four remaining terms; the node sits at
    // cell corner o = (oj, ok, ol) and neighbour d maps to corner o + d.
    struct Acc {
        const float (*X)[8];
        int o;
        SORD_HD float operator()(int c, int m) const {
            int dj = m % 3 - 1, dk = (m / 3) % 3 - 1, dl = m / 9 - 1;
            int oj = o & 1, ok = (o >> 1) & 1, ol = (o >> 2) & 1;
            return X[c][(oj + dj) + 2 * (ok + dk) + 4 * (ol + dl)];
        }
    };
    float B[8];
    {  // term 1: cell (j, k-1, l-1) -> node at corner (0,1,1)
        Acc A{X, 6};
        brackets_cn(A, a, B);
        cn[1] = B[1];
    }
    {  // term 2: cell (j-1, k-1, l) -> node at corner (1,1,0)
        Acc A{X, 3};
        brackets_cn(A, a, B);
        cn[2] = B[2];
    }
    {  // term 5: cell (j, k, l-1) -> node at corner (0,0,1)
        Acc A{X, 4};
        brackets_cn(A, a, B);
        cn[5] = B[5];
    }
    {  // term 6: cell (j-1, k, l) -> node at corner (1,0,0)
        Acc A{X, 1};
        brackets_cn(A, a, B);
        cn[6] = B[6];
    }
}

}  // namespace sordgpu

// Support-operator and hourglass stencils as device functions.
//
// Every expression keeps the operand order of the Fortran it restates; the
// library is compiled with -fmad=false so that each product and sum rounds
// separately, exactly like the reference's (and the oracle's) FP32 code.
#pragma once

namespace sordgpu {

// Cell corners in the term order of diff_nc (diff_nc_op.f90:19-70):
// (0,0,0) (1,0,0) (0,1,0) (1,1,0) (0,0,1) (1,0,1) (1,1,1) (0,1,1).
__device__ __constant__ static const int kTermCorner[8] = {0, 1, 2, 3, 4, 5, 7, 6};  // corner id = dj + 2dk + 4dl

// Brackets of diff_nc for direction a (0-based) at one cell; X[c][n] is
// coordinate c at corner n = dj + 2*dk + 4*dl.  B[t] multiplies term t.
// sord/diff_nc_op.f90:19-70.
__device__ __forceinline__ void brackets_nc(const float (*X)[8], int a, float B[8]) {
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
__device__ __forceinline__ void brackets_cn(const XA& X, int a, float B[8]) {
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
__device__ __forceinline__ float stencil8(const float F[8], const float B[8], float h) {
    float d = h * F[0] * B[0];
#pragma unroll
    for (int t = 1; t < 8; t++) d = d + h * F[t] * B[t];
    return d;
}

// Hourglass sign patterns (hourglass_op.f90): the 8 terms of hourglass_nc
// are the corners 000 111 011 100 101 010 110 001 (offsets), those of
// hourglass_cn the cells at minus the same offsets.
__device__ __constant__ static const int kHgOff[8][3] = {{0, 0, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 0},
                                                         {1, 0, 1}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}};
__device__ __constant__ static const float kHgSign[4][8] = {{1, 1, 1, 1, -1, -1, -1, -1},
                                                            {1, 1, -1, -1, 1, 1, -1, -1},
                                                            {1, 1, -1, -1, -1, -1, 1, 1},
                                                            {1, -1, 1, -1, 1, -1, 1, -1}};

__device__ __forceinline__ float hg_sum(const float A[8], int iq) {
    float r = A[0];
#pragma unroll
    for (int t = 1; t < 8; t++) r = kHgSign[iq][t] > 0.f ? r + A[t] : r - A[t];
    return r;
}

}  // namespace sordgpu

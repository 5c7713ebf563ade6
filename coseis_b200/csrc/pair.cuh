// Two FP32 lanes per instruction (sm_100 packed f32x2 add / sub / fma).
//
// Each lane is rounded to nearest-even exactly like the scalar instruction,
// so evaluating two independent expressions in the two lanes of F2 gives
// bit-identical results to evaluating them one at a time; the stencil
// templates of stencil.cuh instantiated with F2 therefore keep the
// reference's FP32 operation order in each lane while issuing half the
// arithmetic instructions.  An F2 lives in one 64-bit register pair from
// construction to extraction, so chains of operations need no moves.
//
// Products: the assembler fuses a packed multiply whose only use is a packed
// add into one packed fused multiply-add, whatever the contraction settings,
// which changes the rounding.  A product is therefore issued as
// fma(a, b, nz) with nz = (-0.0, -0.0) held in a register pair whose value
// comes from the kernel's arguments: a*b + (-0) is exactly the rounded
// product (signed zeros included), and the assembler cannot see that nz is
// zero, so nothing is fused.  Every F2 carries that pair in `nz`.
#pragma once

namespace sordgpu {

__device__ __forceinline__ unsigned long long f2_pack(float x, float y) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
    return r;
}

struct F2 {
    unsigned long long v;   // lanes (x, y)
    unsigned long long nz;  // (-0.0, -0.0), unknown to the compiler
    __device__ __forceinline__ float x() const {
        float a;
        asm("{\n\t.reg .f32 hi;\n\tmov.b64 {%0, hi}, %1;\n\t}" : "=f"(a) : "l"(v));
        return a;
    }
    __device__ __forceinline__ float y() const {
        float b;
        asm("{\n\t.reg .f32 lo;\n\tmov.b64 {lo, %0}, %1;\n\t}" : "=f"(b) : "l"(v));
        return b;
    }
};

// nz2: f2_pack(-0.0f, -0.0f) of a run-time -0.0
__device__ __forceinline__ F2 f2(float x, float y, unsigned long long nz2) { return F2{f2_pack(x, y), nz2}; }
__device__ __forceinline__ F2 f2(float x, unsigned long long nz2) { return F2{f2_pack(x, x), nz2}; }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.v), "l"(b.v));
    return F2{d, a.nz};
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.v), "l"(b.v));
    return F2{d, a.nz};
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a.v), "l"(b.v), "l"(a.nz));
    return F2{d, a.nz};
}

}  // namespace sordgpu

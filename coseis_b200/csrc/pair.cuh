// Two FP32 lanes per instruction (sm_100 packed f32x2 add / sub / mul).
//
// Each lane is rounded to nearest-even exactly like the scalar instruction,
// so evaluating two independent expressions in the two lanes of F2 gives
// bit-identical results to evaluating them one at a time; the stencil
// templates of stencil.cuh instantiated with F2 therefore keep the
// reference's FP32 operation order in each lane while issuing half the
// arithmetic instructions.
#pragma once

namespace sordgpu {

struct F2 {
    float x, y;
};

__device__ __forceinline__ F2 f2(float x, float y) { return F2{x, y}; }
__device__ __forceinline__ F2 f2(float x) { return F2{x, x}; }

__device__ __forceinline__ unsigned long long f2_pack(F2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ F2 f2_unpack(unsigned long long r) {
    F2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pack(a)), "l"(f2_pack(b)));
    return f2_unpack(d);
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pack(a)), "l"(f2_pack(b)));
    return f2_unpack(d);
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pack(a)), "l"(f2_pack(b)));
    return f2_unpack(d);
}

}  // namespace sordgpu

// fy_common.cuh -- shared device/host helpers for the fysics B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FY_HD __host__ __device__ __forceinline__
#define FY_D __device__ __forceinline__

// Status codes (FY_OK, FY_EINVAL, ...) come from the public header.
#include "fysics_b200.h"

FY_HD float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Complex add and subtract. On the device each is one Blackwell paired FP32 instruction
// (add/sub.rn.f32x2: two IEEE round-to-nearest operations, the same results as two scalar
// ones), which halves the FP issue of the FFT butterflies.
FY_HD float2 cadd(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}
FY_HD float2 csub(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<unsigned long long*>(&a)),
        "l"(*reinterpret_cast<unsigned long long*>(&b)));
    return *reinterpret_cast<float2*>(&r);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// multiply by (i * s), s = +-1
FY_HD float2 cmul_is(float2 a, float s) { return make_float2(-s * a.y, s * a.x); }

// reflect-pad index, paganin.c:121-128 (symmetric "half-sample" reflection)
FY_HD int reflect_idx(int i, int n) {
    if (n == 1) return 0;
    while (i < 0 || i >= n) {
        if (i < 0) i = -i - 1;
        if (i >= n) i = 2 * n - i - 1;
    }
    return i;
}

FY_HD int ceil_div_i(int a, int b) { return (a + b - 1) / b; }

// Unsigned division by a runtime divisor d >= 1 via multiply-high (round-up method):
// q = (umulhi(n, m) + n) >> s, exact for every 32-bit n.
struct FastDiv {
    uint32_t d, m, s;
    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t div) : d(div) {
        s = 0;
        while ((1ull << s) < div) ++s;
        m = (uint32_t)((((1ull << 32) * ((1ull << s) - div)) / div) + 1);
    }
    FY_D uint32_t div(uint32_t n) const {
        return (uint32_t)(((uint64_t)__umulhi(n, m) + n) >> s);
    }
};

// Programmatic dependent launch. A kernel launched with fy_launch_pdl (fy_internal.h) may be
// scheduled while the previous kernel on its stream is finishing; fy_pdl_wait(), its first
// statement, then waits until that kernel has completed and its memory is visible (and is a
// no-op for a normal launch). Nothing before it may touch global memory.
FY_D void fy_pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }


// Shared device helpers of libfpm (B200, sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace fpm {

// Number of SMs on a B200; grids of grid-stride kernels are sized in multiples of it.
constexpr int kB200SMs = 148;

struct cplx {
    float re, im;
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + b.x * a.y);
}

// conj(b) * a, written with the operand order of the reference's gradW / gradP
// (cuFPM_v3/cuda/kernels.cuh:103-105, 122-124): re = a.re*b.re + a.im*b.im,
// im = b.re*a.im - a.re*b.im.
__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, b.x * a.y - a.x * b.y);
}

// copysignf(1, x): sign(+0) = +1 (cuFPM_v3/cuda/kernels.cuh:11-15).
__device__ __forceinline__ float sign1(float x) { return copysignf(1.0f, x); }

// Compensated (Kahan) accumulator for complex FP32 sums.  Compiled without
// fast-math, so the compensation is not re-associated away.
struct KahanC {
    float2 s = make_float2(0.f, 0.f);
    float2 c = make_float2(0.f, 0.f);
    __device__ __forceinline__ void add(float2 v) {
        float yx = v.x - c.x;
        float tx = s.x + yx;
        c.x = (tx - s.x) - yx;
        s.x = tx;
        float yy = v.y - c.y;
        float ty = s.y + yy;
        c.y = (ty - s.y) - yy;
        s.y = ty;
    }
};

struct KahanD {
    double s = 0.0;
    double c = 0.0;
    __device__ __forceinline__ void add(double v) {
        double y = v - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// (a mod m) for possibly negative a, m > 0.
__device__ __forceinline__ int pmod(int a, int m) {
    int r = a % m;
    return r < 0 ? r + m : r;
}

}  // namespace fpm

// The MATLAB optimiser classes of the reference's script-level loop, one fused
// elementwise pass each (optimizer_RMSprop.m, optimizer_adam.m, optimizer_yogi.m,
// optimizer_sgd.m), plus the pupil clamp of that loop
// (benchmark/cuFPM_recon_2025_circular.m:180-186).
//
// MATLAB evaluates these statements on single gpuArrays one operation at a time,
// every double scalar rounded to single first; the kernel does the same with
// explicitly rounded operations (no contraction into FMAs).  abs() of a complex
// value is the correctly rounded hypot, formed in double (exact products and a
// single rounding of the sum before the square root).
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "engine.h"

namespace fpm {

namespace {

__device__ __forceinline__ float cabs_rn(float2 z) {
    const double x = z.x, y = z.y;
    return (float)sqrt(x * x + y * y);
}

__device__ __forceinline__ float2 cscale(float s, float2 z) {
    return make_float2(__fmul_rn(s, z.x), __fmul_rn(s, z.y));
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}

__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}

// r * a + c * g, each product and the sum rounded (the moment updates)
__device__ __forceinline__ float2 ema(float r, float2 a, float c, float2 g) {
    return cadd(cscale(r, a), cscale(c, g));
}

// g ./ (sqrt(sq) + 1e-5) with MATLAB's complex square root of a negative sq
__device__ __forceinline__ float2 div_root(float2 g, float sq) {
    if (sq >= 0.f) {
        const float d = __fadd_rn(__fsqrt_rn(sq), 1e-5f);
        return make_float2(__fdiv_rn(g.x, d), __fdiv_rn(g.y, d));
    }
    // denominator 1e-5 + i sqrt(-sq)
    const float dr = 1e-5f, di = __fsqrt_rn(-sq);
    const float den = __fadd_rn(__fmul_rn(dr, dr), __fmul_rn(di, di));
    return make_float2(__fdiv_rn(__fadd_rn(__fmul_rn(g.x, dr), __fmul_rn(g.y, di)), den),
                       __fdiv_rn(__fsub_rn(__fmul_rn(g.y, dr), __fmul_rn(g.x, di)), den));
}

template <int KIND>
__global__ void __launch_bounds__(256) k_optimizer_step(OptStep o) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < o.n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float2 g = o.g[i];
        float2 p = o.p[i];
        if (KIND == kOptSgd) {
            p = csub(p, cscale(o.lr, g));
        } else {
            const float a = cabs_rn(g);
            const float g2 = __fmul_rn(a, a);              // abs(grad).^2
            if (KIND == kOptRmsprop) {
                float sq = __fadd_rn(o.r1, __fmul_rn(o.c1, g2));
                if (o.mom1) {                               // centered
                    const float2 g0 = ema(o.r1, o.mom1[i], o.c1, g);
                    o.mom1[i] = g0;
                    const float b = cabs_rn(g0);
                    sq = __fsub_rn(sq, __fmul_rn(b, b));
                }
                const float2 u = div_root(g, sq);
                if (o.buffer) {                             // momentum
                    const float2 buf = cadd(cscale(o.mum, o.buffer[i]), u);
                    o.buffer[i] = buf;
                    p = csub(p, cscale(o.lr, buf));
                } else {
                    p = csub(p, cscale(o.lr, u));
                }
            } else {
                const float2 m1 = ema(o.r1, o.mom1[i], o.c1, g);
                float m2 = o.mom2[i];
                if (KIND == kOptAdam) {
                    m2 = __fadd_rn(__fmul_rn(o.r2, m2), __fmul_rn(o.c2, g2));
                } else {                                    // Yogi
                    const float d = __fsub_rn(m2, g2);
                    const float s = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
                    m2 = __fsub_rn(m2, __fmul_rn(__fmul_rn(o.c2, s), g2));
                }
                o.mom1[i] = m1;
                o.mom2[i] = m2;
                const float2 num = KIND == kOptAdam ? cscale(o.bias, m1) : m1;
                const float d = __fadd_rn(__fsqrt_rn(m2), 1e-5f);
                p = csub(p, cscale(o.lr, make_float2(__fdiv_rn(num.x, d), __fdiv_rn(num.y, d))));
            }
        }
        if (o.amp) {
            // max(min(abs(p), a + ac), a - ac) .* sign(p) .* a, sign(p) = p ./ abs(p)
            const float a0 = o.amp[i];
            const float w = cabs_rn(p);
            const float t = fmaxf(fminf(w, __fadd_rn(a0, o.margin)), __fsub_rn(a0, o.margin));
            if (w > 0.f) {
                p = make_float2(__fmul_rn(__fmul_rn(t, __fdiv_rn(p.x, w)), a0),
                                __fmul_rn(__fmul_rn(t, __fdiv_rn(p.y, w)), a0));
            } else {
                p = make_float2(0.f, 0.f);
            }
        }
        o.p[i] = p;
    }
}

}  // namespace

cudaError_t launch_optimizer_step(const OptStep &o, cudaStream_t st) {
    size_t gx = (o.n + 255) / 256;
    if (gx > (size_t)kB200SMs * 8) gx = (size_t)kB200SMs * 8;
    if (gx == 0) gx = 1;
    switch (o.kind) {
        case kOptRmsprop: k_optimizer_step<kOptRmsprop><<<(unsigned)gx, 256, 0, st>>>(o); break;
        case kOptAdam: k_optimizer_step<kOptAdam><<<(unsigned)gx, 256, 0, st>>>(o); break;
        case kOptYogi: k_optimizer_step<kOptYogi><<<(unsigned)gx, 256, 0, st>>>(o); break;
        case kOptSgd: k_optimizer_step<kOptSgd><<<(unsigned)gx, 256, 0, st>>>(o); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace fpm

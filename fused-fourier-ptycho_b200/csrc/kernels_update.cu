// Pupil update, spectrum output, initial object, tiled transposes, and the small
// reductions / ingest kernels.  (The object's RMSprop lives in the column pass of
// pipeline.cu.)
#include "common.cuh"
#include "engine.h"

#include <algorithm>

namespace fpm {

// One RMSprop step (constrained_RMSprop_both, cuFPM_v3/cuda/kernels.cuh:364-382 for
// the object, :384-393 for the pupil): mu = beta*m + (1-beta)|g|^2,
// w -= g * lr/(sqrt(mu)+eps), m = mu.  The column pass of pipeline.cu applies the
// same expression to the object.
__device__ __forceinline__ void rms_one(float gr, float gi, float &wr, float &wi, float &m,
                                        float lr, float beta, float omb, float eps) {
    float mu = gr * gr + gi * gi;
    mu = beta * m + omb * mu;
    const float sq = lr / (sqrtf(mu) + eps);
    wr -= gr * sq;
    wi -= gi * sq;
    m = mu;
}

// RMSprop on the pupil plus the amplitude box constraint
// (kernels.cuh:384-410): |P| <- P0 * clamp(|P|, P0-am, P0+am), phase kept.
__global__ void __launch_bounds__(256) k_rmsprop_pupil(const float2 *__restrict__ dP,
                                                        float2 *__restrict__ P,
                                                        float *__restrict__ m,
                                                        const float *__restrict__ P0, int n,
                                                        float lr, float beta, float eps,
                                                        float am) {
    const float omb = 1.0f - beta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 gv = dP[i];
        float2 w = P[i];
        float mv = m[i];
        rms_one(gv.x, gv.y, w.x, w.y, mv, lr, beta, omb, eps);
        const float p0 = P0[i];
        const float ang = atan2f(w.y, w.x);
        float a = sqrtf(w.x * w.x + w.y * w.y);
        a = p0 * fmaxf(fminf(a, p0 + am), p0 - am);
        w.x = cosf(ang) * a;
        w.y = sinf(ang) * a;
        P[i] = w;
        m[i] = mv;
    }
}

cudaError_t launch_rmsprop_pupil(const float2 *dP, float2 *P, float *m, const float *P0, int n,
                                 float lr, float beta, float eps, float am, cudaStream_t st) {
    int gx = (n + 255) / 256;
    if (gx > kB200SMs * 8) gx = kB200SMs * 8;
    k_rmsprop_pupil<<<gx, 256, 0, st>>>(dP, P, m, P0, n, lr, beta, eps, am);
    return cudaGetLastError();
}

// In-place fftshift of an H x H array (even H): swaps (r, c) with
// ((r + H/2) mod H, (c + H/2) mod H); each pair is visited once from the c < H/2 half.
__global__ void __launch_bounds__(256) k_centre_in_place(float2 *__restrict__ S, int H) {
    const size_t half = (size_t)H * (H / 2);
    const int hh = H >> 1;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < half;
         q += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(q % H);
        const int c = (int)(q / H);
        const int r2 = r + hh >= H ? r + hh - H : r + hh;
        const size_t a = (size_t)c * H + r, b = (size_t)(c + hh) * H + r2;
        const float2 t = S[a];
        S[a] = S[b];
        S[b] = t;
    }
}

cudaError_t launch_centre_in_place(float2 *S, int H, cudaStream_t st) {
    const size_t half = (size_t)H * (H / 2);
    size_t gx = (half + 255) / 256;
    const size_t cap = (size_t)kB200SMs * 8 * 8;
    if (gx > cap) gx = cap;
    k_centre_in_place<<<(unsigned)gx, 256, 0, st>>>(S, H);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Initial object: MATLAB imresize(Y_1, pratio, 'bicubic') with zero phase
// (codes_v2/main_run_FPM.m:47-48).  Output pixel u (1-based) samples input
// x = u/p + (1 - 1/p)/2 with the a = -0.5 cubic on 4 taps, weights normalised
// to sum 1, half-sample-symmetric edges; rows are resized first, in FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double cubic_w(double t) {
    const double a = -0.5;
    t = fabs(t);
    if (t <= 1.0) return (a + 2.0) * t * t * t - (a + 3.0) * t * t + 1.0;
    if (t < 2.0) return a * t * t * t - 5.0 * a * t * t + 8.0 * a * t - 4.0 * a;
    return 0.0;
}

__device__ __forceinline__ void cubic_taps(int u0, int p, int n, int idx[4], double w[4]) {
    const double x = (double)(u0 + 1) / p + 0.5 * (1.0 - 1.0 / p);
    const double left = floor(x - 2.0);
    double s = 0.0;
    for (int k = 0; k < 4; ++k) {
        const double t = left + 1.0 + k;      // 1-based tap
        w[k] = cubic_w(x - t);
        s += w[k];
        int j = (int)t - 1;                   // 0-based, mirror with the edge repeated
        const int period = 2 * n;
        j = ((j % period) + period) % period;
        idx[k] = j < n ? j : period - 1 - j;
    }
    for (int k = 0; k < 4; ++k) w[k] /= s;
}

// The taps and weights depend only on the output index (the same table serves rows
// and columns of the square image), and the amplitude only on the input pixel, so
// both are computed once and the per-pixel work is 16 FP64 multiply-adds.
struct Taps {
    int4 idx;
    double w[4];
};

__global__ void __launch_bounds__(256) k_bicubic_taps(int h, int p, Taps *__restrict__ taps) {
    const int n_out = h * p;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n_out; u += gridDim.x * blockDim.x) {
        int idx[4];
        double w[4];
        cubic_taps(u, p, h, idx, w);
        Taps t;
        t.idx = make_int4(idx[0], idx[1], idx[2], idx[3]);
        for (int k = 0; k < 4; ++k) t.w[k] = w[k];
        taps[u] = t;
    }
}

template <int TYPE>
__global__ void __launch_bounds__(256) k_amplitude_page0(StackView Y, int h, float *__restrict__ amp) {
    float mn = 0.f, range = 0.f;
    if (TYPE == kStackU16) {
        mn = (float)Y.minmax[0];
        range = (float)(Y.minmax[1] - Y.minmax[0]);
    }
    const int n = h * h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float a;
        if (TYPE == kStackF32) {
            a = static_cast<const float *>(Y.ptr)[i];
        } else {
            const float x = (float)static_cast<const uint16_t *>(Y.ptr)[i] - mn;
            a = range > 0.f ? sqrtf(x / range) : sqrtf(x);
        }
        amp[i] = a;
    }
}

__global__ void __launch_bounds__(256) k_bicubic_init(const float *__restrict__ amp,
                                                       const Taps *__restrict__ taps, int h, int H,
                                                       float2 *__restrict__ O) {
    const size_t total = (size_t)H * H;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int R = (int)(q % H);
        const int C = (int)(q / H);
        const Taps tr = taps[R], tc = taps[C];
        const int ir[4] = {tr.idx.x, tr.idx.y, tr.idx.z, tr.idx.w};
        const int ic[4] = {tc.idx.x, tc.idx.y, tc.idx.z, tc.idx.w};
        double acc = 0.0;
        for (int kc = 0; kc < 4; ++kc) {
            double t = 0.0;
            for (int kr = 0; kr < 4; ++kr)
                t += tr.w[kr] * (double)amp[(size_t)ic[kc] * h + ir[kr]];
            acc += tc.w[kc] * t;
        }
        O[q] = make_float2((float)acc, 0.f);
    }
}

size_t bicubic_work_bytes(int h, int pratio) {
    return (size_t)h * pratio * sizeof(Taps) + (size_t)h * h * sizeof(float) + 256;
}

cudaError_t launch_bicubic_init(StackView Y, int h, int pratio, float2 *O, void *work,
                                cudaStream_t st) {
    const int H = h * pratio;
    Taps *taps = static_cast<Taps *>(work);
    float *amp = reinterpret_cast<float *>(
        (reinterpret_cast<uintptr_t>(taps + H) + 255) & ~static_cast<uintptr_t>(255));
    k_bicubic_taps<<<(H + 255) / 256, 256, 0, st>>>(h, pratio, taps);
    const int ga = (h * h + 255) / 256 < kB200SMs * 8 ? (h * h + 255) / 256 : kB200SMs * 8;
    if (Y.type == kStackU16)
        k_amplitude_page0<kStackU16><<<ga, 256, 0, st>>>(Y, h, amp);
    else
        k_amplitude_page0<kStackF32><<<ga, 256, 0, st>>>(Y, h, amp);
    const size_t total = (size_t)H * H;
    size_t gx = (total + 255) / 256;
    const size_t cap = (size_t)kB200SMs * 8 * 8;
    if (gx > cap) gx = cap;
    k_bicubic_init<<<(unsigned)gx, 256, 0, st>>>(amp, taps, h, H, O);
    return cudaGetLastError();
}

// Complex up-sampling: the same bicubic resize of the real and the imaginary part of an
// h x h column-major image (re, im planes), for the learned warm start.
__global__ void __launch_bounds__(256) k_bicubic_complex(const float *__restrict__ re,
                                                          const float *__restrict__ im,
                                                          const Taps *__restrict__ taps, int h,
                                                          int H, float2 *__restrict__ O) {
    const size_t total = (size_t)H * H;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int R = (int)(q % H);
        const int C = (int)(q / H);
        const Taps tr = taps[R], tc = taps[C];
        const int ir[4] = {tr.idx.x, tr.idx.y, tr.idx.z, tr.idx.w};
        const int ic[4] = {tc.idx.x, tc.idx.y, tc.idx.z, tc.idx.w};
        double ar = 0.0, ai = 0.0;
        for (int kc = 0; kc < 4; ++kc) {
            double tr_ = 0.0, ti = 0.0;
            for (int kr = 0; kr < 4; ++kr) {
                const size_t i = (size_t)ic[kc] * h + ir[kr];
                tr_ += tr.w[kr] * (double)re[i];
                ti += tr.w[kr] * (double)im[i];
            }
            ar += tc.w[kc] * tr_;
            ai += tc.w[kc] * ti;
        }
        O[q] = make_float2((float)ar, (float)ai);
    }
}

cudaError_t launch_bicubic_complex(const float *re, const float *im, int h, int pratio, float2 *O,
                                   void *work, cudaStream_t st) {
    const int H = h * pratio;
    Taps *taps = static_cast<Taps *>(work);
    k_bicubic_taps<<<(H + 255) / 256, 256, 0, st>>>(h, pratio, taps);
    const size_t total = (size_t)H * H;
    size_t gx = (total + 255) / 256;
    const size_t cap = (size_t)kB200SMs * 8 * 8;
    if (gx > cap) gx = cap;
    k_bicubic_complex<<<(unsigned)gx, 256, 0, st>>>(re, im, taps, h, H, O);
    return cudaGetLastError();
}

// Amplitudes of stack pages [first, first + count) (h*h each), as the solve normalises them.
template <int TYPE>
__global__ void __launch_bounds__(256) k_stack_pages(StackView Y, size_t first, size_t n,
                                                     float *__restrict__ out) {
    float mn = 0.f, range = 0.f;
    if (TYPE == kStackU16) {
        mn = (float)Y.minmax[0];
        range = (float)(Y.minmax[1] - Y.minmax[0]);
    }
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float a;
        if (TYPE == kStackF32) {
            a = static_cast<const float *>(Y.ptr)[first + i];
        } else {
            const float x = (float)static_cast<const uint16_t *>(Y.ptr)[first + i] - mn;
            a = range > 0.f ? sqrtf(x / range) : sqrtf(x);
        }
        out[i] = a;
    }
}

cudaError_t launch_stack_pages(StackView Y, int h, int first, int count, float *out,
                               cudaStream_t st) {
    const size_t plane = (size_t)h * h, n = plane * count;
    size_t gx = (n + 255) / 256;
    if (gx > (size_t)kB200SMs * 16) gx = (size_t)kB200SMs * 16;
    if (Y.type == kStackU16)
        k_stack_pages<kStackU16><<<(unsigned)gx, 256, 0, st>>>(Y, plane * first, n, out);
    else
        k_stack_pages<kStackF32><<<(unsigned)gx, 256, 0, st>>>(Y, plane * first, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Deterministic FP64 loss reduction: one block sums the per-tile partials in a
// fixed order (Kahan per thread, then a fixed tree) and adds them to *slot.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_loss_accumulate(const double *__restrict__ parts, int n,
                                                           double *__restrict__ slot) {
    __shared__ double s[1024];
    KahanD acc;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc.add(parts[i]);
    s[threadIdx.x] = acc.s;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *slot += s[0];
}

cudaError_t launch_loss_accumulate(const double *parts, int n, double *slot, cudaStream_t st) {
    k_loss_accumulate<<<1, 1024, 0, st>>>(parts, n, slot);
    return cudaGetLastError();
}

// End of a captured epoch: its accumulated loss goes to the slot the counter names, the
// accumulator restarts at zero and the counter moves to the next epoch.
__global__ void k_epoch_end(double *acc, double *loss, int *counter) {
    const int ep = *counter;
    loss[ep] = *acc;
    *acc = 0.0;
    *counter = ep + 1;
}

cudaError_t launch_epoch_end(double *acc, double *loss, int *counter, cudaStream_t st) {
    k_epoch_end<<<1, 1, 0, st>>>(acc, loss, counter);
    return cudaGetLastError();
}

__global__ void k_set_int(int *p, int v) { *p = v; }

cudaError_t launch_set_int(int *p, int v, cudaStream_t st) {
    k_set_int<<<1, 1, 0, st>>>(p, v);
    return cudaGetLastError();
}

// Global min / max of a uint16 stack (integer atomics: order-independent).
__global__ void __launch_bounds__(256) k_stack_minmax(const uint16_t *__restrict__ p, size_t n,
                                                       unsigned *__restrict__ mm) {
    unsigned lo = 0xffffu, hi = 0u;
    // eight values per 16-byte load over the aligned bulk, then the tail
    const size_t n8 = (reinterpret_cast<uintptr_t>(p) & 15u) ? 0 : n / 8;
    const uint4 *p8 = reinterpret_cast<const uint4 *>(p);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n8;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint4 v = p8[i];
        const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const unsigned a = w[k] & 0xffffu, b = w[k] >> 16;
            lo = min(lo, min(a, b));
            hi = max(hi, max(a, b));
        }
    }
    for (size_t i = n8 * 8 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const unsigned v = p[i];
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned a = __shfl_down_sync(0xffffffffu, lo, off);
        const unsigned b = __shfl_down_sync(0xffffffffu, hi, off);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

cudaError_t launch_stack_minmax(const uint16_t *p, size_t n, unsigned *mm, cudaStream_t st) {
    const unsigned init[2] = {0xffffu, 0u};
    cudaError_t e = cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    size_t gx = (n / 8 + 255) / 256;
    if (gx > (size_t)kB200SMs * 16) gx = (size_t)kB200SMs * 16;
    if (gx == 0) gx = 1;
    k_stack_minmax<<<(unsigned)gx, 256, 0, st>>>(p, n, mm);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_normalise(const uint16_t *__restrict__ p, size_t n,
                                                    const unsigned *__restrict__ mm,
                                                    float *__restrict__ out) {
    const float mn = (float)mm[0];
    const float range = (float)(mm[1] - mm[0]);
    auto amp = [&](unsigned v) {
        const float x = (float)v - mn;
        return range > 0.f ? sqrtf(x / range) : sqrtf(x);
    };
    // eight values per 16-byte load and two 16-byte stores over the aligned bulk
    const bool vec = ((reinterpret_cast<uintptr_t>(p) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
    const size_t n8 = vec ? n / 8 : 0;
    const uint4 *p8 = reinterpret_cast<const uint4 *>(p);
    float4 *o4 = reinterpret_cast<float4 *>(out);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n8;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint4 v = p8[i];
        o4[2 * i] = make_float4(amp(v.x & 0xffffu), amp(v.x >> 16), amp(v.y & 0xffffu), amp(v.y >> 16));
        o4[2 * i + 1] = make_float4(amp(v.z & 0xffffu), amp(v.z >> 16), amp(v.w & 0xffffu), amp(v.w >> 16));
    }
    for (size_t i = n8 * 8 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = amp(p[i]);
}

cudaError_t launch_normalise(const uint16_t *p, size_t n, const unsigned *mm, float *out,
                             cudaStream_t st) {
    size_t gx = (n / 8 + 255) / 256;
    if (gx > (size_t)kB200SMs * 16) gx = (size_t)kB200SMs * 16;
    if (gx == 0) gx = 1;
    k_normalise<<<(unsigned)gx, 256, 0, st>>>(p, n, mm, out);
    return cudaGetLastError();
}


// Amplitude of every uint16 count: one table lookup per pixel in the passes instead of
// a division and a square root, with the very floats the formula gives.
__global__ void __launch_bounds__(256) k_amplitude_lut(const unsigned *__restrict__ mm,
                                                        float *__restrict__ lut) {
    const float mn = (float)mm[0];
    const float range = (float)(mm[1] - mm[0]);
    const unsigned v = blockIdx.x * blockDim.x + threadIdx.x;
    const float x = (float)v - mn;
    lut[v] = range > 0.f ? sqrtf(x / range) : sqrtf(x);
}

cudaError_t launch_amplitude_lut(const unsigned *mm, float *lut, cudaStream_t st) {
    k_amplitude_lut<<<65536 / 256, 256, 0, st>>>(mm, lut);
    return cudaGetLastError();
}

// Row-major amplitude copy: 32 x 32 tiles through shared memory, read along the stored
// rows of a page (r), written along c; block (x, y, z) takes tile (x, y) of pages z,
// z + gridDim.z, ...
template <int TYPE>
__global__ void __launch_bounds__(256) k_amplitude_rows(StackView Y, int h, int pages,
                                                        float *__restrict__ out) {
    __shared__ float tile[32][33];
    float mn = 0.f, range = 0.f;
    if (TYPE == kStackU16 && !Y.lut) {
        mn = (float)Y.minmax[0];
        range = (float)(Y.minmax[1] - Y.minmax[0]);
    }
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int p = blockIdx.z; p < pages; p += gridDim.z) {
        const size_t page = (size_t)p * h * h;
        for (int i = threadIdx.y; i < 32; i += 8) {   // column c0 + i, row r0 + threadIdx.x
            const size_t idx = page + (size_t)(c0 + i) * h + r0 + threadIdx.x;
            float a;
            if (TYPE == kStackF32) {
                a = static_cast<const float *>(Y.ptr)[idx];
            } else {
                const uint16_t raw = static_cast<const uint16_t *>(Y.ptr)[idx];
                if (Y.lut) {
                    a = Y.lut[raw];
                } else {
                    const float x = (float)raw - mn;
                    a = range > 0.f ? sqrtf(x / range) : sqrtf(x);
                }
            }
            tile[i][threadIdx.x] = a;
        }
        __syncthreads();
        for (int i = threadIdx.y; i < 32; i += 8)     // row r0 + i, column c0 + threadIdx.x
            out[page + (size_t)(r0 + i) * h + c0 + threadIdx.x] = tile[threadIdx.x][i];
        __syncthreads();
    }
}

cudaError_t launch_amplitude_rows(StackView Y, int h, int pages, float *out, cudaStream_t st) {
    if (h % 32 != 0 || pages < 1) return cudaErrorInvalidValue;
    // about 32 blocks per SM for the whole stack (each walks its tile through many pages)
    const int tiles = (h / 32) * (h / 32);
    const int zc = std::max(1, std::min(pages, (kB200SMs * 32 + tiles - 1) / tiles));
    const dim3 grid((unsigned)(h / 32), (unsigned)(h / 32), (unsigned)std::min(zc, 65535));
    if (Y.type == kStackU16)
        k_amplitude_rows<kStackU16><<<grid, dim3(32, 8), 0, st>>>(Y, h, pages, out);
    else
        k_amplitude_rows<kStackF32><<<grid, dim3(32, 8), 0, st>>>(Y, h, pages, out);
    return cudaGetLastError();
}

// Float stacks (multi-sample frames averaged on ingest): the same min / max and
// sqrt((x - min) / (max - min)), min / max over order-preserving integer keys
// of the float bits (NaN skipped, as MATLAB's min / max omit NaN).
__device__ __forceinline__ unsigned float_key(float x) {
    const unsigned b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void __launch_bounds__(256) k_stack_minmax_f32(const float *__restrict__ p, size_t n,
                                                           unsigned *__restrict__ mm) {
    unsigned lo = 0xffffffffu, hi = 0u;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float x = p[i];
        if (x != x) continue;
        const unsigned k = float_key(x);
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned a = __shfl_down_sync(0xffffffffu, lo, off);
        const unsigned b = __shfl_down_sync(0xffffffffu, hi, off);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

__global__ void __launch_bounds__(256) k_normalise_f32(const float *p, size_t n,
                                                        const unsigned *__restrict__ mm,
                                                        float *out) {  // out may equal p
    const float mn = key_float(mm[0]);
    const float range = key_float(mm[1]) - mn;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float x = p[i] - mn;
        out[i] = range > 0.f ? sqrtf(x / range) : sqrtf(x);  // constant stack: zeros, as for uint16
    }
}

cudaError_t launch_normalise_f32(const float *p, size_t n, unsigned *mm, float *out,
                                 cudaStream_t st) {
    const unsigned init[2] = {0xffffffffu, 0u};
    cudaError_t e = cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    size_t gx = (n + 255) / 256;
    if (gx > (size_t)kB200SMs * 16) gx = (size_t)kB200SMs * 16;
    if (gx == 0) gx = 1;
    k_stack_minmax_f32<<<(unsigned)gx, 256, 0, st>>>(p, n, mm);
    k_normalise_f32<<<(unsigned)gx, 256, 0, st>>>(p, n, mm, out);
    return cudaGetLastError();
}

}  // namespace fpm

namespace fpm {

// ---------------------------------------------------------------------------
// Tiled transpose of a complex matrix: out[c * ldo + r] = in[r * ldi + c] for
// r < rows, c < cols (32 x 32 tiles through shared memory, both sides coalesced).
// With `conj_scale` != 0 the values are conjugated and multiplied by it.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_transpose_c(const float2 *__restrict__ in, size_t ldi,
                                                      float2 *__restrict__ out, size_t ldo,
                                                      int rows, int cols, float conj_scale) {
    __shared__ float2 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = r0 + ty + 8 * k, c = c0 + tx;
        if (r < rows && c < cols) tile[ty + 8 * k][tx] = in[(size_t)r * ldi + c];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = c0 + ty + 8 * k, r = r0 + tx;
        if (r < rows && c < cols) {
            float2 v = tile[tx][ty + 8 * k];
            if (conj_scale != 0.f) v = make_float2(v.x * conj_scale, -v.y * conj_scale);
            out[(size_t)c * ldo + r] = v;
        }
    }
}

cudaError_t launch_transpose(const float2 *in, size_t ldi, float2 *out, size_t ldo, int rows,
                             int cols, float conj_scale, cudaStream_t st) {
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    if (grid.y > 65535u) return cudaErrorInvalidValue;
    k_transpose_c<<<grid, 256, 0, st>>>(in, ldi, out, ldo, rows, cols, conj_scale);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bounding box of the non-zero pixels of a complex h x h pupil and of a real one
// (either may be NULL; NaN counts as non-zero): box = {min row, max row, min col,
// max col}, initialised by the launcher to {h, -1, h, -1} (no pixel).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_support_box(const float2 *__restrict__ P,
                                                      const float *__restrict__ A, int h,
                                                      int *__restrict__ box) {
    int rmin = h, rmax = -1, cmin = h, cmax = -1;
    const size_t n = (size_t)h * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        bool nz = false;
        if (P) {
            const float2 v = P[i];
            nz = !(v.x == 0.f && v.y == 0.f);
        }
        if (A) nz = nz || !(A[i] == 0.f);
        if (nz) {
            const int r = (int)(i % h), c = (int)(i / h);
            rmin = min(rmin, r);
            rmax = max(rmax, r);
            cmin = min(cmin, c);
            cmax = max(cmax, c);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        rmin = min(rmin, __shfl_down_sync(0xffffffffu, rmin, off));
        rmax = max(rmax, __shfl_down_sync(0xffffffffu, rmax, off));
        cmin = min(cmin, __shfl_down_sync(0xffffffffu, cmin, off));
        cmax = max(cmax, __shfl_down_sync(0xffffffffu, cmax, off));
    }
    if ((threadIdx.x & 31) == 0 && rmax >= 0) {
        atomicMin(&box[0], rmin);
        atomicMax(&box[1], rmax);
        atomicMin(&box[2], cmin);
        atomicMax(&box[3], cmax);
    }
}

__global__ void k_support_box_init(int *box, int h) {
    if (threadIdx.x == 0) {
        box[0] = h;
        box[1] = -1;
        box[2] = h;
        box[3] = -1;
    }
}

cudaError_t launch_support_box(const float2 *P, const float *A, int h, int *box, cudaStream_t st) {
    k_support_box_init<<<1, 32, 0, st>>>(box, h);
    const size_t n = (size_t)h * h;
    size_t gx = (n + 255) / 256;
    if (gx > (size_t)kB200SMs * 4) gx = (size_t)kB200SMs * 4;
    k_support_box<<<(unsigned)gx, 256, 0, st>>>(P, A, h, box);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Forward model output (benchmark/gen_img_batch.m:197-199): x = z * scale with z the
// unnormalised inverse FFT and scale = 1 / (h^2 pratio^2); out = |x|^2 (intensity)
// or |x| (amplitude), float.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sim_magnitude(const float4 *__restrict__ z, size_t n2,
                                                        float scale, int amplitude,
                                                        float2 *__restrict__ out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2;
         i += (size_t)gridDim.x * blockDim.x) {
        const float4 v = z[i];
        const float ar = v.x * scale, ai = v.y * scale, br = v.z * scale, bi = v.w * scale;
        float2 o = make_float2(ar * ar + ai * ai, br * br + bi * bi);
        if (amplitude) o = make_float2(sqrtf(o.x), sqrtf(o.y));
        out[i] = o;
    }
}

cudaError_t launch_sim_magnitude(const float2 *z, size_t n, float scale, int amplitude,
                                 float *out, cudaStream_t st) {
    if (n % 2) return cudaErrorInvalidValue;
    const size_t n2 = n / 2;
    size_t gx = (n2 + 255) / 256;
    if (gx > (size_t)kB200SMs * 16) gx = (size_t)kB200SMs * 16;
    k_sim_magnitude<<<(unsigned)gx, 256, 0, st>>>(reinterpret_cast<const float4 *>(z), n2, scale,
                                                  amplitude, reinterpret_cast<float2 *>(out));
    return cudaGetLastError();
}

}  // namespace fpm

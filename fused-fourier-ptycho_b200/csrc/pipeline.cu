// Fused mini-batch pipeline (B200, sm_100a).
//
// Per batch (centred crop box rows [rlo, rlo+rspan), cols [clo, clo+cspan);
// LED l sits at box offset (a_l, b_l) = (kt_l - 1 - rlo, kl_l - 1 - clo) mod H):
//
//  L1 cols_inv   T1[l][c'][:] = IFFT_r(sub_l(r, c) P(r, c)) with (r, c) = ifftshift(r', c')
//                (fused_getSubpupil_shifted + the batched inverse FFT's first half,
//                 cuFPM_v3/cuda/kernels.cuh:19-65, cuFPM_pure_v3.cu:151-156)
//  L2 rows_inv   z = IFFT_c(T1) in place; Rs = |z|/(h^2 p^2) - Y
//  L3 rows_fwd   d = anisotropic sign stencil of Rs, out = d z/|z| (differenceKernel_acc,
//                kernels.cuh:197-275) + loss partials; T1 = FFT_c(out) in place
//  L4 cols_fwd   X = FFT_r(T1); Xs[l][r][c] = X(fftshift(r, c)) row-major
//  pupil grad    dP = sum_l conj(sub_l) Xs_l, LED order, Kahan (kernels.cuh:118-128)
//  A rows_inv    per box row: stitch conj(P) Xs / H^2 of the covering LEDs (LED order,
//                Kahan; kernels.cuh:95-116 as a gather), IFFT along the row -> U
//  B cols        per column: IFFT along r of U (zero outside the box rows) -> object
//                gradient; RMSprop of O and m (kernels.cuh:364-382); FFT along r of the
//                updated column, kept only on the next batch's box rows -> V
//  C rows_fwd    per next-box row: FFT along the row of V, kept on the next box columns
//                -> the next batch's Sbox
//
// Only the box rows / columns of the gradient spectrum are non-zero and only the
// next box is read, so passes A and C touch rspan lines instead of H, and U, V
// hold H x rspan values instead of H x H.  Lines are transformed in shared memory
// by fft::line_fft (one CTA per line of 16384, several lines per CTA below).
#include "common.cuh"
#include "engine.h"
#include "fft_core.cuh"
#include "pipeline.h"

namespace fpm {

using fft::Geo;
using fft::swz;

namespace {

__device__ __forceinline__ int2 led_box_offset(const int2 *led, int l, const BatchGeom &g) {
    const int2 k = led[g.z_off + l];
    return make_int2(pmod(k.y - 1 - g.rlo, g.H), pmod(k.x - 1 - g.clo, g.H));
}

// Box index of crop position (offset + i).  Below H it is the plain sum (the box
// holds every crop); a box clamped to the full spectrum (span H) wraps modulo H.
__device__ __forceinline__ int box_index(int offset, int i, int H) {
    const int v = offset + i;
    return v >= H ? v - H : v;
}

template <int N>
constexpr int smem_bytes() {
    return Geo<N>::LINE_BYTES + Geo<N>::TW_BYTES;
}

template <class K>
cudaError_t set_smem(K kernel, int bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <int TYPE>
__device__ __forceinline__ float amplitude(const StackView &Y, size_t idx, float mn, float range) {
    if (TYPE == kStackF32) return static_cast<const float *>(Y.ptr)[idx];
    const float x = (float)static_cast<const uint16_t *>(Y.ptr)[idx] - mn;
    return range > 0.f ? sqrtf(x / range) : sqrtf(x);
}

// ---------------------------------------------------------------------------
// L1: crop x pupil, ifftshift, inverse FFT along r (contiguous column lines)
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_lr_cols_inv(const float2 *__restrict__ Sbox, const float2 *__restrict__ P,
                  const int2 *__restrict__ led, BatchGeom g, int l0, int nl,
                  float2 *__restrict__ T1, const float2 *__restrict__ thi,
                  const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    const long long total = (long long)nl * N;
    const long long g0 = (long long)blockIdx.x * G::LPC;
    constexpr int hh = N / 2;
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q / N;
        const int e = q % N;
        const long long gl = g0 + ln;
        if (gl < total) {
            const int lloc = (int)(gl / N);
            const int cq = (int)(gl % N);
            const int2 ab = led_box_offset(led, l0 + lloc, g);
            const int r = e + hh >= N ? e + hh - N : e + hh;
            const int c = cq + hh >= N ? cq + hh - N : cq + hh;
            const float2 s = Sbox[(size_t)box_index(ab.y, c, g.H) * g.rspan +
                                  box_index(ab.x, r, g.H)];
            smem[ln * N + swz(e)] = cmul(s, P[(size_t)c * N + r]);
        }
    }
    __syncthreads();
    fft::line_fft<N, +1>(smem + (threadIdx.x / G::T) * N, s_hi, s_lo, threadIdx.x % G::T);
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q / N;
        const int e = q % N;
        const long long gl = g0 + ln;
        if (gl < total) T1[(size_t)gl * N + e] = smem[ln * N + swz(e)];
    }
}

// ---------------------------------------------------------------------------
// L2: inverse FFT along c (strided row lines) -> z (in place) and the residual
// ---------------------------------------------------------------------------
template <int N, int TYPE>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_lr_rows_inv(StackView Y, BatchGeom g, int l0, int nl, float2 *__restrict__ T1,
                  float *__restrict__ Rs, const float2 *__restrict__ thi,
                  const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    const long long total = (long long)nl * N;
    const long long g0 = (long long)blockIdx.x * G::LPC;
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int c = q / G::LPC;
        const long long gl = g0 + ln;
        if (gl < total) {
            const size_t idx = ((size_t)(gl / N) * N + c) * N + (size_t)(gl % N);
            smem[ln * N + swz(c)] = T1[idx];
        }
    }
    __syncthreads();
    fft::line_fft<N, +1>(smem + (threadIdx.x / G::T) * N, s_hi, s_lo, threadIdx.x % G::T);
    float mn = 0.f, range = 0.f;
    if (TYPE == kStackU16) {
        mn = (float)Y.minmax[0];
        range = (float)(Y.minmax[1] - Y.minmax[0]);
    }
    const float ratio = (float)((double)N * N * g.pratio * g.pratio);
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int c = q / G::LPC;
        const long long gl = g0 + ln;
        if (gl < total) {
            const int lloc = (int)(gl / N);
            const int r = (int)(gl % N);
            const size_t idx = ((size_t)lloc * N + c) * N + r;
            const float2 z = smem[ln * N + swz(c)];
            T1[idx] = z;
            const size_t ypix = (size_t)(g.z_off + l0 + lloc) * N * N + (size_t)c * N + r;
            Rs[idx] = sqrtf(z.x * z.x + z.y * z.y) / ratio - amplitude<TYPE>(Y, ypix, mn, range);
        }
    }
}

// ---------------------------------------------------------------------------
// L3: sign stencil of the residual, phase, forward FFT along c (strided rows)
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_lr_rows_fwd(BatchGeom g, int nl, float2 *__restrict__ T1, const float *__restrict__ Rs,
                  double *__restrict__ parts, const float2 *__restrict__ thi,
                  const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    __shared__ double s_red[32];
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    const long long total = (long long)nl * N;
    const long long g0 = (long long)blockIdx.x * G::LPC;
    const float gscale = (float)(g.pratio * g.pratio);
    double lsum = 0.0;
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int c = q / G::LPC;
        const long long gl = g0 + ln;
        if (gl < total) {
            const int lloc = (int)(gl / N);
            const int r = (int)(gl % N);
            const float *rp = Rs + (size_t)lloc * N * N;
            const int cp = c + 1 == N ? 0 : c + 1, cm = c == 0 ? N - 1 : c - 1;
            const int rpp = r + 1 == N ? 0 : r + 1, rmm = r == 0 ? N - 1 : r - 1;
            const float a = rp[(size_t)c * N + r];
            const float rx = rp[(size_t)cp * N + r] - a;     // res(r, c+1) - res(r, c)
            const float ry = rp[(size_t)c * N + rpp] - a;    // res(r+1, c) - res(r, c)
            const float oxm = sign1(a - rp[(size_t)cm * N + r]);
            const float oym = sign1(a - rp[(size_t)c * N + rmm]);
            const float d = (oxm - sign1(rx) + oym - sign1(ry)) * gscale;
            lsum += (double)fabsf(rx) + (double)fabsf(ry);
            const float2 z = T1[((size_t)lloc * N + c) * N + r];
            const float mag = sqrtf(z.x * z.x + z.y * z.y);
            float2 o = make_float2(0.f, 0.f);
            if (mag > 0.f) {
                const float inv = 1.0f / mag;
                o.x = z.x * inv * d;
                o.y = z.y * inv * d;
            }
            smem[ln * N + swz(c)] = o;
        }
    }
    // fixed-order block reduction of the loss partial
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < G::THREADS / 32; ++w) t += s_red[w];
        parts[blockIdx.x] = t;
    }
    fft::line_fft<N, -1>(smem + (threadIdx.x / G::T) * N, s_hi, s_lo, threadIdx.x % G::T);
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int c = q / G::LPC;
        const long long gl = g0 + ln;
        if (gl < total) {
            const size_t idx = ((size_t)(gl / N) * N + c) * N + (size_t)(gl % N);
            T1[idx] = smem[ln * N + swz(c)];
        }
    }
}

// ---------------------------------------------------------------------------
// L4: forward FFT along r (contiguous columns) -> fftshift'ed row-major Xs
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_lr_cols_fwd(int l0, int nl, const float2 *__restrict__ T1, float2 *__restrict__ Xs,
                  const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    const long long total = (long long)nl * N;
    const long long g0 = (long long)blockIdx.x * G::LPC;
    constexpr int hh = N / 2;
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q / N;
        const int e = q % N;
        const long long gl = g0 + ln;
        if (gl < total) smem[ln * N + swz(e)] = T1[(size_t)gl * N + e];
    }
    __syncthreads();
    fft::line_fft<N, -1>(smem + (threadIdx.x / G::T) * N, s_hi, s_lo, threadIdx.x % G::T);
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int r = q / G::LPC;
        const long long gl = g0 + ln;
        if (gl < total) {
            const int lloc = (int)(gl / N);
            const int cf = (int)(gl % N);
            const int c = cf + hh >= N ? cf + hh - N : cf + hh;
            const int rf = r + hh >= N ? r + hh - N : r + hh;
            Xs[((size_t)(l0 + lloc) * N + r) * N + c] = smem[ln * N + swz(rf)];
        }
    }
}

// ---------------------------------------------------------------------------
// pupil gradient: 32 x 32 tiles, LED loop inside, Kahan accumulation
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_lr_pupil_grad(const float2 *__restrict__ Sbox,
                                                        const float2 *__restrict__ Xs,
                                                        const int2 *__restrict__ led, BatchGeom g,
                                                        float2 *__restrict__ dP) {
    __shared__ float2 sA[32][33];   // sub: [c][r]
    __shared__ float2 sB[32][33];   // Xs:  [r][c]
    const int h = g.h;
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    KahanC acc[4];
    for (int l = 0; l < g.nb; ++l) {
        const int2 ab = led_box_offset(led, l, g);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int cl = ty + 8 * k;
            const int r = r0 + tx, c = c0 + cl;       // sub: coalesced along r
            if (r < h && c < h)
                sA[cl][tx] = Sbox[(size_t)box_index(ab.y, c, g.H) * g.rspan + box_index(ab.x, r, g.H)];
            const int rr = r0 + cl, cc = c0 + tx;     // Xs: coalesced along c
            if (rr < h && cc < h) sB[cl][tx] = Xs[((size_t)l * h + rr) * h + cc];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int cl = ty + 8 * k;
            acc[k].add(cmul_conj(sB[tx][cl], sA[cl][tx]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = r0 + tx, c = c0 + ty + 8 * k;
        if (r < h && c < h) dP[(size_t)c * h + r] = acc[k].s;
    }
}

// ---------------------------------------------------------------------------
// Pass A: stitch the box rows of the gradient spectrum, inverse FFT along the row
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_big_rows_inv(BatchGeom g, const int2 *__restrict__ led, const float2 *__restrict__ P,
                   const float2 *__restrict__ Xs, float2 *__restrict__ U, int ldU,
                   const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    int2 *s_ab = reinterpret_cast<int2 *>(s_lo + 128);
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    for (int l = threadIdx.x; l < g.nb; l += G::THREADS) s_ab[l] = led_box_offset(led, l, g);
    const int ln = threadIdx.x / G::T;
    const int t = threadIdx.x % G::T;
    const int i = blockIdx.x * G::LPC + ln;     // box row of this line
    float2 *line = smem + ln * N;
    for (int e = t; e < N; e += G::T) line[swz(e)] = make_float2(0.f, 0.f);
    __syncthreads();
    const int h = g.h;
    const float inv_H2 = 1.0f / (float)((double)N * N);
    if (i < g.rspan) {
        // thread t owns box columns j = t + k*T; four per chunk
        for (int j0 = 0; j0 < g.cspan; j0 += 4 * G::T) {
            KahanC acc[4];
            for (int l = 0; l < g.nb; ++l) {
                const int2 ab = s_ab[l];
                int rr = i - ab.x;
                if (rr < 0) rr += N;
                if (rr >= h) continue;
                const float2 *xrow = Xs + ((size_t)l * h + rr) * h;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    int c = j0 + t + k * G::T - ab.y;
                    if (c < 0) c += N;
                    if (c < h && j0 + t + k * G::T < g.cspan) {
                        float2 v = cmul_conj(xrow[c], P[(size_t)c * h + rr]);
                        v.x *= inv_H2;
                        v.y *= inv_H2;
                        acc[k].add(v);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int j = j0 + t + k * G::T;
                if (j < g.cspan) {
                    int pos = g.Cu0 + j;
                    pos = pos >= N ? pos - N : pos;
                    line[swz(pos)] = acc[k].s;
                }
            }
        }
    }
    __syncthreads();
    fft::line_fft<N, +1>(line, s_hi, s_lo, t);
    if (i < g.rspan)
        for (int e = t; e < N; e += G::T) U[(size_t)e * ldU + i] = line[swz(e)];
}

// ---------------------------------------------------------------------------
// Pass B: columns (contiguous): IFFT of the gradient, RMSprop, FFT of the update
// ---------------------------------------------------------------------------
template <int N, int MODE>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_big_cols(ColsArgs a, const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    const int ln = threadIdx.x / G::T;
    const int t = threadIdx.x % G::T;
    const int c = blockIdx.x * G::LPC + ln;    // column; c >= N only when N < LPC
    const bool live = c < N;
    float2 *line = smem + ln * N;
    const size_t col = (size_t)(live ? c : 0) * N;
    if (MODE == kColsForward) {
        for (int e = t; e < N; e += G::T)
            line[swz(e)] = live ? a.O[col + e] : make_float2(0.f, 0.f);
    } else {
        for (int e = t; e < N; e += G::T) line[swz(e)] = make_float2(0.f, 0.f);
        __syncthreads();
        if (live) {
            const float2 *u = a.U + (size_t)c * a.ldU;
            for (int i = t; i < a.rspan; i += G::T) {
                int pos = a.Ru0 + i;
                pos = pos >= N ? pos - N : pos;
                line[swz(pos)] = u[i];
            }
        }
    }
    __syncthreads();
    if (MODE != kColsForward) {
        fft::line_fft<N, +1>(line, s_hi, s_lo, t);
        if (MODE == kColsGradient) {
            if (live)
                for (int e = t; e < N; e += G::T) a.gout[col + e] = line[swz(e)];
            return;
        }
        // RMSprop on the column (constrained_RMSprop_both, kernels.cuh:364-382)
        const float omb = 1.0f - a.beta;
        if (live) {
            for (int e = t; e < N; e += G::T) {
                const float2 gv = line[swz(e)];
                float2 w = a.O[col + e];
                float mu = gv.x * gv.x + gv.y * gv.y;
                mu = a.beta * a.m[col + e] + omb * mu;
                const float sq = a.lr / (sqrtf(mu) + a.eps);
                w.x -= gv.x * sq;
                w.y -= gv.y * sq;
                a.O[col + e] = w;
                a.m[col + e] = mu;
                line[swz(e)] = w;
            }
        }
        if (a.rspan_n == 0) return;   // uniform over the grid: no next batch
        __syncthreads();
    }
    fft::line_fft<N, -1>(line, s_hi, s_lo, t);
    if (live) {
        float2 *v = a.V + (size_t)c * a.ldV;
        for (int i = t; i < a.rspan_n; i += G::T) {
            int pos = a.Ru0n + i;
            pos = pos >= N ? pos - N : pos;
            v[i] = line[swz(pos)];
        }
    }
}

// ---------------------------------------------------------------------------
// Pass C: rows of V (strided) -> FFT along the row -> the next batch's Sbox
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Geo<N>::THREADS)
    k_big_rows_fwd(const float2 *__restrict__ V, int ldV, int rspan_n, int Cu0n, int cspan_n,
                   float2 *__restrict__ Sbox, const float2 *__restrict__ thi,
                   const float2 *__restrict__ tlo) {
    using G = Geo<N>;
    extern __shared__ float2 smem[];
    float2 *s_hi = smem + G::LPC * N;
    float2 *s_lo = s_hi + 128;
    fft::load_twiddles(s_hi, s_lo, thi, tlo, G::NHI, G::NLO);
    const int i0 = blockIdx.x * G::LPC;
    for (int q = threadIdx.x; q < G::LPC * N; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int e = q / G::LPC;
        if (i0 + ln < rspan_n) smem[ln * N + swz(e)] = V[(size_t)e * ldV + i0 + ln];
    }
    __syncthreads();
    fft::line_fft<N, -1>(smem + (threadIdx.x / G::T) * N, s_hi, s_lo, threadIdx.x % G::T);
    for (int q = threadIdx.x; q < G::LPC * cspan_n; q += G::THREADS) {
        const int ln = q % G::LPC;
        const int j = q / G::LPC;
        if (i0 + ln < rspan_n) {
            int pos = Cu0n + j;
            pos = pos >= N ? pos - N : pos;
            Sbox[(size_t)j * rspan_n + i0 + ln] = smem[ln * N + swz(pos)];
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
bool pipeline_supported(int h, int H) {
    auto p2 = [](int n) { return n >= 16 && n <= 16384 && (n & (n - 1)) == 0; };
    return p2(h) && p2(H) && h <= 8192;
}

#define FPM_DISPATCH_LR(n, F)   \
    switch (n) {                \
        case 16: F(16); break;  \
        case 32: F(32); break;  \
        case 64: F(64); break;  \
        case 128: F(128); break; \
        case 256: F(256); break; \
        case 512: F(512); break; \
        case 1024: F(1024); break; \
        case 2048: F(2048); break; \
        case 4096: F(4096); break; \
        case 8192: F(8192); break; \
        default: return cudaErrorInvalidValue; \
    }

#define FPM_DISPATCH_BIG(n, F)  \
    switch (n) {                \
        case 16: F(16); break;  \
        case 32: F(32); break;  \
        case 64: F(64); break;  \
        case 128: F(128); break; \
        case 256: F(256); break; \
        case 512: F(512); break; \
        case 1024: F(1024); break; \
        case 2048: F(2048); break; \
        case 4096: F(4096); break; \
        case 8192: F(8192); break; \
        case 16384: F(16384); break; \
        default: return cudaErrorInvalidValue; \
    }

static int lpc_of(int n) { return (n * 8 >= 64 * 1024) ? 1 : (64 * 1024) / (n * 8); }

int lr_blocks(int h, int nl) {
    const long long lines = (long long)nl * h;
    const int lpc = lpc_of(h);
    return (int)((lines + lpc - 1) / lpc);
}

cudaError_t launch_lr_cols_inv(const BatchGeom &g, const int2 *led, const float2 *P, BatchBufs b,
                               int l0, int nl, const Twiddles &tw, cudaStream_t st) {
    const int blocks = lr_blocks(g.h, nl);
    cudaError_t e = cudaSuccess;
#define F(N)                                                                              \
    e = set_smem(k_lr_cols_inv<N>, smem_bytes<N>());                                      \
    if (e != cudaSuccess) return e;                                                       \
    k_lr_cols_inv<N><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(                   \
        b.Sbox, P, led, g, l0, nl, b.T1, tw.lo_hi, tw.lo_lo);
    FPM_DISPATCH_LR(g.h, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_lr_rows_inv(const BatchGeom &g, StackView Y, BatchBufs b, int l0, int nl,
                               const Twiddles &tw, cudaStream_t st) {
    const int blocks = lr_blocks(g.h, nl);
    cudaError_t e = cudaSuccess;
#define F(N)                                                                              \
    if (Y.type == kStackU16) {                                                            \
        e = set_smem(k_lr_rows_inv<N, kStackU16>, smem_bytes<N>());                       \
        if (e != cudaSuccess) return e;                                                   \
        k_lr_rows_inv<N, kStackU16><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(    \
            Y, g, l0, nl, b.T1, b.Rs, tw.lo_hi, tw.lo_lo);                                \
    } else {                                                                              \
        e = set_smem(k_lr_rows_inv<N, kStackF32>, smem_bytes<N>());                       \
        if (e != cudaSuccess) return e;                                                   \
        k_lr_rows_inv<N, kStackF32><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(    \
            Y, g, l0, nl, b.T1, b.Rs, tw.lo_hi, tw.lo_lo);                                \
    }
    FPM_DISPATCH_LR(g.h, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_lr_rows_fwd(const BatchGeom &g, BatchBufs b, int l0, int nl, int part_off,
                               const Twiddles &tw, cudaStream_t st) {
    (void)l0;
    const int blocks = lr_blocks(g.h, nl);
    cudaError_t e = cudaSuccess;
#define F(N)                                                                              \
    e = set_smem(k_lr_rows_fwd<N>, smem_bytes<N>());                                      \
    if (e != cudaSuccess) return e;                                                       \
    k_lr_rows_fwd<N><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(                   \
        g, nl, b.T1, b.Rs, b.parts + part_off, tw.lo_hi, tw.lo_lo);
    FPM_DISPATCH_LR(g.h, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_lr_cols_fwd(const BatchGeom &g, BatchBufs b, int l0, int nl,
                               const Twiddles &tw, cudaStream_t st) {
    const int blocks = lr_blocks(g.h, nl);
    cudaError_t e = cudaSuccess;
#define F(N)                                                                              \
    e = set_smem(k_lr_cols_fwd<N>, smem_bytes<N>());                                      \
    if (e != cudaSuccess) return e;                                                       \
    k_lr_cols_fwd<N><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(                   \
        l0, nl, b.T1, b.Xs, tw.lo_hi, tw.lo_lo);
    FPM_DISPATCH_LR(g.h, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_lr_pupil_grad(const BatchGeom &g, const int2 *led, BatchBufs b, float2 *dP,
                                 cudaStream_t st) {
    const int t = (g.h + 31) / 32;
    k_lr_pupil_grad<<<dim3(t, t), 256, 0, st>>>(b.Sbox, b.Xs, led, g, dP);
    return cudaGetLastError();
}

cudaError_t launch_big_rows_inv(const BatchGeom &g, const int2 *led, const float2 *P,
                                const float2 *Xs, float2 *U, int ldU, const Twiddles &tw,
                                cudaStream_t st) {
    cudaError_t e = cudaSuccess;
#define F(N)                                                                                  \
    {                                                                                         \
        const int smem = smem_bytes<N>() + g.nb * (int)sizeof(int2);                          \
        const int blocks = (g.rspan + Geo<N>::LPC - 1) / Geo<N>::LPC;                          \
        e = set_smem(k_big_rows_inv<N>, smem);                                                \
        if (e != cudaSuccess) return e;                                                       \
        k_big_rows_inv<N><<<blocks, Geo<N>::THREADS, smem, st>>>(g, led, P, Xs, U, ldU,       \
                                                                 tw.hi_hi, tw.hi_lo);         \
    }
    FPM_DISPATCH_BIG(g.H, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_big_cols(const ColsArgs &a, const Twiddles &tw, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
#define F(N)                                                                                  \
    {                                                                                         \
        const int blocks = (N + Geo<N>::LPC - 1) / Geo<N>::LPC;                               \
        if (a.mode == kColsForward) {                                                         \
            e = set_smem(k_big_cols<N, kColsForward>, smem_bytes<N>());                       \
            if (e != cudaSuccess) return e;                                                   \
            k_big_cols<N, kColsForward><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(    \
                a, tw.hi_hi, tw.hi_lo);                                                       \
        } else if (a.mode == kColsUpdate) {                                                   \
            e = set_smem(k_big_cols<N, kColsUpdate>, smem_bytes<N>());                        \
            if (e != cudaSuccess) return e;                                                   \
            k_big_cols<N, kColsUpdate><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(     \
                a, tw.hi_hi, tw.hi_lo);                                                       \
        } else {                                                                              \
            e = set_smem(k_big_cols<N, kColsGradient>, smem_bytes<N>());                      \
            if (e != cudaSuccess) return e;                                                   \
            k_big_cols<N, kColsGradient><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(   \
                a, tw.hi_hi, tw.hi_lo);                                                       \
        }                                                                                     \
    }
    FPM_DISPATCH_BIG(a.H, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_big_rows_fwd(int H, const float2 *V, int ldV, int rspan_n, int Cu0n,
                                int cspan_n, float2 *Sbox, const Twiddles &tw, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
#define F(N)                                                                                  \
    {                                                                                         \
        const int blocks = (rspan_n + Geo<N>::LPC - 1) / Geo<N>::LPC;                          \
        e = set_smem(k_big_rows_fwd<N>, smem_bytes<N>());                                     \
        if (e != cudaSuccess) return e;                                                       \
        k_big_rows_fwd<N><<<blocks, Geo<N>::THREADS, smem_bytes<N>(), st>>>(                  \
            V, ldV, rspan_n, Cu0n, cspan_n, Sbox, tw.hi_hi, tw.hi_lo);                        \
    }
    FPM_DISPATCH_BIG(H, F)
#undef F
    return cudaGetLastError();
}

}  // namespace fpm

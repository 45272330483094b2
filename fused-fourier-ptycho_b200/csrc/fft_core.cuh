// Block-level FFT building blocks (power-of-two lengths 16 .. 16384).
//
// A line of N complex values sits in shared memory in natural order at
// swizzled addresses (swz below).  T = N/16 threads cooperate on one line; each
// stage of a radix-R Stockham (self-sorting) decomposition has every thread
// load 16 values, apply the stage twiddles, run 16/R in-register DFTs of
// length R, and store 16 values:
//
//   butterfly i in [0, N/R), k = i mod p (p = product of the radices done):
//     inputs   x[i + r N/R]                          r = 0..R-1
//     twiddle  x_r *= W_{pR}^{r k}   (W_n = exp(DIR 2 pi i / n))
//     outputs  y[(i - k) R + k + r p] = DFT_R(x)_r
//
// (radix-R form of the Stockham algorithm; natural order in and out).  The
// XOR swizzle l ^ ((l >> 4) & 15) makes the strided stores of the first stage
// and all contiguous loads bank-conflict free.  Stage twiddles W_N^m come from
// a two-level table W_N^m = hi[m >> 7] * lo[m & 127] held in shared memory
// (about 1.5 ulp), built on the host in double precision.
#pragma once

#include "common.cuh"

namespace fpm {
namespace fft {

__device__ __forceinline__ int swz(int l) { return l ^ ((l >> 4) & 15); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// cos / sin of 2 pi k / 16, k = 0..4 (the rest follow by symmetry)
__host__ __device__ constexpr float c16(int k) {
    return k == 0 ? 1.0f
         : k == 1 ? 0.92387953251128674f
         : k == 2 ? 0.70710678118654757f
         : k == 3 ? 0.38268343236508978f
                  : 0.0f;
}

// W_16^k = exp(DIR 2 pi i k / 16) for k in [0, 8)
template <int DIR>
__device__ __forceinline__ float2 w16(int k) {
    // cos(2 pi k/16) and sin(2 pi k/16) for k in 0..7
    const float c = k <= 4 ? c16(k) : -c16(8 - k);
    const float s = k <= 4 ? c16(4 - k) : c16(k - 4);
    return make_float2(c, DIR < 0 ? -s : s);
}

// multiply by W_16^k (k compile-time), special-casing the trivial factors
template <int DIR, int K>
__device__ __forceinline__ float2 mul_w16(float2 v) {
    if constexpr (K == 0) {
        return v;
    } else if constexpr (K == 4) {  // exp(DIR i pi/2) = DIR * i
        return DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
    } else {
        return cmulf(v, w16<DIR>(K));
    }
}

__host__ __device__ constexpr int bitrev(int x, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

// In-register DFT of length R in {1, 2, 4, 8, 16}: out_k = sum_j v_j W_R^{jk}.
// Radix-2 decimation in time over a bit-reversed copy; every index and twiddle
// is a compile-time constant after unrolling.
template <int R, int DIR>
__device__ __forceinline__ void dft(float2 (&v)[R]) {
    if constexpr (R == 1) {
        return;
    } else {
        constexpr int B = ilog2(R);
        float2 a[R];
#pragma unroll
        for (int i = 0; i < R; ++i) a[i] = v[bitrev(i, B)];
#pragma unroll
        for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
            for (int i = 0; i < R; i += len) {
#pragma unroll
                for (int j = 0; j < len / 2; ++j) {
                    // W_len^j = W_16^(j * 16 / len)
                    float2 u = a[i + j];
                    float2 t = a[i + j + len / 2];
                    const int kk = j * (16 / len);
                    if (kk == 0) {
                    } else if (kk == 4) {
                        t = mul_w16<DIR, 4>(t);
                    } else {
                        t = cmulf(t, w16<DIR>(kk));
                    }
                    a[i + j] = cadd(u, t);
                    a[i + j + len / 2] = csub(u, t);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = a[i];
    }
}

// W_N^m with the sign of DIR, from the two-level forward table (hi, lo).
template <int DIR>
__device__ __forceinline__ float2 twiddle(const float2 *hi, const float2 *lo, int m) {
    float2 w = cmulf(hi[m >> 7], lo[m & 127]);
    if (DIR > 0) w.y = -w.y;
    return w;
}

// One radix-R stage on a line of N values; t in [0, N/16).
template <int N, int DIR, int P, int R>
__device__ __forceinline__ void stage(float2 *s, const float2 *hi, const float2 *lo, int t) {
    constexpr int T = N / 16;
    constexpr int NB = 16 / R;
    float2 v[NB][R];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const int i = t + j * T;
#pragma unroll
        for (int r = 0; r < R; ++r) v[j][r] = s[swz(i + r * (N / R))];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const int i = t + j * T;
        const int k = i & (P - 1);
        if constexpr (P > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r)
                v[j][r] = cmulf(v[j][r], twiddle<DIR>(hi, lo, r * k * (N / (P * R))));
        }
        dft<R, DIR>(v[j]);
        const int base = (i - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) s[swz(base + r * P)] = v[j][r];
    }
    __syncthreads();
}

template <int N, int DIR, int P>
__device__ __forceinline__ void stages(float2 *s, const float2 *hi, const float2 *lo, int t) {
    if constexpr (P < N) {
        constexpr int REM = N / P;
        constexpr int R = REM >= 16 ? 16 : REM;
        stage<N, DIR, P, R>(s, hi, lo, t);
        stages<N, DIR, P * R>(s, hi, lo, t);
    }
}

// Unnormalised DFT of the N values at s (swizzled, natural order), in place.
// Must be reached by every thread of the block (it synchronises); threads with
// t >= N/16 of a multi-line block run their own line.
template <int N, int DIR>
__device__ __forceinline__ void line_fft(float2 *s, const float2 *hi, const float2 *lo, int t) {
    static_assert(N >= 16 && (N & (N - 1)) == 0, "power-of-two length >= 16");
    stages<N, DIR, 1>(s, hi, lo, t);
}

// Copies the two-level twiddle table of length N into shared memory.
// hi needs max(1, N/128) entries, lo min(N, 128).
__device__ __forceinline__ void load_twiddles(float2 *s_hi, float2 *s_lo, const float2 *g_hi,
                                              const float2 *g_lo, int n_hi, int n_lo) {
    for (int i = threadIdx.x; i < n_hi; i += blockDim.x) s_hi[i] = g_hi[i];
    for (int i = threadIdx.x; i < n_lo; i += blockDim.x) s_lo[i] = g_lo[i];
}

// CTA shape for lines of length N: T = N/16 threads per line, LPC lines per CTA
// (64 KiB of line data per CTA for N <= 8192, one 128 KiB line for N = 16384).
template <int N>
struct Geo {
    static constexpr int T = N / 16;
    static constexpr int LPC = (N * 8 >= 64 * 1024) ? 1 : (64 * 1024) / (N * 8);
    static constexpr int THREADS = T * LPC;
    static constexpr int LINE_BYTES = LPC * N * 8;
    static constexpr int TW_BYTES = 2 * 128 * 8;
    static constexpr int NHI = N >= 128 ? N / 128 : 1;
    static constexpr int NLO = N >= 128 ? 128 : N;
};

}  // namespace fft
}  // namespace fpm

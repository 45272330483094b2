// Block-level FFT building blocks (power-of-two lengths 16 .. 16384).
//
// T = N/16 threads cooperate on a line of N complex values, each holding 16 of
// them in registers; each stage of a radix-R Stockham (self-sorting)
// decomposition applies the stage twiddles, runs 16/R in-register DFTs of
// length R, and exchanges values through shared memory (swizzled addresses,
// swz below):
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
// (about 1.5 ulp), built on the host in double precision; within a butterfly the
// powers W^(r m) beyond r = 1, 2, 4, 8 are products of table values.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace fpm {
namespace fft {

__device__ __forceinline__ int swz(int l) { return l ^ ((l >> 4) & 15); }

// Exchange addresses for E values per thread: E = 16 uses swz above; E = 32 (radix-32
// stages, whose first-stage stores stride 32 values) uses l ^ ((l >> 5) & 15), which
// keeps every store and load of the 16384-point plan 32 x 16 x ... on distinct bank
// pairs.
template <int E>
__device__ __forceinline__ int swz_e(int l) {
    if constexpr (E == 32) {
        return l ^ ((l >> 5) & 15);
    } else {
        return swz(l);
    }
}

// Complex arithmetic on packed float pairs: one sm_100 two-lane instruction
// (FADD2 / FMUL2 / FFMA2) per complex add and two per complex product, half the
// scalar count.  Each lane is an ordinary IEEE round-to-nearest operation.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);   // a - b, exact negation
}
// w * v = (w.x v.x - w.y v.y, w.x v.y + w.y v.x); w is the factor that is
// broadcast (a twiddle or a constant), v the data.
__device__ __forceinline__ float2 cmulf(float2 w, float2 v) {
    const float2 t = __fmul2_rn(make_float2(w.x, w.x), v);
    return __ffma2_rn(make_float2(-w.y, w.y), make_float2(v.y, v.x), t);
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

// cos / sin of 2 pi k / 32, k = 0..8
__host__ __device__ constexpr float c32(int k) {
    return k == 0 ? 1.0f
         : k == 1 ? 0.98078528040323043f
         : k == 2 ? 0.92387953251128674f
         : k == 3 ? 0.83146961230254524f
         : k == 4 ? 0.70710678118654757f
         : k == 5 ? 0.55557023301960218f
         : k == 6 ? 0.38268343236508978f
         : k == 7 ? 0.19509032201612825f
                  : 0.0f;
}

// W_32^k = exp(DIR 2 pi i k / 32) for k in [0, 16)
template <int DIR>
__device__ __forceinline__ float2 w32(int k) {
    const float c = k <= 8 ? c32(k) : -c32(16 - k);
    const float s = k <= 8 ? c32(8 - k) : c32(k - 8);
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
        return cmulf(w16<DIR>(K), v);
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
    } else if constexpr (R == 32) {
        // the 16-point networks of the even and odd halves, then the last level with W_32^j
        float2 e[16], o[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            e[i] = v[2 * i];
            o[i] = v[2 * i + 1];
        }
        dft<16, DIR>(e);
        dft<16, DIR>(o);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            float2 t = o[j];
            if (j == 8) {
                t = mul_w16<DIR, 4>(t);
            } else if (j != 0) {
                t = cmulf(w32<DIR>(j), t);
            }
            v[j] = cadd(e[j], t);
            v[j + 16] = csub(e[j], t);
        }
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
                        t = cmulf(w16<DIR>(kk), t);
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

// Position of table entry i in shared memory: within each block of 16 entries the low
// three bits are XORed with the block number, so that the strided lookups of a stage
// (index stride 1 .. 64 across a warp) fall on distinct banks instead of piling up on
// one (stride 16: eight entries on one bank pair without it).
__device__ __forceinline__ int twpos(int i) { return i ^ ((i >> 4) & 7); }

// W_N^m with the sign of DIR, from the two-level forward table (hi, lo).
template <int DIR>
__device__ __forceinline__ float2 twiddle(const float2 *hi, const float2 *lo, int m) {
    float2 w = cmulf(hi[twpos(m >> 7)], lo[twpos(m & 127)]);
    if (DIR > 0) w.y = -w.y;
    return w;
}

// u[r] *= W^(r m1) for r = 1 .. R-1.  Only W^m1, W^2m1, W^4m1, W^8m1 come from the
// table (two shared-memory loads each); the other powers are products of those
// (at most three products deep, a few ulp), which takes most of the twiddle loads
// and their bank conflicts off the shared-memory pipe.
template <int R, int DIR>
__device__ __forceinline__ void apply_twiddles(float2 (&u)[R], const float2 *hi, const float2 *lo,
                                               int m1) {
    // radix 32: u[16 + q] takes W^((16 + q) m1) = W^(q m1) W^(16 m1), next to u[q]
    float2 w16 = make_float2(1.f, 0.f);
    if constexpr (R >= 32) {
        w16 = twiddle<DIR>(hi, lo, 16 * m1);
        u[16] = cmulf(w16, u[16]);
    }
    auto put = [&](int q, float2 wq) {
        u[q] = cmulf(wq, u[q]);
        if constexpr (R >= 32) u[16 + q] = cmulf(cmulf(wq, w16), u[16 + q]);
    };
    const float2 w1 = twiddle<DIR>(hi, lo, m1);
    put(1, w1);
    if constexpr (R >= 4) {
        const float2 w2 = twiddle<DIR>(hi, lo, 2 * m1);
        put(2, w2);
        const float2 w3 = cmulf(w1, w2);
        put(3, w3);
        if constexpr (R >= 8) {
            const float2 w4 = twiddle<DIR>(hi, lo, 4 * m1);
            put(4, w4);
            put(5, cmulf(w1, w4));
            put(6, cmulf(w2, w4));
            put(7, cmulf(w3, w4));
            if constexpr (R >= 16) {
                const float2 w8 = twiddle<DIR>(hi, lo, 8 * m1);
                put(8, w8);
                put(9, cmulf(w1, w8));
                put(10, cmulf(w2, w8));
                put(11, cmulf(w3, w8));
                const float2 w12 = cmulf(w4, w8);
                put(12, w12);
                put(13, cmulf(w1, w12));
                put(14, cmulf(w2, w12));
                put(15, cmulf(w3, w12));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Register-resident variant.  Thread t of a line owns the 16 elements
// t + m*(N/16), m = 0..15, in v[m] ("canonical" layout) on entry and on exit.
// For any radix R the butterfly j of a first stage (p = 1) reads exactly these
// positions (i + r N/R = t + (j + r*16/R) N/16), and a last stage (p = N/R)
// writes them, so the first stage takes its inputs from registers and the last
// stage leaves its outputs in registers; only the exchanges between stages go
// through shared memory (N values at s, swizzled).  Callers load v straight
// from global memory (16 independent loads per thread) and store it back, or
// hand it to the next computation without a shared-memory round trip.
// ---------------------------------------------------------------------------
// Called by stages_regs between the last stage's reads of the exchange area and its
// arithmetic, after a block barrier: from then on the area is free (e.g. for a copy
// into it that overlaps the last stage's butterflies).
struct NoHook {
    __device__ void operator()() const {}
};

template <int N, int DIR, int P, int E, typename Hook = NoHook>
__device__ __forceinline__ void stages_regs(float2 (&v)[E], float2 *s, const float2 *hi,
                                            const float2 *lo, int t, const Hook &hook = Hook{}) {
    constexpr int REM = N / P;
    constexpr int R = REM >= E ? E : REM;
    constexpr int T = N / E;
    constexpr int NB = E / R;
    constexpr bool FIRST = P == 1;
    constexpr bool LAST = P * R == N;
    if constexpr (!FIRST) {
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int r = 0; r < R; ++r) v[j + r * NB] = s[swz_e<E>(t + j * T + r * (N / R))];
    }
    if constexpr (!LAST) __syncthreads();   // every read of s done before it is rewritten
    if constexpr (LAST && !FIRST && !std::is_same<Hook, NoHook>::value) {
        __syncthreads();                    // every read of s done: the area is free
        hook();
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        float2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[j + r * NB];
        const int i = t + j * T;
        const int k = i & (P - 1);
        if constexpr (P > 1) apply_twiddles<R, DIR>(u, hi, lo, k * (N / (P * R)));
        dft<R, DIR>(u);
        if constexpr (LAST) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[j + r * NB] = u[r];
        } else {
            const int base = (i - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) s[swz_e<E>(base + r * P)] = u[r];
        }
    }
    if constexpr (!LAST) {
        __syncthreads();
        stages_regs<N, DIR, P * R, E, Hook>(v, s, hi, lo, t, hook);
    }
}

// Unnormalised DFT of a line held in canonical registers (see above).  Must be
// reached by every thread of the block when N > 16 (it synchronises); the
// shared-memory line s must not be in use by other threads on entry.
template <int N, int DIR, typename Hook = NoHook>
__device__ __forceinline__ void line_fft_regs(float2 (&v)[16], float2 *s, const float2 *hi,
                                              const float2 *lo, int t, const Hook &hook = Hook{}) {
    static_assert(N >= 16 && (N & (N - 1)) == 0, "power-of-two length >= 16");
    stages_regs<N, DIR, 1, 16, Hook>(v, s, hi, lo, t, hook);
}

// The same with 32 values per thread (t + m N/32, m < 32): radix-32 stages, one
// exchange fewer for N = 16384 (32 x 32 x 16) at N/32 threads per line.
template <int N, int DIR, typename Hook = NoHook>
__device__ __forceinline__ void line_fft_regs32(float2 (&v)[32], float2 *s, const float2 *hi,
                                                const float2 *lo, int t, const Hook &hook = Hook{}) {
    static_assert(N >= 1024 && (N & (N - 1)) == 0, "power-of-two length >= 1024");
    stages_regs<N, DIR, 1, 32, Hook>(v, s, hi, lo, t, hook);
}

// Copies the two-level twiddle table of length N into shared memory.
// hi needs max(1, N/128) entries, lo min(N, 128).
__device__ __forceinline__ void load_twiddles(float2 *s_hi, float2 *s_lo, const float2 *g_hi,
                                              const float2 *g_lo, int n_hi, int n_lo) {
    for (int i = threadIdx.x; i < n_hi; i += blockDim.x) s_hi[twpos(i)] = g_hi[i];
    for (int i = threadIdx.x; i < n_lo; i += blockDim.x) s_lo[twpos(i)] = g_lo[i];
}

// CTA shape for the register-resident kernels: LPC lines of length N per CTA,
// T = N/16 threads per line, lines padded in shared memory by PAD values so that
// the LPC lines of an interleaved warp fall on different banks.
template <int N, int E = 16>
struct LG {
    static constexpr int T = N / E;
    static constexpr int LPC = (N * 8 >= 64 * 1024) ? 1 : (64 * 1024) / (N * 8);
    static constexpr int THREADS = T * LPC;
    // 16 values per thread: 64 registers, two CTAs per SM when they fit; 32 values:
    // up to 128 registers, one CTA
    static constexpr int MINB = (E == 16 && THREADS <= 512) ? 2 : 1;
    static constexpr int PAD = LPC == 1 ? 0 : (16 / LPC > 0 ? 16 / LPC : 1);
    static constexpr int STRIDE = N + PAD;
    static constexpr int SMEM = LPC * STRIDE * 8 + 2 * 128 * 8;
    static constexpr int NHI = N >= 128 ? N / 128 : 1;
    static constexpr int NLO = N >= 128 ? 128 : N;
    // contiguous mapping: a warp walks one line
    __device__ static int cline() { return threadIdx.x / T; }
    __device__ static int ct() { return threadIdx.x % T; }
    // interleaved mapping: a warp spans the LPC lines, LPC consecutive lines per element
    __device__ static int iline() { return threadIdx.x % LPC; }
    __device__ static int it() { return threadIdx.x / LPC; }
    __device__ static float2 *tw_hi(float2 *smem) { return smem + LPC * STRIDE; }
};

}  // namespace fft
}  // namespace fpm

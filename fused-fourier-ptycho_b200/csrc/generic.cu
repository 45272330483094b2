// Any-size path (generic.h): mixed-radix line FFT and the per-batch stages for image
// sides that are not powers of two.
//
// Line FFT: a CTA transforms LPC contiguous lines of n values held in shared memory,
// T = ceil(n/16) threads per line.  Each stage is a radix-R Stockham step (self-sorting,
// natural order in and out, as in fft_core.cuh):
//
//   butterfly j in [0, n/R), k = j mod p (p = product of the radices done):
//     inputs   x[j + r n/R]                          r = 0..R-1
//     twiddle  x_r *= W_{pR}^{r k} = W_n^{r k n/(pR)}
//     outputs  y[(j - k) R + k + r p] = DFT_R(x)_r
//
// A thread holds its butterflies' inputs in registers across a block barrier, so the
// stage runs in place in one shared-memory line.  Twiddles come from a table of W_n^m,
// m < n, built on the host in double precision and read through the read-only cache.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "fft_core.cuh"
#include "generic.h"
#include "tuning.h"

namespace fpm {

namespace {

// cos / sin of 2 pi m / R for the odd radices (m = 1 .. (R-1)/2)
template <int R>
__device__ __forceinline__ float cos_r(int m) {
    if constexpr (R == 3) {
        return -0.5f;
    } else if constexpr (R == 5) {
        return m == 1 ? 0.30901699437494745f : -0.8090169943749473f;
    } else {
        return m == 1 ? 0.6234898018587336f : m == 2 ? -0.22252093395631434f : -0.900968867902419f;
    }
}
template <int R>
__device__ __forceinline__ float sin_r(int m) {
    if constexpr (R == 3) {
        return 0.8660254037844387f;
    } else if constexpr (R == 5) {
        return m == 1 ? 0.9510565162951535f : 0.5877852522924732f;
    } else {
        return m == 1 ? 0.7818314824680298f : m == 2 ? 0.9749279121818236f : 0.43388373911755823f;
    }
}

// DFT of odd length R in {3, 5, 7}: with a_j = v_j + v_{R-j}, b_j = v_j - v_{R-j},
//   out_k     = v_0 + sum_j a_j cos(2 pi j k / R) + i DIR sum_j b_j sin(2 pi j k / R)
//   out_{R-k} = the same with the sine term negated.
template <int R, int DIR>
__device__ __forceinline__ void dft_odd(float2 (&v)[R]) {
    constexpr int H = (R - 1) / 2;
    float2 a[H], b[H];
#pragma unroll
    for (int j = 1; j <= H; ++j) {
        a[j - 1] = make_float2(v[j].x + v[R - j].x, v[j].y + v[R - j].y);
        b[j - 1] = make_float2(v[j].x - v[R - j].x, v[j].y - v[R - j].y);
    }
    float2 out[R];
    float2 s0 = v[0];
#pragma unroll
    for (int j = 0; j < H; ++j) s0 = make_float2(s0.x + a[j].x, s0.y + a[j].y);
    out[0] = s0;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
        float2 t1 = v[0], t2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            const int m = (j * k) % R;                       // compile-time after unrolling
            const int mm = m <= H ? m : R - m;
            const float c = cos_r<R>(mm);
            const float s = m <= H ? sin_r<R>(mm) : -sin_r<R>(mm);
            t1 = make_float2(fmaf(a[j - 1].x, c, t1.x), fmaf(a[j - 1].y, c, t1.y));
            t2 = make_float2(fmaf(b[j - 1].x, s, t2.x), fmaf(b[j - 1].y, s, t2.y));
        }
        // i DIR t2 = DIR (-t2.y, t2.x)
        const float2 it2 = DIR < 0 ? make_float2(t2.y, -t2.x) : make_float2(-t2.y, t2.x);
        out[k] = make_float2(t1.x + it2.x, t1.y + it2.y);
        out[R - k] = make_float2(t1.x - it2.x, t1.y - it2.y);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
}

template <int R, int DIR>
__device__ __forceinline__ void dft_any(float2 (&v)[R]) {
    if constexpr (R == 3 || R == 5 || R == 7) {
        dft_odd<R, DIR>(v);
    } else {
        fft::dft<R, DIR>(v);
    }
}

__device__ __forceinline__ float2 cmul2(float2 w, float2 v) {
    return make_float2(w.x * v.x - w.y * v.y, w.x * v.y + w.y * v.x);
}

// k mod p of a butterfly index j < 2^24: the quotient from the float reciprocal of p,
// corrected to the exact one
__device__ __forceinline__ int mod_p(int j, int p, float pinv) {
    int q = __float2int_rz(__int2float_rn(j) * pinv);
    int r = j - q * p;
    if (r < 0) r += p;
    else if (r >= p) r -= p;
    return r;
}

// One radix-R stage over a line of n values at s (shared memory), T = ceil(n/V) threads,
// thread t; pinv = 1 / p.
template <int R, int DIR, int V>
__device__ __forceinline__ void gen_stage_body(float2 *s, int n, int p, float pinv, int T, int t,
                                               const float2 *__restrict__ tw) {
    constexpr int KMAX = (V + R - 1) / R;    // ceil(n/R / ceil(n/V)) <= ceil(V/R)
    const int nbf = n / R;
    float2 v[KMAX][R];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        const int j = t + k * T;
        if (j < nbf) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[k][r] = s[j + r * nbf];
        }
    }
    __syncthreads();
    const int step = n / (p * R);
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        const int j = t + k * T;
        if (j < nbf) {
            const int kk = p > 1 ? mod_p(j, p, pinv) : 0;
            if (p > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = __ldg(tw + r * kk * step);   // < n: (R-1)(p-1) n/(pR) < n
                    if (DIR > 0) w.y = -w.y;
                    v[k][r] = cmul2(w, v[k][r]);
                }
            }
            dft_any<R, DIR>(v[k]);
            const int base = (j - kk) * R + kk;
#pragma unroll
            for (int r = 0; r < R; ++r) s[base + r * p] = v[k][r];
        }
    }
    __syncthreads();
}

// a call per stage keeps the kernel's registers within 128 (inlined, the six radices'
// bodies spill)
template <int R, int DIR, int V>
__device__ __noinline__ void gen_stage(float2 *s, int n, int p, float pinv, int T, int t,
                                       const float2 *__restrict__ tw) {
    gen_stage_body<R, DIR, V>(s, n, p, pinv, T, t, tw);
}

struct GenPlan {
    int n = 0, nst = 0, T = 0, lpc = 1, v = 8;
    int radix[16] = {};
    float pinv[16] = {};   // 1 / (product of the radices before stage i)
};

// V values per thread: 8 up to n = 4096, 16 up to 8192, 32 beyond (at most 512 threads
// per line, so that a thread may use up to 128 registers)
template <int DIR, int V>
__global__ void __launch_bounds__(512, 1) k_gen_lines(const float2 *__restrict__ in,
                                                    float2 *__restrict__ out, long long count,
                                                    size_t ld, GenPlan pl,
                                                    const float2 *__restrict__ tw) {
    extern __shared__ float2 smem[];
    const int n = pl.n, T = pl.T, lpc = pl.lpc;
    const long long g0 = (long long)blockIdx.x * lpc;
    const int nl = (int)min((long long)lpc, count - g0);
    // coalesced copy of the CTA's lines into shared memory
    for (int q = threadIdx.x; q < nl * n; q += blockDim.x) {
        const int l = q / n, i = q - l * n;
        smem[l * n + i] = in[(size_t)(g0 + l) * ld + i];
    }
    __syncthreads();
    const int line = threadIdx.x / T, t = threadIdx.x - line * T;
    // threads of a line past the last one (the CTA's tail) still join every barrier
    float2 *s = smem + (size_t)min(line, lpc - 1) * n;
    const bool live = line < nl;
    int p = 1;
    for (int st = 0; st < pl.nst; ++st) {
        const int R = pl.radix[st];
        const float pinv = pl.pinv[st];
        const int tt = live ? t : (1 << 29);   // idle threads skip every butterfly
        switch (R) {
            case 2: gen_stage<2, DIR, V>(s, n, p, pinv, T, tt, tw); break;
            case 3: gen_stage<3, DIR, V>(s, n, p, pinv, T, tt, tw); break;
            case 4: gen_stage<4, DIR, V>(s, n, p, pinv, T, tt, tw); break;
            case 5: gen_stage<5, DIR, V>(s, n, p, pinv, T, tt, tw); break;
            case 7: gen_stage<7, DIR, V>(s, n, p, pinv, T, tt, tw); break;
            default: gen_stage<8, DIR, V>(s, n, p, pinv, T, tt, tw); break;
        }
        p *= R;
    }
    for (int q = threadIdx.x; q < nl * n; q += blockDim.x) {
        const int l = q / n, i = q - l * n;
        out[(size_t)(g0 + l) * ld + i] = smem[l * n + i];
    }
}

// Register-resident form, where every stage's radix divides the values per thread V: a
// thread holds the canonical elements t + m T (m < V, T = n / V) of its line, loaded and
// stored straight from global memory.  The first stage's butterflies j = t + k T take
// their inputs x[j + r n/R] = element t + (k + r V/R) T from the thread's own registers,
// the last stage's outputs y[j + r p] land on the same elements, and only the stages in
// between exchange through shared memory; V/R butterflies per thread in every stage.
struct VPlan {
    int n = 0, V = 0, T = 0, lpc = 1, nst = 0;
    int radix[16] = {};
    float pinv[16] = {};
};

// shared-memory position of line element l: l ^ ((l >> 4) & 15) within its 16-element
// block when n is a multiple of 16 (mask 15: the stride-R stores of a stage and the
// contiguous loads fall on distinct banks), l itself otherwise (mask 0)
__device__ __forceinline__ int vswz(int l, int mask) { return l ^ ((l >> 4) & mask); }

template <int R, int DIR, int V>
__device__ __forceinline__ void vstage(float2 (&v)[V], float2 *s, int n, int p, float pinv, int T,
                                       int t, const float2 *__restrict__ tw, bool first,
                                       bool last, int mask) {
    constexpr int NB = V / R;
    const int nbf = n / R;   // = NB T butterflies
    if (!first) {
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
            for (int r = 0; r < R; ++r) v[k + r * NB] = s[vswz(t + k * T + r * nbf, mask)];
        __syncthreads();   // every read of the line done before it is rewritten
    }
    const int step = n / (p * R);
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int j = t + k * T;
        float2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[k + r * NB];
        int kk = 0;
        if (p > 1) {
            kk = mod_p(j, p, pinv);
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(tw + r * kk * step);   // < n: (R-1)(p-1) n/(pR) < n
                if (DIR > 0) w.y = -w.y;
                u[r] = cmul2(w, u[r]);
            }
        }
        dft_any<R, DIR>(u);
        if (last) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[k + r * NB] = u[r];   // y[j + r p], p = n/R
        } else {
            const int base = (j - kk) * R + kk;
#pragma unroll
            for (int r = 0; r < R; ++r) s[vswz(base + r * p, mask)] = u[r];
        }
    }
    if (!last) __syncthreads();   // the stage's outputs visible to the next stage
}

// Line g is column c = (g_lo + g) mod n of page P = g / n (with g_lo = 0: line g at
// in + g*ld, the plain batch of lines).  TOUT: the output is written transposed, for
// n x n pages (ld = n; whole pages, or with g_lo the columns [g_lo, g_lo + count) mod n of
// one page): element e of line g goes to out[P][e][c].  The CTA's lines are staged in
// shared memory as [element][line] and stored as rows of lpc columns.
template <int DIR, int V, bool TOUT>
__global__ void __launch_bounds__(512, 1) k_gen_lines_v(const float2 *__restrict__ in,
                                                      float2 *__restrict__ out, long long count,
                                                      size_t ld, VPlan pl,
                                                      const float2 *__restrict__ tw, int g_lo) {
    extern __shared__ float2 smem[];
    const int n = pl.n, T = pl.T;
    const int line = threadIdx.x / T, t = threadIdx.x - line * T;
    const long long g = (long long)blockIdx.x * pl.lpc + line;
    const bool live = g < count;   // lines past the last one join every barrier on zeros
    float2 *s = smem + (size_t)line * n;
    float2 v[V];
    auto line_of = [&](long long gg) {   // page * n + column of line gg
        const long long page = gg / n;
        const int c = (int)((g_lo + (gg - page * n)) % n);
        return page * n + c;
    };
    const float2 *src = in + (size_t)(live ? (TOUT && g_lo ? line_of(g) : g) : 0) * ld;
#pragma unroll
    for (int m = 0; m < V; ++m) v[m] = live ? src[t + m * T] : make_float2(0.f, 0.f);
    const int mask = n % 16 == 0 ? 15 : 0;
    int p = 1;
    for (int st = 0; st < pl.nst; ++st) {
        const int R = pl.radix[st];
        const float pinv = pl.pinv[st];
        const bool first = st == 0, last = st == pl.nst - 1;
        switch (R) {
            case 2: vstage<2, DIR, V>(v, s, n, p, pinv, T, t, tw, first, last, mask); break;
            case 4: vstage<4, DIR, V>(v, s, n, p, pinv, T, t, tw, first, last, mask); break;
            case 3:
                if constexpr (V % 3 == 0) vstage<3, DIR, V>(v, s, n, p, pinv, T, t, tw, first, last, mask);
                break;
            case 5:
                if constexpr (V % 5 == 0) vstage<5, DIR, V>(v, s, n, p, pinv, T, t, tw, first, last, mask);
                break;
            case 7:
                if constexpr (V % 7 == 0) vstage<7, DIR, V>(v, s, n, p, pinv, T, t, tw, first, last, mask);
                break;
            default:
                if constexpr (V % 8 == 0) vstage<8, DIR, V>(v, s, n, p, pinv, T, t, tw, first, last, mask);
                break;
        }
        p *= R;
    }
    if constexpr (TOUT) {
        __syncthreads();                        // the last stage's reads of the area done
        const int W = pl.lpc + 1;               // padded staging row
#pragma unroll
        for (int m = 0; m < V; ++m) smem[(size_t)(t + m * T) * W + line] = v[m];
        __syncthreads();
        const int l = threadIdx.x % pl.lpc;
        const long long gl = (long long)blockIdx.x * pl.lpc + l;
        if (gl < count) {
            const long long pc = line_of(gl), page = pc / n;
            float2 *dst = out + (size_t)page * n * n + (size_t)(pc - page * n);
            for (int e = threadIdx.x / pl.lpc; e < n; e += T) dst[(size_t)e * n] = smem[(size_t)e * W + l];
        }
    } else if (live) {
        float2 *dst = out + (size_t)g * ld;
#pragma unroll
        for (int m = 0; m < V; ++m) dst[t + m * T] = v[m];
    }
}

GenPlan make_plan(int n) {
    GenPlan pl;
    pl.n = n;
    const std::vector<int> rad = gen_fft_radices(n);
    pl.nst = (int)rad.size();
    int prod = 1;
    for (int i = 0; i < pl.nst; ++i) {
        pl.radix[i] = rad[i];
        pl.pinv[i] = 1.0f / (float)prod;
        prod *= rad[i];
    }
    pl.v = n <= 4096 ? 8 : n <= 8192 ? 16 : 32;
    pl.T = (n + pl.v - 1) / pl.v;
    // lines per CTA: up to 16, within 512 threads and 96 KiB of shared memory
    int lpc = 1;
    while (lpc < 16 && (lpc * 2) * pl.T <= 512 && (size_t)(lpc * 2) * n * 8 <= 96 * 1024) lpc *= 2;
    // a tuned (or forced) count within the same limits
    const int want = knob("FPM_GEN_LPC", tuning().gen_lpc, 0, lpc);
    while (pl.lpc * 2 <= want && pl.lpc * 2 * pl.T <= 512 && (size_t)(pl.lpc * 2) * n * 8 <= 96 * 1024)
        pl.lpc *= 2;
    return pl;
}

__global__ void __launch_bounds__(256) k_transpose_pages(const float2 *__restrict__ in,
                                                         float2 *__restrict__ out, int n) {
    __shared__ float2 tile[32][33];
    const size_t page = (size_t)blockIdx.z * n * n;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    // in[page][c][r]: element (r, c) at c*n + r
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = c0 + ty + 8 * k, r = r0 + tx;
        if (r < n && c < n) tile[ty + 8 * k][tx] = in[page + (size_t)c * n + r];
    }
    __syncthreads();
    // out[page][r][c] = element (r, c) at r*n + c
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = r0 + ty + 8 * k, c = c0 + tx;
        if (r < n && c < n) out[page + (size_t)r * n + c] = tile[tx][ty + 8 * k];
    }
}

// out[c][r] = in[r][c] for the columns [lo, lo + cnt) mod n of in, zero for the others (which
// are never read): the transpose of a page whose other columns count as zeros.
__global__ void __launch_bounds__(256) k_transpose_page_cols(const float2 *__restrict__ in,
                                                             float2 *__restrict__ out, int n,
                                                             int lo, int cnt) {
    __shared__ float2 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    auto inbox = [&](int c) {
        int d = c - lo;
        if (d < 0) d += n;
        return d < cnt;
    };
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = c0 + ty + 8 * k, r = r0 + tx;
        if (r < n && c < n)
            tile[ty + 8 * k][tx] = inbox(c) ? in[(size_t)c * n + r] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = r0 + ty + 8 * k, c = c0 + tx;
        if (r < n && c < n) out[(size_t)r * n + c] = tile[tx][ty + 8 * k];
    }
}

// Rows [lo, lo + cnt) mod n of a column-major n x n page as cnt contiguous lines, and
// back: TO_LINES: lines[i][c] = page[c][(lo + i) mod n]; else page[c][(lo + i) mod n] =
// lines[i][c].  32 x 32 tiles through shared memory, both sides coalesced.
template <bool TO_LINES>
__global__ void __launch_bounds__(256) k_transpose_rows(const float2 *__restrict__ in,
                                                        float2 *__restrict__ out, int n, int lo,
                                                        int cnt) {
    __shared__ float2 tile[32][33];
    const int c0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    auto row = [&](int i) {
        const int r = lo + i;
        return r >= n ? r - n : r;
    };
    if (TO_LINES) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {   // page: consecutive rows of one column
            const int c = c0 + ty + 8 * k, i = i0 + tx;
            if (i < cnt && c < n) tile[ty + 8 * k][tx] = in[(size_t)c * n + row(i)];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) {   // lines: consecutive columns of one line
            const int i = i0 + ty + 8 * k, c = c0 + tx;
            if (i < cnt && c < n) out[(size_t)i * n + c] = tile[tx][ty + 8 * k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = i0 + ty + 8 * k, c = c0 + tx;
            if (i < cnt && c < n) tile[ty + 8 * k][tx] = in[(size_t)i * n + c];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int c = c0 + ty + 8 * k, i = i0 + tx;
            if (i < cnt && c < n) out[(size_t)c * n + row(i)] = tile[tx][ty + 8 * k];
        }
    }
}

// ---------------------------------------------------------------------------
// per-batch stages
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gen_crop_pupil(const float2 *__restrict__ S, int H,
                                                        const float2 *__restrict__ P, int h,
                                                        const int2 *__restrict__ led, int z_off,
                                                        float2 *__restrict__ out) {
    const int l = blockIdx.y;
    const size_t plane = (size_t)h * h;
    const int2 k = led[z_off + l];                 // (kl, kt), 1-based
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < plane;
         i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i % h), c = (int)(i / h);
        const int R = (k.y - 1 + r + H / 2) % H, C = (k.x - 1 + c + H / 2) % H;
        const float2 a = S[(size_t)C * H + R];
        const float2 p = P[i];
        const float2 v = make_float2(a.x * p.x - a.y * p.y, a.x * p.y + p.x * a.y);
        const int rs = (r + h / 2) % h, cs = (c + h / 2) % h;
        out[(size_t)l * plane + (size_t)cs * h + rs] = v;
    }
}

__global__ void __launch_bounds__(256) k_gen_stitch(const float2 *__restrict__ X, int h,
                                                    const float2 *__restrict__ P,
                                                    const int2 *__restrict__ led, int z_off,
                                                    int nb, int H, int rlo, int rspan, int clo,
                                                    int cspan, float inv_h2,
                                                    float2 *__restrict__ G) {
    extern __shared__ int2 s_led[];
    for (int l = threadIdx.x; l < nb; l += blockDim.x) s_led[l] = led[z_off + l];
    __syncthreads();
    const size_t plane = (size_t)h * h;
    const size_t n = (size_t)rspan * cspan;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x) {
        const int br = (int)(q % rspan), bc = (int)(q / rspan);
        const int Rc = (rlo + br) % H, Cc = (clo + bc) % H;     // centred coordinates
        KahanC acc;
        bool any = false;
        for (int l = 0; l < nb; ++l) {
            const int r = pmod(Rc - (s_led[l].y - 1), H);
            const int c = pmod(Cc - (s_led[l].x - 1), H);
            if (r >= h || c >= h) continue;
            const float2 x = X[(size_t)l * plane + (size_t)((c + h / 2) % h) * h + (r + h / 2) % h];
            const float2 g = cmul_conj(x, P[(size_t)c * h + r]);
            acc.add(make_float2(g.x * inv_h2, g.y * inv_h2));
            any = true;
        }
        if (any) {
            const int R = (Rc + H / 2) % H, C = (Cc + H / 2) % H;   // un-shifted position
            G[(size_t)C * H + R] = acc.s;
        }
    }
}

__global__ void __launch_bounds__(256) k_gen_pupil_grad(const float2 *__restrict__ S, int H,
                                                        const float2 *__restrict__ X, int h,
                                                        const int2 *__restrict__ led, int z_off,
                                                        int nb, float2 *__restrict__ dP) {
    extern __shared__ int2 s_led[];
    for (int l = threadIdx.x; l < nb; l += blockDim.x) s_led[l] = led[z_off + l];
    __syncthreads();
    const size_t plane = (size_t)h * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < plane;
         i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i % h), c = (int)(i / h);
        const size_t xs = (size_t)((c + h / 2) % h) * h + (r + h / 2) % h;
        KahanC acc;
        for (int l = 0; l < nb; ++l) {
            const int R = (s_led[l].y - 1 + r + H / 2) % H, C = (s_led[l].x - 1 + c + H / 2) % H;
            acc.add(cmul_conj(X[(size_t)l * plane + xs], S[(size_t)C * H + R]));
        }
        dP[i] = acc.s;
    }
}

__global__ void __launch_bounds__(256) k_rmsprop_object(float2 *__restrict__ O, float *__restrict__ m,
                                                        const float2 *__restrict__ g, size_t n,
                                                        float lr, float beta, float eps) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float2 gr = g[i];
        float2 w = O[i];
        float mu = gr.x * gr.x + gr.y * gr.y;
        mu = beta * m[i] + (1.0f - beta) * mu;
        const float sq = lr / (sqrtf(mu) + eps);
        w.x -= gr.x * sq;
        w.y -= gr.y * sq;
        O[i] = w;
        m[i] = mu;
    }
}

int pmod_host(int a, int m) {
    const int r = a % m;
    return r < 0 ? r + m : r;
}

unsigned grid_for(size_t n, int threads) {
    const size_t b = (n + threads - 1) / threads;
    return (unsigned)std::min<size_t>(b, (size_t)kB200SMs * 16);
}

}  // namespace

std::vector<int> gen_fft_radices(int n) {
    std::vector<int> r;
    if (n < 2 || n > kMaxFftLen) return {};
    int m = n;
    while (m % 8 == 0) r.push_back(8), m /= 8;
    if (m % 4 == 0) r.push_back(4), m /= 4;
    if (m % 2 == 0) r.push_back(2), m /= 2;
    for (int q : {3, 5, 7})
        while (m % q == 0) r.push_back(q), m /= q;
    if (m != 1) return {};
    return r;
}

bool gen_fft_supported(int n) { return !gen_fft_radices(n).empty(); }

GenFft::~GenFft() { release(); }

void GenFft::release() {
    for (auto &kv : tw_) cudaFree(kv.second);
    tw_.clear();
}

cudaError_t GenFft::table(int n, const float2 **tw) {
    auto it = tw_.find(n);
    if (it == tw_.end()) {
        std::vector<float2> h(n);
        const double two_pi = 6.283185307179586476925286766559;
        for (int m = 0; m < n; ++m) {
            const double a = -two_pi * (double)m / n;
            h[m] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        float2 *d = nullptr;
        cudaError_t e = cudaMalloc(&d, (size_t)n * sizeof(float2));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), (size_t)n * sizeof(float2), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d);
            return e;
        }
        it = tw_.emplace(n, d).first;
    }
    *tw = it->second;
    return cudaSuccess;
}

// A register-resident plan for n: V in {16, 24, 20, 28} values per thread (the radices of
// each divide it: 8, 4, 2 and 3 for 24; 4, 2 and 5 for 20; 4, 2 and 7 for 28), at least 8
// and at most 512 threads per line.  False where none fits (odd parts 15, 21, ...): the
// shared-memory form then runs.
bool make_vplan(int n, VPlan &pl) {
    int a = 0, m = n;
    while (m % 2 == 0) m /= 2, ++a;
    int odd[3] = {0, 0, 0};
    const int primes[3] = {3, 5, 7};
    for (int i = 0; i < 3; ++i)
        while (m % primes[i] == 0) m /= primes[i], ++odd[i];
    if (m != 1) return false;
    int V = 0, pmax = 0, q = 0;
    if (odd[1] == 0 && odd[2] == 0) {
        V = odd[0] ? 24 : 16;
        pmax = 8;
        q = 3;
    } else if (odd[0] == 0 && odd[2] == 0) {
        V = 20, pmax = 4, q = 5;
    } else if (odd[0] == 0 && odd[1] == 0) {
        V = 28, pmax = 4, q = 7;
    } else {
        return false;
    }
    if (n % V != 0) return false;
    const int T = n / V;
    if (T < 8 || T > 512) return false;
    // the order of gen_fft_radices (powers of two first, the odd radix last), so that where
    // V holds radix 8 every butterfly computes what the shared-memory form computes
    std::vector<int> rad;
    const int nq = q == 3 ? odd[0] : q == 5 ? odd[1] : odd[2];
    while (a >= 3 && pmax >= 8) rad.push_back(8), a -= 3;
    while (a >= 2) rad.push_back(4), a -= 2;
    if (a == 1) rad.push_back(2);
    for (int i = 0; i < nq; ++i) rad.push_back(q);
    if ((int)rad.size() > 16) return false;
    pl.n = n;
    pl.V = V;
    pl.T = T;
    pl.nst = (int)rad.size();
    int prod = 1;
    for (int i = 0; i < pl.nst; ++i) {
        pl.radix[i] = rad[i];
        pl.pinv[i] = 1.0f / (float)prod;
        prod *= rad[i];
    }
    // lines per CTA: about 256 threads, within 96 KiB of shared memory
    pl.lpc = 1;
    while (pl.lpc < 16 && (pl.lpc * 2) * T <= 256 && (size_t)(pl.lpc * 2) * n * 8 <= 96 * 1024)
        pl.lpc *= 2;
    return prod == n;
}

cudaError_t GenFft::lines(const float2 *in, float2 *out, int n, long long count, size_t ld,
                          FftDir dir, cudaStream_t st) {
    if (!gen_fft_supported(n) || count < 1 || ld < (size_t)n) return cudaErrorInvalidValue;
    const float2 *tw = nullptr;
    cudaError_t e = table(n, &tw);
    if (e != cudaSuccess) return e;
    VPlan vp;
    if (knob("FPM_GEN_REG", 0, 0, 1) != 0 && make_vplan(n, vp)) {
        const long long vblocks = (count + vp.lpc - 1) / vp.lpc;
        if (vblocks > 0x7fffffffLL) return cudaErrorInvalidValue;
        const size_t vsmem = (size_t)vp.lpc * n * sizeof(float2);
        auto vgo = [&](auto kernel) {
            cudaError_t e2 = cudaFuncSetAttribute(
                kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsmem);
            if (e2 != cudaSuccess) return e2;
            kernel<<<(unsigned)vblocks, vp.T * vp.lpc, vsmem, st>>>(in, out, count, ld, vp, tw, 0);
            return cudaGetLastError();
        };
        const bool fwd = dir == kForward;
        switch (vp.V) {
            case 16: return fwd ? vgo(k_gen_lines_v<-1, 16, false>) : vgo(k_gen_lines_v<1, 16, false>);
            case 20: return fwd ? vgo(k_gen_lines_v<-1, 20, false>) : vgo(k_gen_lines_v<1, 20, false>);
            case 24: return fwd ? vgo(k_gen_lines_v<-1, 24, false>) : vgo(k_gen_lines_v<1, 24, false>);
            default: return fwd ? vgo(k_gen_lines_v<-1, 28, false>) : vgo(k_gen_lines_v<1, 28, false>);
        }
    }
    const GenPlan pl = make_plan(n);
    const long long blocks = (count + pl.lpc - 1) / pl.lpc;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const int threads = pl.T * pl.lpc;
    const size_t smem = (size_t)pl.lpc * n * sizeof(float2);
    auto go = [&](auto kernel) {
        cudaError_t e2 = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem);
        if (e2 != cudaSuccess) return e2;
        kernel<<<(unsigned)blocks, threads, smem, st>>>(in, out, count, ld, pl, tw);
        return cudaGetLastError();
    };
    if (dir == kForward)
        return pl.v == 8 ? go(k_gen_lines<-1, 8>) : pl.v == 16 ? go(k_gen_lines<-1, 16>)
                                                               : go(k_gen_lines<-1, 32>);
    return pl.v == 8 ? go(k_gen_lines<1, 8>) : pl.v == 16 ? go(k_gen_lines<1, 16>)
                                                          : go(k_gen_lines<1, 32>);
}

cudaError_t launch_transpose_pages(const float2 *in, float2 *out, int n, int count,
                                   cudaStream_t st) {
    if (n < 1 || count < 1 || count > 65535) return cudaErrorInvalidValue;
    const dim3 grid((n + 31) / 32, (n + 31) / 32, count);
    k_transpose_pages<<<grid, 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

// The register-resident transform of `lines` lines of n x n pages, written transposed (see
// k_gen_lines_v): whole pages (g_lo = 0, lines a multiple of n) or the columns
// [g_lo, g_lo + lines) mod n of one page; cudaErrorNotSupported where its plan does not
// allow it.
cudaError_t GenFft::lines_t(const float2 *in, float2 *out, int n, int g_lo, long long lines,
                            FftDir dir, cudaStream_t st) {
    VPlan vp;
    if (knob("FPM_GEN_REG", 0, 0, 1) == 0 || !make_vplan(n, vp) || n % vp.lpc != 0)
        return cudaErrorNotSupported;
    const size_t smem = (size_t)n * (vp.lpc + 1) * sizeof(float2);
    if (smem > 110 * 1024) return cudaErrorNotSupported;   // two CTAs per SM
    if (lines < 1 || (g_lo != 0 && lines > n) || (g_lo == 0 && lines % n != 0 && lines > n))
        return cudaErrorInvalidValue;
    const long long blocks = (lines + vp.lpc - 1) / vp.lpc;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const float2 *tw = nullptr;
    cudaError_t e = table(n, &tw);
    if (e != cudaSuccess) return e;
    auto go = [&](auto kernel) {
        cudaError_t e2 = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem);
        if (e2 != cudaSuccess) return e2;
        kernel<<<(unsigned)blocks, vp.T * vp.lpc, smem, st>>>(in, out, lines, (size_t)n, vp, tw,
                                                              g_lo);
        return cudaGetLastError();
    };
    const bool fwd = dir == kForward;
    switch (vp.V) {
        case 16: return fwd ? go(k_gen_lines_v<-1, 16, true>) : go(k_gen_lines_v<1, 16, true>);
        case 20: return fwd ? go(k_gen_lines_v<-1, 20, true>) : go(k_gen_lines_v<1, 20, true>);
        case 24: return fwd ? go(k_gen_lines_v<-1, 24, true>) : go(k_gen_lines_v<1, 24, true>);
        default: return fwd ? go(k_gen_lines_v<-1, 28, true>) : go(k_gen_lines_v<1, 28, true>);
    }
}

cudaError_t GenFft::fft2(const float2 *in, float2 *out, float2 *tmp, int n, int count, FftDir dir,
                         cudaStream_t st) {
    const size_t plane = (size_t)n * n;
    if (count >= 1 && gen_fft_supported(n)) {
        // two passes, each writing its pages transposed: along r into tmp, along c back
        const long long lines = (long long)count * n;
        cudaError_t e = lines_t(in, tmp, n, 0, lines, dir, st);
        if (e == cudaSuccess) return lines_t(tmp, out, n, 0, lines, dir, st);
        if (e != cudaErrorNotSupported) return e;
    }
    // transform along r (contiguous), transpose, along c (now contiguous), transpose back;
    // count pages at a time, at most 65535 per transpose launch
    cudaError_t e = lines(in, out, n, (long long)count * n, n, dir, st);
    for (int p0 = 0; e == cudaSuccess && p0 < count; p0 += 65535) {
        const int pc = std::min(65535, count - p0);
        e = launch_transpose_pages(out + p0 * plane, tmp + p0 * plane, n, pc, st);
    }
    if (e == cudaSuccess) e = lines(tmp, tmp, n, (long long)count * n, n, dir, st);
    for (int p0 = 0; e == cudaSuccess && p0 < count; p0 += 65535) {
        const int pc = std::min(65535, count - p0);
        e = launch_transpose_pages(tmp + p0 * plane, out + p0 * plane, n, pc, st);
    }
    return e;
}

cudaError_t GenFft::fft2_box(const float2 *in, float2 *out, float2 *tmp, int n, FftDir dir,
                             int c_lo, int c_cnt, int r_lo, int r_cnt, cudaStream_t st) {
    if (c_cnt < 1 || c_cnt > n || r_cnt < 1 || r_cnt > n || (c_cnt < n && (in != out || r_cnt < n)))
        return cudaErrorInvalidValue;
    // lines [lo, lo + cnt) mod n of a page: one or two contiguous runs
    auto run = [&](const float2 *src, float2 *dst, int lo, int cnt) {
        lo = ((lo % n) + n) % n;
        const int first = std::min(cnt, n - lo);
        cudaError_t e = lines(src + (size_t)lo * n, dst + (size_t)lo * n, n, first, n, dir, st);
        if (e == cudaSuccess && cnt > first) e = lines(src, dst, n, cnt - first, n, dir, st);
        return e;
    };
    cudaError_t e = run(in, out, c_lo, c_cnt);                      // along r, box columns
    if (r_cnt == n) {
        if (e == cudaSuccess && c_cnt < n) {   // only the box columns are read
            const int lo = ((c_lo % n) + n) % n;
            const dim3 grid((n + 31) / 32, (n + 31) / 32);
            k_transpose_page_cols<<<grid, 256, 0, st>>>(out, tmp, n, lo, c_cnt);
            e = cudaGetLastError();
        } else if (e == cudaSuccess) {
            e = launch_transpose_pages(out, tmp, n, 1, st);
        }
        if (e == cudaSuccess) e = run(tmp, tmp, r_lo, r_cnt);      // along c, every row
        if (e == cudaSuccess) e = launch_transpose_pages(tmp, out, n, 1, st);
        return e;
    }
    // only the box rows go through the transform along c: they alone are turned into
    // contiguous lines and back; the other rows of out keep the first pass's values
    const int lo = ((r_lo % n) + n) % n;
    const dim3 grid((n + 31) / 32, (r_cnt + 31) / 32);
    if (e == cudaSuccess) {
        k_transpose_rows<true><<<grid, 256, 0, st>>>(out, tmp, n, lo, r_cnt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = lines(tmp, tmp, n, r_cnt, n, dir, st);   // along c, box rows
    if (e == cudaSuccess) {
        k_transpose_rows<false><<<grid, 256, 0, st>>>(tmp, out, n, lo, r_cnt);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_gen_crop_pupil(const float2 *S, int H, const float2 *P, int h, const int2 *led,
                                  int z_off, int nb, float2 *out, cudaStream_t st) {
    if (nb < 1 || nb > 65535) return cudaErrorInvalidValue;
    const size_t plane = (size_t)h * h;
    const unsigned bx = (unsigned)std::min<size_t>((plane + 255) / 256, 1024);
    k_gen_crop_pupil<<<dim3(bx, nb), 256, 0, st>>>(S, H, P, h, led, z_off, out);
    return cudaGetLastError();
}

cudaError_t launch_gen_stitch(const float2 *X, int h, const float2 *P, const int2 *led, int z_off,
                              int nb, int H, int rlo, int rspan, int clo, int cspan, float2 *G,
                              cudaStream_t st) {
    if (nb < 1 || nb > 1024 || rspan < 1 || cspan < 1) return cudaErrorInvalidValue;
    const size_t n = (size_t)rspan * cspan;
    const float inv_h2 = 1.0f / (float)((unsigned)H * (unsigned)H);
    k_gen_stitch<<<grid_for(n, 256), 256, nb * sizeof(int2), st>>>(
        X, h, P, led, z_off, nb, H, pmod_host(rlo, H), rspan, pmod_host(clo, H), cspan, inv_h2, G);
    return cudaGetLastError();
}

cudaError_t launch_gen_pupil_grad(const float2 *S, int H, const float2 *X, int h, const int2 *led,
                                  int z_off, int nb, float2 *dP, cudaStream_t st) {
    if (nb < 1 || nb > 1024) return cudaErrorInvalidValue;
    const size_t plane = (size_t)h * h;
    k_gen_pupil_grad<<<grid_for(plane, 256), 256, nb * sizeof(int2), st>>>(S, H, X, h, led, z_off,
                                                                          nb, dP);
    return cudaGetLastError();
}

cudaError_t launch_rmsprop_object(float2 *O, float *m, const float2 *g, size_t n, float lr,
                                  float beta, float eps, cudaStream_t st) {
    k_rmsprop_object<<<grid_for(n, 256), 256, 0, st>>>(O, m, g, n, lr, beta, eps);
    return cudaGetLastError();
}

}  // namespace fpm

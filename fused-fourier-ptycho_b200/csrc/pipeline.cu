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
//                Kahan; kernels.cuh:95-116 as a gather), IFFT along the row -> Ur
//                (row-major; a tiled transpose makes it U, column-major)
//  B cols        per column: IFFT along r of U (zero outside the box rows) -> object
//                gradient; RMSprop of O and m (kernels.cuh:364-382); FFT along r of the
//                updated column, kept only on the next batch's box rows -> V
//  C rows_fwd    per next-box row (V transposed to Vr first): FFT along the row,
//                kept on the next box columns -> Sboxr, transposed into the next Sbox
//
// Only the box rows / columns of the gradient spectrum are non-zero and only the
// next box is read, so passes A and C touch rspan lines instead of H, and U, V
// hold H x rspan values instead of H x H.  Lines are transformed in shared memory
// by fft::line_fft (one CTA per line of 16384, several lines per CTA below).
#include "common.cuh"
#include "engine.h"
#include "fft_core.cuh"
#include "pipeline.h"
#include "stencil.cuh"
#include "tuning.h"

#include <algorithm>
#include "tma.cuh"

#include <cudaTypedefs.h>
#include <cstdlib>

namespace fpm {

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
    return fft::LG<N>::SMEM;
}

template <class K>
cudaError_t set_smem(K kernel, int bytes) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
}

template <int TYPE>
__device__ __forceinline__ float amplitude(const StackView &Y, size_t idx, float mn, float range) {
    if (TYPE == kStackF32) return static_cast<const float *>(Y.ptr)[idx];
    if (Y.lut) return Y.lut[static_cast<const uint16_t *>(Y.ptr)[idx]];
    const float x = (float)static_cast<const uint16_t *>(Y.ptr)[idx] - mn;
    return range > 0.f ? sqrtf(x / range) : sqrtf(x);
}

// Shared set-up of every pass kernel: twiddles into shared memory.
template <int N, int E = 16>
__device__ __forceinline__ void setup(float2 *smem, const float2 *thi, const float2 *tlo) {
    using G = fft::LG<N, E>;
    float2 *s_hi = G::tw_hi(smem);
    fft::load_twiddles(s_hi, s_hi + 128, thi, tlo, G::NHI, G::NLO);
    __syncthreads();
}

// E values per thread: 16, or 32 for N = 16384 (radix-32 stages, one exchange fewer)
template <int N, int DIR, int E>
__device__ __forceinline__ void line_fft_e(float2 (&v)[E], float2 *s, const float2 *hi,
                                           const float2 *lo, int t) {
    if constexpr (E == 32) {
        fft::line_fft_regs32<N, DIR>(v, s, hi, lo, t);
    } else {
        fft::line_fft_regs<N, DIR>(v, s, hi, lo, t);
    }
}

// ---------------------------------------------------------------------------
// L1: crop x pupil, ifftshift, inverse FFT along r (contiguous column lines)
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(fft::LG<N>::THREADS, fft::LG<N>::MINB)
    k_lr_cols_inv(const float2 *__restrict__ Sbox, const float2 *__restrict__ P,
                  const int2 *__restrict__ led, BatchGeom g, int l0, int nl,
                  float2 *__restrict__ T1, const float2 *__restrict__ thi,
                  const float2 *__restrict__ tlo) {
    using G = fft::LG<N>;
    extern __shared__ float2 smem[];
    setup<N>(smem, thi, tlo);
    const int ln = G::cline(), t = G::ct();
    const long long gl = (long long)blockIdx.x * G::LPC + ln;
    const bool live = gl < (long long)nl * N;
    constexpr int hh = N / 2;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = make_float2(0.f, 0.f);
    bool nz = false;   // the crop column meets the pupil support
    if (live) {
        const int lloc = (int)(gl / N);
        const int cq = (int)(gl % N);
        const int c = cq + hh >= N ? cq + hh - N : cq + hh;
        nz = c >= g.pc_lo && c < g.pc_hi;
        if (nz) {
            const int2 ab = led_box_offset(led, l0 + lloc, g);
            const float2 *scol = Sbox + (size_t)box_index(ab.y, c, g.H) * g.rspan;
            const float2 *pcol = P + (size_t)c * N;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int e = t + m * G::T;
                const int r = e + hh >= N ? e + hh - N : e + hh;
                if (r >= g.pr_lo && r < g.pr_hi)   // the box holds only the support rows
                    v[m] = cmul(scol[box_index(ab.x, r, g.H)], pcol[r]);
            }
        }
    }
    // columns outside the support transform zeros: a CTA holding only such lines skips
    // the transform and writes the zeros (none when the buffer already holds them)
    if (__syncthreads_or(nz))
        fft::line_fft_regs<N, +1>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128, t);
    if (live && (nz || !g.t1_clean)) {
        float2 *dst = T1 + (size_t)gl * N;
#pragma unroll
        for (int m = 0; m < 16; ++m) dst[t + m * G::T] = v[m];
    }
}

// ---------------------------------------------------------------------------
// L2: inverse FFT along c (strided row lines) -> z (in place) and the residual
// ---------------------------------------------------------------------------
template <int N, int TYPE>
__global__ void __launch_bounds__(fft::LG<N>::THREADS, fft::LG<N>::MINB)
    k_lr_rows_inv(StackView Y, BatchGeom g, int l0, int nl, float2 *__restrict__ T1,
                  float *__restrict__ Rs, const float2 *__restrict__ thi,
                  const float2 *__restrict__ tlo) {
    using G = fft::LG<N>;
    extern __shared__ float2 smem[];
    setup<N>(smem, thi, tlo);
    const int ln = G::iline(), t = G::it();
    const long long gl = (long long)blockIdx.x * G::LPC + ln;
    const bool live = gl < (long long)nl * N;
    const int lloc = live ? (int)(gl / N) : 0;
    const int r = live ? (int)(gl % N) : 0;
    float2 *page = T1 + (size_t)lloc * N * N + r;   // element c at page[c * N]
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m)
        v[m] = live ? page[(size_t)(t + m * G::T) * N] : make_float2(0.f, 0.f);
    fft::line_fft_regs<N, +1>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128, t);
    if (!live) return;
    float mn = 0.f, range = 0.f;
    if (TYPE == kStackU16) {
        mn = (float)Y.minmax[0];
        range = (float)(Y.minmax[1] - Y.minmax[0]);
    }
    // 1 / (h^2 p^2): a power of two, so the product equals the quotient exactly
    const float inv_ratio = (float)(1.0 / ((double)N * N * g.pratio * g.pratio));
    const size_t ypage = (size_t)(g.z_off + l0 + lloc) * N * N + r;
    float *rs = Rs + (size_t)lloc * N * N + r;
    float y[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) y[m] = amplitude<TYPE>(Y, ypage + (size_t)(t + m * G::T) * N, mn, range);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const size_t off = (size_t)(t + m * G::T) * N;
        const float2 z = v[m];
        page[off] = z;
        rs[off] = sqrtf(z.x * z.x + z.y * z.y) * inv_ratio - y[m];
    }
}

// ---------------------------------------------------------------------------
// L3: sign stencil of the residual, phase, forward FFT along c (strided rows)
// ---------------------------------------------------------------------------
template <int N, int LOSS>
__global__ void __launch_bounds__(fft::LG<N>::THREADS, fft::LG<N>::MINB)
    k_lr_rows_fwd(BatchGeom g, int nl, float2 *__restrict__ T1, const float *__restrict__ Rs,
                  double *__restrict__ parts, const float2 *__restrict__ thi,
                  const float2 *__restrict__ tlo) {
    using G = fft::LG<N>;
    extern __shared__ float2 smem[];
    __shared__ double s_red[32];
    setup<N>(smem, thi, tlo);
    const int ln = G::iline(), t = G::it();
    const long long gl = (long long)blockIdx.x * G::LPC + ln;
    const bool live = gl < (long long)nl * N;
    const int lloc = live ? (int)(gl / N) : 0;
    const int r = live ? (int)(gl % N) : 0;
    const float gscale = (float)(g.pratio * g.pratio);
    const float *rp = Rs + (size_t)lloc * N * N;
    float2 *page = T1 + (size_t)lloc * N * N + r;
    const int rpp = r + 1 == N ? 0 : r + 1, rmm = r == 0 ? N - 1 : r - 1;
    double lsum = 0.0;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int c = t + m * G::T;
        float2 o = make_float2(0.f, 0.f);
        if (live) {
            const int cp = c + 1 == N ? 0 : c + 1, cm = c == 0 ? N - 1 : c - 1;
            const float d =
                stencil<LOSS>(rp[(size_t)c * N + r], rp[(size_t)cp * N + r], rp[(size_t)cm * N + r],
                              rp[(size_t)c * N + rpp], rp[(size_t)c * N + rmm],
                              LOSS == kLossAnisotropic ? 0.f : rp[(size_t)cm * N + rpp],
                              LOSS == kLossAnisotropic ? 0.f : rp[(size_t)cp * N + rmm], lsum) *
                gscale;
            const float2 z = page[(size_t)c * N];
            const float mag = sqrtf(z.x * z.x + z.y * z.y);
            if (mag > 0.f) {
                const float inv = 1.0f / mag;
                o.x = z.x * inv * d;
                o.y = z.y * inv * d;
            }
        }
        v[m] = o;
    }
    // fixed-order block reduction of the loss partial
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < G::THREADS / 32; ++w) tot += s_red[w];
        parts[blockIdx.x] = tot;
    }
    fft::line_fft_regs<N, -1>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128, t);
    if (live) {
#pragma unroll
        for (int m = 0; m < 16; ++m) page[(size_t)(t + m * G::T) * N] = v[m];
    }
}

// ---------------------------------------------------------------------------
// L2 + L3 fused.  A cluster of CL CTAs takes CL LIN consecutive row lines of one LED
// (LIN per CTA): every line gets its inverse FFT and its residual |z|/(h^2 p^2) - Y in
// shared memory; the CTAs read their neighbours' boundary residual rows through
// distributed shared memory, and the CL LIN - 2 central lines get the loss stencil, the
// phase and the forward FFT.  The two outer lines are halo: their inverse FFTs are
// recomputed by the neighbouring clusters.  The output goes to a second buffer because
// neighbours still read the halo rows of the input.
//
// Cluster p holds rows p POUT + q (q < CL LIN, taken modulo h); its central lines are
// q in [1, POUT] with p POUT + q <= h, so row 0 is central once (as row h, in the last
// cluster of the LED) and the first row of every CTA, p POUT + j LIN, is even (the
// 16-byte rule of the TMA row coordinate).
//
// The row lines are strided in memory (element c of row r at c h + r): the TMA unit
// copies the CTA's LIN rows x all columns into shared memory (boxes of LIN x 256) and
// the LIN amplitude rows (FP32, a row-major copy of the stack made once per solve) come
// by bulk copy.  Lines past row h - 1 (the last cluster of an LED) read their field
// from global memory.  The residual rows take the exchange area once the inverse FFTs
// are done, so a CTA holds one field tile, the amplitude rows and the twiddles: about
// 100 KB at 512 threads from h = 1024 (two CTAs per SM), 200 KB at 1024 threads below.
// ---------------------------------------------------------------------------
template <int N, int CL>
struct L23 {
    static constexpr int THREADS = N >= 1024 ? 512 : 1024;
    static constexpr int MINB = THREADS == 512 ? 2 : 1;
    static constexpr int T = N / 16;
    static constexpr int LIN = THREADS / T;           // lines per CTA
    static constexpr int POUT = CL * LIN - 2;         // central lines per cluster
    static constexpr int PAD = 16 / LIN > 0 ? 16 / LIN : 1;
    static constexpr int STRIDE = N + PAD;            // FFT exchange line stride (float2)
    // residual and amplitude row strides (float): the (line, t) pairs of a warp on
    // distinct banks where the 16-byte bulk-copy rule allows (LIN <= 8)
    static constexpr int RSTRIDE = N + (LIN >= 32 ? 1 : 32 / LIN);
    static constexpr int ASTRIDE = N + (LIN <= 8 ? 32 / LIN : 4);
    static constexpr int LINE_BYTES = LIN * STRIDE * 8;
    static constexpr int AMP_BYTES = LIN * ASTRIDE * 4;
    static constexpr int CB = N < 256 ? N : 256;      // TMA box width along c
    static constexpr int SMEM = LINE_BYTES + AMP_BYTES + 2 * 128 * 8 + 16;
    static constexpr int PAIRS_PER_LED = (N + POUT - 1) / POUT;   // clusters per LED
    static constexpr int CTAS_PER_LED = CL * PAIRS_PER_LED;
    static constexpr int NHI = N >= 128 ? N / 128 : 1;
    static constexpr int NLO = N >= 128 ? 128 : N;
    static_assert(LIN >= 4 && LIN % 2 == 0 && LIN <= 256, "TMA box rows");
    static_assert(POUT % 2 == 0, "even cluster stride keeps the TMA row start even");
    static_assert(LIN * N * 8 <= LINE_BYTES, "field tile fits the exchange area");
    static_assert((LIN + 2) * RSTRIDE * 4 <= LINE_BYTES, "residual rows fit the exchange area");
    static_assert(LINE_BYTES % 16 == 0 && (ASTRIDE * 4) % 16 == 0, "bulk-copy alignment");
    static_assert(MINB * (SMEM + 1024) <= 228 * 1024, "shared memory per SM");
};

__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
// An arrive that publishes no writes: it only tells the cluster that this CTA's loads of
// the other CTAs' shared memory are finished, and those loads have returned (their values
// are stored in this CTA's own shared memory before a block barrier) when it runs.
__device__ __forceinline__ void cluster_arrive_reads_done() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// value at the same shared-memory location of CTA `rank` of this cluster
__device__ __forceinline__ float cluster_load(const float *p, unsigned rank) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(remote)
                 : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))), "r"(rank));
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(remote) : "memory");
    return v;
}

template <int N, int LOSS, int CL>
__global__ void __launch_bounds__(L23<N, CL>::THREADS, L23<N, CL>::MINB)
    k_lr_rows_fused(const float *__restrict__ amp, BatchGeom g, int l0,
                    const float2 *__restrict__ T1, float2 *__restrict__ T2,
                    double *__restrict__ parts, int *__restrict__ flag,
                    const __grid_constant__ CUtensorMap tm_field, const float2 *__restrict__ thi,
                    const float2 *__restrict__ tlo) {
    using F = L23<N, CL>;
    constexpr int T = F::T, LIN = F::LIN;
    extern __shared__ __align__(128) float2 smem[];
    __shared__ double s_red[32];
    float *ampt = reinterpret_cast<float *>(smem + LIN * F::STRIDE);     // [k][ASTRIDE]
    float2 *s_hi = reinterpret_cast<float2 *>(ampt + LIN * F::ASTRIDE);
    uint64_t *bar = reinterpret_cast<uint64_t *>(s_hi + 256);          // [0] field, [1] rows
    const float2 *tile = smem;                                          // [c][LIN] field tile
    float *res = reinterpret_cast<float *>(smem);   // after the inverse FFTs: row 0 ghost above
    const int k = threadIdx.x % LIN, t = threadIdx.x / LIN;
    const unsigned j = blockIdx.x % CL;                 // rank in the cluster
    const int pair = blockIdx.x / CL;
    const int lloc = pair / F::PAIRS_PER_LED;
    const int x0 = (pair % F::PAIRS_PER_LED) * F::POUT + (int)j * LIN;   // first row (even)
    const int zpage = g.z_off + l0 + lloc;
    // boxes of CB stored columns holding a supported crop column; with a field buffer
    // whose other columns are known zeros (t1_clean) only those are copied
    unsigned boxes = 0;
    if (x0 < N) {
#pragma unroll
        for (int q = 0; q < N / F::CB; ++q) {
            const int lo = (q * F::CB + N / 2) % N, hi = lo + F::CB;   // crop columns of box q
            const bool sup = hi <= N ? (lo < g.pc_hi && hi > g.pc_lo)
                                     : (lo < g.pc_hi || hi - N > g.pc_lo);
            if (sup || !g.t1_clean) boxes |= 1u << q;
        }
    }
    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
        tma::arrive_expect_tx(&bar[0], (uint32_t)__popc(boxes) * LIN * F::CB * 8);
#pragma unroll 1
        for (int q = 0; q < N / F::CB; ++q)
            if (boxes >> q & 1u)
                tma::load_3d(smem + q * F::CB * LIN, &tm_field, x0, q * F::CB, lloc, &bar[0]);
        tma::arrive_expect_tx(&bar[1], (uint32_t)LIN * N * 4);
    }
    fft::load_twiddles(s_hi, s_hi + 128, thi, tlo, F::NHI, F::NLO);
    __syncthreads();                                    // barriers initialised before any use
    if (threadIdx.x >> 5 == 1) {                        // warp 1: the amplitude rows
        for (int kk = threadIdx.x & 31; kk < LIN; kk += 32) {
            const int rr = (x0 + kk) & (N - 1);
            tma::load_1d(ampt + kk * F::ASTRIDE, amp + ((size_t)zpage * N + rr) * N, N * 4,
                         &bar[1]);
        }
    }
    const int rraw = x0 + k;                            // row before the wrap
    const bool wrapped = rraw >= N;
    const int r = rraw & (N - 1);
    const int q = (int)j * LIN + k;                     // line within the cluster
    const bool central = q >= 1 && q <= F::POUT && rraw <= N;
    float *rk = res + (k + 1) * F::RSTRIDE;
    float2 v[16];
    if (wrapped) {   // past the last row: the field from global memory
        const float2 *page = T1 + (size_t)lloc * N * N + r;
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = page[(size_t)(t + m * T) * N];
    }
    // A copy that never completes is flagged for the host; the CTA then skips its work
    // but still passes every cluster barrier, so its partners never wait for ever.
    bool failed = __syncthreads_or(!tma::mbar_wait(&bar[0], 0));
    if (failed && threadIdx.x == 0) {
        atomicExch(flag, 1);
        tma::mbar_wait(&bar[0], 0);
    }
    if (!failed) {
        if (!wrapped) {
#pragma unroll
            for (int m = 0; m < 16; ++m)
                v[m] = boxes >> ((t + m * T) / F::CB) & 1u ? tile[(t + m * T) * LIN + k]
                                                          : make_float2(0.f, 0.f);
        }
        __syncthreads();                                // the tile area becomes FFT scratch
        fft::line_fft_regs<N, +1>(v, smem + k * F::STRIDE, s_hi, s_hi + 128, t);
    }
    // every read of the exchange area done (the residuals take it) and the rows in
    const bool failed_rows = __syncthreads_or(!tma::mbar_wait(&bar[1], 0));
    if (failed_rows && threadIdx.x == 0) {
        atomicExch(flag, 1);
        tma::mbar_wait(&bar[1], 0);
    }
    failed = failed || failed_rows;
    if (!failed) {
        // 1 / (h^2 p^2): a power of two, so the product equals the quotient exactly
        const float inv_ratio = (float)(1.0 / ((double)N * N * g.pratio * g.pratio));
        const float *ak = ampt + k * F::ASTRIDE;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const float2 z = v[m];
            const float mag = sqrtf(z.x * z.x + z.y * z.y);
            rk[t + m * T] = mag * inv_ratio - ak[t + m * T];
            // z / |z| for the phase of the gradient (zero where |z| is): the stencil step
            // multiplies it by d, in the order (z.x / |z|) d
            if (mag > 0.f) {
                const float inv = 1.0f / mag;
                v[m] = make_float2(z.x * inv, z.y * inv);
            } else {
                v[m] = make_float2(0.f, 0.f);
            }
        }
    }
    // residual rows of every CTA written: take the neighbours' boundary rows as ghosts
    cluster_arrive();
    cluster_wait();
    if (!failed) {
        // ghost above: the last line of rank j-1; ghost below: the first line of rank j+1
        for (int c = threadIdx.x; c < N; c += F::THREADS) {
            if (j > 0) res[c] = cluster_load(res + LIN * F::RSTRIDE + c, j - 1);
            if (j + 1 < CL) res[(LIN + 1) * F::RSTRIDE + c] = cluster_load(res + F::RSTRIDE + c, j + 1);
        }
        __syncthreads();
    }
    cluster_arrive_reads_done();   // done with the neighbours' memory; waited for before the area is reused
    double lsum = 0.0;
    if (!failed) {
        const float gscale = (float)(g.pratio * g.pratio);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int c = t + m * T;
            float2 o = make_float2(0.f, 0.f);
            if (central) {
                const int cp = c + 1 == N ? 0 : c + 1, cm = c == 0 ? N - 1 : c - 1;
                const float d =
                    stencil<LOSS>(rk[c], rk[cp], rk[cm], rk[F::RSTRIDE + c], rk[c - F::RSTRIDE],
                                  LOSS == kLossAnisotropic ? 0.f : rk[F::RSTRIDE + cm],
                                  LOSS == kLossAnisotropic ? 0.f : rk[cp - F::RSTRIDE], lsum) *
                    gscale;
                const float2 u = v[m];   // z / |z|, or zero
                if (u.x != 0.f || u.y != 0.f) {
                    o.x = u.x * d;
                    o.y = u.y * d;
                }
            }
            v[m] = o;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < F::THREADS / 32; ++w) tot += s_red[w];
        parts[blockIdx.x] = failed ? 0.0 : tot;
    }
    cluster_wait();     // the neighbours are done with this CTA's residual rows
    if (!failed) {
        fft::line_fft_regs<N, -1>(v, smem + k * F::STRIDE, s_hi, s_hi + 128, t);
        if (central) {   // only the columns the next pass transforms (pupil support, fftshifted)
            float2 *dst = T2 + (size_t)lloc * N * N + r;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int cf = t + m * T;
                const int c = cf + N / 2 >= N ? cf - N / 2 : cf + N / 2;
                if (c >= g.pc_lo && c < g.pc_hi) dst[(size_t)cf * N] = v[m];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// L4: forward FFT along r (column lines, interleaved so the row-major store of
// the fftshift'ed Xs writes LPC consecutive columns per row)
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(fft::LG<N>::THREADS, fft::LG<N>::MINB)
    k_lr_cols_fwd(BatchGeom g, int l0, int nl, const float2 *__restrict__ T1, float2 *__restrict__ Xs,
                  const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = fft::LG<N>;
    extern __shared__ float2 smem[];
    setup<N>(smem, thi, tlo);
    const int ln = G::iline(), t = G::it();
    const long long gl = (long long)blockIdx.x * G::LPC + ln;
    const bool live = gl < (long long)nl * N;
    constexpr int hh = N / 2;
    const int cf = live ? (int)(gl % N) : 0;
    const int c = cf + hh >= N ? cf + hh - N : cf + hh;
    // only gradient-spectrum columns inside the pupil support are ever read
    const bool need = live && c >= g.pc_lo && c < g.pc_hi;
    if (!__syncthreads_or(need)) return;
    const float2 *src = T1 + (size_t)(need ? gl : 0) * N;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = need ? src[t + m * G::T] : make_float2(0.f, 0.f);
    fft::line_fft_regs<N, -1>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128, t);
    if (!need) return;
    const int lloc = (int)(gl / N);
    float2 *xs = Xs + (size_t)(l0 + lloc) * N * N + c;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int e = t + m * G::T;                  // frequency row of X
        const int r = e + hh >= N ? e + hh - N : e + hh;
        xs[(size_t)r * N] = v[m];
    }
}

// L4 persistent (h of 2048): a CTA walks groups of LPC consecutive columns (skipping
// groups with no supported column); the next group's columns are copied into the
// exchange area while this group's last FFT stage runs.  Two CTAs per SM.
template <int N>
__global__ void __launch_bounds__(fft::LG<N>::THREADS, fft::LG<N>::MINB)
    k_lr_cols_fwd_async(BatchGeom g, int l0, int nl, const float2 *__restrict__ T1,
                        float2 *__restrict__ Xs, int *__restrict__ err,
                        const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = fft::LG<N>;
    static_assert(G::LPC > 1 && (G::STRIDE * 8) % 16 == 0, "16-byte aligned line starts");
    extern __shared__ __align__(128) float2 smem[];
    constexpr int hh = N / 2;
    const int ngroups = nl * N / G::LPC;
    uint64_t *bar = reinterpret_cast<uint64_t *>(G::tw_hi(smem) + 256);
    // first group at or after q holding a supported column (block-uniform)
    auto next_group = [&](int q) {
        for (; q < ngroups; q += gridDim.x) {
            const int cf0 = (int)(((long long)q * G::LPC) % N);
            for (int k = 0; k < G::LPC; ++k) {
                const int cf = cf0 + k;
                const int c = cf + hh >= N ? cf + hh - N : cf + hh;
                if (c >= g.pc_lo && c < g.pc_hi) return q;
            }
        }
        return ngroups;
    };
    auto fetch = [&](int q) {   // one thread: the LPC columns of group q into the lines
        tma::arrive_expect_tx(bar, G::LPC * N * 8);
        for (int k = 0; k < G::LPC; ++k)
            tma::load_1d(smem + k * G::STRIDE, T1 + ((size_t)q * G::LPC + k) * N, N * 8, bar);
    };
    const int ln = G::iline(), t = G::it();
    int q = next_group(blockIdx.x);
    if (threadIdx.x == 0) {
        tma::mbar_init(bar, 1);
        tma::fence_barrier_init();
        if (q < ngroups) fetch(q);
    }
    fft::load_twiddles(G::tw_hi(smem), G::tw_hi(smem) + 128, thi, tlo, G::NHI, G::NLO);
    __syncthreads();
    uint32_t parity = 0;
    bool pending = q < ngroups, failed = false;
    while (q < ngroups) {
        failed = __syncthreads_or(!tma::mbar_wait(bar, parity));
        if (failed) break;
        pending = false;
        parity ^= 1u;
        const long long gl = (long long)q * G::LPC + ln;
        const int cf = (int)(gl % N);
        const int c = cf + hh >= N ? cf + hh - N : cf + hh;
        const bool need = c >= g.pc_lo && c < g.pc_hi;
        float2 v[16];
        const float2 *line = smem + ln * G::STRIDE;
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = need ? line[t + m * G::T] : make_float2(0.f, 0.f);
        __syncthreads();                                // every read before the first exchange
        const int qn = next_group(q + gridDim.x);
        fft::line_fft_regs<N, -1>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128,
                                  t, [&] {
                                      if (threadIdx.x == 0 && qn < ngroups) {
                                          tma::fence_proxy_async();
                                          fetch(qn);
                                      }
                                  });
        pending = qn < ngroups;
        if (need) {
            const int lloc = (int)(gl / N);
            float2 *xs = Xs + (size_t)(l0 + lloc) * N * N + c;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int e = t + m * G::T;             // frequency row of X
                const int r = e + hh >= N ? e + hh - N : e + hh;
                xs[(size_t)r * N] = v[m];
            }
        }
        q = qn;
    }
    if (failed && threadIdx.x == 0) {
        atomicExch(err, 1);
        if (pending) tma::mbar_wait(bar, parity);      // bounded drain of the copies in flight
    }
}

// ---------------------------------------------------------------------------
// pupil gradient: 32 x 32 tiles, LED loop inside, Kahan accumulation
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_lr_pupil_grad(const float2 *__restrict__ Sbox,
                                                        const float2 *__restrict__ Xs,
                                                        const int2 *__restrict__ led, BatchGeom g,
                                                        float2 *__restrict__ dP,
                                                        const unsigned *__restrict__ pie) {
    __shared__ float2 sA[32][33];   // sub: [c][r]
    __shared__ float2 sB[32][33];   // Xs:  [r][c]
    const int h = g.h;
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    KahanC acc[4];
    // outside the pupil support the gradient is never used (the amplitude clamp keeps
    // the pupil at zero there): tiles beyond it only write zeros
    const bool any = r0 < g.pr_hi && r0 + 32 > g.pr_lo && c0 < g.pc_hi && c0 + 32 > g.pc_lo;
    // LED l's tile values into registers; LED l + 1's loads are in flight while LED l's
    // products are summed
    float2 na[4], nx[4];
    auto load = [&](int l) {
        const int2 ab = led_box_offset(led, l, g);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int cl = ty + 8 * k;
            const int r = r0 + tx, c = c0 + cl;       // sub: coalesced along r
            const bool a_in = r >= g.pr_lo && r < g.pr_hi && c >= g.pc_lo && c < g.pc_hi;
            na[k] = a_in ? Sbox[(size_t)box_index(ab.y, c, g.H) * g.rspan + box_index(ab.x, r, g.H)]
                         : make_float2(0.f, 0.f);
            const int rr = r0 + cl, cc = c0 + tx;     // Xs: coalesced along c
            const bool b_in = rr >= g.pr_lo && rr < g.pr_hi && cc >= g.pc_lo && cc < g.pc_hi;
            nx[k] = b_in ? Xs[((size_t)l * h + rr) * h + cc] : make_float2(0.f, 0.f);
        }
    };
    if (any && g.nb > 0) load(0);
    for (int l = 0; any && l < g.nb; ++l) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            sA[ty + 8 * k][tx] = na[k];
            sB[ty + 8 * k][tx] = nx[k];
        }
        __syncthreads();
        if (l + 1 < g.nb) load(l + 1);
        // ePIE: the LED's term over max|sub_l|^2 of its whole crop
        const float emax = g.pie == 1 ? __uint_as_float(pie[1 + l]) : 1.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int cl = ty + 8 * k;
            const float2 a = sA[cl][tx];
            float2 term = cmul_conj(sB[tx][cl], a);
            if (g.pie != 0) {   // deconv_pie (fpm_forward_GPU.m:64-76): conj(sub) X ./ weight
                const float den = g.pie == 1 ? emax : a.x * a.x + a.y * a.y + 1e-5f;
                term = make_float2(term.x / den, term.y / den);
            }
            acc[k].add(term);
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
template <int N, int E, bool OWNED>
__global__ void __launch_bounds__(fft::LG<N, E>::THREADS, fft::LG<N, E>::MINB)
    k_big_rows_inv(BatchGeom g, const int2 *__restrict__ led, const float2 *__restrict__ Pt,
                   const float2 *__restrict__ Xs, float2 *__restrict__ Ur,
                   const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = fft::LG<N, E>;
    extern __shared__ float2 smem[];
    int2 *s_ab = reinterpret_cast<int2 *>(G::tw_hi(smem) + 256);
    for (int l = threadIdx.x; l < g.nb; l += G::THREADS) s_ab[l] = led_box_offset(led, l, g);
    setup<N, E>(smem, thi, tlo);
    const int ln = G::cline(), t = G::ct();
    const int h = g.h;
    // persistent: the CTA walks groups of LPC box rows (its set-up done once; a row's store
    // drains while the next row's gathers are in flight)
    for (int grp = blockIdx.x; grp * G::LPC < g.rspan; grp += gridDim.x) {
        if (grp != (int)blockIdx.x) __syncthreads();   // the last transform's reads of the lines done
        const int i = grp * G::LPC + ln;            // box row of this line
        const bool live = i < g.rspan;
        float2 v[E];
        if constexpr (OWNED) {
            // Per covering LED, only its supported crop columns: they land on the contiguous
            // (mod N) line positions e = pc_lo + ab.y + Cu0 + idx.  Thread t owns the positions
            // e = t (mod T), accumulated in LED order in this line's exchange area, so no two
            // threads touch one position and no barrier is needed until the transform.
            float2 *acc = smem + ln * G::STRIDE;
#pragma unroll
            for (int m = 0; m < E; ++m) acc[t + m * G::T] = make_float2(0.f, 0.f);
            const int W = g.pc_hi - g.pc_lo;
            // one covering LED's share of this line: its rows of Xs and Pt and the position
            // of its first supported column; four of this thread's positions per pass
            struct Src {
                const float2 *x = nullptr, *p = nullptr;
                int es = 0, base = 0x7fffffff;
            };
            auto src_of = [&](int l) {
                Src q;
                const int2 ab = s_ab[l];
                int rr = i - ab.x;
                if (rr < 0) rr += N;
                if (rr < g.pr_lo || rr >= g.pr_hi) return q;   // pupil zero on that crop row
                q.x = Xs + ((size_t)l * h + rr) * h + g.pc_lo;
                q.p = Pt + (size_t)rr * h + g.pc_lo;
                q.es = (int)(((long long)g.pc_lo + ab.y + g.Cu0) % N);   // position of idx 0
                q.base = (t - q.es) & (G::T - 1);
                return q;
            };
            auto load4 = [&](const Src &q, int base, float2 (&x)[4], float2 (&pp)[4]) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int idx = base + u * G::T;
                    x[u] = idx < W ? q.x[idx] : make_float2(0.f, 0.f);
                    pp[u] = idx < W ? q.p[idx] : make_float2(0.f, 0.f);
                }
            };
            auto add4 = [&](const Src &q, int base, const float2 (&x)[4], const float2 (&pp)[4]) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int idx = base + u * G::T;
                    if (idx < W) {
                        int e = q.es + idx;
                        if (e >= N) e -= N;
                        int j = e - g.Cu0;                  // box column
                        if (j < 0) j += N;
                        if (j < g.cspan) {
                            const float2 pr = cmul(x[u], pp[u]);
                            float2 a = acc[e];
                            a.x += pr.x;
                            a.y += pr.y;
                            acc[e] = a;
                        }
                    }
                }
            };
            if (W <= 4 * G::T) {
                // every LED in one pass: two covering LEDs' loads in flight together, each
                // position still summed in LED order (four in flight measured no faster)
                int l = 0;
                while (live) {
                    Src qa, qb;
                    for (; l < g.nb && !(qa = src_of(l)).x; ++l) {}
                    if (l >= g.nb) break;
                    for (++l; l < g.nb && !(qb = src_of(l)).x; ++l) {}
                    ++l;
                    float2 xa[4], pa[4], xb[4], pb[4];
                    load4(qa, qa.base, xa, pa);
                    if (qb.x) load4(qb, qb.base, xb, pb);
                    add4(qa, qa.base, xa, pa);
                    if (qb.x) add4(qb, qb.base, xb, pb);
                    if (!qb.x) break;
                }
            } else {
                for (int l = 0; live && l < g.nb; ++l) {
                    const Src q = src_of(l);
                    if (!q.x) continue;
                    for (int base = q.base; base < W; base += 4 * G::T) {
                        float2 x[4], pp[4];
                        load4(q, base, x, pp);
                        add4(q, base, x, pp);
                    }
                }
            }
#pragma unroll
            for (int m = 0; m < E; ++m) v[m] = acc[t + m * G::T];
            __syncthreads();                        // every accumulator read before the exchanges
        } else {
        // four elements per LED sweep: four independent gathers in flight per thread
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += 4) {
            int jj[4];
            bool any = false;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                int j = t + (m0 + k) * G::T - g.Cu0;     // box column of element e
                if (j < 0) j += N;
                jj[k] = (live && j < g.cspan) ? j : -1;
                any |= jj[k] >= 0;
            }
            KahanC acc[4];
            if (__any_sync(0xffffffffu, any)) {
                for (int l = 0; l < g.nb; ++l) {
                    const int2 ab = s_ab[l];
                    int rr = i - ab.x;
                    if (rr < 0) rr += N;
                    if (rr < g.pr_lo || rr >= g.pr_hi) continue;   // pupil zero on that crop row
                    const float2 *xrow = Xs + ((size_t)l * h + rr) * h;
                    const float2 *prow = Pt + (size_t)rr * h;
                    float2 x[4], pp[4];
                    bool in[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        int c = jj[k] - ab.y;
                        if (c < 0) c += N;
                        in[k] = jj[k] >= 0 && c >= g.pc_lo && c < g.pc_hi;
                        x[k] = in[k] ? xrow[c] : make_float2(0.f, 0.f);
                        pp[k] = in[k] ? prow[c] : make_float2(0.f, 0.f);
                    }
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if (in[k]) acc[k].add(cmul(x[k], pp[k]));
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) v[m0 + k] = acc[k].s;
        }
        }
        line_fft_e<N, +1, E>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128, t);
        if (live) {
            float2 *row = Ur + (size_t)i * N;
#pragma unroll
            for (int m = 0; m < E; ++m) row[t + m * G::T] = v[m];
        }
    }
}

// ---------------------------------------------------------------------------
// Pass B: columns (contiguous): IFFT of the gradient, RMSprop in registers,
// FFT of the updated column; the IFFT's last stage hands its registers to the
// RMSprop and the FFT's first stage without a shared-memory round trip.
// ---------------------------------------------------------------------------
template <int N, int MODE, int E>
__global__ void __launch_bounds__(fft::LG<N, E>::THREADS, fft::LG<N, E>::MINB)
    k_big_cols(ColsArgs a, const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = fft::LG<N, E>;
    extern __shared__ float2 smem[];
    setup<N, E>(smem, thi, tlo);
    const int ln = G::cline(), t = G::ct();
    const int c = blockIdx.x * G::LPC + ln;    // column; c >= N only when N < LPC
    const bool live = c < N;
    float2 *line = smem + ln * G::STRIDE;
    const float2 *s_hi = G::tw_hi(smem);
    const size_t col = (size_t)(live ? c : 0) * N;
    float2 v[E];
    if (MODE == kColsForward) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = live ? a.O[col + t + m * G::T] : make_float2(0.f, 0.f);
    } else {
        const float2 *u = a.U + (size_t)(live ? c : 0) * a.ldU;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            int i = t + m * G::T - a.Ru0;          // box row of element e
            if (i < 0) i += N;
            v[m] = (live && i < a.rspan) ? u[i] : make_float2(0.f, 0.f);
        }
        line_fft_e<N, +1, E>(v, line, s_hi, s_hi + 128, t);
        if (MODE == kColsGradient) {
            if (live) {
#pragma unroll
                for (int m = 0; m < E; ++m) a.gout[col + t + m * G::T] = v[m];
            }
            return;
        }
        // RMSprop on the column (constrained_RMSprop_both, kernels.cuh:364-382)
        const float omb = 1.0f - a.beta;
        if (live) {
#pragma unroll
            for (int m0 = 0; m0 < E; m0 += 4) {
                float2 w[4];
                float mv[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    w[k] = a.O[col + t + (m0 + k) * G::T];
                    mv[k] = a.m[col + t + (m0 + k) * G::T];
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float2 gv = v[m0 + k];
                    float mu = gv.x * gv.x + gv.y * gv.y;
                    mu = a.beta * mv[k] + omb * mu;
                    const float sq = a.lr / (sqrtf(mu) + a.eps);
                    w[k].x -= gv.x * sq;
                    w[k].y -= gv.y * sq;
                    a.O[col + t + (m0 + k) * G::T] = w[k];
                    a.m[col + t + (m0 + k) * G::T] = mu;
                    v[m0 + k] = w[k];
                }
            }
        }
        if (a.rspan_n == 0) return;   // uniform over the grid: no next batch
    }
    line_fft_e<N, -1, E>(v, line, s_hi, s_hi + 128, t);
    if (live) {
        float2 *vv = a.V + (size_t)c * a.ldV;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            int i = t + m * G::T - a.Ru0n;
            if (i < 0) i += N;
            if (i < a.rspan_n) vv[i] = v[m];
        }
    }
}

// ---------------------------------------------------------------------------
// Pass B, update mode, persistent with prefetch (N = 16384, 32 values per thread).
// A CTA per SM walks the columns c = blockIdx.x + k gridDim.x; while it transforms
// one column, bulk copies bring the next column's RMSprop moment (64 KiB) and, when
// they fit, its gradient rows into shared memory, so those loads leave the critical
// path.  Waits are bounded; a copy that never completes sets the device flag and the
// CTA drains its copies in flight and stops.
// ---------------------------------------------------------------------------
constexpr int kColsUCap = 4096;   // gradient rows staged in shared memory (32 KiB)

template <int N, int E>
struct ColsAsync {
    static constexpr int SMEM = N * 8 + 2 * 128 * 8 + N * 4 + kColsUCap * 8 + 32;
    static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
    static_assert(fft::LG<N, E>::LPC == 1, "one line per CTA");
};

template <int N, int E>
__global__ void __launch_bounds__(fft::LG<N, E>::THREADS, 1)
    k_big_cols_async(ColsArgs a, const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = fft::LG<N, E>;
    extern __shared__ __align__(128) float2 smem[];
    float2 *line = smem;
    float2 *s_hi = smem + N;
    float *mbuf = reinterpret_cast<float *>(smem + N + 256);
    float2 *ubuf = reinterpret_cast<float2 *>(mbuf + N);
    // [0] moment, [1] gradient rows, [2] object column (into the exchange area)
    uint64_t *bar = reinterpret_cast<uint64_t *>(ubuf + kColsUCap);
    const int t = threadIdx.x;
    const bool u_async = a.rspan > 0 && a.rspan <= kColsUCap;
    const uint32_t ubytes = (uint32_t)((a.rspan + 1) & ~1) * 8u;
    int c = blockIdx.x;
    if (t == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::mbar_init(&bar[2], 1);
        tma::fence_barrier_init();
        if (c < N) {
            tma::arrive_expect_tx(&bar[0], N * 4);
            tma::load_1d(mbuf, a.m + (size_t)c * N, N * 4, &bar[0]);
            if (u_async) {
                tma::arrive_expect_tx(&bar[1], ubytes);
                tma::load_1d(ubuf, a.U + (size_t)c * a.ldU, ubytes, &bar[1]);
            }
        }
    }
    fft::load_twiddles(s_hi, s_hi + 128, thi, tlo, G::NHI, G::NLO);
    __syncthreads();
    // each barrier completes once per column: the parity of the copy in flight, and
    // whether one is in flight (block-uniform)
    uint32_t pm = 0, pu = 0, po = 0;
    bool mp = c < N, up = c < N && u_async, op = false;
    bool failed = false;
    const float omb = 1.0f - a.beta;
    for (; c < N; c += gridDim.x) {
        const int cn = c + gridDim.x;
        const size_t col = (size_t)c * N;
        float2 v[E];
        if (u_async) {
            failed = __syncthreads_or(!tma::mbar_wait(&bar[1], pu));
            if (failed) break;
            up = false;
            pu ^= 1u;
#pragma unroll
            for (int m = 0; m < E; ++m) {
                int i = t + m * G::T - a.Ru0;          // box row of element e
                if (i < 0) i += N;
                v[m] = i < a.rspan ? ubuf[i] : make_float2(0.f, 0.f);
            }
            __syncthreads();                           // the rows buffer is free
            if (cn < N) {
                if (t == 0) {
                    tma::fence_proxy_async();
                    tma::arrive_expect_tx(&bar[1], ubytes);
                    tma::load_1d(ubuf, a.U + (size_t)cn * a.ldU, ubytes, &bar[1]);
                }
                up = true;
            }
        } else {
            const float2 *u = a.U + (size_t)c * a.ldU;
#pragma unroll
            for (int m = 0; m < E; ++m) {
                int i = t + m * G::T - a.Ru0;
                if (i < 0) i += N;
                v[m] = i < a.rspan ? u[i] : make_float2(0.f, 0.f);
            }
        }
        // once the inverse FFT's last stage has read the exchange area, the object column
        // is copied into it while that stage's butterflies run
        const float2 *ocol = a.O + col;
        fft::line_fft_regs32<N, +1>(v, line, s_hi, s_hi + 128, t, [&] {
            if (t == 0) {
                tma::fence_proxy_async();
                tma::arrive_expect_tx(&bar[2], N * 8);
                tma::load_1d(line, ocol, N * 8, &bar[2]);
            }
        });
        op = true;
        failed = __syncthreads_or(!tma::mbar_wait(&bar[0], pm) || !tma::mbar_wait(&bar[2], po));
        if (failed) break;
        mp = false;
        pm ^= 1u;
        op = false;
        po ^= 1u;
        // RMSprop on the column (constrained_RMSprop_both, kernels.cuh:364-382)
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += 4) {
            float2 w[4];
            float mv[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                w[k] = line[t + (m0 + k) * G::T];
                mv[k] = mbuf[t + (m0 + k) * G::T];
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float2 gv = v[m0 + k];
                float mu = gv.x * gv.x + gv.y * gv.y;
                mu = a.beta * mv[k] + omb * mu;
                const float sq = a.lr / (sqrtf(mu) + a.eps);
                w[k].x -= gv.x * sq;
                w[k].y -= gv.y * sq;
                a.O[col + t + (m0 + k) * G::T] = w[k];
                a.m[col + t + (m0 + k) * G::T] = mu;
                v[m0 + k] = w[k];
            }
        }
        __syncthreads();                               // the moment buffer and the area are free
        if (cn < N) {
            if (t == 0) {
                tma::fence_proxy_async();
                tma::arrive_expect_tx(&bar[0], N * 4);
                tma::load_1d(mbuf, a.m + (size_t)cn * N, N * 4, &bar[0]);
            }
            mp = true;
        }
        if (a.rspan_n == 0) continue;                  // uniform: no next batch
        line_fft_e<N, -1, E>(v, line, s_hi, s_hi + 128, t);
        float2 *vv = a.V + (size_t)c * a.ldV;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            int i = t + m * G::T - a.Ru0n;
            if (i < 0) i += N;
            if (i < a.rspan_n) vv[i] = v[m];
        }
    }
    if (failed && t == 0) {
        atomicExch(a.err, 1);
        if (mp) tma::mbar_wait(&bar[0], pm);           // bounded drains of copies in flight
        if (up) tma::mbar_wait(&bar[1], pu);
        if (op) tma::mbar_wait(&bar[2], po);
    }
}

// ---------------------------------------------------------------------------
// Pass C: rows of V (strided) -> FFT along the row -> the next batch's Sbox
// ---------------------------------------------------------------------------
template <int N, int E>
__global__ void __launch_bounds__(fft::LG<N, E>::THREADS, fft::LG<N, E>::MINB)
    k_big_rows_fwd(const float2 *__restrict__ Vr, int rspan_n, int Cu0n, int cspan_n,
                   float2 *__restrict__ Sboxr, const float2 *__restrict__ thi,
                   const float2 *__restrict__ tlo) {
    using G = fft::LG<N, E>;
    extern __shared__ float2 smem[];
    setup<N, E>(smem, thi, tlo);
    const int ln = G::cline(), t = G::ct();
    const int i = blockIdx.x * G::LPC + ln;
    const bool live = i < rspan_n;
    const float2 *row = Vr + (size_t)(live ? i : 0) * N;
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = live ? row[t + m * G::T] : make_float2(0.f, 0.f);
    line_fft_e<N, -1, E>(v, smem + ln * G::STRIDE, G::tw_hi(smem), G::tw_hi(smem) + 128, t);
    if (live) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
            int j = t + m * G::T - Cu0n;
            if (j < 0) j += N;
            if (j < cspan_n) Sboxr[(size_t)i * cspan_n + j] = v[m];
        }
    }
}

// Pass C persistent (16384-point rows, 32 values per thread): a CTA per SM walks the
// rows i = blockIdx.x + k gridDim.x; the next row is copied into the exchange area
// while the current row's last FFT stage runs (bounded waits, device flag on failure).
template <int N, int E>
__global__ void __launch_bounds__(fft::LG<N, E>::THREADS, 1)
    k_big_rows_fwd_async(const float2 *__restrict__ Vr, int rspan_n, int Cu0n, int cspan_n,
                         float2 *__restrict__ Sboxr, int *__restrict__ err,
                         const float2 *__restrict__ thi, const float2 *__restrict__ tlo) {
    using G = fft::LG<N, E>;
    static_assert(G::LPC == 1 && E == 32, "one 32-values-per-thread line per CTA");
    extern __shared__ __align__(128) float2 smem[];
    float2 *line = smem;
    float2 *s_hi = smem + N;
    uint64_t *bar = reinterpret_cast<uint64_t *>(s_hi + 256);
    const int t = threadIdx.x;
    int i = blockIdx.x;
    if (t == 0) {
        tma::mbar_init(bar, 1);
        tma::fence_barrier_init();
        if (i < rspan_n) {
            tma::arrive_expect_tx(bar, N * 8);
            tma::load_1d(line, Vr + (size_t)i * N, N * 8, bar);
        }
    }
    fft::load_twiddles(s_hi, s_hi + 128, thi, tlo, G::NHI, G::NLO);
    __syncthreads();
    uint32_t parity = 0;
    bool pending = i < rspan_n, failed = false;
    for (; i < rspan_n; i += gridDim.x) {
        failed = __syncthreads_or(!tma::mbar_wait(bar, parity));
        if (failed) break;
        pending = false;
        parity ^= 1u;
        float2 v[E];
        const int in = i + gridDim.x;
        // the next row's DRAM read starts under this row's FFT; its copy into the exchange
        // area during the last stage then reads L2
        if (t == 0 && in < rspan_n) tma::prefetch_l2(Vr + (size_t)in * N, N * 8);
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = line[t + m * G::T];
        __syncthreads();                               // every read before the first exchange
        fft::line_fft_regs32<N, -1>(v, line, s_hi, s_hi + 128, t, [&] {
            if (t == 0 && in < rspan_n) {
                tma::fence_proxy_async();
                tma::arrive_expect_tx(bar, N * 8);
                tma::load_1d(line, Vr + (size_t)in * N, N * 8, bar);
            }
        });
        pending = in < rspan_n;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            int j = t + m * G::T - Cu0n;
            if (j < 0) j += N;
            if (j < cspan_n) Sboxr[(size_t)i * cspan_n + j] = v[m];
        }
    }
    if (failed && t == 0) {
        atomicExch(err, 1);
        if (pending) tma::mbar_wait(bar, parity);      // bounded drain of the copy in flight
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Self-check of the bounded waits: one thread arms an mbarrier for 16 bytes that no copy
// delivers and waits with the given limit; the wait gives up, the kernel sets the flag
// every pass uses for a wait that ran out, and returns.  No copy is in flight at any time.
// ---------------------------------------------------------------------------
__global__ void k_wait_selftest(int *flag, long long limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tma::mbar_init(&bar, 1);
        tma::fence_barrier_init();
        tma::arrive_expect_tx(&bar, 16);
        if (!tma::mbar_wait(&bar, 0, limit)) atomicExch(flag, 1);
    }
}

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

static int lpc_of(int n) { return (n * 8 >= 64 * 1024) ? 1 : (64 * 1024) / (n * 8); }  // fft::LG<n>::LPC

int lr_blocks(int h, int nl) {
    const long long lines = (long long)nl * h;
    const int lpc = lpc_of(h);
    return (int)((lines + lpc - 1) / lpc);
}

static bool cols_async();

cudaError_t launch_lr_cols_inv(const BatchGeom &g, const int2 *led, const float2 *P, BatchBufs b,
                               int l0, int nl, const Twiddles &tw, cudaStream_t st) {
    const int blocks = lr_blocks(g.h, nl);
    cudaError_t e = cudaSuccess;
#define F(N)                                                                              \
    e = set_smem(k_lr_cols_inv<N>, smem_bytes<N>());                                      \
    if (e != cudaSuccess) return e;                                                       \
    k_lr_cols_inv<N><<<blocks, fft::LG<N>::THREADS, smem_bytes<N>(), st>>>(                   \
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
        k_lr_rows_inv<N, kStackU16><<<blocks, fft::LG<N>::THREADS, smem_bytes<N>(), st>>>(    \
            Y, g, l0, nl, b.T1, b.Rs, tw.lo_hi, tw.lo_lo);                                \
    } else {                                                                              \
        e = set_smem(k_lr_rows_inv<N, kStackF32>, smem_bytes<N>());                       \
        if (e != cudaSuccess) return e;                                                   \
        k_lr_rows_inv<N, kStackF32><<<blocks, fft::LG<N>::THREADS, smem_bytes<N>(), st>>>(    \
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
    if (g.loss == kLossIsotropic) {                                                       \
        e = set_smem(k_lr_rows_fwd<N, kLossIsotropic>, smem_bytes<N>());                  \
        if (e != cudaSuccess) return e;                                                   \
        k_lr_rows_fwd<N, kLossIsotropic><<<blocks, fft::LG<N>::THREADS, smem_bytes<N>(), st>>>( \
            g, nl, b.T1, b.Rs, b.parts + part_off, tw.lo_hi, tw.lo_lo);                   \
    } else {                                                                              \
        e = set_smem(k_lr_rows_fwd<N, kLossAnisotropic>, smem_bytes<N>());                \
        if (e != cudaSuccess) return e;                                                   \
        k_lr_rows_fwd<N, kLossAnisotropic><<<blocks, fft::LG<N>::THREADS, smem_bytes<N>(), st>>>( \
            g, nl, b.T1, b.Rs, b.parts + part_off, tw.lo_hi, tw.lo_lo);                   \
    }
    FPM_DISPATCH_LR(g.h, F)
#undef F
    return cudaGetLastError();
}

bool lr_rows_fused_supported(int h) { return h >= 128 && h <= 2048 && (h & (h - 1)) == 0; }

static int fused_cluster(int h);

static int ctas_per_led_fused(int h) {   // L23<h, CL>::CTAS_PER_LED
    const int cl = fused_cluster(h);
    const int pout = cl * ((h >= 1024 ? 512 : 1024) / (h / 16)) - 2;
    return cl * ((h + pout - 1) / pout);
}

int lr_rows_fused_blocks(int h, int nl) { return nl * ctas_per_led_fused(h); }

#define FPM_DISPATCH_FUSED(n, F) \
    switch (n) {                 \
        case 128: F(128); break;  \
        case 256: F(256); break;  \
        case 512: F(512); break;  \
        case 1024: F(1024); break; \
        case 2048: F(2048); break; \
        default: return cudaErrorInvalidValue; \
    }

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library links the runtime only).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// 3-D tile map over pages of n x n column-major images (x = row, y = column, z = page).
static cudaError_t page_tile_map(CUtensorMap *map, CUtensorMapDataType type, size_t esz,
                                 const void *base, int n, int pages, int box_rows, int box_cols) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)pages};
    const cuuint64_t strides[2] = {(cuuint64_t)n * esz, (cuuint64_t)n * n * esz};
    const cuuint32_t box[3] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(map, type, 3, const_cast<void *>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int N, int LOSS, int CL>
static cudaError_t launch_fused_cl(int nl, const float *amp, const BatchGeom &g, int l0,
                                   const BatchBufs &b, int part_off, const CUtensorMap &tm_field,
                                   const Twiddles &tw, cudaStream_t st) {
    using F = L23<N, CL>;
    auto kern = k_lr_rows_fused<N, LOSS, CL>;
    cudaError_t e = set_smem(kern, F::SMEM);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nl * F::CTAS_PER_LED));
    cfg.blockDim = dim3(F::THREADS);
    cfg.dynamicSmemBytes = F::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, amp, g, l0, (const float2 *)b.T1, b.T2,
                              b.parts + part_off, b.flag, tm_field, tw.lo_hi, tw.lo_lo);
}

// cluster size of the fused row pass: 16 lines per cluster by default (4 CTAs of 4 lines
// at h = 2048, 2 CTAs below); FPM_L23_CLUSTER (or the tuner) picks 2, 4 or 8
static int fused_cluster(int h) {
    const int v = knob("FPM_L23_CLUSTER", tuning().l23_cluster, 0, h == 2048 ? 4 : 2);
    return v == 8 ? 8 : (v == 4 ? 4 : 2);
}

template <int N, int LOSS>
static cudaError_t launch_fused_k(int nl, const float *amp, const BatchGeom &g, int l0,
                                  const BatchBufs &b, int part_off, const CUtensorMap &tm_field,
                                  const Twiddles &tw, cudaStream_t st) {
    switch (fused_cluster(N)) {
        case 8: return launch_fused_cl<N, LOSS, 8>(nl, amp, g, l0, b, part_off, tm_field, tw, st);
        case 4: return launch_fused_cl<N, LOSS, 4>(nl, amp, g, l0, b, part_off, tm_field, tw, st);
        default: return launch_fused_cl<N, LOSS, 2>(nl, amp, g, l0, b, part_off, tm_field, tw, st);
    }
}

cudaError_t launch_lr_rows_fused(const BatchGeom &g, StackView Y, BatchBufs b, int l0, int nl,
                                 int part_off, const Twiddles &tw, cudaStream_t st) {
    if (!Y.rows) return cudaErrorInvalidValue;   // the amplitude rows are made per solve
    cudaError_t e = cudaSuccess;
    CUtensorMap tm_field{};
#define F(N)                                                                              \
    static_assert(L23<N, 2>::LIN == (N >= 1024 ? 512 : 1024) / (N / 16), "host CTA count");  \
    e = page_tile_map(&tm_field, CU_TENSOR_MAP_DATA_TYPE_UINT64, 8, b.T1, N, nl,          \
                      L23<N, 2>::LIN, L23<N, 2>::CB);                                     \
    if (e != cudaSuccess) return e;                                                       \
    e = g.loss == kLossIsotropic                                                          \
            ? launch_fused_k<N, kLossIsotropic>(nl, Y.rows, g, l0, b, part_off, tm_field, tw, st) \
            : launch_fused_k<N, kLossAnisotropic>(nl, Y.rows, g, l0, b, part_off, tm_field, tw, st); \
    if (e != cudaSuccess) return e;
    FPM_DISPATCH_FUSED(g.h, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_lr_cols_fwd(const BatchGeom &g, const float2 *src, BatchBufs b, int l0,
                               int nl, const Twiddles &tw, cudaStream_t st) {
    const int blocks = lr_blocks(g.h, nl);
    cudaError_t e = cudaSuccess;
    if (g.h == 2048 && b.flag && cols_async()) {
        using G = fft::LG<2048>;
        constexpr int smem = G::SMEM + 16;
        e = set_smem(k_lr_cols_fwd_async<2048>, smem);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        const int ngroups = nl * 2048 / G::LPC;
        const int grid = ngroups < 2 * sms ? ngroups : 2 * sms;
        k_lr_cols_fwd_async<2048><<<grid, G::THREADS, smem, st>>>(g, l0, nl, src, b.Xs, b.flag,
                                                                  tw.lo_hi, tw.lo_lo);
        return cudaGetLastError();
    }
#define F(N)                                                                              \
    e = set_smem(k_lr_cols_fwd<N>, smem_bytes<N>());                                      \
    if (e != cudaSuccess) return e;                                                       \
    k_lr_cols_fwd<N><<<blocks, fft::LG<N>::THREADS, smem_bytes<N>(), st>>>(                   \
        g, l0, nl, src, b.Xs, tw.lo_hi, tw.lo_lo);
    FPM_DISPATCH_LR(g.h, F)
#undef F
    return cudaGetLastError();
}

cudaError_t launch_lr_pupil_grad(const BatchGeom &g, const int2 *led, BatchBufs b, float2 *dP,
                                 cudaStream_t st, const unsigned *pie_scratch) {
    if (g.pie == 1 && !pie_scratch) return cudaErrorInvalidValue;
    const int t = (g.h + 31) / 32;
    k_lr_pupil_grad<<<dim3(t, t), 256, 0, st>>>(b.Sbox, b.Xs, led, g, dP, pie_scratch);
    return cudaGetLastError();
}

// max |x|^2 of non-negative floats through integer atomics on their bit patterns
__device__ __forceinline__ void max_abs2(unsigned *slot, float v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) atomicMax(slot, __float_as_uint(v));
}

__global__ void __launch_bounds__(256) k_pupil_abs2_max(const float2 *__restrict__ P, int n,
                                                         unsigned *__restrict__ slot) {
    float m = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 p = P[i];
        m = fmaxf(m, p.x * p.x + p.y * p.y);
    }
    max_abs2(slot, m);
}

// per LED of the batch (blockIdx.y): max |sub|^2 over its whole h x h crop of the box
__global__ void __launch_bounds__(256) k_crop_abs2_max(const float2 *__restrict__ Sbox,
                                                        const int2 *__restrict__ led, BatchGeom g,
                                                        unsigned *__restrict__ slots) {
    const int l = blockIdx.y;
    const int2 ab = led_box_offset(led, l, g);
    const int n = g.h * g.h;
    float m = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = i % g.h, c = i / g.h;
        const float2 v = Sbox[(size_t)box_index(ab.y, c, g.H) * g.rspan + box_index(ab.x, r, g.H)];
        m = fmaxf(m, v.x * v.x + v.y * v.y);
    }
    max_abs2(&slots[l], m);
}

// object term: Pt = conj(P) / H^2 (row-major) over max|P|^2 (ePIE) or (|P|^2 + 1e-5) (tPIE)
__global__ void __launch_bounds__(256) k_pie_object_weights(float2 *__restrict__ Pt, int n,
                                                             float H2, int pie,
                                                             const unsigned *__restrict__ scratch) {
    const float pmax = __uint_as_float(scratch[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float2 w = Pt[i];
        float den = pmax;
        if (pie == 2) {   // |P|^2 from conj(P) / H^2: H^2 is a power of two, so exactly
            const float ax = w.x * H2, ay = w.y * H2;
            den = ax * ax + ay * ay + 1e-5f;
        }
        Pt[i] = make_float2(w.x / den, w.y / den);
    }
}

cudaError_t launch_pie_prepare(const BatchGeom &g, const float2 *P, const int2 *led,
                               const float2 *Sbox, unsigned *scratch, cudaStream_t st) {
    if (g.pie != 1) return cudaSuccess;   // tPIE needs no reductions
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned) * (1 + g.nb), st);
    if (e != cudaSuccess) return e;
    const int n = g.h * g.h;
    const int gx = std::min((n + 255) / 256, kB200SMs * 4);
    k_pupil_abs2_max<<<gx, 256, 0, st>>>(P, n, scratch);
    k_crop_abs2_max<<<dim3(std::min((n + 255) / 256, 64), g.nb), 256, 0, st>>>(Sbox, led, g,
                                                                             scratch + 1);
    return cudaGetLastError();
}

cudaError_t launch_pie_object_weights(const BatchGeom &g, float2 *Pt, const unsigned *scratch,
                                      cudaStream_t st) {
    if (g.pie == 0) return cudaSuccess;
    const int n = g.h * g.h;
    const int gx = std::min((n + 255) / 256, kB200SMs * 8);
    k_pie_object_weights<<<gx, 256, 0, st>>>(Pt, n, (float)((double)g.H * g.H), g.pie, scratch);
    return cudaGetLastError();
}

// Pass A's stitch over each LED's supported columns only, each line position owned by
// one thread; FPM_STITCH_OWNED=0 (measurements) loops every position over every LED
// with Kahan sums instead
static bool stitch_owned() {
    const char *e = std::getenv("FPM_STITCH_OWNED");
    return !(e && std::atoi(e) == 0);
}

template <int N, int E>
static cudaError_t launch_rows_inv_e(const BatchGeom &g, const int2 *led, const float2 *Pt,
                                     const float2 *Xs, float2 *Ur, const Twiddles &tw,
                                     cudaStream_t st) {
    using G = fft::LG<N, E>;
    const int smem = G::SMEM + g.nb * (int)sizeof(int2);
    const int groups = (g.rspan + G::LPC - 1) / G::LPC;
    auto kern = stitch_owned() ? k_big_rows_inv<N, E, true> : k_big_rows_inv<N, E, false>;
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, dev = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, G::THREADS, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int grid = std::max(1, std::min(groups, std::max(1, per_sm) * sms));
    kern<<<grid, G::THREADS, smem, st>>>(g, led, Pt, Xs, Ur, tw.hi_hi, tw.hi_lo);
    return cudaGetLastError();
}

static bool cols_e16();

cudaError_t launch_big_rows_inv(const BatchGeom &g, const int2 *led, const float2 *Pt,
                                const float2 *Xs, float2 *Ur, const Twiddles &tw,
                                cudaStream_t st) {
    cudaError_t e = cudaSuccess;
#define F(N)                                                                                  \
    if (N == 16384 && !cols_e16())                                                            \
        e = launch_rows_inv_e<N, (N == 16384 ? 32 : 16)>(g, led, Pt, Xs, Ur, tw, st);       \
    else                                                                                      \
        e = launch_rows_inv_e<N, 16>(g, led, Pt, Xs, Ur, tw, st);
    FPM_DISPATCH_BIG(g.H, F)
#undef F
    return e;
}

template <int N, int MODE, int E>
static cudaError_t launch_cols_k(const ColsArgs &a, const Twiddles &tw, cudaStream_t st) {
    using G = fft::LG<N, E>;
    const int blocks = (N + G::LPC - 1) / G::LPC;
    cudaError_t e = set_smem(k_big_cols<N, MODE, E>, G::SMEM);
    if (e != cudaSuccess) return e;
    k_big_cols<N, MODE, E><<<blocks, G::THREADS, G::SMEM, st>>>(a, tw.hi_hi, tw.hi_lo);
    return cudaGetLastError();
}

template <int N, int E>
static cudaError_t launch_cols_e(const ColsArgs &a, const Twiddles &tw, cudaStream_t st) {
    if (a.mode == kColsForward) return launch_cols_k<N, kColsForward, E>(a, tw, st);
    if (a.mode == kColsUpdate) return launch_cols_k<N, kColsUpdate, E>(a, tw, st);
    return launch_cols_k<N, kColsGradient, E>(a, tw, st);
}

// 16384-point lines (passes A, B, C) run with 32 values per thread; FPM_COLS_E16=1
// keeps 16 (measurements).
static bool cols_e16() { return knob("FPM_COLS_E16", tuning().cols_e16, -1, 0) != 0; }

// FPM_COLS_ASYNC=0 runs the update with plain loads (measurements)
static bool cols_async() { return knob("FPM_COLS_ASYNC", tuning().cols_async, -1, 1) != 0; }

static cudaError_t launch_cols_async(const ColsArgs &a, const Twiddles &tw, cudaStream_t st) {
    constexpr int N = 16384, E = 32;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = set_smem(k_big_cols_async<N, E>, ColsAsync<N, E>::SMEM);
    if (e != cudaSuccess) return e;
    const int grid = sms < N ? sms : N;
    k_big_cols_async<N, E><<<grid, fft::LG<N, E>::THREADS, ColsAsync<N, E>::SMEM, st>>>(
        a, tw.hi_hi, tw.hi_lo);
    return cudaGetLastError();
}

cudaError_t launch_big_cols(const ColsArgs &a, const Twiddles &tw, cudaStream_t st) {
    if (a.H == 16384 && a.mode == kColsUpdate && a.err && !cols_e16() && cols_async())
        return launch_cols_async(a, tw, st);
    cudaError_t e = cudaSuccess;
#define F(N)                                                                                  \
    if (N == 16384 && !cols_e16())                                                            \
        e = launch_cols_e<N, (N == 16384 ? 32 : 16)>(a, tw, st);                             \
    else                                                                                      \
        e = launch_cols_e<N, 16>(a, tw, st);
    FPM_DISPATCH_BIG(a.H, F)
#undef F
    return e;
}

template <int N, int E>
static cudaError_t launch_rows_fwd_e(int rspan_n, int Cu0n, int cspan_n, const float2 *Vr,
                                     float2 *Sboxr, const Twiddles &tw, cudaStream_t st) {
    using G = fft::LG<N, E>;
    const int blocks = (rspan_n + G::LPC - 1) / G::LPC;
    cudaError_t e = set_smem(k_big_rows_fwd<N, E>, G::SMEM);
    if (e != cudaSuccess) return e;
    k_big_rows_fwd<N, E><<<blocks, G::THREADS, G::SMEM, st>>>(Vr, rspan_n, Cu0n, cspan_n, Sboxr,
                                                             tw.hi_hi, tw.hi_lo);
    return cudaGetLastError();
}

cudaError_t launch_big_rows_fwd(int H, const float2 *Vr, int rspan_n, int Cu0n, int cspan_n,
                                float2 *Sboxr, const Twiddles &tw, cudaStream_t st, int *err) {
    cudaError_t e = cudaSuccess;
    if (H == 16384 && !cols_e16() && err && cols_async() && rspan_n > 0) {
        using G = fft::LG<16384, 32>;
        constexpr int smem = 16384 * 8 + 256 * 8 + 16;
        e = set_smem(k_big_rows_fwd_async<16384, 32>, smem);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        const int grid = rspan_n < sms ? rspan_n : sms;
        k_big_rows_fwd_async<16384, 32><<<grid, G::THREADS, smem, st>>>(
            Vr, rspan_n, Cu0n, cspan_n, Sboxr, err, tw.hi_hi, tw.hi_lo);
        return cudaGetLastError();
    }
#define F(N)                                                                                  \
    if (N == 16384 && !cols_e16())                                                            \
        e = launch_rows_fwd_e<N, (N == 16384 ? 32 : 16)>(rspan_n, Cu0n, cspan_n, Vr, Sboxr, tw, st); \
    else                                                                                      \
        e = launch_rows_fwd_e<N, 16>(rspan_n, Cu0n, cspan_n, Vr, Sboxr, tw, st);
    FPM_DISPATCH_BIG(H, F)
#undef F
    return e;
}

cudaError_t launch_wait_selftest(int *flag, long long limit, cudaStream_t st) {
    k_wait_selftest<<<1, 32, 0, st>>>(flag, limit);
    return cudaGetLastError();
}

}  // namespace fpm

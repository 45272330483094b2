// 2-D FFT passes built on the shared-memory line FFT of fft_core.cuh.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "fft.h"
#include "fft_core.cuh"
#include "tuning.h"

namespace fpm {

namespace {

template <int N, int E = 16>
using LG = fft::LG<N, E>;

template <int N, int DIR, int E>
__device__ __forceinline__ void line_fft_e(float2 (&v)[E], float2 *s, const float2 *hi,
                                           const float2 *lo, int t) {
    if constexpr (E == 32) {
        fft::line_fft_regs32<N, DIR>(v, s, hi, lo, t);
    } else {
        fft::line_fft_regs<N, DIR>(v, s, hi, lo, t);
    }
}

template <class K>
cudaError_t set_smem(K kernel, int bytes) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
}

// Lines along the contiguous axis: line L (over all pages) = elements [L*N, (L+1)*N).
template <int N, int DIR, int E>
__global__ void __launch_bounds__(LG<N, E>::THREADS, LG<N, E>::MINB)
    k_fft_contig(const float2 *__restrict__ in, float2 *__restrict__ out, long long n_lines,
                 const float2 *__restrict__ g_hi, const float2 *__restrict__ g_lo) {
    using G = LG<N, E>;
    extern __shared__ float2 smem[];
    float2 *s_hi = G::tw_hi(smem);
    fft::load_twiddles(s_hi, s_hi + 128, g_hi, g_lo, G::NHI, G::NLO);
    __syncthreads();
    const int ln = G::cline(), t = G::ct();
    const long long L = (long long)blockIdx.x * G::LPC + ln;
    const bool live = L < n_lines;
    const float2 *src = in + (size_t)(live ? L : 0) * N;
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = live ? src[t + m * G::T] : make_float2(0.f, 0.f);
    line_fft_e<N, DIR, E>(v, smem + ln * G::STRIDE, s_hi, s_hi + 128, t);
    if (live) {
        float2 *dst = out + (size_t)L * N;
#pragma unroll
        for (int m = 0; m < E; ++m) dst[t + m * G::T] = v[m];
    }
}

// Lines along the strided axis: line (p, r) = elements p*N*N + c*N + r, c = 0..N-1,
// numbered g = p*N + r; a CTA takes LPC consecutive g with its warps interleaved
// over them, so each c contributes LPC*8 contiguous bytes.
template <int N, int DIR, int E>
__global__ void __launch_bounds__(LG<N, E>::THREADS, LG<N, E>::MINB)
    k_fft_strided(const float2 *__restrict__ in, float2 *__restrict__ out, long long n_lines,
                  const float2 *__restrict__ g_hi, const float2 *__restrict__ g_lo) {
    using G = LG<N, E>;
    extern __shared__ float2 smem[];
    float2 *s_hi = G::tw_hi(smem);
    fft::load_twiddles(s_hi, s_hi + 128, g_hi, g_lo, G::NHI, G::NLO);
    __syncthreads();
    const int ln = G::iline(), t = G::it();
    const long long g = (long long)blockIdx.x * G::LPC + ln;
    const bool live = g < n_lines;
    const size_t base = live ? (size_t)(g / N) * N * N + (size_t)(g % N) : 0;
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; ++m)
        v[m] = live ? in[base + (size_t)(t + m * G::T) * N] : make_float2(0.f, 0.f);
    line_fft_e<N, DIR, E>(v, smem + ln * G::STRIDE, s_hi, s_hi + 128, t);
    if (live) {
#pragma unroll
        for (int m = 0; m < E; ++m) out[base + (size_t)(t + m * G::T) * N] = v[m];
    }
}

// axes: bit 0 = the contiguous pass, bit 1 = the strided pass (run in that order; the
// strided pass reads the contiguous pass's output when both run)
template <int N, int DIR, int E>
cudaError_t run_ne(const float2 *in, float2 *out, int count, int axes, const float2 *hi,
                   const float2 *lo, cudaStream_t st) {
    using G = LG<N, E>;
    cudaError_t e = set_smem(k_fft_contig<N, DIR, E>, G::SMEM);
    if (e != cudaSuccess) return e;
    e = set_smem(k_fft_strided<N, DIR, E>, G::SMEM);
    if (e != cudaSuccess) return e;
    const long long lines = (long long)count * N;
    const long long blocks = (lines + G::LPC - 1) / G::LPC;
    if (axes & 1) {
        k_fft_contig<N, DIR, E><<<(unsigned)blocks, G::THREADS, G::SMEM, st>>>(in, out, lines, hi, lo);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (axes & 2) {
        k_fft_strided<N, DIR, E><<<(unsigned)blocks, G::THREADS, G::SMEM, st>>>(
            (axes & 1) ? out : in, out, lines, hi, lo);
        e = cudaGetLastError();
    }
    return e;
}

// 16384-point lines run with 32 values per thread (FPM_COLS_E16=1 keeps 16, for
// measurements); shorter lines with 16
template <int N, int DIR>
cudaError_t run_n(const float2 *in, float2 *out, int count, int axes, const float2 *hi,
                  const float2 *lo, cudaStream_t st) {
    if constexpr (N == 16384) {
        if (knob("FPM_COLS_E16", tuning().cols_e16, -1, 0) == 0)
            return run_ne<N, DIR, 32>(in, out, count, axes, hi, lo, st);
    }
    return run_ne<N, DIR, 16>(in, out, count, axes, hi, lo, st);
}

template <int DIR>
cudaError_t dispatch(int n, const float2 *in, float2 *out, int count, int axes, const float2 *hi,
                     const float2 *lo, cudaStream_t st) {
    switch (n) {
        case 16: return run_n<16, DIR>(in, out, count, axes, hi, lo, st);
        case 32: return run_n<32, DIR>(in, out, count, axes, hi, lo, st);
        case 64: return run_n<64, DIR>(in, out, count, axes, hi, lo, st);
        case 128: return run_n<128, DIR>(in, out, count, axes, hi, lo, st);
        case 256: return run_n<256, DIR>(in, out, count, axes, hi, lo, st);
        case 512: return run_n<512, DIR>(in, out, count, axes, hi, lo, st);
        case 1024: return run_n<1024, DIR>(in, out, count, axes, hi, lo, st);
        case 2048: return run_n<2048, DIR>(in, out, count, axes, hi, lo, st);
        case 4096: return run_n<4096, DIR>(in, out, count, axes, hi, lo, st);
        case 8192: return run_n<8192, DIR>(in, out, count, axes, hi, lo, st);
        case 16384: return run_n<16384, DIR>(in, out, count, axes, hi, lo, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool fft_supported(int n) { return n >= 16 && n <= kMaxFftLen && (n & (n - 1)) == 0; }

FftEngine::~FftEngine() { release(); }

void FftEngine::release() {
    for (auto &kv : tw_) cudaFree(kv.second);
    tw_.clear();
}

cudaError_t FftEngine::tables(int n, const float2 **hi, const float2 **lo) {
    auto it = tw_.find(n);
    const int nhi = n >= 128 ? n / 128 : 1;
    const int nlo = n >= 128 ? 128 : n;
    if (it == tw_.end()) {
        std::vector<float2> h(nhi + nlo);
        const double two_pi = 6.283185307179586476925286766559;
        for (int j = 0; j < nhi; ++j) {
            const double a = -two_pi * (double)(j * 128) / n;
            h[j] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        for (int j = 0; j < nlo; ++j) {
            const double a = -two_pi * (double)j / n;
            h[nhi + j] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        float2 *d = nullptr;
        cudaError_t e = cudaMalloc(&d, h.size() * sizeof(float2));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d);
            return e;
        }
        it = tw_.emplace(n, d).first;
    }
    *hi = it->second;
    *lo = it->second + nhi;
    return cudaSuccess;
}

cudaError_t FftEngine::run(const float2 *in, float2 *out, int n, int count, FftDir dir,
                           cudaStream_t st) {
    if (!fft_supported(n) || count < 1) return cudaErrorInvalidValue;
    const float2 *hi, *lo;
    cudaError_t e = tables(n, &hi, &lo);
    if (e != cudaSuccess) return e;
    return dir == kForward ? dispatch<-1>(n, in, out, count, 3, hi, lo, st)
                           : dispatch<+1>(n, in, out, count, 3, hi, lo, st);
}

cudaError_t FftEngine::run_axis(const float2 *in, float2 *out, int n, int count, int axis,
                                FftDir dir, cudaStream_t st) {
    if (!fft_supported(n) || count < 1 || (axis != 0 && axis != 1)) return cudaErrorInvalidValue;
    const float2 *hi, *lo;
    cudaError_t e = tables(n, &hi, &lo);
    if (e != cudaSuccess) return e;
    const int axes = axis == 0 ? 1 : 2;
    return dir == kForward ? dispatch<-1>(n, in, out, count, axes, hi, lo, st)
                           : dispatch<+1>(n, in, out, count, axes, hi, lo, st);
}

}  // namespace fpm

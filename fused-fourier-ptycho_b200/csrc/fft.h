// 2-D complex FFTs of square column-major arrays (pages of n x n), unnormalised
// in both directions, like the cuFFT C2C transforms the reference calls at
// cuFPM_v3/cuFPM_pure_v3.cu:116-126,135-187.  Hand-written sm_100a kernels:
// one pass along the contiguous axis, one along the strided axis, each line
// transformed in shared memory (fft_core.cuh).
#pragma once

#include <cuda_runtime.h>
#include <map>

namespace fpm {

enum FftDir : int { kForward = -1, kInverse = +1 };

// Largest supported line length (one line per CTA in 128 KiB of shared memory).
constexpr int kMaxFftLen = 16384;

bool fft_supported(int n);

class FftEngine {
public:
    FftEngine() = default;
    ~FftEngine();
    FftEngine(const FftEngine &) = delete;
    FftEngine &operator=(const FftEngine &) = delete;

    // n x n transform of `count` pages of n*n elements; in may equal out.
    cudaError_t run(const float2 *in, float2 *out, int n, int count, FftDir dir, cudaStream_t st);
    // One axis only: axis 0 transforms the contiguous lines (along rows r), axis 1 the
    // strided ones (along columns c).
    cudaError_t run_axis(const float2 *in, float2 *out, int n, int count, int axis, FftDir dir,
                         cudaStream_t st);
    // Device two-level twiddle table of length n: hi (max(1, n/128) entries)
    // followed by lo (min(n, 128) entries), W_n^m = hi[m >> 7] * lo[m & 127].
    cudaError_t tables(int n, const float2 **hi, const float2 **lo);
    size_t workspace_bytes(int, int) const { return 0; }
    void release();

private:
    std::map<int, float2 *> tw_;
};

}  // namespace fpm

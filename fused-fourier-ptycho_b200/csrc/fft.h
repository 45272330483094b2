// 2-D complex FFTs of square column-major arrays, unnormalised in both
// directions (as cuFFT's C2C, which the reference calls at
// cuFPM_v3/cuFPM_pure_v3.cu:116-126,135-187).
#pragma once

#include <cuda_runtime.h>
#include <map>
#include <utility>

namespace fpm {

enum FftDir : int { kForward = -1, kInverse = +1 };

class FftEngine {
public:
    FftEngine() = default;
    ~FftEngine();
    FftEngine(const FftEngine &) = delete;
    FftEngine &operator=(const FftEngine &) = delete;

    // n x n transform of `count` pages of n*n elements; in may equal out.
    cudaError_t run(const float2 *in, float2 *out, int n, int count, FftDir dir, cudaStream_t st);
    // device bytes the plans for (n, count) need (for the memory budget).
    size_t workspace_bytes(int n, int count);
    void release();

private:
    std::map<std::pair<int, int>, int> plans_;  // (n, count) -> cufftHandle
};

}  // namespace fpm

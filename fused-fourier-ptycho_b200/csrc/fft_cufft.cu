// Temporary FFT back end on cuFFT plans; the hand-written sm_100a FFT kernels
// replace it.
#include "fft.h"

#include <cufft.h>

namespace fpm {

static cudaError_t to_cuda(cufftResult r) {
    if (r == CUFFT_SUCCESS) return cudaSuccess;
    if (r == CUFFT_ALLOC_FAILED) return cudaErrorMemoryAllocation;
    return cudaErrorUnknown;
}

FftEngine::~FftEngine() { release(); }

void FftEngine::release() {
    for (auto &kv : plans_) cufftDestroy((cufftHandle)kv.second);
    plans_.clear();
}

size_t FftEngine::workspace_bytes(int n, int count) {
    size_t ws = 0;
    int dims[2] = {n, n};
    if (cufftEstimateMany(2, dims, nullptr, 1, n * n, nullptr, 1, n * n, CUFFT_C2C, count, &ws) !=
        CUFFT_SUCCESS)
        return 0;
    return ws;
}

cudaError_t FftEngine::run(const float2 *in, float2 *out, int n, int count, FftDir dir,
                           cudaStream_t st) {
    auto key = std::make_pair(n, count);
    auto it = plans_.find(key);
    cufftHandle plan;
    if (it == plans_.end()) {
        int dims[2] = {n, n};
        cufftResult r = cufftPlanMany(&plan, 2, dims, nullptr, 1, n * n, nullptr, 1, n * n,
                                      CUFFT_C2C, count);
        if (r != CUFFT_SUCCESS) return to_cuda(r);
        plans_[key] = (int)plan;
    } else {
        plan = (cufftHandle)it->second;
    }
    cufftResult r = cufftSetStream(plan, st);
    if (r != CUFFT_SUCCESS) return to_cuda(r);
    r = cufftExecC2C(plan, (cufftComplex *)const_cast<float2 *>(in), (cufftComplex *)out,
                     dir == kForward ? CUFFT_FORWARD : CUFFT_INVERSE);
    return to_cuda(r);
}

}  // namespace fpm

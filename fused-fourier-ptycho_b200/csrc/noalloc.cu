// Loss-gradient stage for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a mex function living inside MATLAB's GPU
// memory manager (memory it does not hand out through gpuArrays is invisible to
// it and can exhaust the device under it), a framework whose caching allocator
// owns the device (a raw cudaMalloc there can fail under memory pressure and
// synchronises the device), or an acquisition loop that must not stall on an
// implicit device-wide synchronisation.  This entry point computes the same
// result as the loss-gradient stage inside fpm_solve / fpm_batch_gradients,
// but its only scratch (the per-tile loss partials) lives in the fixed device
// array below, so the call allocates nothing: the caller passes every input
// and output buffer.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fpm.h"
#include "engine.h"

namespace {

// Per-tile FP64 loss partials, one per 32 x 32 tile of every image
// (FPM_NOALLOC_MAX_TILES x 8 B = 512 KiB).  Every GPU that loads the library holds
// this array until the process exits.
__device__ __align__(256) double g_noalloc_tile_partials[FPM_NOALLOC_MAX_TILES];

constexpr int kMaxDevices = 64;
double *g_partials_addr[kMaxDevices] = {};
std::mutex g_partials_mutex;

// Device address of the array on the current device.  In host code the symbol
// is only a host-side stand-in; the address comes from cudaGetSymbolAddress,
// once per device, with that device current.
fpm_status partials_on_current_device(double **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return FPM_ERR_NO_DEVICE;
    }
    if (dev >= kMaxDevices) return FPM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_partials_mutex);
    if (!g_partials_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tile_partials);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return FPM_ERR_CUDA;
        }
        g_partials_addr[dev] = static_cast<double *>(p);
    }
    *out = g_partials_addr[dev];
    return FPM_OK;
}

bool on_current_device(const void *p) {
    int dev = -1;
    cudaPointerAttributes a;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

extern "C" fpm_status fpm_feature_gradient_noalloc(const float *z, const float *amplitude,
                                                   int32_t h, int32_t n_images, int32_t pratio,
                                                   float *gradient, double *loss, void *stream) {
    if (!z || !amplitude || !gradient || !loss) return FPM_ERR_INVALID_ARGUMENT;
    if (h < 2 || (h & 1) || n_images < 1 || pratio < 1) return FPM_ERR_INVALID_ARGUMENT;
    // size limit of the fixed scratch, checked before anything touches the device; the
    // side bound keeps the 64-bit tile count and the launch grid far from any overflow
    // whatever h the caller passes (a single image of 8192^2 already fills the array)
    if (h > FPM_NOALLOC_MAX_SIDE || n_images > 65535) return FPM_ERR_UNSUPPORTED;
    const long long tiles = (long long)n_images * fpm::feature_grad_blocks_per_image(h);
    if (tiles < 1 || tiles > FPM_NOALLOC_MAX_TILES) return FPM_ERR_UNSUPPORTED;
    if (!on_current_device(z) || !on_current_device(amplitude) || !on_current_device(gradient) ||
        !on_current_device(loss))
        return FPM_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(z) | reinterpret_cast<uintptr_t>(gradient)) & 7u ||
        reinterpret_cast<uintptr_t>(loss) & 7u || reinterpret_cast<uintptr_t>(amplitude) & 3u)
        return FPM_ERR_INVALID_ARGUMENT;
    double *partials = nullptr;
    fpm_status st = partials_on_current_device(&partials);
    if (st != FPM_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    fpm::StackView Y;
    Y.ptr = amplitude;
    Y.type = fpm::kStackF32;
    // every tile overwrites its own partial; only the loss accumulator starts at zero
    if (fpm::launch_feature_grad(reinterpret_cast<const float2 *>(z), Y, 0, n_images, h, pratio,
                                 reinterpret_cast<float2 *>(gradient), partials, s) != cudaSuccess)
        return FPM_ERR_CUDA;
    if (cudaMemsetAsync(loss, 0, sizeof(double), s) != cudaSuccess) return FPM_ERR_CUDA;
    if (fpm::launch_loss_accumulate(partials, (int)tiles, loss, s) != cudaSuccess)
        return FPM_ERR_CUDA;
    return FPM_OK;
}

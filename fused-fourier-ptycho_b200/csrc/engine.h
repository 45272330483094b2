// Internal (C++) interface between the C ABI / solver loop and the CUDA kernels.
// Every launcher enqueues on `st` and returns the launch status; nothing here
// synchronises.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace fpm {

enum StackType : int { kStackF32 = 0, kStackU16 = 1 };

// The measured stack as the kernels see it: float amplitude, or uint16 counts
// normalised on the fly with the stack's global (min, max) held on the device.
struct StackView {
    const void *ptr = nullptr;
    int type = kStackF32;
    const unsigned *minmax = nullptr;  // device [min, max] for kStackU16
};

// Half-open box of centred-spectrum rows/cols [lo, lo + span) taken modulo H.
struct Box {
    int r_lo = 0, r_span = 0, c_lo = 0, c_span = 0;
};

// ---- low-resolution (per-LED) stages -------------------------------------
cudaError_t launch_crop_pupil(const float2 *S, const float2 *P, const int2 *led, int z_off,
                              int nb, int h, int H, float2 *T, cudaStream_t st);
int feature_grad_blocks_per_image(int h);
cudaError_t launch_feature_grad(const float2 *Z, StackView Y, int z_off, int nb, int h,
                                int pratio, float2 *out, double *loss_part, cudaStream_t st);
cudaError_t launch_stitch_gather(const float2 *X, const float2 *P, const int2 *led, int z_off,
                                 int nb, int h, int H, Box box, float2 *G, cudaStream_t st);
cudaError_t launch_pupil_grad(const float2 *S, const float2 *X, const int2 *led, int z_off,
                              int nb, int h, int H, float2 *dP, cudaStream_t st);

// ---- large-array stages ---------------------------------------------------
cudaError_t launch_rmsprop_object(const float2 *g, float2 *O, float *m, size_t n, float lr,
                                  float beta, float eps, cudaStream_t st);
cudaError_t launch_rmsprop_pupil(const float2 *dP, float2 *P, float *m, const float *P0, int n,
                                 float lr, float beta, float eps, float am, cudaStream_t st);
cudaError_t launch_centre_spectrum(const float2 *S, int H, float2 *out, cudaStream_t st);
cudaError_t launch_centre_in_place(float2 *S, int H, cudaStream_t st);
// out[c*ldo + r] = in[r*ldi + c] (r < rows, c < cols); conj_scale != 0 conjugates and scales.
cudaError_t launch_transpose(const float2 *in, size_t ldi, float2 *out, size_t ldo, int rows,
                             int cols, float conj_scale, cudaStream_t st);
cudaError_t launch_bicubic_init(StackView Y, int h, int pratio, float2 *O, cudaStream_t st);

// ---- reductions and ingest ------------------------------------------------
cudaError_t launch_loss_accumulate(const double *parts, int n, double *slot, cudaStream_t st);
cudaError_t launch_stack_minmax(const uint16_t *p, size_t n, unsigned *minmax, cudaStream_t st);
cudaError_t launch_normalise(const uint16_t *p, size_t n, const unsigned *minmax, float *out,
                             cudaStream_t st);

}  // namespace fpm

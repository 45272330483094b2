// Internal (C++) interface between the C ABI / solver loop and the CUDA kernels.
// Every launcher enqueues on `st` and returns the launch status; nothing here
// synchronises.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <vector>

struct fpm_context;   // the C ABI's context (include/fpm.h)

namespace fpm {

enum StackType : int { kStackF32 = 0, kStackU16 = 1 };

// The measured stack as the kernels see it: float amplitude, or uint16 counts
// normalised on the fly with the stack's global (min, max) held on the device.
struct StackView {
    const void *ptr = nullptr;
    int type = kStackF32;
    const unsigned *minmax = nullptr;  // device [min, max] for kStackU16
    // device amplitude sqrt((v - min) / (max - min)) of every uint16 value v, the same
    // float the formula gives (kStackU16; null: kernels evaluate the formula)
    const float *lut = nullptr;
    // row-major FP32 copy of those amplitudes, page p row r at rows + (p h + r) h (the
    // fused row pass reads it; null until launch_amplitude_rows has made it)
    const float *rows = nullptr;
};

// Half-open box of centred-spectrum rows/cols [lo, lo + span) taken modulo H.
struct Box {
    int r_lo = 0, r_span = 0, c_lo = 0, c_span = 0;
};

// ---- low-resolution (per-LED) stages -------------------------------------
long long feature_grad_blocks_per_image(int h);
// loss: 0 anisotropic (the v3 loss), 1 isotropic
cudaError_t launch_feature_grad(const float2 *Z, StackView Y, int z_off, int nb, int h,
                                int pratio, float2 *out, double *loss_part, cudaStream_t st,
                                int loss = 0);

// ---- large-array stages ---------------------------------------------------
cudaError_t launch_rmsprop_pupil(const float2 *dP, float2 *P, float *m, const float *P0, int n,
                                 float lr, float beta, float eps, float am, cudaStream_t st);
cudaError_t launch_centre_in_place(float2 *S, int H, cudaStream_t st);
// out[c*ldo + r] = in[r*ldi + c] (r < rows, c < cols); conj_scale != 0 conjugates and scales.
cudaError_t launch_transpose(const float2 *in, size_t ldi, float2 *out, size_t ldo, int rows,
                             int cols, float conj_scale, cudaStream_t st);
// work: bicubic_work_bytes(h, pratio) bytes of device scratch (tap table + amplitude image)
size_t bicubic_work_bytes(int h, int pratio);
cudaError_t launch_bicubic_init(StackView Y, int h, int pratio, float2 *O, void *work,
                                cudaStream_t st);
// O = bicubic resize (as above) of re + i im, both h x h column-major; work as above
cudaError_t launch_bicubic_complex(const float *re, const float *im, int h, int pratio, float2 *O,
                                   void *work, cudaStream_t st);
// normalised amplitudes of stack pages [first, first + count) into out (count * h*h floats)
cudaError_t launch_stack_pages(StackView Y, int h, int first, int count, float *out,
                               cudaStream_t st);

// ---- reductions and ingest ------------------------------------------------
cudaError_t launch_loss_accumulate(const double *parts, int n, double *slot, cudaStream_t st);
// a captured epoch's end: loss[*counter] = *acc, *acc = 0, ++*counter
cudaError_t launch_epoch_end(double *acc, double *loss, int *counter, cudaStream_t st);
cudaError_t launch_set_int(int *p, int v, cudaStream_t st);
cudaError_t launch_stack_minmax(const uint16_t *p, size_t n, unsigned *minmax, cudaStream_t st);
cudaError_t launch_normalise(const uint16_t *p, size_t n, const unsigned *minmax, float *out,
                             cudaStream_t st);
// One step of a MATLAB optimiser class over n complex parameters (optimizers.cu).
enum OptKind { kOptRmsprop = 0, kOptAdam = 1, kOptYogi = 2, kOptSgd = 3 };
struct OptStep {
    int kind = kOptRmsprop;
    size_t n = 0;
    float2 *p = nullptr;
    const float2 *g = nullptr;
    float2 *mom1 = nullptr;    // Adam / Yogi first moment; RMSprop g0 (centered), else null
    float *mom2 = nullptr;     // Adam / Yogi second moment
    float2 *buffer = nullptr;  // RMSprop momentum buffer (momentum > 0), else null
    const float *amp = nullptr;  // pupil clamp amplitude, null = no clamp
    // scalars rounded to single from the double values: r1, 1 - r1, r2, 1 - r2, lr,
    // momentum, Adam's bias sqrt(1 - r2^t) / (1 - r1^t), clamp margin
    float r1 = 0, c1 = 0, r2 = 0, c2 = 0, lr = 0, mum = 0, bias = 1, margin = 0;
};
cudaError_t launch_optimizer_step(const OptStep &o, cudaStream_t st);

// amplitude of each of the 65536 uint16 values for the stack's (min, max)
cudaError_t launch_amplitude_lut(const unsigned *minmax, float *lut, cudaStream_t st);
// out[p][r][c] = amplitude of element (r, c) of page p of Y (pages of h x h, column-major,
// h a multiple of 32), the float every other pass takes for it
cudaError_t launch_amplitude_rows(StackView Y, int h, int pages, float *out, cudaStream_t st);
// float stack: min / max and normalise in two launches; mm: 2 unsigned of scratch
cudaError_t launch_normalise_f32(const float *p, size_t n, unsigned *mm, float *out,
                                 cudaStream_t st);

// box = {min row, max row, min col, max col} of the non-zero pixels of P (complex) or A
// (real), either may be NULL; {h, -1, h, -1} when none
cudaError_t launch_support_box(const float2 *P, const float *A, int h, int *box, cudaStream_t st);

// out[i] = |z[i] scale|^2, or its square root when amplitude != 0 (n even, 16-byte aligned)
cudaError_t launch_sim_magnitude(const float2 *z, size_t n, float scale, int amplitude,
                                 float *out, cudaStream_t st);

// ---- LED geometry (FP64) -----------------------------------------------------
struct LedGeom {
    int grid = 0, h = 0, NN = 0;     // LEDs per side, low-res side, high-res side
    double pitch = 0, height = 0;    // D_led, LED-plane height (um)
    double dx = 0, dy = 0;           // objdx, objdy (um)
    double k_lamuda = 0;             // 2 pi / lambda
    double ND = 0;                   // N * D_pixel
    double two_pi = 0;               // 2 pi
};
// (i, j) 1-based grid cells of an odd n x n array in the centre-out spiral order
void spiral_grid_order(int n, std::vector<int2> &order);
// led_idx[2l], led_idx[2l+1] = (kl, kt) of the LED at grid cell pos[l]
cudaError_t launch_led_nearest(const int2 *pos, int n_leds, const LedGeom &p, int32_t *led_idx,
                               cudaStream_t st);

// the stream and device of a C-ABI context (fpm_api.cpp), for the other ABI units
void *context_stream(::fpm_context *ctx);
int context_device(::fpm_context *ctx);

}  // namespace fpm

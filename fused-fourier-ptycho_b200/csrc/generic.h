// Any-size path: mixed-radix line FFTs (radices 2, 3, 4, 5, 7, 8) and the per-batch
// stages of the reconstruction for image sides that are not powers of two (the reference
// accepts any even size, README.md:9; its cuFFT plans take any h and H,
// cuFPM_v3/cuFPM_pure_v3.cu:116-126).  Every kernel enqueues on `st` and returns the
// launch status.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <vector>

#include "engine.h"
#include "fft.h"

namespace fpm {

// n >= 2 whose prime factors are all in {2, 3, 5, 7}, n <= kMaxFftLen.
bool gen_fft_supported(int n);
// the radices of n's stages in execution order (empty when unsupported)
std::vector<int> gen_fft_radices(int n);

// Unnormalised line FFTs of any supported length on contiguous lines, and 2-D FFTs of
// column-major n x n pages built from them (contiguous pass, page transpose, contiguous
// pass, transpose back).  Twiddle tables are built once per length in double precision.
class GenFft {
public:
    GenFft() = default;
    ~GenFft();
    GenFft(const GenFft &) = delete;
    GenFft &operator=(const GenFft &) = delete;
    // `count` lines of n values, line g at in + g*ld -> out + g*ld (in may equal out)
    cudaError_t lines(const float2 *in, float2 *out, int n, long long count, size_t ld, FftDir dir,
                      cudaStream_t st);
    // `count` column-major n x n pages; tmp holds count*n*n values; in may equal out
    cudaError_t fft2(const float2 *in, float2 *out, float2 *tmp, int n, int count, FftDir dir,
                     cudaStream_t st);
    // One n x n page with the work limited to a box: the transform along r runs only on
    // columns [c_lo, c_lo + c_cnt) mod n (with c_cnt < n: in == out, r_cnt == n, and the
    // other columns count as zeros whatever they hold) and the transform along c only on
    // rows [r_lo, r_lo + r_cnt) mod n (the other rows of out are left as the first pass
    // made them).  Exact on the box rows.
    cudaError_t fft2_box(const float2 *in, float2 *out, float2 *tmp, int n, FftDir dir, int c_lo,
                         int c_cnt, int r_lo, int r_cnt, cudaStream_t st);
    void release();

private:
    cudaError_t table(int n, const float2 **tw);
    cudaError_t lines_t(const float2 *in, float2 *out, int n, int g_lo, long long lines,
                        FftDir dir, cudaStream_t st);
    std::map<int, float2 *> tw_;
};

// out[p][c][r] = in[p][r][c] for count pages of n x n (column-major both).
cudaError_t launch_transpose_pages(const float2 *in, float2 *out, int n, int count,
                                   cudaStream_t st);

// Crop x pupil with the inverse shift (fused_getSubpupil_shifted, kernels.cuh:19-65): for
// LED l of [z_off, z_off + nb), pixel (r, c) of the h x h crop at the 1-based corner
// led[l] = (kl, kt) of the centred spectrum, read from the un-shifted spectrum S at
// ((kt-1+r+H/2) mod H, (kl-1+c+H/2) mod H), times P(r, c), stored at page l - z_off,
// position ((r+h/2) mod h, (c+h/2) mod h).
cudaError_t launch_gen_crop_pupil(const float2 *S, int H, const float2 *P, int h, const int2 *led,
                                  int z_off, int nb, float2 *out, cudaStream_t st);

// Stitch (fused_deconvPIE_shifted, kernels.cuh:95-116, as a gather): G[u] = sum over the
// batch's LEDs covering spectrum pixel u, in LED order with compensated summation, of
// conj(P(r, c)) X_l(shift(r, c)) / H^2.  Only the centred box rows [rlo, rlo + rspan) x
// cols [clo, clo + cspan) (modulo H) are written; the caller clears G first.
cudaError_t launch_gen_stitch(const float2 *X, int h, const float2 *P, const int2 *led, int z_off,
                              int nb, int H, int rlo, int rspan, int clo, int cspan, float2 *G,
                              cudaStream_t st);

// Pupil gradient (kernels.cuh:118-128): dP(r, c) = sum_l conj(sub_l(r, c)) X_l(shift(r, c)),
// LED order, compensated, sub_l the LED's crop of S.
cudaError_t launch_gen_pupil_grad(const float2 *S, int H, const float2 *X, int h, const int2 *led,
                                  int z_off, int nb, float2 *dP, cudaStream_t st);

// Object RMSprop (constrained_RMSprop_both, kernels.cuh:364-382): m = beta m + (1-beta)|g|^2,
// O -= g lr / (sqrt(m) + eps).
cudaError_t launch_rmsprop_object(float2 *O, float *m, const float2 *g, size_t n, float lr,
                                  float beta, float eps, cudaStream_t st);

}  // namespace fpm

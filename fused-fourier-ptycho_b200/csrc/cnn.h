// Learned warm start: a small convolutional encoder-decoder that maps the central
// bright-field frames of a stack to the real and imaginary parts of a low-resolution
// object estimate, trained on pairs the plain reconstruction produces.  No counterpart
// in the reference (its initial object is imresize(Y_1, pratio) with zero phase,
// codes_v2/main_run_FPM.m:48).
//
// Kernels (cnn.cu): 3x3 convolutions (stride 1, zero padding 1) as implicit GEMMs on the
// fifth-generation tensor cores (tcgen05: BF16 operands staged in shared memory, FP32
// accumulators in tensor memory), their data and weight gradients (the weight gradient
// split over the pixel axis into ordered partials), bias gradients, ReLU, 2x2 average
// pooling, 2x nearest up-sampling, additions, the mean-squared loss and an Adam step on
// FP32 master weights with BF16 copies.  Activations are FP32 in memory, NCHW; operands
// are rounded to BF16 as they are staged into shared memory.
//
// BF16 weights are kept in padded tap-major rows: layer weights W[co][ci][ky][kx] of a
// convolution with Cin inputs and Cout outputs as padded_rows(Cout) rows of
// padded_taps(Cin) values, W[co][ci][ky][kx] at co * padded_taps(Cin) + (3 ky + kx) Cin + ci,
// zero in every pad.  Every convolution takes
// a device int *flag that a tensor-core wait which runs out sets to 1.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstddef>

namespace fpm {
namespace cnn {

int padded_taps(int cin);   // 9 cin rounded up to 64
int padded_rows(int c);     // c rounded up to 16
// out[n][co][y][x] = bias[co] + sum_{ci,ky,kx} W[co][ci][ky][kx] in[n][ci][y+ky-1][x+kx-1]
// (W: BF16 padded rows; bias may be null; Cout <= 256), then max(out, 0) with relu
cudaError_t conv3x3_forward(const float *in, int N, int Cin, int Hh, int Ww,
                            const __nv_bfloat16 *W, const float *bias, int Cout, float *out,
                            bool relu, int *flag, cudaStream_t st);
// Wt[ci][co][2-ky][2-kx] = W[co][ci][ky][kx], both in padded tap-major rows (Wt:
// padded_rows(Cin) rows of padded_taps(Cout), pads left as they are): the data gradient is
// conv3x3_forward of the output gradient with Wt
cudaError_t conv3x3_flip(const __nv_bfloat16 *W, int Cout, int Cin, __nv_bfloat16 *Wt,
                         cudaStream_t st);
// dW[co][ci][ky][kx] = sum_{n,y,x} dout[n][co][y][x] in[n][ci][y+ky-1][x+kx-1], FP32;
// work: splits * Cout * Cin * 9 floats of partials, summed in split order
cudaError_t conv3x3_weight_grad(const float *in, const float *dout, int N, int Cin, int Hh,
                                int Ww, int Cout, float *dW, float *work, int splits, int *flag,
                                cudaStream_t st);
// the split count conv3x3_weight_grad is meant to get (work holds that many partials)
int conv3x3_weight_grad_splits(int N, int Hh, int Ww, int Cin);
// db[c] = sum_{n,p} dout[n][c][p] (ordered: bias_grad_splits(N, HW) partials per channel in
// work, C times that many floats)
int bias_grad_splits(int N, int HW);
cudaError_t bias_grad(const float *dout, int N, int C, int HW, float *db, float *work,
                      cudaStream_t st);

// dx = dy where y > 0 else 0 (in place on dy)
cudaError_t relu_backward(float *dy, const float *y, size_t n, cudaStream_t st);
// out = a + b (out may alias a)
cudaError_t add(const float *a, const float *b, float *out, size_t n, cudaStream_t st);
// 2x2 average pooling of planes of Hh x Ww (even) -> Hh/2 x Ww/2, and its gradient
cudaError_t pool_forward(const float *in, int planes, int Hh, int Ww, float *out, cudaStream_t st);
cudaError_t pool_backward(const float *dout, int planes, int Hh, int Ww, float *din,
                          cudaStream_t st);
// 2x nearest up-sampling of planes of Hh x Ww -> 2Hh x 2Ww, and its gradient (sum of 4)
cudaError_t up_forward(const float *in, int planes, int Hh, int Ww, float *out, cudaStream_t st);
cudaError_t up_backward(const float *dout, int planes, int Hh, int Ww, float *din,
                        cudaStream_t st);
// loss = sum (y - t)^2 / n (FP64, ordered), dy = 2 (y - t) / n
cudaError_t mse(const float *y, const float *t, size_t n, float *dy, double *loss,
                double *work, cudaStream_t st);
// Adam on FP32 master weights w (m, v moments) of a convolution with cin inputs, their BF16
// copy wb (may be null) in padded tap-major rows of ldb, step t >= 1
cudaError_t adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, size_t n,
                 int cin, int ldb, float lr, float b1, float b2, float eps, int t,
                 cudaStream_t st);
cudaError_t to_bf16(const float *w, __nv_bfloat16 *wb, size_t n, int cin, int ldb,
                    cudaStream_t st);

}  // namespace cnn
}  // namespace fpm

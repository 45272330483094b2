// Fused per-batch pipeline: low-resolution passes L1-L4 and the pruned
// large-array passes A, B, C (see pipeline.cu for the data flow).
#pragma once

#include <cuda_runtime.h>

#include "engine.h"

namespace fpm {

enum LossKind : int { kLossAnisotropic = 0, kLossIsotropic = 1 };

// One mini-batch's crop box.  Centred rows [rlo, rlo + rspan) and columns
// [clo, clo + cspan), modulo H; Ru0 / Cu0 are the matching un-shifted starts.
struct BatchGeom {
    int H = 0, h = 0, pratio = 0;
    int z_off = 0, nb = 0;
    int rlo = 0, rspan = 0, clo = 0, cspan = 0;
    int Ru0 = 0, Cu0 = 0;
    // crop rows / columns [pr_lo, pr_hi) x [pc_lo, pc_hi) (centred h x h frame) outside
    // which the pupil is zero: the crop there contributes nothing and the gradient
    // spectrum there is never used, so the box above covers only this part of each crop
    int pr_lo = 0, pr_hi = 0, pc_lo = 0, pc_hi = 0;
    int loss = 0;   // LossKind
    // the per-LED field buffer already holds zeros in the crop columns outside
    // [pc_lo, pc_hi) (cleared once per solve), so L1 writes only the supported columns
    int t1_clean = 0;
    // weights of the gradient terms (fpm_pie_weights): 0 none, 1 ePIE, 2 tPIE
    int pie = 0;
};

// Two-level twiddle tables (fft_core.cuh) for the low-res length h and the large length H.
struct Twiddles {
    const float2 *lo_hi = nullptr, *lo_lo = nullptr;  // length h
    const float2 *hi_hi = nullptr, *hi_lo = nullptr;  // length H
};

// Workspace of one batch.
struct BatchBufs {
    const float2 *Sbox = nullptr;  // [cspan][rspan] spectrum inside the box (leading dim rspan)
    float2 *T1 = nullptr;          // [group][h][h] per-LED field (group-local pages)
    float *Rs = nullptr;           // [group][h][h] residual |z|/(h^2 p^2) - Y (separate L2, L3)
    float2 *T2 = nullptr;          // [group][h][h] output of the fused L2 + L3 pass
    float2 *Xs = nullptr;          // [nb][h][h] row-major fftshift'ed gradient spectrum
    double *parts = nullptr;       // loss partials of the batch
    int *flag = nullptr;           // set by a kernel whose bounded wait gave up
};

bool pipeline_supported(int h, int H);
int lr_blocks(int h, int nl);  // CTAs of one L-pass over nl LEDs

// low-resolution passes over LEDs [l0, l0 + nl) of the batch (T1 / Rs group-local)
cudaError_t launch_lr_cols_inv(const BatchGeom &g, const int2 *led, const float2 *P, BatchBufs b,
                               int l0, int nl, const Twiddles &tw, cudaStream_t st);
cudaError_t launch_lr_rows_inv(const BatchGeom &g, StackView Y, BatchBufs b, int l0, int nl,
                               const Twiddles &tw, cudaStream_t st);
cudaError_t launch_lr_rows_fwd(const BatchGeom &g, BatchBufs b, int l0, int nl, int part_off,
                               const Twiddles &tw, cudaStream_t st);
// L2 + L3 in one pass (h in [128, 2048]): T1 -> T2, loss partials at parts + part_off,
// lr_rows_fused_blocks(h, nl) of them; reads the amplitude rows Y.rows
// (launch_amplitude_rows), not the stack itself.
bool lr_rows_fused_supported(int h);
int lr_rows_fused_blocks(int h, int nl);
cudaError_t launch_lr_rows_fused(const BatchGeom &g, StackView Y, BatchBufs b, int l0, int nl,
                                 int part_off, const Twiddles &tw, cudaStream_t st);
// L4 over src (T1 after separate L2, L3; T2 after the fused pass) -> Xs
cudaError_t launch_lr_cols_fwd(const BatchGeom &g, const float2 *src, BatchBufs b, int l0,
                               int nl, const Twiddles &tw, cudaStream_t st);
// ePIE / tPIE weights of the gradient terms (fpm_forward_GPU.m:64-76).  scratch: 1 + nb
// unsigned, zeroed by launch_pie_prepare; [0] max|P|^2, [1 + l] max|sub_l|^2 (float bits)
cudaError_t launch_pie_prepare(const BatchGeom &g, const float2 *P, const int2 *led,
                               const float2 *Sbox, unsigned *scratch, cudaStream_t st);
// Pt (row-major conj(P)/H^2) times the object-term weight of g.pie
cudaError_t launch_pie_object_weights(const BatchGeom &g, float2 *Pt, const unsigned *scratch,
                                      cudaStream_t st);
cudaError_t launch_lr_pupil_grad(const BatchGeom &g, const int2 *led, BatchBufs b, float2 *dP,
                                 cudaStream_t st,
                                 const unsigned *pie_scratch = nullptr);

// Pass A: gradient spectrum rows of the box -> inverse FFT along the rows ->
// Ur [rspan][H] (row-major).  Pt is the conjugated pupil transposed to row-major
// and scaled by 1/H^2: Pt[r*h + c] = conj(P[c*h + r]) / H^2.
cudaError_t launch_big_rows_inv(const BatchGeom &g, const int2 *led, const float2 *Pt,
                                const float2 *Xs, float2 *Ur, const Twiddles &tw,
                                cudaStream_t st);

enum BigColsMode : int { kColsForward = 0, kColsUpdate = 1, kColsGradient = 2 };
// Pass B over every column c:
//   kColsForward : V[c][i] = FFT_r(O[c])[(Ru0n + i) mod H], i < rspan_n
//   kColsUpdate  : g = IFFT_r(U[c] placed at rows Ru0 + i); RMSprop(O, m); V from FFT_r(O')
//                  (no V when rspan_n == 0)
//   kColsGradient: g = IFFT_r(U[c]) written to out[c]
struct ColsArgs {
    int mode = kColsForward;
    int H = 0;
    const float2 *U = nullptr;
    int ldU = 0, Ru0 = 0, rspan = 0;
    float2 *O = nullptr;
    float *m = nullptr;
    float lr = 0.f, beta = 0.f, eps = 0.f;
    float2 *V = nullptr;
    int ldV = 0, Ru0n = 0, rspan_n = 0;
    float2 *gout = nullptr;
    int *err = nullptr;   // device flag set when a bounded wait gives up (update mode)
};
cudaError_t launch_big_cols(const ColsArgs &a, const Twiddles &tw, cudaStream_t st);

// Pass C: rows i < rspan_n of Vr [rspan_n][H] -> FFT along the rows ->
// Sboxr[i][j] = row[(Cu0n + j) mod H] (row-major, leading dim cspan_n).
// err: device flag for the persistent form's bounded waits (null: the one-row-per-CTA form)
cudaError_t launch_big_rows_fwd(int H, const float2 *Vr, int rspan_n, int Cu0n, int cspan_n,
                                float2 *Sboxr, const Twiddles &tw, cudaStream_t st,
                                int *err = nullptr);

// A bounded wait that runs out on purpose (no copy delivers the bytes it waits for): sets
// *flag after `limit` SM clocks and returns.
cudaError_t launch_wait_selftest(int *flag, long long limit, cudaStream_t st);

}  // namespace fpm

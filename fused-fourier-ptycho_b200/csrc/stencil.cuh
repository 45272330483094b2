// Loss-gradient stencil of the feature-domain loss, shared by the fused row pass
// (pipeline.cu) and the standalone loss-gradient kernel (kernels_lowres.cu).
#pragma once

#include "common.cuh"
#include "pipeline.h"

namespace fpm {

// Loss-gradient stencil at one pixel from the residuals around it:
// a = res(r, c), right = res(r, c+1), left = res(r, c-1), down = res(r+1, c),
// up = res(r-1, c), dl = res(r+1, c-1), ur = res(r-1, c+1).  Returns d (before the
// pratio^2 scale) and adds the pixel's loss term to lsum.
//   anisotropic (v3, kernels.cuh:234-263): sign(Rx(c-1)) - sign(Rx) + sign(Ry(r-1)) - sign(Ry)
//   isotropic (codes/func_ware/misc/ret_loss.m:7-11,18-19): ox = Rx / (|R| + 1e-5),
//     oy = Ry / (|R| + 1e-5), d = (ox(c-1) - ox) + (oy(r-1) - oy), loss |R| = sqrt(Rx²+Ry²)
template <int LOSS>
__device__ __forceinline__ float stencil(float a, float right, float left, float down, float up,
                                         float dl, float ur, double &lsum) {
    const float rx = right - a;                  // Rx(r, c)
    const float ry = down - a;                   // Ry(r, c)
    if (LOSS == kLossAnisotropic) {
        const float oxm = sign1(a - left);       // sign Rx(r, c-1)
        const float oym = sign1(a - up);         // sign Ry(r-1, c)
        lsum += (double)fabsf(rx) + (double)fabsf(ry);
        return oxm - sign1(rx) + oym - sign1(ry);
    } else {
        const float n = sqrtf(__fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)));
        const float den = n + 1e-5f;
        const float ox = rx / den, oy = ry / den;
        const float rxm = a - left, rym = dl - left;       // R(r, c-1) differences
        const float oxm = rxm / (sqrtf(__fadd_rn(__fmul_rn(rxm, rxm), __fmul_rn(rym, rym))) + 1e-5f);
        const float ryu = a - up, rxu = ur - up;           // R(r-1, c) differences
        const float oyu = ryu / (sqrtf(__fadd_rn(__fmul_rn(rxu, rxu), __fmul_rn(ryu, ryu))) + 1e-5f);
        lsum += (double)n;
        return (oxm - ox) + (oyu - oy);
    }
}

}  // namespace fpm

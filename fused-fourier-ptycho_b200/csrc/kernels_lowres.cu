// Standalone loss-gradient stage on whole h x h fields: the kernel of the
// allocation-free entry point (noalloc.cu).  The reconstruction itself runs the
// same arithmetic fused into the low-resolution row pass of pipeline.cu.
//
// Layout: every h x h image is column-major (index c*h + r); threads of a warp
// walk the row index r, so global accesses are coalesced.  Batches are pages
// of h*h elements.
#include "common.cuh"
#include "engine.h"
#include "stencil.cuh"

namespace fpm {

// ---------------------------------------------------------------------------
// feature-domain loss gradient (differenceKernel_acc, cuFPM_v3/cuda/kernels.cuh:197-275)
//   res   = |z| / (h² p²) - Y
//   ox(c) = sign(res(r, c+1) - res(r, c)),  oy(r) = sign(res(r+1, c) - res(r, c))  (periodic)
//   d     = (ox(c-1) - ox(c) + oy(r-1) - oy(r)) * p²
//   out   = d * z/|z|  (0 where |z| = 0)
// plus the loss partial sum of |res(c+1)-res(c)| + |res(r+1)-res(r)| per tile
// (benchmark/func_ware/ret_loss.m:13, the reference never forms it).
// Tile: 32 rows x 32 cols, 256 threads (32 along r, 8 along c, 4 cols each);
// the residual tile with a one-pixel periodic halo is staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int kTR = 32;
constexpr int kTC = 32;

template <int TYPE>
__device__ __forceinline__ float load_amp(const StackView &Y, size_t idx, float mn, float inv_den,
                                          float range) {
    if (TYPE == kStackF32) {
        return static_cast<const float *>(Y.ptr)[idx];
    } else {
        // single-precision (I - min) / (max - min), then sqrt: codes_v2/main_run_FPM.m:43-45
        const float x = (float)static_cast<const uint16_t *>(Y.ptr)[idx] - mn;
        return range > 0.f ? sqrtf(x / range) : sqrtf(x);
    }
}

template <int TYPE, int LOSS>
__global__ void __launch_bounds__(256) k_feature_grad(const float2 *__restrict__ Z, StackView Y,
                                                       int z_off, int h, int pratio,
                                                       float2 *__restrict__ out,
                                                       double *__restrict__ loss_part) {
    __shared__ float s_res[kTC + 2][kTR + 2];
    __shared__ double s_red[8];
    const int l = blockIdx.z;
    const size_t plane = (size_t)h * h;
    const int r0 = blockIdx.x * kTR;
    const int c0 = blockIdx.y * kTC;
    const float2 *z = Z + l * plane;
    const size_t ypage = (size_t)(z_off + l) * plane;
    const float ratio = (float)((double)h * h * pratio * pratio);
    const float gscale = (float)(pratio * pratio);
    float mn = 0.f, range = 0.f;
    if (TYPE == kStackU16) {
        mn = (float)Y.minmax[0];
        range = (float)(Y.minmax[1] - Y.minmax[0]);
    }
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < (kTR + 2) * (kTC + 2); i += 256) {
        const int lr = i % (kTR + 2);
        const int lc = i / (kTR + 2);
        const int r = pmod(r0 - 1 + lr, h);
        const int c = pmod(c0 - 1 + lc, h);
        const size_t idx = (size_t)c * h + r;
        const float2 v = z[idx];
        const float a = sqrtf(v.x * v.x + v.y * v.y) / ratio;
        s_res[lc][lr] = a - load_amp<TYPE>(Y, ypage + idx, mn, 0.f, range);
    }
    __syncthreads();

    double lsum = 0.0;
    const int lr = threadIdx.x + 1;
    const int r = r0 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kTC / 8; ++k) {
        const int lc = threadIdx.y + 8 * k + 1;
        const int c = c0 + threadIdx.y + 8 * k;
        if (r < h && c < h) {
            // right, left, down, up, down-left, up-right neighbours of (r, c)
            const float d = stencil<LOSS>(s_res[lc][lr], s_res[lc + 1][lr], s_res[lc - 1][lr],
                                          s_res[lc][lr + 1], s_res[lc][lr - 1],
                                          s_res[lc - 1][lr + 1], s_res[lc + 1][lr - 1], lsum) *
                            gscale;
            const size_t idx = (size_t)c * h + r;
            const float2 v = z[idx];
            const float mag = sqrtf(v.x * v.x + v.y * v.y);
            float2 o = make_float2(0.f, 0.f);
            if (mag > 0.f) {
                const float inv = 1.0f / mag;
                o.x = v.x * inv * d;
                o.y = v.y * inv * d;
            }
            out[l * plane + idx] = o;
        }
    }
    // fixed-order block reduction of the loss partial
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if (threadIdx.x == 0) s_red[threadIdx.y] = lsum;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += s_red[w];
        loss_part[((size_t)l * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
    }
}

long long feature_grad_blocks_per_image(int h) {
    const long long t = ((long long)h + kTR - 1) / kTR;   // 64-bit: t * t overflows int past h ~ 1.48e6
    return t * t;
}

cudaError_t launch_feature_grad(const float2 *Z, StackView Y, int z_off, int nb, int h,
                                int pratio, float2 *out, double *loss_part, cudaStream_t st,
                                int loss) {
    const int t = (h + kTR - 1) / kTR;
    dim3 grid(t, t, nb), block(32, 8);
    const bool u16 = Y.type == kStackU16, iso = loss == kLossIsotropic;
    if (u16 && !iso)
        k_feature_grad<kStackU16, kLossAnisotropic><<<grid, block, 0, st>>>(Z, Y, z_off, h, pratio,
                                                                          out, loss_part);
    else if (u16)
        k_feature_grad<kStackU16, kLossIsotropic><<<grid, block, 0, st>>>(Z, Y, z_off, h, pratio,
                                                                        out, loss_part);
    else if (!iso)
        k_feature_grad<kStackF32, kLossAnisotropic><<<grid, block, 0, st>>>(Z, Y, z_off, h, pratio,
                                                                          out, loss_part);
    else
        k_feature_grad<kStackF32, kLossIsotropic><<<grid, block, 0, st>>>(Z, Y, z_off, h, pratio,
                                                                        out, loss_part);
    return cudaGetLastError();
}

}  // namespace fpm

// Per-LED (low-resolution) stages of one mini-batch.
//
// Layout: every h x h image is column-major (index c*h + r); threads of a warp
// walk the row index r, so global accesses are coalesced.  Batches are pages
// of h*h elements.  The crop of LED l covers centred-spectrum rows
// kt-1 .. kt-2+h and columns kl-1 .. kl-2+h, taken modulo H and mapped to the
// un-shifted spectrum by +H/2 (cuFPM_v3/cuda/kernels.cuh:43-47).
#include "common.cuh"
#include "engine.h"

namespace fpm {

// ---------------------------------------------------------------------------
// crop x pupil, stored ifftshift'ed, ready for the inverse FFT
// (fused_getSubpupil_shifted, cuFPM_v3/cuda/kernels.cuh:19-65).
// T[l][q] = S[crop_l(p)] * P[p] with q = (p + h/2) mod h on both axes.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_crop_pupil(const float2 *__restrict__ S,
                                                     const float2 *__restrict__ P,
                                                     const int2 *__restrict__ led, int z_off,
                                                     int h, int H, float2 *__restrict__ T) {
    const int l = blockIdx.y;
    const size_t plane = (size_t)h * h;
    const int2 k = led[z_off + l];           // (kl, kt)
    const int hh = h >> 1;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < plane;
         q += (size_t)gridDim.x * blockDim.x) {
        const int rq = (int)(q % h);
        const int cq = (int)(q / h);
        const int r = rq + hh >= h ? rq + hh - h : rq + hh;
        const int c = cq + hh >= h ? cq + hh - h : cq + hh;
        const int R = pmod(k.y - 1 + r + (H >> 1), H);
        const int C = pmod(k.x - 1 + c + (H >> 1), H);
        const float2 s = S[(size_t)C * H + R];
        const float2 p = P[(size_t)c * h + r];
        T[l * plane + q] = cmul(s, p);
    }
}

cudaError_t launch_crop_pupil(const float2 *S, const float2 *P, const int2 *led, int z_off,
                              int nb, int h, int H, float2 *T, cudaStream_t st) {
    const size_t plane = (size_t)h * h;
    unsigned gx = (unsigned)((plane + 255) / 256);
    if (gx > 4096u) gx = 4096u;
    k_crop_pupil<<<dim3(gx, nb), 256, 0, st>>>(S, P, led, z_off, h, H, T);
    return cudaGetLastError();
}

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

template <int TYPE>
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
            const float a = s_res[lc][lr];
            const float rx = s_res[lc + 1][lr] - a;
            const float ry = s_res[lc][lr + 1] - a;
            const float ox = sign1(rx);
            const float oy = sign1(ry);
            const float ox_m = sign1(a - s_res[lc - 1][lr]);
            const float oy_m = sign1(a - s_res[lc][lr - 1]);
            const float d = (ox_m - ox + oy_m - oy) * gscale;
            lsum += (double)fabsf(rx) + (double)fabsf(ry);
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

int feature_grad_blocks_per_image(int h) {
    const int t = (h + kTR - 1) / kTR;
    return t * t;
}

cudaError_t launch_feature_grad(const float2 *Z, StackView Y, int z_off, int nb, int h,
                                int pratio, float2 *out, double *loss_part, cudaStream_t st) {
    const int t = (h + kTR - 1) / kTR;
    dim3 grid(t, t, nb), block(32, 8);
    if (Y.type == kStackU16)
        k_feature_grad<kStackU16><<<grid, block, 0, st>>>(Z, Y, z_off, h, pratio, out, loss_part);
    else
        k_feature_grad<kStackF32><<<grid, block, 0, st>>>(Z, Y, z_off, h, pratio, out, loss_part);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// stitch (fused_deconvPIE_shifted's dldw part, cuFPM_v3/cuda/kernels.cuh:95-116), as a
// deterministic gather: every un-shifted G pixel is written exactly once with
//   G = sum over the batch's LEDs, in LED order, of conj(P) * X_l / H²
// (X_l read at the fftshift'ed index), Kahan-compensated; pixels outside the
// crop box are written 0, so G needs no separate clearing.
// ---------------------------------------------------------------------------
constexpr int kMaxBatch = 1024;

__global__ void __launch_bounds__(256) k_stitch_gather(const float2 *__restrict__ X,
                                                        const float2 *__restrict__ P,
                                                        const int2 *__restrict__ led, int z_off,
                                                        int nb, int h, int H, Box box,
                                                        float2 *__restrict__ G) {
    extern __shared__ int2 s_led[];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_led[i] = led[z_off + i];
    __syncthreads();
    const size_t plane = (size_t)h * h;
    const int hh = h >> 1;
    const float inv_H2 = 1.0f / (float)((double)H * H);
    const size_t total = (size_t)H * H;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (size_t)gridDim.x * blockDim.x) {
        const int Ru = (int)(g % H);
        const int Cu = (int)(g / H);
        const int R = Ru + (H >> 1) >= H ? Ru + (H >> 1) - H : Ru + (H >> 1);   // centred row
        const int C = Cu + (H >> 1) >= H ? Cu + (H >> 1) - H : Cu + (H >> 1);
        KahanC acc;
        if (pmod(R - box.r_lo, H) < box.r_span && pmod(C - box.c_lo, H) < box.c_span) {
            for (int i = 0; i < nb; ++i) {
                const int2 k = s_led[i];
                const int r = pmod(R - (k.y - 1), H);
                const int c = pmod(C - (k.x - 1), H);
                if (r < h && c < h) {
                    const int rs = r + hh >= h ? r + hh - h : r + hh;
                    const int cs = c + hh >= h ? c + hh - h : c + hh;
                    const float2 x = X[i * plane + (size_t)cs * h + rs];
                    const float2 p = P[(size_t)c * h + r];
                    float2 gw = cmul_conj(x, p);
                    gw.x *= inv_H2;
                    gw.y *= inv_H2;
                    acc.add(gw);
                }
            }
        }
        G[g] = acc.s;
    }
}

cudaError_t launch_stitch_gather(const float2 *X, const float2 *P, const int2 *led, int z_off,
                                 int nb, int h, int H, Box box, float2 *G, cudaStream_t st) {
    if (nb > kMaxBatch) return cudaErrorInvalidValue;
    const size_t total = (size_t)H * H;
    size_t gx = (total + 255) / 256;
    const size_t cap = (size_t)kB200SMs * 8 * 16;
    if (gx > cap) gx = cap;
    k_stitch_gather<<<(unsigned)gx, 256, nb * sizeof(int2), st>>>(X, P, led, z_off, nb, h, H, box,
                                                                  G);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// pupil gradient (fused_deconvPIE_shifted's dldp part, kernels.cuh:118-128):
//   dP(p) = sum over the batch's LEDs, in order, of conj(sub_l(p)) * X_l(p)
// with sub_l re-read from the spectrum (the reference keeps a copy, `subwave`).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_pupil_grad(const float2 *__restrict__ S,
                                                     const float2 *__restrict__ X,
                                                     const int2 *__restrict__ led, int z_off,
                                                     int nb, int h, int H,
                                                     float2 *__restrict__ dP) {
    extern __shared__ int2 s_led[];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_led[i] = led[z_off + i];
    __syncthreads();
    const size_t plane = (size_t)h * h;
    const int hh = h >> 1;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < plane;
         p += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(p % h);
        const int c = (int)(p / h);
        const int rs = r + hh >= h ? r + hh - h : r + hh;
        const int cs = c + hh >= h ? c + hh - h : c + hh;
        const size_t xs = (size_t)cs * h + rs;
        KahanC acc;
        for (int i = 0; i < nb; ++i) {
            const int2 k = s_led[i];
            const int R = pmod(k.y - 1 + r + (H >> 1), H);
            const int C = pmod(k.x - 1 + c + (H >> 1), H);
            const float2 s = S[(size_t)C * H + R];
            const float2 x = X[i * plane + xs];
            acc.add(cmul_conj(x, s));
        }
        dP[p] = acc.s;
    }
}

cudaError_t launch_pupil_grad(const float2 *S, const float2 *X, const int2 *led, int z_off,
                              int nb, int h, int H, float2 *dP, cudaStream_t st) {
    if (nb > kMaxBatch) return cudaErrorInvalidValue;
    const size_t plane = (size_t)h * h;
    size_t gx = (plane + 255) / 256;
    if (gx > (size_t)kB200SMs * 16) gx = (size_t)kB200SMs * 16;
    k_pupil_grad<<<(unsigned)gx, 256, nb * sizeof(int2), st>>>(S, X, led, z_off, nb, h, H, dP);
    return cudaGetLastError();
}

}  // namespace fpm

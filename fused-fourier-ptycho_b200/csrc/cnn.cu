// Kernels of the learned warm start (cnn.h).
//
// Convolutions are implicit GEMMs on the tensor cores: a CTA of four warps computes a
// 64 x 64 tile of C = A B, staging 64 x 32 and 32 x 64 BF16 tiles of A and B in shared
// memory (rounded from the FP32 activations as they are gathered), each warp a 32 x 32
// block of 2 x 2 WMMA 16x16x16 fragments with FP32 accumulators; the tile goes back
// through shared memory to a per-GEMM epilogue.  Gathers and stores run with consecutive
// threads on consecutive pixels.
//   forward      M = N*H*W pixels, N = Cout, K = Cin*9: A = im2col(in), B = W^T
//   data grad    the forward GEMM on the output gradient with the flipped weights
//   weight grad  M = Cout, N = Cin*9, K = N*H*W: A = dout, B = im2col(in)^T, split over K
//                into partials that one more pass sums in split order (deterministic)
#include <mma.h>

#include <algorithm>

#include "cnn.h"
#include "common.cuh"

namespace fpm {
namespace cnn {

namespace {

using namespace nvcuda;

constexpr int BM = 64, BN = 64, BK = 32, GT = 128;
constexpr int LDA = BK + 8, LDB = BN + 8, LDC = BN + 4;

unsigned grid_1d(size_t n) {
    return (unsigned)std::min<size_t>((n + 255) / 256, (size_t)kB200SMs * 16);
}

// Generic tile GEMM; Op supplies a(m, k), b(k, n) as floats, c(m, n, value, split) and
// which index varies fastest across threads when gathering / storing.
template <class Op>
__global__ void __launch_bounds__(GT) k_gemm(Op op, int M, int N, int K, int kchunk) {
    __shared__ __align__(32) __nv_bfloat16 sA[BM * LDA];
    __shared__ __align__(32) __nv_bfloat16 sB[BK * LDB];
    __shared__ __align__(32) float sC[BM * LDC];
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
    const int warp = threadIdx.x >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.0f);
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        for (int i = threadIdx.x; i < BM * BK; i += GT) {
            const int r = Op::A_ROW_FAST ? i % BM : i / BK;
            const int c = Op::A_ROW_FAST ? i / BM : i % BK;
            const int m = m0 + r, k = k0 + c;
            sA[r * LDA + c] = __float2bfloat16_rn(m < M && k < kend ? op.a(m, k) : 0.f);
        }
        for (int i = threadIdx.x; i < BK * BN; i += GT) {
            const int r = Op::B_ROW_FAST ? i % BK : i / BN;
            const int c = Op::B_ROW_FAST ? i / BK : i % BN;
            const int k = k0 + r, n = n0 + c;
            sB[r * LDB + c] = __float2bfloat16_rn(k < kend && n < N ? op.b(k, n) : 0.f);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa[2];
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) wmma::load_matrix_sync(fa[i], sA + (wm + 16 * i) * LDA + kk, LDA);
#pragma unroll
            for (int j = 0; j < 2; ++j) wmma::load_matrix_sync(fb[j], sB + kk * LDB + wn + 16 * j, LDB);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
            wmma::store_matrix_sync(sC + (wm + 16 * i) * LDC + wn + 16 * j, acc[i][j], LDC,
                                    wmma::mem_row_major);
    __syncthreads();
    for (int i = threadIdx.x; i < BM * BN; i += GT) {
        const int r = Op::C_ROW_FAST ? i % BM : i / BN;
        const int c = Op::C_ROW_FAST ? i / BM : i % BN;
        const int m = m0 + r, n = n0 + c;
        if (m < M && n < N) op.c(m, n, sC[r * LDC + c], blockIdx.z);
    }
}

// in[n][ci][y+ky-1][x+kx-1] for pixel q = (n, y, x) and tap j = (ci, ky, kx), 0 outside
__device__ __forceinline__ float im2col(const float *in, int Cin, int Hh, int Ww, int q, int j) {
    const int HW = Hh * Ww;
    const int n = q / HW, p = q - n * HW;
    const int y = p / Ww, x = p - y * Ww;
    const int ci = j / 9, t = j - ci * 9;
    const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
    if (yy < 0 || yy >= Hh || xx < 0 || xx >= Ww) return 0.f;
    return in[((size_t)(n * Cin + ci) * Hh + yy) * Ww + xx];
}

struct ConvFwd {
    static constexpr bool A_ROW_FAST = true, B_ROW_FAST = true, C_ROW_FAST = true;
    const float *in;
    const __nv_bfloat16 *W;
    const float *bias;
    float *out;
    int Cin, Hh, Ww, Cout;
    __device__ float a(int m, int k) const { return im2col(in, Cin, Hh, Ww, m, k); }
    __device__ float b(int k, int co) const { return __bfloat162float(W[(size_t)co * Cin * 9 + k]); }
    __device__ void c(int m, int co, float v, int) const {
        const int HW = Hh * Ww;
        const int n = m / HW, p = m - n * HW;
        out[(size_t)(n * Cout + co) * HW + p] = bias ? v + bias[co] : v;
    }
};

struct ConvWgrad {
    static constexpr bool A_ROW_FAST = false, B_ROW_FAST = true, C_ROW_FAST = false;
    const float *in, *dout;
    float *part;
    int Cin, Hh, Ww, Cout;
    __device__ float a(int co, int q) const {
        const int HW = Hh * Ww;
        const int n = q / HW, p = q - n * HW;
        return dout[(size_t)(n * Cout + co) * HW + p];
    }
    __device__ float b(int q, int j) const { return im2col(in, Cin, Hh, Ww, q, j); }
    __device__ void c(int co, int j, float v, int z) const {
        part[((size_t)z * Cout + co) * Cin * 9 + j] = v;
    }
};

__global__ void k_flip(const __nv_bfloat16 *W, int Cout, int Cin, __nv_bfloat16 *Wt) {
    const int total = Cout * Cin * 9;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int co = i / (Cin * 9), rem = i - co * Cin * 9;
        const int ci = rem / 9, t = rem - ci * 9;
        Wt[((size_t)ci * Cout + co) * 9 + (8 - t)] = W[i];    // (ky, kx) -> (2-ky, 2-kx)
    }
}

__global__ void k_sum_parts(const float *part, int splits, size_t n, float *out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < splits; ++z) s += part[(size_t)z * n + i];
        out[i] = s;
    }
}

// one block per channel, fixed order: thread-strided sums then a tree in shared memory
__global__ void __launch_bounds__(256) k_bias_grad(const float *dout, int N, int C, int HW,
                                                   float *db) {
    __shared__ float s[256];
    const int c = blockIdx.x;
    float acc = 0.f;
    for (int n = 0; n < N; ++n)
        for (int p = threadIdx.x; p < HW; p += 256) acc += dout[(size_t)(n * C + c) * HW + p];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[c] = s[0];
}

__global__ void k_relu(float *x, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = fmaxf(x[i], 0.f);
}

__global__ void k_relu_bwd(float *dy, const float *y, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        if (!(y[i] > 0.f)) dy[i] = 0.f;
}

__global__ void k_add(const float *a, const float *b, float *out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = a[i] + b[i];
}

__global__ void k_pool(const float *in, int planes, int Hh, int Ww, float *out) {
    const int ho = Hh / 2, wo = Ww / 2;
    const size_t total = (size_t)planes * ho * wo;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = i / ((size_t)ho * wo);
        const int q = (int)(i - pl * ho * wo), y = q / wo, x = q - y * wo;
        const float *s = in + pl * Hh * Ww + (size_t)(2 * y) * Ww + 2 * x;
        out[i] = 0.25f * ((s[0] + s[1]) + (s[Ww] + s[Ww + 1]));
    }
}

__global__ void k_pool_bwd(const float *dout, int planes, int Hh, int Ww, float *din) {
    const size_t total = (size_t)planes * Hh * Ww;
    const int wo = Ww / 2, ho = Hh / 2;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = i / ((size_t)Hh * Ww);
        const int q = (int)(i - pl * Hh * Ww), y = q / Ww, x = q - y * Ww;
        din[i] = 0.25f * dout[pl * ho * wo + (size_t)(y / 2) * wo + x / 2];
    }
}

__global__ void k_up(const float *in, int planes, int Hh, int Ww, float *out) {
    const int Ho = 2 * Hh, Wo = 2 * Ww;
    const size_t total = (size_t)planes * Ho * Wo;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = i / ((size_t)Ho * Wo);
        const int q = (int)(i - pl * Ho * Wo), y = q / Wo, x = q - y * Wo;
        out[i] = in[pl * Hh * Ww + (size_t)(y / 2) * Ww + x / 2];
    }
}

__global__ void k_up_bwd(const float *dout, int planes, int Hh, int Ww, float *din) {
    const size_t total = (size_t)planes * Hh * Ww;
    const int Wo = 2 * Ww;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = i / ((size_t)Hh * Ww);
        const int q = (int)(i - pl * Hh * Ww), y = q / Ww, x = q - y * Ww;
        const float *s = dout + pl * 4 * Hh * Ww + (size_t)(2 * y) * Wo + 2 * x;
        din[i] = (s[0] + s[1]) + (s[Wo] + s[Wo + 1]);
    }
}

constexpr int kMseBlocks = 256;

__global__ void __launch_bounds__(256) k_mse(const float *y, const float *t, size_t n, float *dy,
                                             double *work) {
    __shared__ double s[256];
    const float scale = (float)(2.0 / (double)n);
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        acc += (double)d * d;
        dy[i] = scale * d;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) work[blockIdx.x] = s[0];
}

__global__ void k_mse_final(const double *work, int nb, size_t n, double *loss) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += work[b];
        *loss = s / (double)n;
    }
}

__global__ void k_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, size_t n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void k_to_bf16(const float *w, __nv_bfloat16 *wb, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

template <class Op>
cudaError_t gemm(const Op &op, int M, int N, int K, int splits, cudaStream_t st) {
    if (M < 1 || N < 1 || K < 1) return cudaErrorInvalidValue;
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    const int sp = (K + kchunk - 1) / kchunk;
    const dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, sp);
    if (grid.y > 65535u || grid.z > 65535u) return cudaErrorInvalidValue;
    k_gemm<Op><<<grid, GT, 0, st>>>(op, M, N, K, kchunk);
    return cudaGetLastError();
}

}  // namespace

cudaError_t conv3x3_forward(const float *in, int N, int Cin, int Hh, int Ww,
                            const __nv_bfloat16 *W, const float *bias, int Cout, float *out,
                            cudaStream_t st) {
    ConvFwd op{in, W, bias, out, Cin, Hh, Ww, Cout};
    return gemm(op, N * Hh * Ww, Cout, Cin * 9, 1, st);
}

cudaError_t conv3x3_flip(const __nv_bfloat16 *W, int Cout, int Cin, __nv_bfloat16 *Wt,
                         cudaStream_t st) {
    k_flip<<<grid_1d((size_t)Cout * Cin * 9), 256, 0, st>>>(W, Cout, Cin, Wt);
    return cudaGetLastError();
}

int conv3x3_weight_grad_splits(int N, int Hh, int Ww) {
    const int K = N * Hh * Ww;
    return std::max(1, std::min(64, K / 2048));   // at least 2048 pixels per split
}

cudaError_t conv3x3_weight_grad(const float *in, const float *dout, int N, int Cin, int Hh,
                                int Ww, int Cout, float *dW, float *work, int splits,
                                cudaStream_t st) {
    const int K = N * Hh * Ww;
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    const int sp = (K + kchunk - 1) / kchunk;   // the splits the GEMM actually makes
    ConvWgrad op{in, dout, work, Cin, Hh, Ww, Cout};
    cudaError_t e = gemm(op, Cout, Cin * 9, K, splits, st);
    if (e != cudaSuccess) return e;
    const size_t n = (size_t)Cout * Cin * 9;
    k_sum_parts<<<grid_1d(n), 256, 0, st>>>(work, sp, n, dW);
    return cudaGetLastError();
}

cudaError_t bias_grad(const float *dout, int N, int C, int HW, float *db, cudaStream_t st) {
    k_bias_grad<<<C, 256, 0, st>>>(dout, N, C, HW, db);
    return cudaGetLastError();
}

cudaError_t relu_forward(float *x, size_t n, cudaStream_t st) {
    k_relu<<<grid_1d(n), 256, 0, st>>>(x, n);
    return cudaGetLastError();
}

cudaError_t relu_backward(float *dy, const float *y, size_t n, cudaStream_t st) {
    k_relu_bwd<<<grid_1d(n), 256, 0, st>>>(dy, y, n);
    return cudaGetLastError();
}

cudaError_t add(const float *a, const float *b, float *out, size_t n, cudaStream_t st) {
    k_add<<<grid_1d(n), 256, 0, st>>>(a, b, out, n);
    return cudaGetLastError();
}

cudaError_t pool_forward(const float *in, int planes, int Hh, int Ww, float *out, cudaStream_t st) {
    k_pool<<<grid_1d((size_t)planes * Hh * Ww / 4), 256, 0, st>>>(in, planes, Hh, Ww, out);
    return cudaGetLastError();
}

cudaError_t pool_backward(const float *dout, int planes, int Hh, int Ww, float *din,
                          cudaStream_t st) {
    k_pool_bwd<<<grid_1d((size_t)planes * Hh * Ww), 256, 0, st>>>(dout, planes, Hh, Ww, din);
    return cudaGetLastError();
}

cudaError_t up_forward(const float *in, int planes, int Hh, int Ww, float *out, cudaStream_t st) {
    k_up<<<grid_1d((size_t)planes * Hh * Ww * 4), 256, 0, st>>>(in, planes, Hh, Ww, out);
    return cudaGetLastError();
}

cudaError_t up_backward(const float *dout, int planes, int Hh, int Ww, float *din,
                        cudaStream_t st) {
    k_up_bwd<<<grid_1d((size_t)planes * Hh * Ww), 256, 0, st>>>(dout, planes, Hh, Ww, din);
    return cudaGetLastError();
}

cudaError_t mse(const float *y, const float *t, size_t n, float *dy, double *loss, double *work,
                cudaStream_t st) {
    k_mse<<<kMseBlocks, 256, 0, st>>>(y, t, n, dy, work);
    k_mse_final<<<1, 32, 0, st>>>(work, kMseBlocks, n, loss);
    return cudaGetLastError();
}

cudaError_t adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, size_t n,
                 float lr, float b1, float b2, float eps, int t, cudaStream_t st) {
    const float c1 = (float)(1.0 - std::pow((double)b1, t));
    const float c2 = (float)(1.0 - std::pow((double)b2, t));
    k_adam<<<grid_1d(n), 256, 0, st>>>(w, m, v, g, wb, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t to_bf16(const float *w, __nv_bfloat16 *wb, size_t n, cudaStream_t st) {
    k_to_bf16<<<grid_1d(n), 256, 0, st>>>(w, wb, n);
    return cudaGetLastError();
}

}  // namespace cnn
}  // namespace fpm

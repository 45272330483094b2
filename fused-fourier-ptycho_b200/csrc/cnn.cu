// Kernels of the learned warm start (cnn.h).
//
// Convolutions are implicit GEMMs on the fifth-generation tensor cores (tcgen05, umma.cuh):
// a CTA of 128 threads computes a 128-row tile of D = A B^T with all of B's rows (at most
// 256) as the MMA's N, the FP32 accumulator in tensor memory.  The threads stage the
// operands as BF16 (rounded from the FP32 activations as they are gathered, the weights
// already BF16) into two shared-memory stages of 64 K columns in the 128-byte swizzled
// K-major layout while one thread issues the MMAs of the other stage; the epilogue reads
// the accumulator back with tcgen05.ld, one TMEM lane per tile row.
//   forward      rows = N*H*W pixels, K = Cin*9, B = W (rows co): D = im2col(in) W^T
//   data grad    the forward GEMM on the output gradient with the flipped weights
//   weight grad  rows = Cin*9 taps, K = N*H*W pixels, B = dout (rows co): D = dW^T, split
//                over the pixels into partials that one more pass sums in split order
//                (deterministic)
// Gathers run with consecutive threads on consecutive pixels where the layout allows.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "cnn.h"
#include "common.cuh"
#include "tma.cuh"
#include "umma.cuh"

namespace fpm {
namespace cnn {

namespace {

constexpr int kTM = 128;              // MMA M: rows of a tile, one thread per row
constexpr int kTK = 64;               // K per stage: one 128-byte row of BF16
constexpr int kThreads = 128;
constexpr int kATile = kTM * 128;     // bytes of one A stage

unsigned grid_1d(size_t n) {
    return (unsigned)std::min<size_t>((n + 255) / 256, (size_t)kB200SMs * 16);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);   // lo at the lower address
    return *reinterpret_cast<const uint32_t *>(&p);
}

// 16-byte chunk c of row r of a swizzled K-major operand tile (umma.cuh)
__device__ __forceinline__ uint4 *chunk(uint8_t *tile, int r, int c) {
    return reinterpret_cast<uint4 *>(tile + r * 128 + ((c ^ (r & 7)) << 4));
}

// One tile of D = A B^T on the tensor cores: D (kTM rows x bn columns, FP32) in TMEM;
// A (kTM x K) and B (bn x K) staged as BF16 by the CTA's threads through two shared-
// memory stages of kTK columns each while the MMAs of the other stage run (one thread
// issues them, completion on one mbarrier per stage).  Op supplies
//   kdim()                         the GEMM's K (its M is the host's `rows`)
//   build_a(tile, m0, k0, scratch) row threadIdx.x of A, K columns k0 .. k0 + 63 (called by
//                                  every thread; scratch: kScratch floats of shared memory)
//   build_b(tile, bn, k0)          all bn rows of B, the same K columns
//   store(m, n0, v[16], split)     D(m, n0 .. n0 + 15) of K split `split`
// Blocks: x = M tile, z = K split (kchunk columns, a multiple of kTK).  A wait that
// runs out sets *flag and skips the epilogue; TMEM is always freed.
template <class Op>
__global__ void __launch_bounds__(kThreads) k_umma_gemm(Op op, int bn, int kchunk, int *flag) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t pad = (1024u - (umma::saddr(smem_raw) & 1023u)) & 1023u;
    uint8_t *base = smem_raw + pad;                      // swizzle atoms need 1024-byte bases
    uint8_t *sa[2] = {base, base + kATile};
    uint8_t *sb[2] = {base + 2 * kATile, base + 2 * kATile + bn * 128};
    uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * kATile + 2 * bn * 128);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 2);
    float *scratch = reinterpret_cast<float *>(bar + 4);   // Op::kScratch floats (16-byte aligned)
    const int warp = threadIdx.x >> 5;
    const int m0 = blockIdx.x * kTM;
    const int K = op.kdim();
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    const int ntiles = (ke - kb + kTK - 1) / kTK;
    const uint32_t ncols = umma::tmem_cols(bn);
    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
    }
    if (warp == 0) umma::alloc(slot, ncols);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t idesc = umma::idesc_bf16_f32(kTM, bn);
    bool failed = false;
    int issued = 0;
    for (int t = 0; t < ntiles; ++t) {
        const int s = t & 1;
        if (t >= 2) {   // the MMAs of tile t - 2 are done with stage s
            failed = __syncthreads_or(!tma::mbar_wait(&bar[s], ((t - 2) >> 1) & 1));
            if (failed) break;
        }
        const int k0 = kb + t * kTK;
        op.build_a(sa[s], m0, k0, scratch);
        op.build_b(sb[s], bn, k0);
        tma::fence_proxy_async();   // the stores above, visible to the tensor cores
        __syncthreads();
        if (threadIdx.x == 0) {
            umma::fence_after_sync();
            const uint32_t a = umma::saddr(sa[s]), b = umma::saddr(sb[s]);
#pragma unroll
            for (int kk = 0; kk < kTK / 16; ++kk)
                umma::mma_bf16(tmem, umma::sw128_desc(a + 32 * kk), umma::sw128_desc(b + 32 * kk),
                               idesc, (t > 0 || kk > 0) ? 1u : 0u);
            umma::commit(&bar[s]);
        }
        issued = t + 1;
    }
    if (!failed && issued > 0) {   // the last commit covers every MMA before it
        const int tl = issued - 1;
        failed = __syncthreads_or(!tma::mbar_wait(&bar[tl & 1], (tl >> 1) & 1));
    }
    if (failed) {
        if (threadIdx.x == 0) {
            atomicExch(flag, 1);
            if (issued > 0) tma::mbar_wait(&bar[(issued - 1) & 1], ((issued - 1) >> 1) & 1);
        }
    } else {
        umma::fence_after_sync();
        const int row = warp * 32 + (threadIdx.x & 31);   // TMEM lane = tile row
        for (int c0 = 0; c0 < bn; c0 += 16) {
            float v[16];
            umma::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            op.store(m0 + row, c0, v, blockIdx.z);
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::dealloc(tmem, ncols);
    }
}

// Forward convolution: rows = pixels q = (n, y, x), K = taps k = tap Cin + ci (tap = 3 ky +
// kx); B = the BF16 weights in that order, rows co (ldw >= 9 Cin per row, zero beyond
// 9 Cin, zero rows up to the padded bn); out[n][co][y][x] = bias[co] + D.
struct ConvFwd {
    const float *in;
    const __nv_bfloat16 *W;
    int ldw;
    const float *bias;
    float *out;
    int N, Cin, Hh, Ww, Cout;
    int relu;   // ReLU of the output in the epilogue
    static constexpr int kScratch = 0;
    __device__ int kdim() const { return Cin * 9; }
    __device__ void build_a(uint8_t *tile, int m0, int k0, float *) const {
        const int r = threadIdx.x, q = m0 + r;
        const int HW = Hh * Ww;
        const bool live = q < N * HW;
        int n = 0, y = 0, x = 0;
        if (live) {
            n = q / HW;
            const int p = q - n * HW;
            y = p / Ww;
            x = p - y * Ww;
        }
        const float *src = in + (size_t)n * Cin * HW;
        // K = tap Cin + ci: the tap's offset and bounds hold over a run of channels.  Per
        // group of 16 values the offsets and a validity mask come first (the bookkeeping's
        // branches depend on no load), then the 16 loads go out together.
        int tap = k0 / Cin, ci = k0 - tap * Cin;
        int off = 0;
        bool ok = false;
        auto enter_tap = [&]() {
            const int ky = tap / 3, yy = y + ky - 1, xx = x + (tap - 3 * ky) - 1;
            ok = live && tap < 9 && yy >= 0 && yy < Hh && xx >= 0 && xx < Ww;
            off = ci * HW + yy * Ww + xx;
        };
        enter_tap();
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            int o[16];
            unsigned mask = 0;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                o[j] = off;
                mask |= ok ? 1u << j : 0u;
                off += HW;
                if (++ci == Cin) {
                    ci = 0;
                    ++tap;
                    enter_tap();
                }
            }
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = mask >> j & 1u ? src[o[j]] : 0.f;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
                *chunk(tile, r, 2 * g + cc) =
                    make_uint4(pack_bf16(v[8 * cc], v[8 * cc + 1]), pack_bf16(v[8 * cc + 2], v[8 * cc + 3]),
                               pack_bf16(v[8 * cc + 4], v[8 * cc + 5]),
                               pack_bf16(v[8 * cc + 6], v[8 * cc + 7]));
        }
    }
    __device__ void build_b(uint8_t *tile, int nrows, int k0) const {
        for (int i = threadIdx.x; i < nrows * 8; i += kThreads) {
            const int r = i >> 3, c = i & 7;
            *chunk(tile, r, c) = *reinterpret_cast<const uint4 *>(W + (size_t)r * ldw + k0 + c * 8);
        }
    }
    __device__ void store(int m, int co0, const float (&v)[16], int) const {
        const int HW = Hh * Ww;
        if (m >= N * HW) return;
        const int n = m / HW, p = m - n * HW;
        float *o = out + (size_t)n * Cout * HW + p;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int co = co0 + j;
            if (co < Cout) {
                const float y = bias ? v[j] + bias[co] : v[j];
                o[(size_t)co * HW] = relu ? fmaxf(y, 0.f) : y;
            }
        }
    }
};

// Weight gradient, transposed: rows = taps k = ci 9 + tap (the order of W[co][ci][ky][kx]),
// K = pixels q; A = im2col(in)^T, B = dout (rows co, zero rows up to bn); D(k, co) =
// dW[co][k] of the split's pixels, into part[split][co][k].
struct ConvWgrad {
    const float *in, *dout;
    float *part;
    int N, Cin, Hh, Ww, Cout;
    static constexpr int kScratch = 0;
    __device__ int kdim() const { return N * Hh * Ww; }
    __device__ void build_a(uint8_t *tile, int m0, int q0, float *) const {
        const int r = threadIdx.x, k = m0 + r;
        const int HW = Hh * Ww, Q = N * HW;
        const bool live = k < Cin * 9;
        const int ci = live ? k / 9 : 0, t = k - ci * 9;       // k = ci 9 + tap: a warp's rows
        const int ky = t / 3, dy = ky - 1, dx = t - 3 * ky - 1;  // read nearby pixels
        int n = q0 / HW, p = q0 - n * HW;
        int y = p / Ww, x = p - y * Ww;
        const bool full = q0 + kTK <= Q;                       // no pixel past the end
        int q = q0;
        // offset of the current image's plane of channel ci, and row y + dy of it (pixel x
        // of the run at rowo + x); both change only when the run wraps to the next row.
        // Per group of 16 values the offsets and a validity mask come first, then the loads.
        int plane = (n * Cin + ci) * HW, rowo = 0;
        bool rowok = false;
        auto enter_row = [&]() {
            const int yy = y + dy;
            rowok = live && yy >= 0 && yy < Hh;
            rowo = plane + yy * Ww + dx;
        };
        enter_row();
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            int o[16];
            unsigned mask = 0;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                o[j] = rowo + x;
                const bool in_x = (unsigned)(x + dx) < (unsigned)Ww;
                mask |= rowok && in_x && (full || q < Q) ? 1u << j : 0u;
                ++q;
                if (++x == Ww) {
                    x = 0;
                    if (++y == Hh) {
                        y = 0;
                        plane += Cin * HW;                     // next image
                    }
                    enter_row();
                }
            }
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = mask >> j & 1u ? in[o[j]] : 0.f;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
                *chunk(tile, r, 2 * g + cc) =
                    make_uint4(pack_bf16(v[8 * cc], v[8 * cc + 1]), pack_bf16(v[8 * cc + 2], v[8 * cc + 3]),
                               pack_bf16(v[8 * cc + 4], v[8 * cc + 5]),
                               pack_bf16(v[8 * cc + 6], v[8 * cc + 7]));
        }
    }
    __device__ void build_b(uint8_t *tile, int nrows, int q0) const {
        const int HW = Hh * Ww, Q = N * HW;
        const bool vec = (HW & 7) == 0;   // a chunk of 8 pixels lies in one image, 32-byte aligned
        for (int i = threadIdx.x; i < nrows * 8; i += kThreads) {
            const int r = i >> 3, c = i & 7;   // row co, pixels q0 + 8 c .. + 7
            int q = q0 + c * 8;
            int n = q / HW, p = q - n * HW;
            uint32_t w[4];
            if (vec) {
                float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
                if (r < Cout && q < Q) {
                    const float4 *src =
                        reinterpret_cast<const float4 *>(dout + ((size_t)n * Cout + r) * HW + p);
                    lo = src[0];
                    hi = src[1];
                }
                w[0] = pack_bf16(lo.x, lo.y);
                w[1] = pack_bf16(lo.z, lo.w);
                w[2] = pack_bf16(hi.x, hi.y);
                w[3] = pack_bf16(hi.z, hi.w);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    float v2[2];
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        v2[hh] = r < Cout && q < Q ? dout[((size_t)n * Cout + r) * HW + p] : 0.f;
                        ++q;
                        if (++p == HW) {
                            p = 0;
                            ++n;
                        }
                    }
                    w[e] = pack_bf16(v2[0], v2[1]);
                }
            }
            *chunk(tile, r, c) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    __device__ void store(int k, int co0, const float (&v)[16], int z) const {
        const int K = Cin * 9;
        if (k >= K) return;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int co = co0 + j;
            if (co < Cout) part[((size_t)z * Cout + co) * K + k] = v[j];
        }
    }
};

// Wt[ci][(8 - t) Cout + co] = W[co][t Cin + ci] (tap-major rows of ldw and ldt values, pads
// untouched): the transposed convolution's weights, (ky, kx) -> (2-ky, 2-kx)
__global__ void k_flip(const __nv_bfloat16 *W, int ldw, int Cout, int Cin, __nv_bfloat16 *Wt,
                       int ldt) {
    const int total = Cout * Cin * 9;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int co = i / (Cin * 9), rem = i - co * Cin * 9;
        const int t = rem / Cin, ci = rem - t * Cin;
        Wt[(size_t)ci * ldt + (8 - t) * Cout + co] = W[(size_t)co * ldw + rem];
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
// db[c] = sum over n, p of dout[n][c][p], in a fixed order: block (c, s) sums the pixels
// q = 256 s + t, + 256 S, ... of the N images (thread t), then a tree, into work[c S + s];
// k_bias_grad_sum adds the S partials of a channel in order
__global__ void __launch_bounds__(256) k_bias_grad_part(const float *dout, int N, int C, int HW,
                                                        int S, float *work) {
    __shared__ float s[256];
    const int c = blockIdx.x, sp = blockIdx.y;
    const size_t P = (size_t)N * HW;
    float acc = 0.f;
    for (size_t q = (size_t)sp * 256 + threadIdx.x; q < P; q += (size_t)S * 256) {
        const size_t n = q / HW, p = q - n * HW;
        acc += dout[(n * C + c) * HW + p];
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) work[(size_t)c * S + sp] = s[0];
}

__global__ void k_bias_grad_sum(const float *work, int C, int S, float *db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    float acc = 0.f;
    for (int i = 0; i < S; ++i) acc += work[(size_t)c * S + i];
    db[c] = acc;
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

// position in the padded tap-major BF16 rows of FP32 weight i = co 9 Cin + ci 9 + t
__device__ __forceinline__ size_t bf16_slot(size_t i, int cin, int ldb) {
    const size_t K = (size_t)cin * 9, co = i / K;
    const int rem = (int)(i - co * K), ci = rem / 9, t = rem - ci * 9;
    return co * ldb + (size_t)t * cin + ci;
}

// Adam on n FP32 weights; the BF16 copy (if any) of weight i goes to bf16_slot(i)
__global__ void k_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, size_t n,
                       int cin, int ldb, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[bf16_slot(i, cin, ldb)] = __float2bfloat16_rn(wi);
    }
}

__global__ void k_to_bf16(const float *w, __nv_bfloat16 *wb, size_t n, int cin, int ldb) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        wb[bf16_slot(i, cin, ldb)] = __float2bfloat16_rn(w[i]);
}

constexpr int kMaxScratch = 0;   // the largest Op::kScratch (floats)
constexpr int kMaxSmem = 1024 + 2 * kATile + 2 * 256 * 128 + 32 + 4 * kMaxScratch;

template <class Op>
cudaError_t umma_gemm(const Op &op, int rows, int K, int bn, int splits, int *flag,
                      cudaStream_t st) {
    if (rows < 1 || K < 1 || bn < 16 || bn > 256 || bn % 16 != 0 || !flag)
        return cudaErrorInvalidValue;
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + kTK - 1) / kTK * kTK;
    const int sp = (K + kchunk - 1) / kchunk;
    const dim3 grid((unsigned)((rows + kTM - 1) / kTM), 1, (unsigned)sp);
    if (grid.z > 65535u) return cudaErrorInvalidValue;
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_umma_gemm<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
    if (attr != cudaSuccess) return attr;
    static_assert(Op::kScratch <= kMaxScratch, "scratch fits the attribute");
    const int smem = 1024 + 2 * kATile + 2 * bn * 128 + 32 + 4 * Op::kScratch;
    k_umma_gemm<Op><<<grid, kThreads, smem, st>>>(op, bn, kchunk, flag);
    return cudaGetLastError();
}

}  // namespace

int padded_taps(int cin) { return (cin * 9 + kTK - 1) / kTK * kTK; }
int padded_rows(int c) { return (c + 15) / 16 * 16; }

cudaError_t conv3x3_forward(const float *in, int N, int Cin, int Hh, int Ww,
                            const __nv_bfloat16 *W, const float *bias, int Cout, float *out,
                            bool relu, int *flag, cudaStream_t st) {
    // the operand staging addresses an image's channels with 32-bit offsets
    if (Cout > 256 || (long long)Cin * Hh * Ww >= (1LL << 31)) return cudaErrorInvalidValue;
    ConvFwd op{in, W, padded_taps(Cin), bias, out, N, Cin, Hh, Ww, Cout, relu ? 1 : 0};
    return umma_gemm(op, N * Hh * Ww, Cin * 9, padded_rows(Cout), 1, flag, st);
}

cudaError_t conv3x3_flip(const __nv_bfloat16 *W, int Cout, int Cin, __nv_bfloat16 *Wt,
                         cudaStream_t st) {
    k_flip<<<grid_1d((size_t)Cout * Cin * 9), 256, 0, st>>>(W, padded_taps(Cin), Cout, Cin, Wt,
                                                           padded_taps(Cout));
    return cudaGetLastError();
}

int conv3x3_weight_grad_splits(int N, int Hh, int Ww, int Cin) {
    // about four waves of 128-tap tiles x splits over the SMs, each split at least 8 stages
    // of 64 pixels
    const long long K = (long long)N * Hh * Ww;
    const int mtiles = (Cin * 9 + kTM - 1) / kTM;
    const long long want = (4LL * kB200SMs + mtiles - 1) / mtiles;
    const long long most = std::max<long long>(1, K / (8 * kTK));
    return (int)std::max<long long>(1, std::min<long long>({want, most, 1024}));
}

cudaError_t conv3x3_weight_grad(const float *in, const float *dout, int N, int Cin, int Hh,
                                int Ww, int Cout, float *dW, float *work, int splits, int *flag,
                                cudaStream_t st) {
    // the operand staging addresses the whole input with 32-bit offsets
    if (Cout > 256 || (long long)N * Cin * Hh * Ww >= (1LL << 31)) return cudaErrorInvalidValue;
    const int K = N * Hh * Ww;
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + kTK - 1) / kTK * kTK;
    const int sp = (K + kchunk - 1) / kchunk;   // the splits the GEMM actually makes
    ConvWgrad op{in, dout, work, N, Cin, Hh, Ww, Cout};
    cudaError_t e = umma_gemm(op, Cin * 9, K, padded_rows(Cout), splits, flag, st);
    if (e != cudaSuccess) return e;
    const size_t n = (size_t)Cout * Cin * 9;
    k_sum_parts<<<grid_1d(n), 256, 0, st>>>(work, sp, n, dW);
    return cudaGetLastError();
}

int bias_grad_splits(int N, int HW) {
    return (int)std::max<long long>(1, std::min<long long>(64, (long long)N * HW / 8192));
}

cudaError_t bias_grad(const float *dout, int N, int C, int HW, float *db, float *work,
                      cudaStream_t st) {
    const int S = bias_grad_splits(N, HW);
    k_bias_grad_part<<<dim3((unsigned)C, (unsigned)S), 256, 0, st>>>(dout, N, C, HW, S, work);
    k_bias_grad_sum<<<(C + 127) / 128, 128, 0, st>>>(work, C, S, db);
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
                 int cin, int ldb, float lr, float b1, float b2, float eps, int t,
                 cudaStream_t st) {
    if (wb && (cin < 1 || ldb < 9 * cin)) return cudaErrorInvalidValue;
    const float c1 = (float)(1.0 - std::pow((double)b1, t));
    const float c2 = (float)(1.0 - std::pow((double)b2, t));
    k_adam<<<grid_1d(n), 256, 0, st>>>(w, m, v, g, wb, n, cin, ldb, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t to_bf16(const float *w, __nv_bfloat16 *wb, size_t n, int cin, int ldb,
                    cudaStream_t st) {
    if (cin < 1 || ldb < 9 * cin) return cudaErrorInvalidValue;
    k_to_bf16<<<grid_1d(n), 256, 0, st>>>(w, wb, n, cin, ldb);
    return cudaGetLastError();
}

}  // namespace cnn
}  // namespace fpm

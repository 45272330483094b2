// LED illumination geometry on the device, in FP64.
//
// For every LED of a square array (visited in the centre-out spiral order) the
// illumination angle gives a target spatial frequency; the LED's crop corner is
// the nearest point of the high-res frequency axis (the first one on ties),
// exactly the statements of codes_v2/func_ware/init_environment_rgb.m:15-46 and
// :64-106, and the corner offsets of codes_v2/main_run_FPM.m:21-31,51-55.
//
// Every floating-point operation is an explicitly rounded intrinsic (no fused
// multiply-add), evaluated in MATLAB's left-to-right order, so the integer
// results equal an IEEE double evaluation of the MATLAB statements.
#include <cfloat>
#include <climits>
#include <cmath>

#include "engine.h"

namespace fpm {

namespace {

// One CTA per (LED, axis): the target frequency, then a scan of the NN-point
// axis F_k = ((k - NN/2) / (h * D_pixel)) * 2 pi for min |F_k - target|.
__global__ void __launch_bounds__(256) k_led_nearest(const int2 *__restrict__ pos, LedGeom p,
                                                     int32_t *__restrict__ led_idx) {
    const int l = blockIdx.x >> 1, axis = blockIdx.x & 1;
    __shared__ double s_tgt;
    __shared__ double s_best[8];
    __shared__ int s_idx[8];
    if (threadIdx.x == 0) {
        const double cen = (double)(p.grid - 1) / 2.0;               // (ledMM - 1) / 2
        const double vv = __dsub_rn((double)(pos[l].x - 1), cen);   // vled(i)
        const double hh = __dsub_rn((double)(pos[l].y - 1), cen);   // hled(j)
        const double a = __dadd_rn(__dmul_rn(-vv, p.pitch), p.dx);  // -vvled*D_led + objdx
        const double b = __dadd_rn(__dmul_rn(-hh, p.pitch), p.dy);  // -hhled*D_led + objdy
        const double den = __dsqrt_rn(
            __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(p.height, p.height)));
        const double v0 = __ddiv_rn(a, den);                         // v (before the swap)
        const double u0 = __ddiv_rn(-b, den);                        // u (before the swap)
        // after the swap u <- v0 drives the column (kl) axis, v <- u0 the row (kt) axis
        s_tgt = __dmul_rn(p.k_lamuda, axis == 0 ? v0 : u0);
    }
    __syncthreads();
    const double tgt = s_tgt;
    double best = DBL_MAX;
    int bi = INT_MAX;
    for (int k = threadIdx.x; k < p.NN; k += blockDim.x) {
        const double f = __dmul_rn(__ddiv_rn((double)(k - p.NN / 2), p.ND), p.two_pi);
        const double d = fabs(__dsub_rn(f, tgt));
        if (d < best) {   // k grows along the thread's walk: the first minimum stays
            best = d;
            bi = k;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob < best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        s_best[threadIdx.x >> 5] = best;
        s_idx[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            if (s_best[w] < best || (s_best[w] == best && s_idx[w] < bi)) {
                best = s_best[w];
                bi = s_idx[w];
            }
        // 1-based find index minus N/2 (kl = kc(3) + uo, kt = kc(1) + vo)
        led_idx[2 * l + axis] = bi + 1 - p.h / 2;
    }
}

}  // namespace

void spiral_grid_order(int n, std::vector<int2> &order) {
    // init_environment_rgb.m:111-133: start at the centre; at every step turn to
    // direction + 1 (steps (sin, cos)(pi/2 * direction)) if that cell is unvisited,
    // then step once.  n is odd.
    std::vector<char> seen((size_t)(n + 2) * (n + 2), 0);
    auto at = [&](int i, int j) -> char & { return seen[(size_t)i * (n + 2) + j]; };
    int i = (n + 1) / 2, j = (n + 1) / 2, d = 0;
    order.clear();
    order.push_back(make_int2(i, j));
    at(i, j) = 1;
    const double half_pi = M_PI / 2;
    while ((int)order.size() < n * n) {
        const int d2 = d + 1;
        const int i2 = (int)std::round(i + std::sin(half_pi * d2));
        const int j2 = (int)std::round(j + std::cos(half_pi * d2));
        if (i2 >= 1 && i2 <= n && j2 >= 1 && j2 <= n && !at(i2, j2)) d = d2;
        i = (int)std::round(i + std::sin(half_pi * d));
        j = (int)std::round(j + std::cos(half_pi * d));
        if (i < 1 || i > n || j < 1 || j > n || at(i, j)) break;   // not reached for odd n
        at(i, j) = 1;
        order.push_back(make_int2(i, j));
    }
}

cudaError_t launch_led_nearest(const int2 *pos, int n_leds, const LedGeom &p, int32_t *led_idx,
                               cudaStream_t st) {
    k_led_nearest<<<2 * n_leds, 256, 0, st>>>(pos, p, led_idx);
    return cudaGetLastError();
}

}  // namespace fpm

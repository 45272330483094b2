// C ABI (include/fpm.h) and the reconstruction loop.
//
// The loop is the reference's epoch x mini-batch schedule
// (cuFPM_v3/cuFPM_pure_v3.cu:128-207): per batch, spectrum of the current
// object -> per-LED forward model, loss gradient and back-propagation ->
// gradient spectrum -> object gradient -> RMSprop on object and pupil; the
// learning rate halves after epochs with index > lr_halve_after.  Unlike the
// reference it never synchronises inside the loop: everything is queued on one
// stream and the host waits once, at the end.  Each batch runs the fused
// pipeline of pipeline.cu (low-resolution passes, stitch + row inverse FFT,
// column pass with the object RMSprop, row forward FFT of the next batch's box).
#include "../../include/fpm.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "fft.h"
#include "generic.h"
#include "pipeline.h"
#include "tiff.h"
#include "tuning.h"

using namespace fpm;

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // grow-only: keeps an existing allocation that is large enough
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        if (n == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();  // clear the sticky-free allocation error
            return e;
        }
        bytes = n;
        return cudaSuccess;
    }
    template <class T>
    T *as() const {
        return static_cast<T *>(p);
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// per-stage device timing
// ---------------------------------------------------------------------------
namespace {

enum Stage : int {
    ST_COLS_FORWARD, ST_ROWS_FORWARD, ST_LR_COLS_INV, ST_LR_ROWS_INV, ST_LR_ROWS_FWD,
    ST_LR_COLS_FWD, ST_LOSS, ST_PUPIL_GRAD, ST_ROWS_INV, ST_COLS_UPDATE, ST_RMS_PUPIL,
    ST_SPECTRUM, ST_TRANSPOSE, ST_LR_ROWS_FUSED, ST_SIM_ROWS_INV, ST_SIM_MAGNITUDE, ST_H2D,
    ST_D2H, ST_GEN_LR_FFT, ST_GEN_LOSS, ST_GEN_STITCH, ST_GEN_OBJ_FFT, ST_GEN_RMS_OBJ,
    ST_STACK_ROWS, ST_COUNT
};
const char *const kStageName[ST_COUNT] = {
    "cols_forward", "rows_forward", "lr_cols_inverse", "lr_rows_inverse", "lr_rows_forward",
    "lr_cols_forward", "loss_reduce", "pupil_grad", "rows_inverse_stitch", "cols_update",
    "rmsprop_pupil", "spectrum_fft2", "transpose", "lr_rows_fused", "sim_rows_inverse",
    "sim_magnitude", "copy_inputs_h2d", "copy_outputs_d2h", "any_size_lr_fft2",
    "any_size_loss_gradient", "any_size_stitch", "any_size_object_fft2",
    "any_size_rmsprop_object", "stack_rows"};
// 0: a host <-> device copy of the caller's buffers (host-memory calls), not a kernel
const int kStageOwn[ST_COUNT] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0,
                                 1, 1, 1, 1, 1, 1};

struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<int> rec_stage;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> rec;
    double ms[ST_COUNT] = {};
    int n[ST_COUNT] = {};
    cudaEvent_t open = nullptr;

    ~Profiler() {
        for (auto e : pool) cudaEventDestroy(e);
    }
    void reset() {
        used = 0;
        rec.clear();
        rec_stage.clear();
        for (int i = 0; i < ST_COUNT; ++i) ms[i] = 0.0, n[i] = 0;
    }
    cudaEvent_t get() {
        if (used == pool.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            pool.push_back(e);
        }
        return pool[used++];
    }
    void begin(cudaStream_t st) {
        if (!on) return;
        open = get();
        if (open) cudaEventRecord(open, st);
    }
    void end(int stage, cudaStream_t st) {
        if (!on || !open) return;
        cudaEvent_t e = get();
        if (!e) return;
        cudaEventRecord(e, st);
        rec.emplace_back(open, e);
        rec_stage.push_back(stage);
        open = nullptr;
    }
    // after the stream has been synchronised
    void collect() {
        if (!on) return;
        for (size_t i = 0; i < rec.size(); ++i) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, rec[i].first, rec[i].second) == cudaSuccess) {
                ms[rec_stage[i]] += t;
                n[rec_stage[i]] += 1;
            }
        }
        rec.clear();
        rec_stage.clear();
        used = 0;
    }
};

}  // namespace

struct fpm_context {
    Profiler prof;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t entry = nullptr;   // orders device-memory calls after the legacy default stream
    size_t mem_limit = 0;
    std::string err;
    FftEngine fft;
    GenFft gfft;   // line FFTs of lengths that are not powers of two
    // work buffers, kept between calls
    DevBuf O, m1, S, P, m2, P0, dP, Pt, T1, T2, Rs, Xs, Sbox, Sboxr, U, V, W, Y, led, parts, loss,
        minmax, lut, spec, flag, pie, rows;
    DevBuf opt[6];   // device copies of an optimiser step's host arrays
    // the last captured epoch; a later capture of the same topology updates it in place
    cudaGraphExec_t epoch_graph = nullptr;
    // fpm_solve_batch: one worker context per instance, on a pool of streams
    std::vector<fpm_context *> workers;
    std::vector<cudaStream_t> pool;
    // autotuner: the chosen launch choices per problem shape
    int flags = 0;
    std::map<std::vector<int>, Tuning> tuned;
};

namespace {

// detail of the last failure of a call made without a context, per host thread
thread_local std::string t_err;

fpm_status fail(fpm_context *ctx, fpm_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    (ctx ? ctx->err : t_err) = buf;
    return s;
}

fpm_status fail_cuda(fpm_context *ctx, cudaError_t e, const char *what, int line) {
    if (e == cudaErrorMemoryAllocation)
        return fail(ctx, FPM_ERR_OUT_OF_MEMORY, "%s: out of device memory (line %d)", what, line);
    return fail(ctx, FPM_ERR_CUDA, "%s failed: %s (line %d)", what, cudaGetErrorString(e), line);
}

#define FPM_CK(call)                                                   \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) return fail_cuda(ctx, e_, #call, __LINE__); \
    } while (0)

// Runs one stage launch, bracketed by profiling events when enabled.
#define FPM_STAGE(id, call)                 \
    do {                                    \
        ctx->prof.begin(ctx->stream);       \
        FPM_CK(call);                       \
        ctx->prof.end((id), ctx->stream);   \
    } while (0)

bool is_device_ptr(const void *p, int device) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) &&
           a.device == device;
}

bool is_host_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered || a.type == cudaMemoryTypeHost;
}

// crop box of one batch in centred coordinates, taken modulo H
// Pupil support: crop rows / columns [r_lo, r_hi) x [c_lo, c_hi) outside which the
// pupil is zero for the whole solve.
struct Support {
    int r_lo = 0, r_hi = 0, c_lo = 0, c_hi = 0;
};

// Centred-spectrum box of one batch: the union of its LEDs' crops restricted to the
// pupil support (the only part of a crop the batch reads or writes).
Box batch_box(const std::vector<int32_t> &led, int first, int nb, const Support &sup, int H) {
    int rlo = 1 << 30, rhi = -(1 << 30), clo = 1 << 30, chi = -(1 << 30);
    for (int i = first; i < first + nb; ++i) {
        const int kl = led[2 * i], kt = led[2 * i + 1];
        rlo = std::min(rlo, kt - 1 + sup.r_lo);
        rhi = std::max(rhi, kt - 1 + sup.r_hi);
        clo = std::min(clo, kl - 1 + sup.c_lo);
        chi = std::max(chi, kl - 1 + sup.c_hi);
    }
    Box b;
    b.r_lo = rlo;
    b.r_span = rhi - rlo;
    b.c_lo = clo;
    b.c_span = chi - clo;
    if (b.r_span >= H) b.r_lo = 0, b.r_span = H;
    if (b.c_span >= H) b.c_lo = 0, b.c_span = H;
    return b;
}

struct Shape {
    int h, H, L, B, pratio;
    size_t plane, big;
};

fpm_status validate(fpm_context *ctx, const fpm_problem *p, bool need_batch) {
    if (!p) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "problem is NULL");
    if (p->h < 2 || (p->h & 1))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "h = %d: must be even and >= 2", p->h);
    if (p->pratio < 1) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pratio = %d < 1", p->pratio);
    const long long H = (long long)p->h * p->pratio;
    if (H > kMaxFftLen ||
        !(pipeline_supported(p->h, (int)H) || (gen_fft_supported(p->h) && gen_fft_supported((int)H))))
        return fail(ctx, FPM_ERR_UNSUPPORTED,
                    "h = %d, H = %lld: h and H must have no prime factor above 7, H <= %d",
                    p->h, H, kMaxFftLen);
    if (!pipeline_supported(p->h, (int)H) && p->pie_weights != FPM_PIE_NONE)
        return fail(ctx, FPM_ERR_UNSUPPORTED,
                    "ePIE / tPIE weights need power-of-two sizes (h = %d, H = %lld)", p->h, H);
    if (p->n_leds < 1) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "n_leds = %d < 1", p->n_leds);
    if (need_batch) {
        if (p->batch < 1) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "batch = %d < 1", p->batch);
        if (p->epochs < 0)
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "epochs = %d < 0", p->epochs);
        if (!std::isfinite(p->lr) || !std::isfinite(p->beta) || !std::isfinite(p->eps) ||
            !std::isfinite(p->pupil_margin) || !std::isfinite(p->lr_decay))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "non-finite optimiser parameter");
        if (p->beta < 0.f || p->beta > 1.f)
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "beta = %g outside [0, 1]", p->beta);
        if (p->eps < 0.f) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "eps = %g < 0", p->eps);
    }
    if (std::min(p->batch, p->n_leds) > 1024 && need_batch)
        return fail(ctx, FPM_ERR_UNSUPPORTED, "batch of %d LEDs exceeds 1024",
                    std::min(p->batch, p->n_leds));
    if (p->loss_kind != FPM_LOSS_ANISOTROPIC && p->loss_kind != FPM_LOSS_ISOTROPIC)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "loss_kind %d", p->loss_kind);
    if (p->pie_weights < FPM_PIE_NONE || p->pie_weights > FPM_PIE_TPIE)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pie_weights %d", p->pie_weights);
    if (p->memory != FPM_MEM_HOST && p->memory != FPM_MEM_DEVICE)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "memory = %d", p->memory);
    if (p->stack_type != FPM_STACK_F32_AMPLITUDE && p->stack_type != FPM_STACK_U16_COUNTS)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "stack_type = %d", p->stack_type);
    if (!p->stack || !p->led_idx || !p->pupil_init || !p->pupil_amp)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT,
                    "stack, led_idx, pupil_init and pupil_amp are required");
    const void *ptrs[5] = {p->stack, p->led_idx, p->pupil_init, p->pupil_amp, p->object_init};
    const char *names[5] = {"stack", "led_idx", "pupil_init", "pupil_amp", "object_init"};
    for (int i = 0; i < 5; ++i) {
        if (!ptrs[i]) continue;
        if (p->memory == FPM_MEM_DEVICE && !is_device_ptr(ptrs[i], ctx->device))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT,
                        "%s is not device memory of device %d", names[i], ctx->device);
        // kernels use 64/128-bit accesses on device buffers
        if (p->memory == FPM_MEM_DEVICE && (reinterpret_cast<uintptr_t>(ptrs[i]) & 15u))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "%s is not 16-byte aligned", names[i]);
        if (p->memory == FPM_MEM_HOST && !is_host_ptr(ptrs[i]))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "%s is not host memory", names[i]);
    }
    return FPM_OK;
}

fpm_status check_leds(fpm_context *ctx, const std::vector<int32_t> &led, int L, int H) {
    for (int i = 0; i < L; ++i) {
        const int kl = led[2 * i], kt = led[2 * i + 1];
        if (kl < 1 || kl > H || kt < 1 || kt > H)
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT,
                        "led_idx[%d] = (%d, %d) outside [1, %d]", i, kl, kt, H);
    }
    return FPM_OK;
}

struct Inputs {
    StackView Y;
    int stack_pages = 0;
    const int2 *led = nullptr;
    std::vector<int32_t> led_host;
};

// Brings every input to the device (or adopts device pointers) and fills `in`.
fpm_status stage_inputs(fpm_context *ctx, const fpm_problem *p, const Shape &s, Inputs &in) {
    cudaStream_t st = ctx->stream;
    in.stack_pages = s.L;
    const size_t ybytes = s.plane * s.L * (p->stack_type == FPM_STACK_U16_COUNTS ? 2 : 4);
    in.led_host.resize(2 * (size_t)s.L);
    if (p->memory == FPM_MEM_HOST) {
        std::memcpy(in.led_host.data(), p->led_idx, 2 * sizeof(int32_t) * s.L);
    } else {
        FPM_CK(cudaMemcpyAsync(in.led_host.data(), p->led_idx, 2 * sizeof(int32_t) * s.L,
                               cudaMemcpyDeviceToHost, st));
        FPM_CK(cudaStreamSynchronize(st));
    }
    fpm_status rc = check_leds(ctx, in.led_host, s.L, s.H);
    if (rc != FPM_OK) return rc;
    if (p->memory == FPM_MEM_HOST) {
        FPM_CK(ctx->Y.ensure(ybytes));
        FPM_STAGE(ST_H2D, cudaMemcpyAsync(ctx->Y.p, p->stack, ybytes, cudaMemcpyHostToDevice, st));
        FPM_CK(ctx->led.ensure(2 * sizeof(int32_t) * s.L));
        FPM_STAGE(ST_H2D, cudaMemcpyAsync(ctx->led.p, p->led_idx, 2 * sizeof(int32_t) * s.L,
                                          cudaMemcpyHostToDevice, st));
        in.Y.ptr = ctx->Y.p;
        in.led = ctx->led.as<int2>();
    } else {
        in.Y.ptr = p->stack;
        in.led = reinterpret_cast<const int2 *>(p->led_idx);
    }
    in.Y.type = p->stack_type == FPM_STACK_U16_COUNTS ? kStackU16 : kStackF32;
    if (in.Y.type == kStackU16) {
        FPM_CK(ctx->minmax.ensure(2 * sizeof(unsigned)));
        FPM_CK(launch_stack_minmax(static_cast<const uint16_t *>(in.Y.ptr), s.plane * s.L,
                                   ctx->minmax.as<unsigned>(), st));
        in.Y.minmax = ctx->minmax.as<unsigned>();
        FPM_CK(ctx->lut.ensure(65536 * sizeof(float)));
        FPM_CK(launch_amplitude_lut(in.Y.minmax, ctx->lut.as<float>(), st));
        in.Y.lut = ctx->lut.as<float>();
    }
    return FPM_OK;
}

// The row-major amplitude copy of the whole stack the fused row pass reads (once per
// call: 4 bytes per pixel beside the stack).
fpm_status stack_rows(fpm_context *ctx, const Shape &s, Inputs &in) {
    FPM_CK(ctx->rows.ensure(s.plane * s.L * sizeof(float)));
    FPM_STAGE(ST_STACK_ROWS,
              launch_amplitude_rows(in.Y, s.h, s.L, ctx->rows.as<float>(), ctx->stream));
    in.Y.rows = ctx->rows.as<float>();
    return FPM_OK;
}

// Pupil support of a solve: the amplitude clamp (|P| <- P0 clamp(|P|, P0 -/+ am))
// keeps the pupil at zero wherever P0 is zero, so after the initial pupil P0c the
// pupil is non-zero only inside supp(P0c) u supp(P0).  FPM_PUPIL_SUPPORT=0 keeps whole
// crops (measurements).
// bit pattern of a float
static inline uint32_t fbits(const float *x) {
    uint32_t b;
    std::memcpy(&b, x, 4);
    return b;
}

// Rows / columns [box[0], box[1]] x [box[2], box[3]] holding every pixel where the host
// pupil P (complex, column-major h x h) or the amplitude A is not +-0 (NaN counts as
// non-zero).  A column is tested with one OR of its bit patterns (the sign bit masked
// afterwards), and only the non-zero columns are searched from both ends for their
// first and last non-zero rows.
static void host_support_cols(const float *P, const float *A, int h, int c0, int c1, int box[4]) {
    const auto nz = [&](size_t i) {
        return ((fbits(P + 2 * i) | fbits(P + 2 * i + 1) | fbits(A + i)) & 0x7fffffffu) != 0;
    };
    for (int c = c0; c < c1; ++c) {
        const float *pc = P + 2 * (size_t)c * h, *ac = A + (size_t)c * h;
        uint32_t any = 0;
        for (int i = 0; i < 2 * h; ++i) any |= fbits(pc + i) & 0x7fffffffu;
        for (int i = 0; i < h; ++i) any |= fbits(ac + i) & 0x7fffffffu;
        if (any == 0) continue;
        int lo = 0, hi = h - 1;
        while (!nz((size_t)c * h + lo)) ++lo;
        while (!nz((size_t)c * h + hi)) --hi;
        box[0] = std::min(box[0], lo);
        box[1] = std::max(box[1], hi);
        box[2] = std::min(box[2], c);
        box[3] = std::max(box[3], c);
    }
}

// the columns split over up to 8 host threads (the arrays are 12 h^2 bytes)
static void host_support_box(const float *P, const float *A, int h, int box[4]) {
    const int nt = std::max(1, std::min({8, (int)std::thread::hardware_concurrency(), h / 64}));
    std::vector<std::array<int, 4>> part(nt, std::array<int, 4>{h, -1, h, -1});
    std::vector<std::thread> pool;
    for (int i = 1; i < nt; ++i)
        pool.emplace_back(host_support_cols, P, A, h, (int)((long long)h * i / nt),
                          (int)((long long)h * (i + 1) / nt), part[i].data());
    host_support_cols(P, A, h, 0, h / nt, part[0].data());
    for (std::thread &t : pool) t.join();
    for (const auto &b : part) {
        box[0] = std::min(box[0], b[0]);
        box[1] = std::max(box[1], b[1]);
        box[2] = std::min(box[2], b[2]);
        box[3] = std::max(box[3], b[3]);
    }
}

fpm_status pupil_support(fpm_context *ctx, const fpm_problem *p, const Shape &s, Support &sup) {
    sup.r_lo = sup.c_lo = 0;
    sup.r_hi = sup.c_hi = s.h;
    if (const char *env = std::getenv("FPM_PUPIL_SUPPORT"))
        if (std::atoi(env) == 0) return FPM_OK;
    // ePIE scales each pupil term by the maximum over the LED's whole crop
    if (p->pie_weights == FPM_PIE_EPIE) return FPM_OK;
    int box[4] = {s.h, -1, s.h, -1};
    if (p->memory == FPM_MEM_HOST) {
        host_support_box(p->pupil_init, p->pupil_amp, s.h, box);
    } else {
        FPM_CK(ctx->flag.ensure(sizeof(int) * 4));
        FPM_CK(launch_support_box(reinterpret_cast<const float2 *>(p->pupil_init), p->pupil_amp,
                                  s.h, ctx->flag.as<int>(), ctx->stream));
        FPM_CK(cudaMemcpyAsync(box, ctx->flag.p, sizeof(box), cudaMemcpyDeviceToHost, ctx->stream));
        FPM_CK(cudaStreamSynchronize(ctx->stream));
    }
    if (box[1] < 0) return FPM_OK;   // an all-zero pupil: keep whole crops
    sup.r_lo = box[0];
    sup.r_hi = box[1] + 1;
    sup.c_lo = box[2];
    sup.c_hi = box[3] + 1;
    return FPM_OK;
}

// Crop boxes of every mini-batch of an epoch (the same every epoch).
struct Plan {
    std::vector<BatchGeom> geoms;
    int ldU = 0;        // max box rows
    size_t sbox = 0;    // max box rows x cols
    int group = 1;      // LEDs per low-resolution launch group
    int parts = 0;      // loss partial slots of the largest batch
    bool fused_rows = false;  // L2 + L3 as one pass (T2 instead of Rs)
};


Plan make_plan(const Shape &s, const std::vector<int32_t> &led, int batch, const Support &sup,
               int loss, int pie) {
    Plan pl;
    for (int cur = 0; cur < s.L; cur += batch) {
        const int nb = std::min(batch, s.L - cur);
        const Box b = batch_box(led, cur, nb, sup, s.H);
        BatchGeom g;
        g.H = s.H;
        g.h = s.h;
        g.pratio = s.pratio;
        g.z_off = cur;
        g.nb = nb;
        g.rlo = b.r_lo;
        g.rspan = b.r_span;
        g.clo = b.c_lo;
        g.cspan = b.c_span;
        g.Ru0 = (g.rlo + s.H / 2) % s.H;
        g.Cu0 = (g.clo + s.H / 2) % s.H;
        g.pr_lo = sup.r_lo;
        g.pr_hi = sup.r_hi;
        g.pc_lo = sup.c_lo;
        g.pc_hi = sup.c_hi;
        g.loss = loss == FPM_LOSS_ISOTROPIC ? kLossIsotropic : kLossAnisotropic;
        g.pie = pie;
        pl.geoms.push_back(g);
        pl.ldU = std::max(pl.ldU, (g.rspan + 3) & ~3);   // columns 32-byte aligned (bulk copies)
        pl.sbox = std::max(pl.sbox, (size_t)g.rspan * g.cspan);
    }
    // LEDs per low-resolution launch: the whole batch (measured fastest: large
    // grids, no tails; the field + residual of 26 LEDs of 2048^2 take 1.3 GB), capped
    // at 4 GiB of field + residual; FPM_LR_GROUP overrides it (tuning).
    const size_t per = s.plane * 16;
    pl.group = (int)std::max<size_t>(1, std::min<size_t>(s.B, (4ull << 30) / per));
    {
        const int v = knob("FPM_LR_GROUP", tuning().lr_group, 0, 0);
        if (v > 0) pl.group = std::min(v, pl.group);
    }
    // fused L2 + L3 where its CTA shape exists; FPM_LR_FUSED=0 keeps the separate passes
    pl.fused_rows = lr_rows_fused_supported(s.h) &&
                    knob("FPM_LR_FUSED", tuning().lr_fused, -1, 1) != 0;
    // with the fused row pass the field buffer is written by L1 alone: its unsupported
    // columns, cleared once per solve, stay zero and L1 skips them
    const bool pruned_cols = sup.c_lo > 0 || sup.c_hi < s.h;
    for (BatchGeom &g : pl.geoms) g.t1_clean = pl.fused_rows && pruned_cols ? 1 : 0;
    int parts = 0;
    for (int l0 = 0; l0 < s.B; l0 += pl.group) {
        const int nl = std::min(pl.group, s.B - l0);
        parts += pl.fused_rows ? lr_rows_fused_blocks(s.h, nl) : lr_blocks(s.h, nl);
    }
    pl.parts = parts;
    return pl;
}

size_t solve_bytes(const fpm_problem *p, const Shape &s, const Plan &pl, bool host, bool spec) {
    size_t b = 0;
    b += s.big * 8 + s.big * 4;                       // O, m1
    b += (size_t)s.H * pl.ldU * 8 * 3;                // U, V and their row-major twin
    b += pl.sbox * 8 * 2;                             // Sbox and its row-major twin
    b += s.plane * 8 * s.B;                           // Xs
    b += s.plane * (pl.fused_rows ? 16 : 12) * pl.group;   // T1 and T2 or Rs
    b += s.plane * (8 * 4 + 4 * 2);                   // P, dP, Pt, m2, P0
    if (spec) b += s.big * 8;                         // spectrum / gradient staging
    if (host) b += s.plane * s.L * (p->stack_type == FPM_STACK_U16_COUNTS ? 2 : 4);
    return b;
}

fpm_status alloc_pipeline(fpm_context *ctx, const fpm_problem *p, const Shape &s, const Plan &pl,
                          bool spec) {
    const size_t need = solve_bytes(p, s, pl, p->memory == FPM_MEM_HOST, spec);
    if (ctx->mem_limit && need > ctx->mem_limit)
        return fail(ctx, FPM_ERR_OUT_OF_MEMORY,
                    "solve needs %zu bytes of device memory, limit is %zu", need,
                    ctx->mem_limit);
    FPM_CK(ctx->U.ensure((size_t)s.H * pl.ldU * 8));
    FPM_CK(ctx->V.ensure((size_t)s.H * pl.ldU * 8));
    FPM_CK(ctx->W.ensure((size_t)s.H * pl.ldU * 8));
    FPM_CK(ctx->Sbox.ensure(pl.sbox * 8));
    FPM_CK(ctx->Sboxr.ensure(pl.sbox * 8));
    FPM_CK(ctx->Pt.ensure(s.plane * 8));
    FPM_CK(ctx->Xs.ensure(s.plane * 8 * s.B));
    FPM_CK(ctx->T1.ensure(s.plane * 8 * pl.group));
    if (!pl.geoms.empty() && pl.geoms[0].t1_clean)
        FPM_CK(cudaMemsetAsync(ctx->T1.p, 0, s.plane * 8 * pl.group, ctx->stream));
    if (pl.fused_rows)
        FPM_CK(ctx->T2.ensure(s.plane * 8 * pl.group));
    else
        FPM_CK(ctx->Rs.ensure(s.plane * 4 * pl.group));
    FPM_CK(ctx->dP.ensure(s.plane * 8));
    FPM_CK(ctx->parts.ensure(sizeof(double) * (size_t)std::max(pl.parts, 1)));
    FPM_CK(ctx->flag.ensure(sizeof(int) * 4));
    FPM_CK(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), ctx->stream));
    return FPM_OK;
}

fpm_status twiddles_of(fpm_context *ctx, const Shape &s, Twiddles &tw) {
    FPM_CK(ctx->fft.tables(s.h, &tw.lo_hi, &tw.lo_lo));
    FPM_CK(ctx->fft.tables(s.H, &tw.hi_hi, &tw.hi_lo));
    return FPM_OK;
}

BatchBufs bufs_of(fpm_context *ctx) {
    BatchBufs b;
    b.Sbox = ctx->Sbox.as<float2>();
    b.T1 = ctx->T1.as<float2>();
    b.Rs = ctx->Rs.as<float>();
    b.T2 = ctx->T2.as<float2>();
    b.flag = ctx->flag.as<int>();
    b.Xs = ctx->Xs.as<float2>();
    b.parts = ctx->parts.as<double>();
    return b;
}

// Row pass of the next box: V (column-major) -> Vr (row-major, in W) -> row FFTs ->
// Sboxr (row-major) -> Sbox (column-major), every access coalesced.
fpm_status rows_forward(fpm_context *ctx, const Plan &pl, const Twiddles &tw,
                        const BatchGeom &gn) {
    cudaStream_t st = ctx->stream;
    float2 *W = ctx->W.as<float2>();
    FPM_STAGE(ST_TRANSPOSE, launch_transpose(ctx->V.as<float2>(), pl.ldU, W, gn.H, gn.H, gn.rspan,
                                             0.f, st));
    FPM_STAGE(ST_ROWS_FORWARD, launch_big_rows_fwd(gn.H, W, gn.rspan, gn.Cu0, gn.cspan,
                                                   ctx->Sboxr.as<float2>(), tw, st,
                                                   ctx->flag.as<int>()));
    FPM_STAGE(ST_TRANSPOSE, launch_transpose(ctx->Sboxr.as<float2>(), gn.cspan,
                                             ctx->Sbox.as<float2>(), gn.rspan, gn.rspan, gn.cspan,
                                             0.f, st));
    return FPM_OK;
}

// S inside the first batch's box, from the object: column forward FFT pass, row pass.
fpm_status spectrum_box(fpm_context *ctx, const Plan &pl, const Twiddles &tw, float2 *O,
                        const BatchGeom &g) {
    ColsArgs a;
    a.mode = kColsForward;
    a.H = g.H;
    a.O = O;
    a.V = ctx->V.as<float2>();
    a.ldV = pl.ldU;
    a.Ru0n = g.Ru0;
    a.rspan_n = g.rspan;
    FPM_STAGE(ST_COLS_FORWARD, launch_big_cols(a, tw, ctx->stream));
    return rows_forward(ctx, pl, tw, g);
}

// Low-resolution passes of one batch (Xs, loss, pupil gradient) and pass A (U).
fpm_status lowres_and_stitch(fpm_context *ctx, const Plan &pl, const Twiddles &tw,
                             const Inputs &in, const float2 *P, const BatchGeom &g,
                             double *loss_slot) {
    cudaStream_t st = ctx->stream;
    BatchBufs b = bufs_of(ctx);
    int part_off = 0;
    for (int l0 = 0; l0 < g.nb; l0 += pl.group) {
        const int nl = std::min(pl.group, g.nb - l0);
        FPM_STAGE(ST_LR_COLS_INV, launch_lr_cols_inv(g, in.led, P, b, l0, nl, tw, st));
        if (pl.fused_rows) {
            FPM_STAGE(ST_LR_ROWS_FUSED,
                      launch_lr_rows_fused(g, in.Y, b, l0, nl, part_off, tw, st));
            FPM_STAGE(ST_LR_COLS_FWD, launch_lr_cols_fwd(g, b.T2, b, l0, nl, tw, st));
            part_off += lr_rows_fused_blocks(g.h, nl);
        } else {
            FPM_STAGE(ST_LR_ROWS_INV, launch_lr_rows_inv(g, in.Y, b, l0, nl, tw, st));
            FPM_STAGE(ST_LR_ROWS_FWD, launch_lr_rows_fwd(g, b, l0, nl, part_off, tw, st));
            FPM_STAGE(ST_LR_COLS_FWD, launch_lr_cols_fwd(g, b.T1, b, l0, nl, tw, st));
            part_off += lr_blocks(g.h, nl);
        }
    }
    FPM_STAGE(ST_LOSS, launch_loss_accumulate(b.parts, part_off, loss_slot, st));
    unsigned *pie = nullptr;
    if (g.pie != FPM_PIE_NONE) {   // ePIE / tPIE weights of the two gradient terms
        FPM_CK(ctx->pie.ensure(sizeof(unsigned) * (1 + (size_t)g.nb)));
        pie = ctx->pie.as<unsigned>();
        FPM_STAGE(ST_PUPIL_GRAD, launch_pie_prepare(g, P, in.led, b.Sbox, pie, st));
    }
    FPM_STAGE(ST_PUPIL_GRAD, launch_lr_pupil_grad(g, in.led, b, ctx->dP.as<float2>(), st, pie));
    // conj(P) / H^2, row-major, for coalesced pupil reads in the stitch
    FPM_STAGE(ST_TRANSPOSE, launch_transpose(P, g.h, ctx->Pt.as<float2>(), g.h, g.h, g.h,
                                             (float)(1.0 / ((double)g.H * g.H)), st));
    if (pie) FPM_STAGE(ST_TRANSPOSE, launch_pie_object_weights(g, ctx->Pt.as<float2>(), pie, st));
    float2 *W = ctx->W.as<float2>();
    FPM_STAGE(ST_ROWS_INV, launch_big_rows_inv(g, in.led, ctx->Pt.as<float2>(), b.Xs, W, tw, st));
    FPM_STAGE(ST_TRANSPOSE, launch_transpose(W, g.H, ctx->U.as<float2>(), pl.ldU, g.rspan, g.H,
                                             0.f, st));
    return FPM_OK;
}

fpm_status shape_of(fpm_context *ctx, const fpm_problem *p, Shape &s, bool need_batch) {
    fpm_status rc = validate(ctx, p, need_batch);
    if (rc != FPM_OK) return rc;
    s.h = p->h;
    s.pratio = p->pratio;
    s.H = p->h * p->pratio;
    s.L = p->n_leds;
    s.B = need_batch ? std::min(p->batch, p->n_leds) : p->n_leds;
    s.plane = (size_t)s.h * s.h;
    s.big = (size_t)s.H * s.H;
    return FPM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// ABI
// ---------------------------------------------------------------------------
extern "C" {

int32_t fpm_abi_version(void) { return FPM_ABI_VERSION; }

const char *fpm_status_string(fpm_status s) {
    switch (s) {
        case FPM_OK: return "ok";
        case FPM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case FPM_ERR_UNSUPPORTED: return "unsupported";
        case FPM_ERR_OUT_OF_MEMORY: return "out of device memory";
        case FPM_ERR_CUDA: return "CUDA error";
        case FPM_ERR_NONFINITE: return "non-finite loss";
        case FPM_ERR_NO_DEVICE: return "no CUDA device";
        case FPM_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

const char *fpm_last_error(const fpm_context *ctx) { return ctx ? ctx->err.c_str() : t_err.c_str(); }

fpm_status fpm_set_profiling(fpm_context *ctx, int32_t enable) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->prof.on = enable != 0;
    ctx->prof.reset();
    return FPM_OK;
}

int32_t fpm_stage_times(const fpm_context *ctx, fpm_stage_time *out, int32_t cap) {
    if (!ctx) return 0;
    int32_t k = 0;
    for (int i = 0; i < ST_COUNT; ++i) {
        if (ctx->prof.n[i] == 0) continue;
        if (out && k < cap) {
            out[k].name = kStageName[i];
            out[k].launches = ctx->prof.n[i];
            out[k].own_kernel = kStageOwn[i];
            out[k].ms = ctx->prof.ms[i];
        }
        ++k;
    }
    return k;
}

fpm_status fpm_create(fpm_context **out, const fpm_device_opts *opts) {
    if (!out) return FPM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FPM_ERR_NO_DEVICE;
    }
    const int dev = opts ? opts->device : 0;
    if (dev < 0 || dev >= ndev) return FPM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return FPM_ERR_NO_DEVICE;
    }
    fpm_context *ctx = new fpm_context();
    ctx->device = dev;
    ctx->mem_limit = opts ? opts->mem_limit_bytes : 0;
    ctx->flags = opts ? opts->flags : 0;
    if (opts && opts->stream) {
        ctx->stream = static_cast<cudaStream_t>(opts->stream);
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            delete ctx;
            return FPM_ERR_CUDA;
        }
        ctx->own_stream = true;
    }
    if (cudaEventCreateWithFlags(&ctx->entry, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return FPM_ERR_CUDA;
    }
    *out = ctx;
    return FPM_OK;
}

void fpm_destroy(fpm_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (fpm_context *w : ctx->workers) fpm_destroy(w);
    for (cudaStream_t sp : ctx->pool) cudaStreamDestroy(sp);
    if (ctx->epoch_graph) cudaGraphExecDestroy(ctx->epoch_graph);
    ctx->fft.release();
    ctx->gfft.release();
    if (ctx->entry) cudaEventDestroy(ctx->entry);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// Device-memory inputs are usually written on the legacy default stream (a MATLAB
// gpuArray, a torch tensor on torch's default stream), which a non-blocking context
// stream does not wait for: every call that reads device memory first makes the
// context's stream wait for the work already queued there.  Work on other streams
// must be complete before the call (the caller's responsibility, as in any CUDA API).
static fpm_status order_after_default_stream(fpm_context *ctx) {
    FPM_CK(cudaEventRecord(ctx->entry, cudaStreamLegacy));
    FPM_CK(cudaStreamWaitEvent(ctx->stream, ctx->entry, 0));
    return FPM_OK;
}

// A kernel whose bounded wait on an asynchronous copy gave up sets the context's
// device flag and skips its work; the call then fails instead of returning
// results computed from incomplete data.
static fpm_status check_device_flag(fpm_context *ctx) {
    int f = 0;
    FPM_CK(cudaMemcpy(&f, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) return fail(ctx, FPM_ERR_INTERNAL, "a device-side wait for a tile copy timed out");
    return FPM_OK;
}

// LED corners on the host (the crop boxes are planned from them), validated.
static fpm_status fetch_leds(fpm_context *ctx, const fpm_problem *p, const Shape &s,
                             std::vector<int32_t> &led) {
    led.resize(2 * (size_t)s.L);
    if (p->memory == FPM_MEM_HOST) {
        std::memcpy(led.data(), p->led_idx, 2 * sizeof(int32_t) * s.L);
    } else {
        FPM_CK(cudaMemcpyAsync(led.data(), p->led_idx, 2 * sizeof(int32_t) * s.L,
                               cudaMemcpyDeviceToHost, ctx->stream));
        FPM_CK(cudaStreamSynchronize(ctx->stream));
    }
    return check_leds(ctx, led, s.L, s.H);
}

// out = fftshift(fft2(O)) (out may not alias O).
static fpm_status centred_spectrum(fpm_context *ctx, const Shape &s, const float2 *O,
                                   float2 *out) {
    FPM_STAGE(ST_SPECTRUM, ctx->fft.run(O, out, s.H, 1, kForward, ctx->stream));
    FPM_CK(launch_centre_in_place(out, s.H, ctx->stream));
    return FPM_OK;
}

// Copy of a caller's input into a work buffer; host-to-device copies are timed as the
// copy_inputs_h2d stage when profiling.
static cudaError_t copy_in(fpm_context *ctx, void *dst, const void *src, size_t bytes,
                           cudaMemcpyKind kind) {
    const bool timed = kind == cudaMemcpyHostToDevice;
    if (timed) ctx->prof.begin(ctx->stream);
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, ctx->stream);
    if (timed && e == cudaSuccess) ctx->prof.end(ST_H2D, ctx->stream);
    return e;
}

// ---------------------------------------------------------------------------
// Any-size path (generic.cu): sides h, H with prime factors up to 7 that are not both
// powers of two.  Per batch, the reference's structure (cuFPM_pure_v3.cu:135-199) with
// the engine's own transforms: S = FFT2(O); per LED crop x pupil, inverse FFT2, loss
// gradient, forward FFT2; stitch of the gradient spectrum (an LED-ordered compensated
// gather over the batch's box, no atomics) and pupil gradient; g = IFFT2(G); RMSprop.
// Work buffers: S in ctx->S, G in ctx->U, the large transposes' scratch in ctx->W, the
// per-LED fields in ctx->T1 / ctx->T2 and their transposes' scratch in ctx->Xs.
// ---------------------------------------------------------------------------
static size_t gen_loss_parts(int h, int nb) {
    return (size_t)nb * (size_t)feature_grad_blocks_per_image(h);
}

static fpm_status gen_alloc(fpm_context *ctx, const fpm_problem *p, const Shape &s, bool host,
                            bool spec) {
    size_t need = s.big * 8 * 3 + s.plane * 8 * (size_t)s.B * 3 + s.plane * (8 * 3 + 4 * 2) +
                  sizeof(double) * gen_loss_parts(s.h, s.B);
    need += s.big * (8 + 4);                         // O, m1
    if (spec) need += s.big * 8;
    if (host) need += s.plane * s.L * (p->stack_type == FPM_STACK_U16_COUNTS ? 2 : 4);
    if (ctx->mem_limit && need > ctx->mem_limit)
        return fail(ctx, FPM_ERR_OUT_OF_MEMORY,
                    "solve needs %zu bytes of device memory, limit is %zu", need, ctx->mem_limit);
    FPM_CK(ctx->S.ensure(s.big * 8));
    FPM_CK(ctx->U.ensure(s.big * 8));
    FPM_CK(ctx->W.ensure(s.big * 8));
    FPM_CK(ctx->T1.ensure(s.plane * 8 * s.B));
    FPM_CK(ctx->T2.ensure(s.plane * 8 * s.B));
    FPM_CK(ctx->Xs.ensure(s.plane * 8 * s.B));
    FPM_CK(ctx->dP.ensure(s.plane * 8));
    FPM_CK(ctx->parts.ensure(sizeof(double) * std::max<size_t>(gen_loss_parts(s.h, s.B), 1)));
    FPM_CK(ctx->flag.ensure(sizeof(int) * 4));
    FPM_CK(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), ctx->stream));
    return FPM_OK;
}

// Gradients of LEDs [z_off, z_off + nb) at (O, P): the object gradient g = IFFT2(G) in
// ctx->U, the pupil gradient in ctx->dP, the batch loss added to *loss_slot.
static fpm_status gen_batch(fpm_context *ctx, const Shape &s, const Inputs &in, const float2 *O,
                            const float2 *P, int z_off, int nb, const Box &box, double *loss_slot,
                            int loss) {
    cudaStream_t st = ctx->stream;
    float2 *S = ctx->S.as<float2>(), *G = ctx->U.as<float2>(), *W = ctx->W.as<float2>();
    float2 *T1 = ctx->T1.as<float2>(), *T2 = ctx->T2.as<float2>(), *Tt = ctx->Xs.as<float2>();
    // the batch's crops read the spectrum on the box rows only (un-shifted: centred + H/2),
    // and the gradient spectrum is zero outside the box columns
    const int box_r = box.r_lo + s.H / 2, box_c = box.c_lo + s.H / 2;
    FPM_STAGE(ST_SPECTRUM,
              ctx->gfft.fft2_box(O, S, W, s.H, kForward, 0, s.H, box_r, box.r_span, st));   // K1
    FPM_STAGE(ST_LR_COLS_INV, launch_gen_crop_pupil(S, s.H, P, s.h, in.led, z_off, nb, T1, st));
    FPM_STAGE(ST_GEN_LR_FFT, ctx->gfft.fft2(T1, T1, Tt, s.h, nb, kInverse, st));        // K3
    FPM_STAGE(ST_GEN_LOSS, launch_feature_grad(T1, in.Y, z_off, nb, s.h, s.pratio, T2,
                                               ctx->parts.as<double>(), st, loss));     // K4
    FPM_STAGE(ST_LOSS, launch_loss_accumulate(ctx->parts.as<double>(),
                                              (int)gen_loss_parts(s.h, nb), loss_slot, st));
    FPM_STAGE(ST_GEN_LR_FFT, ctx->gfft.fft2(T2, T2, Tt, s.h, nb, kForward, st));        // K5
    {   // the inverse transform reads only the box columns (every row of them): those are
        // cleared, one or two contiguous runs, and the stitch fills its covered positions
        const int c0 = ((box_c % s.H) + s.H) % s.H, first = std::min(box.c_span, s.H - c0);
        FPM_CK(cudaMemsetAsync(G + (size_t)c0 * s.H, 0, (size_t)first * s.H * 8, st));
        if (box.c_span > first)
            FPM_CK(cudaMemsetAsync(G, 0, (size_t)(box.c_span - first) * s.H * 8, st));
    }
    FPM_STAGE(ST_GEN_STITCH, launch_gen_stitch(T2, s.h, P, in.led, z_off, nb, s.H, box.r_lo,
                                               box.r_span, box.c_lo, box.c_span, G, st));
    FPM_STAGE(ST_PUPIL_GRAD,
              launch_gen_pupil_grad(S, s.H, T2, s.h, in.led, z_off, nb, ctx->dP.as<float2>(), st));
    FPM_STAGE(ST_GEN_OBJ_FFT,
              ctx->gfft.fft2_box(G, G, W, s.H, kInverse, box_c, box.c_span, 0, s.H, st));   // K8
    return FPM_OK;
}

static fpm_status gradients_generic(fpm_context *ctx, const fpm_problem *p, const Shape &s,
                                    const std::vector<int32_t> &led_host, float *d_object,
                                    float *d_pupil, double *loss) {
    const bool dev = p->memory == FPM_MEM_DEVICE;
    fpm_status rc = gen_alloc(ctx, p, s, !dev, false);
    if (rc != FPM_OK) return rc;
    cudaStream_t st = ctx->stream;
    ctx->prof.reset();
    Inputs in;
    rc = stage_inputs(ctx, p, s, in);
    if (rc != FPM_OK) return rc;
    const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    FPM_CK(ctx->O.ensure(s.big * 8));
    FPM_CK(ctx->P.ensure(s.plane * 8));
    FPM_CK(copy_in(ctx, ctx->O.p, p->object_init, s.big * 8, kin));
    FPM_CK(copy_in(ctx, ctx->P.p, p->pupil_init, s.plane * 8, kin));
    FPM_CK(ctx->loss.ensure(sizeof(double)));
    FPM_CK(cudaMemsetAsync(ctx->loss.p, 0, sizeof(double), st));
    Support whole;
    whole.r_hi = whole.c_hi = s.h;
    const Box box = batch_box(led_host, 0, s.L, whole, s.H);
    rc = gen_batch(ctx, s, in, ctx->O.as<float2>(), ctx->P.as<float2>(), 0, s.L, box,
                   ctx->loss.as<double>(), p->loss_kind);
    if (rc != FPM_OK) return rc;
    const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (d_object) FPM_CK(cudaMemcpyAsync(d_object, ctx->U.p, s.big * 8, kout, st));
    if (d_pupil) FPM_CK(cudaMemcpyAsync(d_pupil, ctx->dP.p, s.plane * 8, kout, st));
    if (loss) FPM_CK(cudaMemcpyAsync(loss, ctx->loss.p, sizeof(double), kout, st));
    FPM_CK(cudaStreamSynchronize(st));
    FPM_CK(cudaGetLastError());
    ctx->prof.collect();
    return FPM_OK;
}

// ---------------------------------------------------------------------------
// One reconstruction in three phases: prepare (validation, plan, buffers, inputs, the
// initial object), epochs (enqueued one at a time, eagerly or replayed from a captured
// CUDA graph), finish (outputs, the one synchronisation, status).  fpm_solve runs the
// phases back to back; fpm_solve_batch interleaves them over many instances.
// ---------------------------------------------------------------------------
struct SolveJob {
    const fpm_problem *p = nullptr;
    fpm_result res{};
    Shape s{};
    bool dev = false, generic = false;
    std::vector<int32_t> led_host;
    Plan pl;                    // power-of-two path
    std::vector<Box> boxes;     // any-size path: the crop box of every mini-batch
    Inputs in;
    Twiddles tw;
    float2 *O = nullptr, *P = nullptr;
    const float *P0 = nullptr;
    float lr = 0.f;
    double *loss = nullptr;     // device: E epoch slots, then a captured epoch's accumulator
    int *epoch_counter = nullptr;   // device: the slot a captured epoch writes its loss to
};

static fpm_status job_prepare(fpm_context *ctx, const fpm_problem *p, fpm_result *res,
                              SolveJob &j) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    FPM_CK(cudaSetDevice(ctx->device));
    fpm_status rc = shape_of(ctx, p, j.s, true);
    if (rc != FPM_OK) return rc;
    const Shape &s = j.s;
    j.p = p;
    if (res) j.res = *res;
    j.dev = p->memory == FPM_MEM_DEVICE;
    const bool dev = j.dev;
    if (dev) {
        void *outs[4] = {j.res.object, j.res.spectrum, j.res.pupil, j.res.loss};
        for (int i = 0; i < 4; ++i) {
            if (outs[i] && !is_device_ptr(outs[i], ctx->device))
                return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "result pointer %d is not device memory",
                            i);
            if (outs[i] && (reinterpret_cast<uintptr_t>(outs[i]) & 15u))
                return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "result pointer %d is not 16-byte aligned",
                            i);
        }
        rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    rc = fetch_leds(ctx, p, s, j.led_host);
    if (rc != FPM_OK) return rc;
    j.generic = !pipeline_supported(s.h, s.H);
    if (j.generic) {
        rc = gen_alloc(ctx, p, s, !dev, j.res.spectrum != nullptr);
        if (rc != FPM_OK) return rc;
        Support whole;
        whole.r_hi = whole.c_hi = s.h;
        for (int cur = 0; cur < s.L; cur += s.B)
            j.boxes.push_back(batch_box(j.led_host, cur, std::min(s.B, s.L - cur), whole, s.H));
    } else {
        Support sup;
        rc = pupil_support(ctx, p, s, sup);
        if (rc != FPM_OK) return rc;
        j.pl = make_plan(s, j.led_host, p->batch, sup, p->loss_kind, p->pie_weights);
        rc = alloc_pipeline(ctx, p, s, j.pl, j.res.spectrum != nullptr);
        if (rc != FPM_OK) return rc;
    }
    cudaStream_t st = ctx->stream;
    ctx->prof.reset();
    rc = stage_inputs(ctx, p, s, j.in);
    if (rc != FPM_OK) return rc;
    if (!j.generic) {
        rc = twiddles_of(ctx, s, j.tw);
        if (rc != FPM_OK) return rc;
        if (j.pl.fused_rows) {
            rc = stack_rows(ctx, s, j.in);
            if (rc != FPM_OK) return rc;
        }
    }
    // object and pupil: work in the caller's device outputs when given, else internal
    if (dev && j.res.object) {
        j.O = reinterpret_cast<float2 *>(j.res.object);
    } else {
        FPM_CK(ctx->O.ensure(s.big * 8));
        j.O = ctx->O.as<float2>();
    }
    if (dev && j.res.pupil) {
        j.P = reinterpret_cast<float2 *>(j.res.pupil);
    } else {
        FPM_CK(ctx->P.ensure(s.plane * 8));
        j.P = ctx->P.as<float2>();
    }
    const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (p->object_init) {
        if ((const void *)p->object_init != (const void *)j.O)
            FPM_CK(copy_in(ctx, j.O, p->object_init, s.big * 8, kin));
    } else {
        DevBuf &scratch = j.generic ? ctx->Rs : ctx->T2;   // not in use before the loop
        FPM_CK(scratch.ensure(bicubic_work_bytes(s.h, s.pratio)));
        FPM_CK(launch_bicubic_init(j.in.Y, s.h, s.pratio, j.O, scratch.p, st));
    }
    if ((const void *)p->pupil_init != (const void *)j.P)
        FPM_CK(copy_in(ctx, j.P, p->pupil_init, s.plane * 8, kin));
    if (dev) {
        j.P0 = p->pupil_amp;
    } else {
        FPM_CK(ctx->P0.ensure(s.plane * 4));
        FPM_CK(copy_in(ctx, ctx->P0.p, p->pupil_amp, s.plane * 4, kin));
        j.P0 = ctx->P0.as<float>();
    }
    FPM_CK(ctx->m1.ensure(s.big * 4));
    FPM_CK(ctx->m2.ensure(s.plane * 4));
    FPM_CK(cudaMemsetAsync(ctx->m1.p, 0, s.big * 4, st));
    FPM_CK(cudaMemsetAsync(ctx->m2.p, 0, s.plane * 4, st));
    const int E = p->epochs;
    // E epoch slots, the accumulator of a captured epoch, and (as an int) its slot index
    FPM_CK(ctx->loss.ensure(sizeof(double) * (E + 2)));
    FPM_CK(cudaMemsetAsync(ctx->loss.p, 0, sizeof(double) * (E + 2), st));
    j.loss = ctx->loss.as<double>();
    j.epoch_counter = reinterpret_cast<int *>(j.loss + E + 1);
    if (!j.generic && E > 0) {
        rc = spectrum_box(ctx, j.pl, j.tw, j.O, j.pl.geoms[0]);
        if (rc != FPM_OK) return rc;
    }
    j.lr = p->lr;
    return FPM_OK;
}

// Enqueues one epoch; the batches' losses are added to *loss_slot.  In the final epoch
// (final) the last batch skips the spectrum of the next box, which nothing reads.
static fpm_status job_epoch(fpm_context *ctx, SolveJob &j, double *loss_slot, bool final) {
    const Shape &s = j.s;
    const fpm_problem *p = j.p;
    cudaStream_t st = ctx->stream;
    fpm_status rc;
    if (j.generic) {
        for (int bi = 0, cur = 0; cur < s.L; ++bi, cur += s.B) {   // cuFPM_pure_v3.cu:131-141
            const int nb = std::min(s.B, s.L - cur);
            rc = gen_batch(ctx, s, j.in, j.O, j.P, cur, nb, j.boxes[bi], loss_slot, p->loss_kind);
            if (rc != FPM_OK) return rc;
            FPM_STAGE(ST_GEN_RMS_OBJ, launch_rmsprop_object(j.O, ctx->m1.as<float>(),
                                                            ctx->U.as<float2>(), s.big, j.lr,
                                                            p->beta, p->eps, st));
            FPM_STAGE(ST_RMS_PUPIL,
                      launch_rmsprop_pupil(ctx->dP.as<float2>(), j.P, ctx->m2.as<float>(), j.P0,
                                           (int)s.plane, j.lr, p->beta, p->eps, p->pupil_margin,
                                           st));
        }
        return FPM_OK;
    }
    const Plan &pl = j.pl;
    const int nbatch = (int)pl.geoms.size();
    for (int bi = 0; bi < nbatch; ++bi) {
        const BatchGeom &g = pl.geoms[bi];
        const bool last = final && bi == nbatch - 1;
        const BatchGeom &gn = pl.geoms[(bi + 1) % nbatch];
        rc = lowres_and_stitch(ctx, pl, j.tw, j.in, j.P, g, loss_slot);
        if (rc != FPM_OK) return rc;
        ColsArgs a;
        a.mode = kColsUpdate;
        a.H = s.H;
        a.U = ctx->U.as<float2>();
        a.ldU = pl.ldU;
        a.Ru0 = g.Ru0;
        a.rspan = g.rspan;
        a.O = j.O;
        a.m = ctx->m1.as<float>();
        a.lr = j.lr;
        a.beta = p->beta;
        a.eps = p->eps;
        a.V = ctx->V.as<float2>();
        a.ldV = pl.ldU;
        a.Ru0n = last ? 0 : gn.Ru0;
        a.rspan_n = last ? 0 : gn.rspan;
        a.err = ctx->flag.as<int>();
        FPM_STAGE(ST_COLS_UPDATE, launch_big_cols(a, j.tw, st));
        if (!last) {
            rc = rows_forward(ctx, pl, j.tw, gn);
            if (rc != FPM_OK) return rc;
        }
        FPM_STAGE(ST_RMS_PUPIL,
                  launch_rmsprop_pupil(ctx->dP.as<float2>(), j.P, ctx->m2.as<float>(), j.P0,
                                       (int)s.plane, j.lr, p->beta, p->eps, p->pupil_margin, st));
    }
    return FPM_OK;
}

// lr schedule after epoch `ep` (cuFPM_pure_v3.cu:204-206)
static void job_lr_after(SolveJob &j, int ep) {
    if (ep > j.p->lr_halve_after) j.lr = (float)(j.lr * (double)j.p->lr_decay);
}

// One epoch captured from the context's stream into an executable graph.  Every replay
// adds its batches' losses to the accumulator slot, then moves the accumulator to the slot
// the device-side epoch counter names and advances the counter, so one graph serves every
// epoch that shares the learning rate.  *exec stays null when the capture did not succeed
// (a call the capture refused, or any failure while recording: nothing ran, and the caller
// runs the epochs eagerly, where a genuine error shows up again).  The executable graph
// belongs to the context and outlives the call: a capture with the same nodes and edges
// (a later learning rate, or a later solve of the same plan) writes its parameters into it
// instead of instantiating a new one; launches already enqueued keep the old parameters.
static fpm_status job_capture(fpm_context *ctx, SolveJob &j, cudaGraphExec_t *exec) {
    *exec = nullptr;
    cudaStream_t st = ctx->stream;
    const bool prof = ctx->prof.on;
    ctx->prof.on = false;   // no stage events inside a graph
    const int E = j.p->epochs;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->prof.on = prof;
        return FPM_OK;
    }
    const fpm_status rc = job_epoch(ctx, j, j.loss + E, false);
    cudaError_t le = cudaSuccess;
    if (rc == FPM_OK) le = launch_epoch_end(j.loss + E, j.loss, j.epoch_counter, st);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    ctx->prof.on = prof;
    if (rc != FPM_OK || le != cudaSuccess || e != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        ctx->err.clear();
        return FPM_OK;
    }
    if (ctx->epoch_graph) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ctx->epoch_graph, graph, &info) == cudaSuccess) {
            cudaGraphDestroy(graph);
            *exec = ctx->epoch_graph;
            return FPM_OK;
        }
        cudaGetLastError();   // another topology: a new executable graph replaces it
        cudaGraphExecDestroy(ctx->epoch_graph);
        ctx->epoch_graph = nullptr;
    }
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        *exec = nullptr;
        cudaGetLastError();
    } else {
        ctx->epoch_graph = *exec;
    }
    return FPM_OK;
}

static fpm_status job_finish(fpm_context *ctx, SolveJob &j) {
    const Shape &s = j.s;
    const bool dev = j.dev;
    cudaStream_t st = ctx->stream;
    fpm_result *res = &j.res;
    const int E = j.p->epochs;
    fpm_status rc;
    if (res->spectrum) {
        float2 *dst = reinterpret_cast<float2 *>(res->spectrum);
        if (!dev) {  // stage through a full-size device buffer
            FPM_CK(ctx->S.ensure(s.big * 8));
            dst = ctx->S.as<float2>();
        }
        if (j.generic) {
            FPM_STAGE(ST_SPECTRUM,
                      ctx->gfft.fft2(j.O, dst, ctx->W.as<float2>(), s.H, 1, kForward, st));
            FPM_CK(launch_centre_in_place(dst, s.H, st));
        } else {
            rc = centred_spectrum(ctx, s, j.O, dst);
            if (rc != FPM_OK) return rc;
        }
        if (!dev)
            FPM_STAGE(ST_D2H, cudaMemcpyAsync(res->spectrum, dst, s.big * 8,
                                              cudaMemcpyDeviceToHost, st));
    }
    if (!dev && res->object)
        FPM_STAGE(ST_D2H, cudaMemcpyAsync(res->object, j.O, s.big * 8, cudaMemcpyDeviceToHost, st));
    if (!dev && res->pupil)
        FPM_STAGE(ST_D2H, cudaMemcpyAsync(res->pupil, j.P, s.plane * 8, cudaMemcpyDeviceToHost, st));
    std::vector<double> loss_h(std::max(E, 1));
    FPM_CK(cudaMemcpyAsync(loss_h.data(), j.loss, sizeof(double) * std::max(E, 1),
                           cudaMemcpyDeviceToHost, st));
    if (res->loss && dev && E > 0)
        FPM_CK(cudaMemcpyAsync(res->loss, j.loss, sizeof(double) * E, cudaMemcpyDeviceToDevice, st));
    FPM_CK(cudaStreamSynchronize(st));
    FPM_CK(cudaGetLastError());
    ctx->prof.collect();
    {
        const fpm_status fr = check_device_flag(ctx);
        if (fr != FPM_OK) return fr;
    }
    if (res->loss && !dev) std::memcpy(res->loss, loss_h.data(), sizeof(double) * E);
    for (int ep = 0; ep < E; ++ep)
        if (!std::isfinite(loss_h[ep]))
            return fail(ctx, FPM_ERR_NONFINITE, "loss of epoch %d is not finite", ep);
    return FPM_OK;
}

// The epochs of a prepared job: epoch 0 eagerly (it builds every table and sets every
// kernel attribute the capture would otherwise meet), then one captured graph per learning
// rate, replayed once per epoch.  Without graphs (FPM_GRAPHS=0, stage profiling on, or a
// stream that cannot be captured) every epoch launches its kernels directly.
static fpm_status job_run_epochs(fpm_context *ctx, SolveJob &j, bool graphs) {
    const int E = j.p->epochs;
    cudaStream_t st = ctx->stream;
    fpm_status rc;
    if (E <= 0) return FPM_OK;
    rc = job_epoch(ctx, j, j.loss, E == 1);
    if (rc != FPM_OK) return rc;
    job_lr_after(j, 0);
    cudaGraphExec_t exec = nullptr;   // owned by the context (job_capture)
    float exec_lr = 0.f;
    for (int ep = 1; ep < E; ++ep) {
        if (graphs && (!exec || exec_lr != j.lr)) {
            exec = nullptr;
            FPM_CK(launch_set_int(j.epoch_counter, ep, st));   // the slot of the next replay
            rc = job_capture(ctx, j, &exec);
            if (rc != FPM_OK) return rc;
            exec_lr = j.lr;
            if (!exec) graphs = false;
        }
        if (exec) {
            const cudaError_t e = cudaGraphLaunch(exec, st);
            if (e != cudaSuccess) {
                cudaGraphExecDestroy(ctx->epoch_graph);
                ctx->epoch_graph = nullptr;
                return fail_cuda(ctx, e, "cudaGraphLaunch", __LINE__);
            }
        } else {
            rc = job_epoch(ctx, j, j.loss + ep, ep == E - 1);
            if (rc != FPM_OK) return rc;
        }
        job_lr_after(j, ep);
    }
    return FPM_OK;
}

static bool graphs_enabled(const fpm_context *ctx) {
    if (ctx->prof.on) return false;
    const char *env = std::getenv("FPM_GRAPHS");
    return !(env && std::atoi(env) == 0);
}

// ---------------------------------------------------------------------------
// Autotuner: one epoch per candidate launch choice on the caller's own problem,
// coordinate search from the defaults, the fastest kept per problem shape.
// ---------------------------------------------------------------------------
static std::vector<int> tune_key(const fpm_problem *p) {
    return {p->h, p->pratio, p->n_leds, std::min(p->batch, p->n_leds), p->stack_type,
            p->loss_kind, p->pie_weights};
}

// Device time of one eager epoch of p under tuning t (set-up excluded), outputs internal.
static fpm_status time_epoch(fpm_context *ctx, const fpm_problem *p, const Tuning &t, float *ms) {
    fpm_problem q = *p;
    q.epochs = 1;
    TuningScope scope(&t);
    SolveJob j;
    fpm_status rc = job_prepare(ctx, &q, nullptr, j);
    if (rc != FPM_OK) return rc;
    cudaEvent_t a = nullptr, b = nullptr;
    FPM_CK(cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return fail(ctx, FPM_ERR_CUDA, "cudaEventCreate");
    }
    cudaEventRecord(a, ctx->stream);
    rc = job_run_epochs(ctx, j, false);
    cudaEventRecord(b, ctx->stream);
    if (rc == FPM_OK) rc = job_finish(ctx, j);
    if (rc == FPM_OK && cudaEventElapsedTime(ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(ctx, FPM_ERR_CUDA, "cudaEventElapsedTime");
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

static std::string tuning_text(const Tuning &t) {
    char buf[256];
    snprintf(buf, sizeof buf, "lr_group=%d lr_fused=%d l23_cluster=%d cols_async=%d cols_e16=%d "
             "gen_lpc=%d", t.lr_group, t.lr_fused, t.l23_cluster, t.cols_async, t.cols_e16,
             t.gen_lpc);
    return buf;
}

}  // extern "C"

void *fpm::context_stream(fpm_context *ctx) { return ctx ? ctx->stream : nullptr; }
int fpm::context_device(fpm_context *ctx) { return ctx ? ctx->device : 0; }

extern "C" {

fpm_status fpm_selftest_bounded_wait(fpm_context *ctx, int64_t limit_cycles) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (limit_cycles < 1 || limit_cycles > (1ll << 32))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "limit_cycles = %lld", (long long)limit_cycles);
    FPM_CK(cudaSetDevice(ctx->device));
    FPM_CK(ctx->flag.ensure(sizeof(int) * 4));
    FPM_CK(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), ctx->stream));
    FPM_CK(launch_wait_selftest(ctx->flag.as<int>(), (long long)limit_cycles, ctx->stream));
    FPM_CK(cudaStreamSynchronize(ctx->stream));
    const fpm_status rc = check_device_flag(ctx);   // the path every solve takes
    FPM_CK(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), ctx->stream));
    FPM_CK(cudaStreamSynchronize(ctx->stream));
    return rc;
}

fpm_status fpm_autotune(fpm_context *ctx, const fpm_problem *p, char *report, size_t report_cap) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    Shape s;
    fpm_status rc = shape_of(ctx, p, s, true);
    if (rc != FPM_OK) return rc;
    const std::vector<int> key = tune_key(p);
    auto it = ctx->tuned.find(key);
    std::string text;
    if (it == ctx->tuned.end()) {
        // candidate values of each knob, tried one knob at a time from the best so far
        std::vector<std::pair<int Tuning::*, std::vector<int>>> knobs;
        const bool generic = !pipeline_supported(s.h, s.H);
        if (generic) {
            knobs.push_back({&Tuning::gen_lpc, {1, 2, 4, 8, 16}});
        } else {
            std::vector<int> groups;
            for (int g : {s.B / 2, 8, 4})
                if (g >= 1 && g < s.B) groups.push_back(g);
            knobs.push_back({&Tuning::lr_group, groups});
            if (lr_rows_fused_supported(s.h)) {
                knobs.push_back({&Tuning::lr_fused, {0}});
                if (s.h == 2048)
                    knobs.push_back({&Tuning::l23_cluster, {2, 8}});
                else
                    knobs.push_back({&Tuning::l23_cluster, {4}});
            }
            if (s.H == 16384) {
                knobs.push_back({&Tuning::cols_async, {0}});
                knobs.push_back({&Tuning::cols_e16, {1}});
            }
        }
        Tuning best;
        float best_ms = 0.f, first_ms = 0.f;
        rc = time_epoch(ctx, p, best, &best_ms);        // warm-up: tables, attributes, buffers
        if (rc == FPM_OK) rc = time_epoch(ctx, p, best, &best_ms);
        if (rc != FPM_OK) return rc;
        first_ms = best_ms;
        int trials = 2;
        for (const auto &kv : knobs) {
            const Tuning base = best;
            for (int v : kv.second) {
                Tuning t = base;
                t.*(kv.first) = v;
                float ms = 0.f;
                rc = time_epoch(ctx, p, t, &ms);
                if (rc != FPM_OK) return rc;
                ++trials;
                if (ms < 0.98f * best_ms) best_ms = ms, best = t;   // 2%: beyond the noise
            }
        }
        it = ctx->tuned.emplace(key, best).first;
        char buf[512];
        snprintf(buf, sizeof buf, "%s: %.3f ms/epoch (defaults %.3f ms, %d timed epochs)",
                 tuning_text(best).c_str(), best_ms, first_ms, trials);
        text = buf;
    } else {
        text = tuning_text(it->second) + " (cached)";
    }
    if (report && report_cap) {
        std::strncpy(report, text.c_str(), report_cap - 1);
        report[report_cap - 1] = '\0';
    }
    return FPM_OK;
}

// The tuning of p's shape: tuned now when the context asks for it, else the cached one.
static const Tuning *tuning_for(fpm_context *ctx, const fpm_problem *p, fpm_status *rc) {
    *rc = FPM_OK;
    if (!p) return nullptr;
    auto it = ctx->tuned.find(tune_key(p));
    if (it == ctx->tuned.end() && (ctx->flags & FPM_CTX_AUTOTUNE)) {
        *rc = fpm_autotune(ctx, p, nullptr, 0);
        if (*rc != FPM_OK) return nullptr;
        it = ctx->tuned.find(tune_key(p));
    }
    return it == ctx->tuned.end() ? nullptr : &it->second;
}

fpm_status fpm_solve(fpm_context *ctx, const fpm_problem *p, fpm_result *res) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    fpm_status rc;
    const Tuning *t = tuning_for(ctx, p, &rc);
    if (rc != FPM_OK) return rc;
    TuningScope scope(t);
    SolveJob j;
    rc = job_prepare(ctx, p, res, j);
    if (rc != FPM_OK) return rc;
    rc = job_run_epochs(ctx, j, graphs_enabled(ctx));
    if (rc != FPM_OK) return rc;
    return job_finish(ctx, j);
}

// Worker contexts of fpm_solve_batch: one per instance (its buffers stay allocated for
// the next call), on a pool of kBatchStreams streams owned by the parent context.
static constexpr int kBatchStreams = 8;

fpm_status fpm_solve_batch(fpm_context *ctx, const fpm_problem *problems, fpm_result *results,
                           int32_t n, int32_t flags, fpm_status *statuses) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!problems || n < 1) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "no problems (n = %d)", n);
    if (flags & ~FPM_BATCH_EAGER) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "flags = %d", flags);
    FPM_CK(cudaSetDevice(ctx->device));
    while ((int)ctx->pool.size() < std::min(n, kBatchStreams)) {
        cudaStream_t sp = nullptr;
        FPM_CK(cudaStreamCreateWithFlags(&sp, cudaStreamNonBlocking));
        ctx->pool.push_back(sp);
    }
    while ((int)ctx->workers.size() < n) {
        const int i = (int)ctx->workers.size();
        fpm_device_opts o{};
        o.device = ctx->device;
        o.mem_limit_bytes = ctx->mem_limit;
        o.stream = ctx->pool[i % ctx->pool.size()];
        fpm_context *w = nullptr;
        const fpm_status cs = fpm_create(&w, &o);
        if (cs != FPM_OK) return fail(ctx, cs, "worker context %d: %s", i, fpm_status_string(cs));
        ctx->workers.push_back(w);
    }
    const bool graphs = !(flags & FPM_BATCH_EAGER) && graphs_enabled(ctx);
    std::vector<SolveJob> jobs(n);
    std::vector<fpm_status> st(n, FPM_OK);
    // prepare every instance, then enqueue every instance's epochs (no host waits between
    // them: the instances run concurrently on the pool's streams), then finish each
    std::vector<const Tuning *> tun(n, nullptr);
    for (int i = 0; i < n; ++i) {
        tun[i] = tuning_for(ctx, &problems[i], &st[i]);
        if (st[i] != FPM_OK) continue;
        TuningScope scope(tun[i]);
        st[i] = job_prepare(ctx->workers[i], &problems[i], results ? &results[i] : nullptr, jobs[i]);
    }
    for (int i = 0; i < n; ++i) {
        if (st[i] != FPM_OK) continue;
        TuningScope scope(tun[i]);
        st[i] = job_run_epochs(ctx->workers[i], jobs[i], graphs);
    }
    fpm_status first = FPM_OK;
    for (int i = 0; i < n; ++i) {
        if (st[i] == FPM_OK) {
            st[i] = job_finish(ctx->workers[i], jobs[i]);
        } else {
            cudaStreamSynchronize(ctx->workers[i]->stream);   // nothing left in flight
            cudaGetLastError();
        }
        if (st[i] != FPM_OK && first == FPM_OK) {
            first = st[i];
            fail(ctx, st[i], "instance %d: %s", i, ctx->workers[i]->err.c_str());
        }
        if (statuses) statuses[i] = st[i];
    }
    return first;
}

fpm_status fpm_batch_gradients(fpm_context *ctx, const fpm_problem *p, float *d_object,
                               float *d_pupil, double *loss) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    FPM_CK(cudaSetDevice(ctx->device));
    Shape s;
    fpm_status rc = shape_of(ctx, p, s, false);
    if (rc != FPM_OK) return rc;
    if (!p->object_init)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "object_init is required for gradients");
    if (s.L > 1024) return fail(ctx, FPM_ERR_UNSUPPORTED, "batch of %d LEDs exceeds 1024", s.L);
    const bool dev = p->memory == FPM_MEM_DEVICE;
    void *outs[3] = {d_object, d_pupil, loss};
    for (int i = 0; i < 3; ++i) {
        if (!outs[i]) continue;
        if (dev && !is_device_ptr(outs[i], ctx->device))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "output %d is not device memory", i);
        if (dev && (reinterpret_cast<uintptr_t>(outs[i]) & 15u))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "output %d is not 16-byte aligned", i);
        if (!dev && !is_host_ptr(outs[i]))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "output %d is not host memory", i);
    }
    if (dev) {
        rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    std::vector<int32_t> led_host;
    rc = fetch_leds(ctx, p, s, led_host);
    if (rc != FPM_OK) return rc;
    if (!pipeline_supported(s.h, s.H))
        return gradients_generic(ctx, p, s, led_host, d_object, d_pupil, loss);
    Support full;   // the pupil gradient is an output here: whole crops
    full.r_hi = full.c_hi = s.h;
    const Plan pl = make_plan(s, led_host, s.L, full, p->loss_kind, p->pie_weights);
    rc = alloc_pipeline(ctx, p, s, pl, true);
    if (rc != FPM_OK) return rc;
    cudaStream_t st = ctx->stream;
    ctx->prof.reset();
    Inputs in;
    rc = stage_inputs(ctx, p, s, in);
    if (rc != FPM_OK) return rc;
    if (pl.fused_rows) {
        rc = stack_rows(ctx, s, in);
        if (rc != FPM_OK) return rc;
    }
    Twiddles tw;
    rc = twiddles_of(ctx, s, tw);
    if (rc != FPM_OK) return rc;
    const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    FPM_CK(ctx->O.ensure(s.big * 8));
    FPM_CK(ctx->P.ensure(s.plane * 8));
    FPM_CK(cudaMemcpyAsync(ctx->O.p, p->object_init, s.big * 8, kin, st));
    FPM_CK(cudaMemcpyAsync(ctx->P.p, p->pupil_init, s.plane * 8, kin, st));
    FPM_CK(ctx->loss.ensure(sizeof(double)));
    FPM_CK(cudaMemsetAsync(ctx->loss.p, 0, sizeof(double), st));
    const BatchGeom &g = pl.geoms[0];
    rc = spectrum_box(ctx, pl, tw, ctx->O.as<float2>(), g);
    if (rc != FPM_OK) return rc;
    rc = lowres_and_stitch(ctx, pl, tw, in, ctx->P.as<float2>(), g, ctx->loss.as<double>());
    if (rc != FPM_OK) return rc;
    FPM_CK(ctx->S.ensure(s.big * 8));
    float2 *gout = dev && d_object ? reinterpret_cast<float2 *>(d_object) : ctx->S.as<float2>();
    ColsArgs a;
    a.mode = kColsGradient;
    a.H = s.H;
    a.U = ctx->U.as<float2>();
    a.ldU = pl.ldU;
    a.Ru0 = g.Ru0;
    a.rspan = g.rspan;
    a.gout = gout;
    FPM_STAGE(ST_COLS_UPDATE, launch_big_cols(a, tw, st));
    const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (d_object && !dev) FPM_CK(cudaMemcpyAsync(d_object, gout, s.big * 8, kout, st));
    if (d_pupil) FPM_CK(cudaMemcpyAsync(d_pupil, ctx->dP.p, s.plane * 8, kout, st));
    if (loss) FPM_CK(cudaMemcpyAsync(loss, ctx->loss.p, sizeof(double), kout, st));
    FPM_CK(cudaStreamSynchronize(st));
    ctx->prof.collect();
    {
        const fpm_status fr = check_device_flag(ctx);
        if (fr != FPM_OK) return fr;
    }
    return FPM_OK;
}

fpm_status fpm_fft2(fpm_context *ctx, const float *in, float *out, int32_t n, int32_t count,
                    int32_t direction, int32_t memory) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!in || !out || count < 1 || (direction != -1 && direction != 1))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "bad fft2 arguments");
    if (!fft_supported(n) && !gen_fft_supported(n))
        return fail(ctx, FPM_ERR_UNSUPPORTED, "n = %d: 2 <= n <= %d with no prime factor above 7",
                    n, kMaxFftLen);
    if (memory != FPM_MEM_DEVICE && memory != FPM_MEM_HOST)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "memory = %d", memory);
    FPM_CK(cudaSetDevice(ctx->device));
    const bool dev = memory == FPM_MEM_DEVICE;
    const size_t bytes = (size_t)n * n * count * 8;
    if (dev) {
        if (!is_device_ptr(in, ctx->device) || !is_device_ptr(out, ctx->device) ||
            ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "in/out: 16-byte aligned device memory");
    } else if (!is_host_ptr(in) || !is_host_ptr(out)) {
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "in/out are not host memory");
    }
    if (ctx->mem_limit && !dev && bytes > ctx->mem_limit)
        return fail(ctx, FPM_ERR_OUT_OF_MEMORY, "fft2 needs %zu bytes", bytes);
    if (dev) {
        const fpm_status rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    cudaStream_t st = ctx->stream;
    const float2 *src = reinterpret_cast<const float2 *>(in);
    float2 *dst = reinterpret_cast<float2 *>(out);
    if (!dev) {
        FPM_CK(ctx->spec.ensure(bytes));
        FPM_CK(cudaMemcpyAsync(ctx->spec.p, in, bytes, cudaMemcpyHostToDevice, st));
        src = dst = ctx->spec.as<float2>();
    }
    const FftDir fdir = direction < 0 ? kForward : kInverse;
    if (fft_supported(n)) {
        FPM_CK(ctx->fft.run(src, dst, n, count, fdir, st));
    } else {   // any-size transform: its transposes need a scratch of the same size
        FPM_CK(ctx->W.ensure(bytes));
        FPM_CK(ctx->gfft.fft2(src, dst, ctx->W.as<float2>(), n, count, fdir, st));
    }
    if (!dev) FPM_CK(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, st));
    FPM_CK(cudaStreamSynchronize(st));
    return FPM_OK;
}

fpm_status fpm_led_indices(fpm_context *ctx, const fpm_led_geometry *geo, int32_t *led_idx,
                           int32_t *grid_pos) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!geo || !led_idx) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "geo or led_idx is NULL");
    const fpm_led_geometry &g = *geo;
    if (g.grid < 1 || g.grid > 255 || g.grid % 2 == 0)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "grid = %d: an odd LED count per side, 1..255",
                    g.grid);
    if (g.h < 2 || g.h % 2 || g.pratio < 1 || (long long)g.h * g.pratio > (1 << 20))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "h = %d, pratio = %d", g.h, g.pratio);
    const double pos[] = {g.wavelength_um, g.led_height_um, g.camera_pixel_um, g.magnification};
    for (double v : pos)
        if (!(v > 0) || !std::isfinite(v))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT,
                        "wavelength, LED height, camera pixel and magnification must be > 0");
    if (!std::isfinite(g.led_pitch_um) || !std::isfinite(g.sample_dx_um) ||
        !std::isfinite(g.sample_dy_um))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "non-finite LED pitch or sample offset");
    if (!is_host_ptr(led_idx) || (grid_pos && !is_host_ptr(grid_pos)))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "led_idx / grid_pos must be host memory");
    FPM_CK(cudaSetDevice(ctx->device));
    std::vector<int2> order;
    spiral_grid_order(g.grid, order);
    const int L = g.grid * g.grid;
    if ((int)order.size() != L) return fail(ctx, FPM_ERR_INTERNAL, "spiral order incomplete");
    LedGeom p;
    p.grid = g.grid;
    p.h = g.h;
    p.NN = g.h * g.pratio;
    p.pitch = g.led_pitch_um;
    p.height = g.led_height_um;
    p.dx = g.sample_dx_um;
    p.dy = g.sample_dy_um;
    p.two_pi = 2 * M_PI;
    p.k_lamuda = p.two_pi / g.wavelength_um;          // k_lamuda = 2*pi/lamuda
    const double d_pixel = g.camera_pixel_um / g.magnification;   // D_pixel
    p.ND = (double)g.h * d_pixel;                       // N * D_pixel
    cudaStream_t st = ctx->stream;
    FPM_CK(ctx->led.ensure((size_t)L * 16));
    int2 *d_pos = ctx->led.as<int2>();
    int32_t *d_idx = reinterpret_cast<int32_t *>(d_pos + L);
    FPM_CK(cudaMemcpyAsync(d_pos, order.data(), (size_t)L * 8, cudaMemcpyHostToDevice, st));
    FPM_CK(launch_led_nearest(d_pos, L, p, d_idx, st));
    FPM_CK(cudaMemcpyAsync(led_idx, d_idx, (size_t)L * 8, cudaMemcpyDeviceToHost, st));
    FPM_CK(cudaStreamSynchronize(st));
    if (grid_pos) std::memcpy(grid_pos, order.data(), (size_t)L * 8);
    return FPM_OK;
}

fpm_status fpm_simulate(fpm_context *ctx, const float *object, const float *pupil,
                        const int32_t *led_idx, int32_t h, int32_t pratio, int32_t n_leds,
                        int32_t output, float *out, int32_t memory) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!object || !pupil || !led_idx || !out)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "object, pupil, led_idx and out are required");
    if (n_leds < 1) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "n_leds = %d", n_leds);
    if (output != FPM_SIM_INTENSITY && output != FPM_SIM_AMPLITUDE)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "output = %d", output);
    if (memory != FPM_MEM_DEVICE && memory != FPM_MEM_HOST)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "memory = %d", memory);
    if (h < 2 || (h & 1) || pratio < 1 || (long long)h * pratio > kMaxFftLen ||
        !(pipeline_supported(h, h * pratio) ||
          (gen_fft_supported(h) && gen_fft_supported(h * pratio))))
        return fail(ctx, FPM_ERR_UNSUPPORTED,
                    "h = %d, pratio = %d: even h, h and h*pratio <= %d with no prime factor "
                    "above 7", h, pratio, kMaxFftLen);
    FPM_CK(cudaSetDevice(ctx->device));
    const bool dev = memory == FPM_MEM_DEVICE;
    const void *ptrs[4] = {object, pupil, led_idx, out};
    for (int i = 0; i < 4; ++i) {
        if (dev && (!is_device_ptr(ptrs[i], ctx->device) ||
                    (reinterpret_cast<uintptr_t>(ptrs[i]) & 15u)))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT,
                        "pointer %d: 16-byte aligned device memory expected", i);
        if (!dev && !is_host_ptr(ptrs[i]))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointer %d is not host memory", i);
    }
    const int H = h * pratio;
    const size_t plane = (size_t)h * h, big = (size_t)H * H;
    const int group = (int)std::max<size_t>(1, std::min<size_t>(n_leds, (2ull << 30) / (plane * 8)));
    const size_t need = big * 8 * (dev ? 1 : 2) + plane * 8 * (group + (dev ? 0 : 1)) +
                        (dev ? 0 : plane * 4 * group);
    if (ctx->mem_limit && need > ctx->mem_limit)
        return fail(ctx, FPM_ERR_OUT_OF_MEMORY, "simulation needs %zu bytes, limit is %zu", need,
                    ctx->mem_limit);
    cudaStream_t st = ctx->stream;
    if (dev) {
        const fpm_status rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    std::vector<int32_t> led_host(2 * (size_t)n_leds);
    FPM_CK(cudaMemcpyAsync(led_host.data(), led_idx, led_host.size() * 4,
                           dev ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost, st));
    FPM_CK(cudaStreamSynchronize(st));
    fpm_status rc = check_leds(ctx, led_host, n_leds, H);
    if (rc != FPM_OK) return rc;
    ctx->prof.reset();
    const float2 *O = reinterpret_cast<const float2 *>(object);
    const float2 *P = reinterpret_cast<const float2 *>(pupil);
    const int2 *led = reinterpret_cast<const int2 *>(led_idx);
    if (!dev) {
        FPM_CK(ctx->O.ensure(big * 8));
        FPM_CK(ctx->P.ensure(plane * 8));
        FPM_CK(ctx->led.ensure(led_host.size() * 4));
        FPM_CK(cudaMemcpyAsync(ctx->O.p, object, big * 8, cudaMemcpyHostToDevice, st));
        FPM_CK(cudaMemcpyAsync(ctx->P.p, pupil, plane * 8, cudaMemcpyHostToDevice, st));
        FPM_CK(cudaMemcpyAsync(ctx->led.p, led_host.data(), led_host.size() * 4,
                               cudaMemcpyHostToDevice, st));
        O = ctx->O.as<float2>();
        P = ctx->P.as<float2>();
        led = ctx->led.as<int2>();
    }
    const float scale = (float)(1.0 / ((double)plane * pratio * pratio));
    if (!pipeline_supported(h, H)) {
        // any size: spectrum (un-shifted), crop x pupil with the inverse shift, inverse 2-D
        // FFT of each LED's page, magnitude
        FPM_CK(ctx->S.ensure(big * 8));
        FPM_CK(ctx->W.ensure(std::max(big, plane * group) * 8));
        FPM_CK(ctx->T1.ensure(plane * 8 * group));
        if (!dev) FPM_CK(ctx->Rs.ensure(plane * 4 * group));
        float2 *S = ctx->S.as<float2>(), *W = ctx->W.as<float2>(), *T1 = ctx->T1.as<float2>();
        FPM_STAGE(ST_SPECTRUM, ctx->gfft.fft2(O, S, W, H, 1, kForward, st));
        for (int l0 = 0; l0 < n_leds; l0 += group) {
            const int nl = std::min(group, n_leds - l0);
            FPM_STAGE(ST_LR_COLS_INV, launch_gen_crop_pupil(S, H, P, h, led, l0, nl, T1, st));
            FPM_STAGE(ST_SIM_ROWS_INV, ctx->gfft.fft2(T1, T1, W, h, nl, kInverse, st));
            float *dst = dev ? out + plane * l0 : ctx->Rs.as<float>();
            FPM_STAGE(ST_SIM_MAGNITUDE, launch_sim_magnitude(T1, plane * nl, scale,
                                                             output == FPM_SIM_AMPLITUDE, dst, st));
            if (!dev)
                FPM_CK(cudaMemcpyAsync(out + plane * l0, dst, plane * 4 * nl,
                                       cudaMemcpyDeviceToHost, st));
        }
        FPM_CK(cudaStreamSynchronize(st));
        ctx->prof.collect();
        return FPM_OK;
    }
    // centred spectrum of the object (gen_img_batch.m:184, fftshift(fft2(wavefront1)))
    FPM_CK(ctx->S.ensure(big * 8));
    float2 *Sc = ctx->S.as<float2>();
    FPM_STAGE(ST_SPECTRUM, ctx->fft.run(O, Sc, H, 1, kForward, st));
    FPM_CK(launch_centre_in_place(Sc, H, st));
    // the whole centred spectrum as the box of every LED, whole crops
    BatchGeom g;
    g.H = H;
    g.h = h;
    g.pratio = pratio;
    g.z_off = 0;
    g.nb = n_leds;
    g.rlo = g.clo = 0;
    g.rspan = g.cspan = H;
    g.Ru0 = g.Cu0 = H / 2;
    g.pr_lo = g.pc_lo = 0;
    g.pr_hi = g.pc_hi = h;
    Twiddles tw;
    FPM_CK(ctx->fft.tables(h, &tw.lo_hi, &tw.lo_lo));
    FPM_CK(ctx->T1.ensure(plane * 8 * group));
    if (!dev) FPM_CK(ctx->Rs.ensure(plane * 4 * group));
    BatchBufs b;
    b.Sbox = Sc;
    b.T1 = ctx->T1.as<float2>();
    for (int l0 = 0; l0 < n_leds; l0 += group) {
        const int nl = std::min(group, n_leds - l0);
        // crop x pupil, ifftshift, inverse FFT along r; then along c
        FPM_STAGE(ST_LR_COLS_INV, launch_lr_cols_inv(g, led, P, b, l0, nl, tw, st));
        FPM_STAGE(ST_SIM_ROWS_INV, ctx->fft.run_axis(b.T1, b.T1, h, nl, 1, kInverse, st));
        float *dst = dev ? out + plane * l0 : ctx->Rs.as<float>();
        FPM_STAGE(ST_SIM_MAGNITUDE, launch_sim_magnitude(b.T1, plane * nl, scale,
                                                         output == FPM_SIM_AMPLITUDE, dst, st));
        if (!dev)
            FPM_CK(cudaMemcpyAsync(out + plane * l0, dst, plane * 4 * nl, cudaMemcpyDeviceToHost,
                                   st));
    }
    FPM_CK(cudaStreamSynchronize(st));
    ctx->prof.collect();
    return FPM_OK;
}

fpm_status fpm_normalise_stack(fpm_context *ctx, const uint16_t *counts, size_t n,
                               float *amplitude, int32_t memory) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!counts || !amplitude || n == 0)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "counts/amplitude NULL or n == 0");
    FPM_CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool dev = memory == FPM_MEM_DEVICE;
    if (memory != FPM_MEM_DEVICE && memory != FPM_MEM_HOST)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "memory = %d", memory);
    if (dev && (!is_device_ptr(counts, ctx->device) || !is_device_ptr(amplitude, ctx->device)))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointers are not device memory");
    if (!dev && (!is_host_ptr(counts) || !is_host_ptr(amplitude)))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointers are not host memory");
    if (dev) {
        const fpm_status rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    const uint16_t *src = counts;
    float *dst = amplitude;
    if (!dev) {
        FPM_CK(ctx->Y.ensure(n * 2));
        FPM_CK(ctx->spec.ensure(n * 4));
        FPM_CK(cudaMemcpyAsync(ctx->Y.p, counts, n * 2, cudaMemcpyHostToDevice, st));
        src = ctx->Y.as<uint16_t>();
        dst = ctx->spec.as<float>();
    }
    FPM_CK(ctx->minmax.ensure(2 * sizeof(unsigned)));
    FPM_CK(launch_stack_minmax(src, n, ctx->minmax.as<unsigned>(), st));
    FPM_CK(launch_normalise(src, n, ctx->minmax.as<unsigned>(), dst, st));
    if (!dev) FPM_CK(cudaMemcpyAsync(amplitude, dst, n * 4, cudaMemcpyDeviceToHost, st));
    FPM_CK(cudaStreamSynchronize(st));
    return FPM_OK;
}

fpm_status fpm_normalise_stack_f32(fpm_context *ctx, const float *values, size_t n,
                                   float *amplitude, int32_t memory) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!values || !amplitude || n == 0)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "values/amplitude NULL or n == 0");
    FPM_CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool dev = memory == FPM_MEM_DEVICE;
    if (memory != FPM_MEM_DEVICE && memory != FPM_MEM_HOST)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "memory = %d", memory);
    if (dev && (!is_device_ptr(values, ctx->device) || !is_device_ptr(amplitude, ctx->device)))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointers are not device memory");
    if (!dev && (!is_host_ptr(values) || !is_host_ptr(amplitude)))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointers are not host memory");
    if (dev) {
        const fpm_status rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    const float *src = values;
    float *dst = amplitude;
    if (!dev) {
        // normalised in place in one device buffer
        FPM_CK(ctx->spec.ensure(n * 4));
        FPM_CK(cudaMemcpyAsync(ctx->spec.p, values, n * 4, cudaMemcpyHostToDevice, st));
        src = dst = ctx->spec.as<float>();
    }
    FPM_CK(ctx->minmax.ensure(2 * sizeof(unsigned)));
    FPM_CK(launch_normalise_f32(src, n, ctx->minmax.as<unsigned>(), dst, st));
    if (!dev) FPM_CK(cudaMemcpyAsync(amplitude, dst, n * 4, cudaMemcpyDeviceToHost, st));
    FPM_CK(cudaStreamSynchronize(st));
    return FPM_OK;
}

fpm_status fpm_read_tiff_stack(fpm_context *ctx, const char *const *paths, int32_t n_images,
                               int32_t row0, int32_t col0, int32_t h, int32_t type, void *stack,
                               int32_t threads) {
    (ctx ? ctx->err : t_err).clear();
    if (!paths || !stack || n_images <= 0 || h <= 0)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "paths/stack NULL, n_images <= 0 or h <= 0");
    if (type != FPM_INGEST_U16 && type != FPM_INGEST_F32_MEAN)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "type = %d", type);
    if (row0 < 0 || col0 < 0)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "row0 = %d, col0 = %d", row0, col0);
    const std::string err =
        read_tiff_stack(paths, n_images, row0, col0, h,
                        type == FPM_INGEST_U16 ? TiffOut::kU16 : TiffOut::kF32Mean, stack, threads);
    if (!err.empty()) return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "%s", err.c_str());
    return FPM_OK;
}

fpm_status fpm_optimizer_step(fpm_context *ctx, const fpm_optimizer *opt, float *param,
                              const float *grad, size_t n, int32_t memory) {
    if (!ctx) return FPM_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    if (!opt || !param || !grad || n == 0)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "opt/param/grad NULL or n == 0");
    if (memory != FPM_MEM_DEVICE && memory != FPM_MEM_HOST)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "memory = %d", memory);
    const int kind = opt->kind;
    if (kind < FPM_OPT_RMSPROP || kind > FPM_OPT_SGD)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "optimizer kind = %d", kind);
    if (!std::isfinite(opt->lr) || !std::isfinite(opt->beta1) || !std::isfinite(opt->beta2) ||
        !std::isfinite(opt->momentum) || !std::isfinite(opt->clamp_margin))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "non-finite hyper-parameter");
    const bool rms = kind == FPM_OPT_RMSPROP, moments = kind == FPM_OPT_ADAM || kind == FPM_OPT_YOGI;
    const bool use_g0 = rms && opt->centered, use_buf = rms && opt->momentum > 0;
    if (moments && (!opt->mom1 || !opt->mom2))
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "Adam / Yogi need mom1 and mom2");
    if (use_g0 && !opt->mom1)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "centered RMSprop needs mom1 (g0)");
    if (use_buf && !opt->buffer)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "RMSprop with momentum needs buffer");
    if (kind == FPM_OPT_ADAM && opt->iter < 1)
        return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "Adam needs iter >= 1");
    FPM_CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool dev = memory == FPM_MEM_DEVICE;
    // (pointer, bytes, written back) of every array the step touches
    struct Arr {
        const void *p;
        size_t bytes;
        bool out;
    } arrs[6] = {{param, n * 8, true},
                 {grad, n * 8, false},
                 {(moments || use_g0) ? opt->mom1 : nullptr, n * 8, true},
                 {moments ? opt->mom2 : nullptr, n * 4, true},
                 {use_buf ? opt->buffer : nullptr, n * 8, true},
                 {opt->clamp_amp, n * 4, false}};
    for (const Arr &a : arrs) {
        if (!a.p) continue;
        if (dev && !is_device_ptr(a.p, ctx->device))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointers are not device memory");
        if (dev && (reinterpret_cast<uintptr_t>(a.p) & 7))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "device pointers must be 8-byte aligned");
        if (!dev && !is_host_ptr(a.p))
            return fail(ctx, FPM_ERR_INVALID_ARGUMENT, "pointers are not host memory");
    }
    if (dev) {
        const fpm_status rc = order_after_default_stream(ctx);
        if (rc != FPM_OK) return rc;
    }
    void *d[6] = {};
    for (int k = 0; k < 6; ++k) {
        if (!arrs[k].p) continue;
        if (dev) {
            d[k] = const_cast<void *>(arrs[k].p);
        } else {
            FPM_CK(ctx->opt[k].ensure(arrs[k].bytes));
            FPM_CK(cudaMemcpyAsync(ctx->opt[k].p, arrs[k].p, arrs[k].bytes, cudaMemcpyHostToDevice,
                                   st));
            d[k] = ctx->opt[k].p;
        }
    }
    OptStep o;
    o.kind = kind;
    o.n = n;
    o.p = static_cast<float2 *>(d[0]);
    o.g = static_cast<const float2 *>(d[1]);
    o.mom1 = static_cast<float2 *>(d[2]);
    o.mom2 = static_cast<float *>(d[3]);
    o.buffer = static_cast<float2 *>(d[4]);
    o.amp = static_cast<const float *>(d[5]);
    o.r1 = (float)opt->beta1;
    o.c1 = (float)(1.0 - opt->beta1);
    o.r2 = (float)opt->beta2;
    o.c2 = (float)(1.0 - opt->beta2);
    o.lr = (float)opt->lr;
    o.mum = (float)opt->momentum;
    o.margin = (float)opt->clamp_margin;
    if (kind == FPM_OPT_ADAM) {
        const double t = (double)opt->iter;
        o.bias = (float)(std::sqrt(1.0 - std::pow(opt->beta2, t)) / (1.0 - std::pow(opt->beta1, t)));
    }
    FPM_CK(launch_optimizer_step(o, st));
    if (!dev)
        for (int k = 0; k < 6; ++k)
            if (arrs[k].p && arrs[k].out)
                FPM_CK(cudaMemcpyAsync(const_cast<void *>(arrs[k].p), d[k], arrs[k].bytes,
                                       cudaMemcpyDeviceToHost, st));
    FPM_CK(cudaStreamSynchronize(st));
    return FPM_OK;
}

}  // extern "C"

/*
 * fpm.h - C ABI of the B200 Fourier-ptychographic reconstruction engine.
 *
 * The engine is a drop-in for the reference's MATLAB mex call
 *
 *     [O, P] = cuFPM_pure_v3(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, [lr beta eps])
 *
 * (cuFPM_v3/cuFPM_pure_v3.cu:44-228; call site codes_v2/main_run_FPM.m:77-106)
 * and for the gradient-only call of the first generation
 *
 *     [dldw1, dldw2] = fullyfusedFPM(O, P, Y, ledIdx, pratio)
 *
 * (codes/fusedfpm/fullyfusedFPM.cu:24-169), computed with the v3 loss.
 *
 * Conventions
 *   - All images are square and column-major (MATLAB layout): element (row r,
 *     col c) of an n x n image sits at index c*n + r.  Stacks are pages of
 *     h*h elements, page l = LED l.
 *   - Complex arrays are interleaved {float re, float im} (MATLAB creal32_T).
 *   - led_idx holds 2*L int32: (kl, kt) per LED, the 1-based column and row of
 *     the top-left corner of the LED's h x h crop in the centred H x H
 *     spectrum (MATLAB int32([kl; kt]), codes_v2/main_run_FPM.m:53-55).  A
 *     crop that runs past the spectrum edge wraps modulo H, as in v3
 *     (cuFPM_v3/cuda/kernels.cuh:43-47).  1 <= kl, kt <= H is required.
 *   - h must be even; h and H = h * pratio may have no prime factor above 7, and
 *     H <= 16384 (FPM_ERR_UNSUPPORTED otherwise).  Powers of two (h >= 16) run the
 *     fused pipeline, other sizes the any-size path (mixed-radix transforms with the
 *     reference's per-batch structure).  The caller owns every buffer.
 *   - Every function returns an fpm_status; nothing throws across the ABI.
 *   - A context is bound to one CUDA device and is not thread-safe: use one
 *     context per host thread.
 *   - There is no CPU fallback: without a usable CUDA device fpm_create fails
 *     with FPM_ERR_NO_DEVICE.
 */
#ifndef FPM_H
#define FPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FPM_ABI_VERSION 2

typedef enum fpm_status {
    FPM_OK = 0,
    FPM_ERR_INVALID_ARGUMENT = 1, /* shapes, sizes, pointers or hyper-parameters rejected */
    FPM_ERR_UNSUPPORTED = 2,      /* valid request this build does not implement */
    FPM_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed or exceeded mem_limit_bytes */
    FPM_ERR_CUDA = 4,             /* a CUDA runtime call or kernel launch failed */
    FPM_ERR_NONFINITE = 5,        /* the loss became NaN/Inf; outputs hold the last state */
    FPM_ERR_NO_DEVICE = 6,        /* no usable CUDA device */
    FPM_ERR_INTERNAL = 7
} fpm_status;

/* Where the pointers of a problem / result live. */
typedef enum fpm_memory {
    FPM_MEM_HOST = 0,   /* ordinary or pinned host memory: copied in and out by the engine */
    FPM_MEM_DEVICE = 1  /* device memory of the context's device, 16-byte aligned: used in
                           place (zero copy) */
} fpm_memory;

/* Element type of the measured stack. */
typedef enum fpm_stack_type {
    /* float amplitude, already normalised: the reference mex input Y (prhs[2]) */
    FPM_STACK_F32_AMPLITUDE = 0,
    /* raw uint16 counts; the engine applies Y = sqrt((I - min) / (max - min)) over
       the whole stack on the device, bit-identical to codes_v2/main_run_FPM.m:43-45
       in single precision, and keeps the stack resident as uint16 (2 B/px). */
    FPM_STACK_U16_COUNTS = 1
} fpm_stack_type;

typedef enum fpm_loss_kind {
    /* sum |d/dx (|x| - Y)| + |d/dy (|x| - Y)| with periodic forward differences,
       sign(0) = +1 (cuFPM_v3/cuda/kernels.cuh:197-275, benchmark/func_ware/ret_loss.m) */
    FPM_LOSS_ANISOTROPIC = 0,
    /* sum sqrt(Rx^2 + Ry^2) of the same differences, gradient through
       R/(|R| + 1e-5) (codes/func_ware/misc/ret_loss.m 'isotropic', the loss of
       benchmark/func_ware/fpm_forward_GPU.m:38); no counterpart in the v3 mex */
    FPM_LOSS_ISOTROPIC = 1
} fpm_loss_kind;

/* Weights of the two gradient terms, the `type` of deconv_pie in the reference's
   conventional MATLAB gradient (benchmark/func_ware/fpm_forward_GPU.m:48,60,64-76),
   applied to the gradients of the v3 mex: object term conj(P) X / H^2, pupil term
   sum_l conj(sub_l) X_l. */
typedef enum fpm_pie_weights {
    FPM_PIE_NONE = 0,  /* 'none': the v3 mex's gradients */
    FPM_PIE_EPIE = 1,  /* 'ePIE': object term / max|P|^2, each pupil term / max|sub_l|^2
                          over the LED's whole crop (disables pupil-support pruning) */
    FPM_PIE_TPIE = 2   /* 'tPIE': object term / (|P|^2 + 1e-5), pupil term
                          / (|sub_l|^2 + 1e-5), per pixel */
} fpm_pie_weights;

/* fpm_device_opts.flags */
#define FPM_CTX_AUTOTUNE 1   /* the first solve of every new problem shape runs fpm_autotune */

typedef struct fpm_device_opts {
    int32_t device;          /* CUDA device ordinal */
    int32_t flags;           /* FPM_CTX_* bits */
    size_t mem_limit_bytes;  /* 0 = no cap; otherwise solves needing more fail with
                                FPM_ERR_OUT_OF_MEMORY before allocating anything */
    void *stream;            /* cudaStream_t to run on, or NULL for a context-owned stream */
} fpm_device_opts;

/* Inputs of one reconstruction (the nine mex arguments, cuFPM_pure_v3.cu:51-65). */
typedef struct fpm_problem {
    int32_t h;               /* low-res side (rows == cols), even */
    int32_t n_leds;          /* L: pages of the stack and entries of led_idx */
    int32_t pratio;          /* up-sampling ratio; H = h * pratio (prhs[5]) */
    int32_t batch;           /* LEDs per mini-batch B (prhs[7]); the last batch holds L mod B */
    int32_t epochs;          /* prhs[6] */
    float lr;                /* RMSprop learning rate (prhs[8][0]) */
    float beta;              /* second-moment decay (prhs[8][1]) */
    float eps;               /* added outside the square root (prhs[8][2]) */
    float pupil_margin;      /* am: |P| clamped to P0 * [P0 - am, P0 + am]; reference 0.2 */
    int32_t lr_halve_after;  /* lr *= lr_decay after each epoch whose 0-based index
                                exceeds this; reference 12 (cuFPM_pure_v3.cu:204-206) */
    float lr_decay;          /* reference 0.5 */
    int32_t loss_kind;       /* fpm_loss_kind */
    int32_t memory;          /* fpm_memory of every pointer below */
    int32_t stack_type;      /* fpm_stack_type */
    const void *stack;       /* h*h*L measured stack (prhs[2]) */
    const int32_t *led_idx;  /* 2*L int32 (kl, kt) (prhs[3]) */
    const float *pupil_init; /* complex h*h initial pupil P0c (prhs[1]) */
    const float *pupil_amp;  /* real h*h pupil amplitude P0 (prhs[4]) */
    const float *object_init;/* complex H*H initial object O0 (prhs[0]); NULL = bicubic
                                up-sampling of stack page 0 with zero phase
                                (codes_v2/main_run_FPM.m:48) */
    int32_t pie_weights;     /* fpm_pie_weights; FPM_PIE_NONE for the mex's behaviour */
    int32_t reserved0;
} fpm_problem;

/* Outputs.  Any pointer may be NULL to skip that output.  Pointers follow the
   problem's fpm_memory.  With FPM_MEM_DEVICE, object may alias object_init and
   pupil may alias pupil_init (updated in place). */
typedef struct fpm_result {
    float *object;    /* complex H*H reconstructed object (plhs[0]) */
    float *spectrum;  /* complex H*H centred spectrum fftshift(fft2(object)) */
    float *pupil;     /* complex h*h reconstructed pupil (plhs[1]) */
    double *loss;     /* epochs values: feature-domain loss summed over each epoch's
                         batches, each batch evaluated before its update */
} fpm_result;

typedef struct fpm_context fpm_context;

/* Replaces mxInitGPU + the per-call set-up of cuFPM_pure_v3.cu:49-126. */
fpm_status fpm_create(fpm_context **ctx, const fpm_device_opts *opts);

/* Replaces the body of mexFunction, cuFPM_pure_v3.cu:44-228.  Every epoch after the
   first is replayed from a CUDA graph captured once per learning rate (the reference
   launches every kernel and synchronises after every mini-batch,
   cuFPM_pure_v3.cu:202); with stage profiling on (fpm_set_profiling) the epochs run
   eagerly.  The context keeps the executable graph: a later capture with the same
   kernels in the same order (the next learning rate, or a later solve of the same
   shape) updates it in place; every capture carries that solve's own arguments. */
fpm_status fpm_solve(fpm_context *ctx, const fpm_problem *prob, fpm_result *res);

/* Many independent reconstructions in one call: tiles of a large field of view, or
   instances of different sizes (h, L, pratio, B may differ).  No counterpart in the
   reference, which runs one reconstruction per mex call (cuFPM_pure_v3.cu:44).
   problems[i] / results[i] follow fpm_solve's rules one by one.  The instances run
   concurrently: each on a worker context of its own (its buffers stay allocated for
   the next call; the parent's mem_limit_bytes caps each instance) over a pool of up to
   8 streams, every instance's epochs after the first replayed from one captured CUDA
   graph per learning rate.  flags: FPM_BATCH_EAGER launches every epoch's kernels
   directly instead.  statuses (optional, n entries) receives each instance's status;
   the return value is the first failing instance's (FPM_OK when all succeed), with its
   detail in fpm_last_error(ctx).  Results equal those of n separate fpm_solve calls. */
#define FPM_BATCH_EAGER 1
fpm_status fpm_solve_batch(fpm_context *ctx, const fpm_problem *problems, fpm_result *results,
                           int32_t n, int32_t flags, fpm_status *statuses);

/* Autotuner (no counterpart in the reference, whose launch shapes are fixed 16 x 16
   blocks, cuFPM_v3/cuda/addon.h:4-5, and whose README reports the LED batch moving the
   time by 1.5x, README.md:47-49).  Times one epoch of `prob` on the caller's own data
   for each candidate launch choice, searching one choice at a time: LEDs per
   low-resolution launch group, the fused or two-pass row transform and its cluster
   size, the 16384-point passes' prefetch and values per thread, the any-size line
   FFT's lines per block.  None of these changes the result beyond the rounding of an
   alternative radix split.  The fastest choice is kept in the context for the
   problem's shape (h, H, LED count, batch, stack type, loss, weights) and used by every
   later fpm_solve / fpm_solve_batch of that shape.  The LED batch B stays the caller's:
   it changes the reconstruction itself.  Outputs nothing but `report` (optional, a
   one-line summary, truncated to report_cap bytes); the inputs are only read.  Costs
   about (number of candidates + 1) epochs. */
fpm_status fpm_autotune(fpm_context *ctx, const fpm_problem *prob, char *report,
                        size_t report_cap);

/* Self-check of the failure path of the device-side waits (no counterpart in the
   reference, which has no waits).  The engine's passes wait for their tile copies with a
   bound (about two seconds); a wait that runs out sets a device flag, the pass stops, and
   the call returns FPM_ERR_INTERNAL instead of results built from incomplete data.  This
   runs one such wait on purpose, with the given bound in SM clocks (1 .. 2^32), on an
   mbarrier armed for bytes that no copy delivers, and returns what a solve would return
   (FPM_ERR_INTERNAL, detail in fpm_last_error); the context stays usable. */
fpm_status fpm_selftest_bounded_wait(fpm_context *ctx, int64_t limit_cycles);

/* Gradients of one LED batch at (object, pupil), v3 loss: replaces
   fullyfusedFPM (codes/fusedfpm/fullyfusedFPM.cu:24-169).  prob->n_leds LEDs
   form one batch (prob->batch, epochs and optimiser fields are ignored);
   object_init / pupil_init give the current estimate (object_init must not be
   NULL).  d_object receives IFFT2 of the stitched gradient spectrum
   (complex H*H, the dldw1 the RMSprop of cuFPM_pure_v3.cu:189 consumes),
   d_pupil the pupil gradient (complex h*h, dldw2), loss the batch loss.
   Any output may be NULL. */
fpm_status fpm_batch_gradients(fpm_context *ctx, const fpm_problem *prob,
                               float *d_object, float *d_pupil, double *loss);

/* Ingest helper (codes_v2/main_run_FPM.m:43-45): amplitude = sqrt((I-min)/(max-min))
   over a whole uint16 stack of n elements, computed on the device in single
   precision.  Pointers follow `memory`. */
fpm_status fpm_normalise_stack(fpm_context *ctx, const uint16_t *counts, size_t n,
                               float *amplitude, int32_t memory);

/* fpm_normalise_stack for a float stack (fpm_read_tiff_stack with
   FPM_INGEST_F32_MEAN): amplitude = sqrt((x-min)/(max-min)) over all n values,
   NaN left out of the min / max as MATLAB's min / max do. */
fpm_status fpm_normalise_stack_f32(fpm_context *ctx, const float *values, size_t n,
                                   float *amplitude, int32_t memory);

/* Element type fpm_read_tiff_stack writes. */
typedef enum fpm_ingest_type {
    FPM_INGEST_U16 = 0,      /* uint16 counts (single-sample frames): the stack of
                                FPM_STACK_U16_COUNTS, normalised inside fpm_solve */
    FPM_INGEST_F32_MEAN = 1  /* float mean over each pixel's samples, mean(single(x), 3) */
} fpm_ingest_type;

/* Ingest of the measured frames (codes_v2/main_run_FPM.m:26-41): for each of the
   n_images files, in LED order, the h x h pixel region whose top-left pixel is
   (row0, col0), 0-based (the reference's imread 'PixelRegion' {[rect(2),
   rect(2)+pix-1], [rect(1), rect(1)+pix-1]} is row0 = rect(2)-1, col0 = rect(1)-1),
   into page i of the host array `stack` (column-major h*h per page).  Reads the
   first image of baseline TIFF files: uncompressed strips, 8- or 16-bit unsigned
   samples, 1 to 4 samples per pixel (chunky), either byte order; anything else,
   a region outside the image or a short file fails with FPM_ERR_INVALID_ARGUMENT
   naming the file.  Host-side only: the files are read on `threads` host threads
   (<= 0: one per hardware thread, at most 32).  ctx may be NULL (no device is
   needed); the failure detail then goes to fpm_last_error(NULL). */
fpm_status fpm_read_tiff_stack(fpm_context *ctx, const char *const *paths, int32_t n_images,
                               int32_t row0, int32_t col0, int32_t h, int32_t type, void *stack,
                               int32_t threads);

/* The engine's own unnormalised 2-D FFT of `count` column-major n x n complex
   pages (direction -1 forward, +1 inverse), the transform behind the cuFFT calls
   of cuFPM_pure_v3.cu:135-187.  n: 2 <= n <= 16384, no prime factor above 7.  in may equal
   out.  Pointers follow `memory`. */
fpm_status fpm_fft2(fpm_context *ctx, const float *in, float *out, int32_t n, int32_t count,
                    int32_t direction, int32_t memory);

/* Loss-gradient stage that allocates nothing.  No counterpart in the reference.
   For callers that cannot call cudaMalloc (a mex inside MATLAB's GPU memory
   manager, a framework whose caching allocator owns the device, an acquisition
   loop that must not stall on the device-wide synchronisation an allocation
   implies).  For n_images fields z (complex h*h each, the unnormalised inverse
   FFT of crop x pupil, as after cuFPM_pure_v3.cu:151) and their amplitudes
   (float h*h each) it writes gradient = d * z/|z| (complex h*h each, the
   loss-gradient stage of fpm_solve) and *loss = the feature-domain loss summed
   over all images.  All pointers: device memory of the current device, on
   `stream` (a cudaStream_t; NULL = legacy default stream).
   Scratch: a fixed device array of FPM_NOALLOC_MAX_TILES FP64 tile partials
   (512 KiB), held by every GPU that loads the library until exit.  The first
   call on a device looks up its address (cudaGetSymbolAddress, with that device
   current); make that first call before any stream capture.  Limit: n_images *
   ceil(h/32)^2 <= FPM_NOALLOC_MAX_TILES (e.g. 16 images of 2048^2, 256 of 512^2),
   h <= FPM_NOALLOC_MAX_SIDE and n_images <= 65535, else FPM_ERR_UNSUPPORTED
   before any device work.  Every call shares the one array: calls whose work
   overlaps on the GPU (other streams, other host threads) race and must be
   serialised by the caller. */
#define FPM_NOALLOC_MAX_TILES 65536
#define FPM_NOALLOC_MAX_SIDE 8192
fpm_status fpm_feature_gradient_noalloc(const float *z, const float *amplitude, int32_t h,
                                        int32_t n_images, int32_t pratio, float *gradient,
                                        double *loss, void *stream);

/* Geometry of a square LED array (codes_v2/func_ware/init_environment_rgb.m:1-25). */
typedef struct fpm_led_geometry {
    int32_t grid;             /* LEDs per side (ledMM = ledNN), odd, 1..255 */
    int32_t h;                /* low-res image side (pix), even */
    int32_t pratio;           /* up-sampling ratio (MAGimg); H = h * pratio */
    int32_t reserved0;
    double wavelength_um;     /* lamuda */
    double led_pitch_um;      /* D_led: distance between neighbouring LEDs */
    double led_height_um;     /* h: distance from the LED plane to the sample */
    double camera_pixel_um;   /* pixel_size */
    double magnification;     /* mag */
    double sample_dx_um;      /* objdx: offset of the reconstructed area (x * D_pixel) */
    double sample_dy_um;      /* objdy */
} fpm_led_geometry;

/* LED corners for fpm_problem.led_idx, computed on the device in FP64: the
   illumination angle of every LED (visited centre-out in the spiral order of
   init_environment_rgb.m:111-133), the nearest point of the high-res frequency
   axis (first on ties; :98-106) and the crop corner kl = uo - h/2, kt = vo - h/2
   (codes_v2/main_run_FPM.m:21-31,51-55), bit-identical to an IEEE double
   evaluation of those MATLAB statements.  led_idx: host array of
   2 * grid * grid int32, (kl, kt) per LED; grid_pos (optional, host, same size):
   the 1-based (row i, column j) grid cell of each LED. */
fpm_status fpm_led_indices(fpm_context *ctx, const fpm_led_geometry *geo, int32_t *led_idx,
                           int32_t *grid_pos);

/* Forward model of the reference's data generator (benchmark/gen_img_batch.m:178-201,
   fpm_forward_gen): for every LED l,
       x_l = ifft2(ifftshift(crop_l(fftshift(fft2(object))) .* pupil)) / pratio^2
   with crop_l the h x h window at led_idx[l] = (kl, kt) of the centred spectrum
   (1-based corner, wrapping modulo H as in fpm_problem), and out page l = |x_l|^2
   (FPM_SIM_INTENSITY) or |x_l| (FPM_SIM_AMPLITUDE).  object: complex H*H (H = h *
   pratio), pupil: complex h*h, led_idx: 2*n_leds int32, out: float h*h*n_leds; all
   column-major, pointers follow `memory`.  h even, h and H with no prime factor above 7, H <= 16384.
   The transforms are the engine's own; used to make training / test data and to
   check a reconstruction against its measurements. */
typedef enum fpm_sim_output { FPM_SIM_INTENSITY = 0, FPM_SIM_AMPLITUDE = 1 } fpm_sim_output;
fpm_status fpm_simulate(fpm_context *ctx, const float *object, const float *pupil,
                        const int32_t *led_idx, int32_t h, int32_t pratio, int32_t n_leds,
                        int32_t output, float *out, int32_t memory);

/* The optimiser classes of the reference's script-level loop, which pairs
   fullyfusedFPM (fpm_batch_gradients here) with a MATLAB optimiser step and a pupil
   amplitude clamp per mini-batch (benchmark/cuFPM_recon_2025_circular.m:108-113,
   180-186; codes/main_run_FPM.m:85-86).  One step is one fused elementwise pass on
   the device over a complex parameter of n elements, single precision as MATLAB's
   gpuArray single, every scalar (lr, betas, Adam's bias) rounded from double. */
typedef enum fpm_optimizer_kind {
    /* optimizer_RMSprop.m:30-47 as written: squave = r1 + (1-r1)|g|^2 (recomputed
       every step, no running average), centered: g0 = r1 g0 + (1-r1) g and
       squave -= |g0|^2, then with momentum mum > 0: buffer = mum buffer +
       g/(sqrt(squave)+1e-5), p -= lr buffer; else p -= lr g/(sqrt(squave)+1e-5).
       A negative squave takes MATLAB's complex square root. */
    FPM_OPT_RMSPROP = 0,
    /* codes/func_ware/optimizers/optimizer_adam.m:25-38: mom1 = r1 mom1 + (1-r1) g,
       mom2 = r2 mom2 + (1-r2)|g|^2, p -= lr sqrt(1-r2^t)/(1-r1^t) mom1/(sqrt(mom2)+1e-5) */
    FPM_OPT_ADAM = 1,
    /* codes_v2/func_ware/optimizers/optimizer_yogi.m:25-36: mom1 as Adam,
       mom2 -= (1-r2) sign(mom2 - |g|^2)|g|^2 (sign(0) = 0), p -= lr mom1/(sqrt(mom2)+1e-5) */
    FPM_OPT_YOGI = 2,
    /* optimizer_sgd.m: p -= lr g (the class's step names an undefined variable
       `update`, so MATLAB cannot run it; this is its evident intent) */
    FPM_OPT_SGD = 3
} fpm_optimizer_kind;

typedef struct fpm_optimizer {
    int32_t kind;          /* fpm_optimizer_kind */
    int32_t centered;      /* RMSprop: 1 = centred */
    double lr;
    double beta1;          /* r1 (RMSprop, Adam, Yogi) */
    double beta2;          /* r2 (Adam, Yogi) */
    double momentum;       /* RMSprop mum; > 0 uses `buffer` */
    int64_t iter;          /* Adam: step count t >= 1 of the bias correction */
    /* state, updated in place; NULL where the kind does not use it.  MATLAB starts
       every state at 0 (the classes are built with zeros): pass zeroed arrays. */
    float *mom1;           /* complex n: Adam / Yogi first moment; RMSprop g0 (centered) */
    float *mom2;           /* real n: Adam / Yogi second moment */
    float *buffer;         /* complex n: RMSprop momentum buffer (momentum > 0) */
    /* optional pupil clamp after the step (cuFPM_recon_2025_circular.m:183-186):
       p = max(min(|p|, a + margin), a - margin) .* sign(p) .* a, sign(p) = p/|p|
       (0 at 0); a: real n, NULL = no clamp */
    const float *clamp_amp;
    double clamp_margin;
} fpm_optimizer;

/* param (complex n) -= the step of opt for gradient grad (complex n).  Pointers
   (param, grad, states, clamp_amp) follow `memory`; device pointers 8-byte aligned. */
fpm_status fpm_optimizer_step(fpm_context *ctx, const fpm_optimizer *opt, float *param,
                              const float *grad, size_t n, int32_t memory);

/* Learned warm start (no counterpart in the reference, whose initial object is
   imresize(Y_1, pratio) with zero phase, codes_v2/main_run_FPM.m:48).
   A 4-level convolutional encoder-decoder (channels base, 2 base, 4 base, 8 base; base a
   multiple of 8 up to 32; 3x3 convolutions on the tcgen05 tensor cores with BF16 operands
   and FP32 accumulation in tensor memory; FP32 master weights) maps the first in_channels frames of a stack (the central bright-field block
   of the spiral order: 25 frames = the central 5 x 5 LEDs) to the real and imaginary parts
   of a low-resolution object, which fpm_cnn_initial_object up-samples bicubically to the
   H x H starting object.  Trained by fpm_cnn_train_step on pairs the plain
   reconstruction produces.  All arrays: device memory of the context's device, FP32,
   planes of h x h (h a multiple of 8), [n][channels][h*h]; the network keeps the
   context's stream and device.  Parameter order: for each of the 14 layers, weights
   [Cout][Cin][3][3] then biases [Cout]. */
typedef struct fpm_cnn fpm_cnn;
/* a network must be destroyed before its context */
fpm_status fpm_cnn_create(fpm_context *ctx, int32_t in_channels, int32_t base_channels,
                          uint64_t seed, fpm_cnn **net);
void fpm_cnn_destroy(fpm_cnn *net);
int64_t fpm_cnn_parameter_count(const fpm_cnn *net);
const char *fpm_cnn_last_error(const fpm_cnn *net);
/* host arrays of fpm_cnn_parameter_count floats; setting also resets the Adam state */
fpm_status fpm_cnn_set_parameters(fpm_cnn *net, const float *params, int64_t n);
fpm_status fpm_cnn_get_parameters(fpm_cnn *net, float *params, int64_t n);
/* y [n][2][h*h] = network(x [n][in_channels][h*h]) */
fpm_status fpm_cnn_forward(fpm_cnn *net, const float *x, int32_t n, int32_t h, float *y);
/* loss = mean over all n*2*h*h outputs of (y - t)^2, and (host array or NULL) its
   gradient with respect to every parameter; the parameters are not changed */
fpm_status fpm_cnn_gradients(fpm_cnn *net, const float *x, const float *t, int32_t n,
                             int32_t h, double *loss, float *grads);
/* fpm_cnn_gradients, then one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) of rate lr */
fpm_status fpm_cnn_train_step(fpm_cnn *net, const float *x, const float *t, int32_t n,
                              int32_t h, float lr, double *loss);
/* the starting object of a device-memory problem (complex H*H, column-major): the network
   on the problem's first in_channels frames, normalised as fpm_solve normalises them */
fpm_status fpm_cnn_initial_object(fpm_cnn *net, const fpm_problem *prob, float *object);
/* fpm_solve from the learned start with the plain start as the fallback: one epoch from
   each of the network's object (fpm_cnn_initial_object) and the plain start (object_init,
   or the bicubic start when NULL), then the full solve from the start whose first-epoch
   loss is lower (the network's on a tie).  *used_network (may be NULL) tells which.
   Device-memory problems; costs two extra epochs and one network evaluation. */
fpm_status fpm_solve_warm(fpm_context *ctx, fpm_cnn *net, const fpm_problem *prob,
                          fpm_result *res, int32_t *used_network);

void fpm_destroy(fpm_context *ctx);

/* Per-stage device timing (no counterpart in the reference, which only times
   the whole mex call with tic/toc, benchmark/cuFPM_recon_2025_circular.m:152-169).
   When enabled, every stage launch of the next fpm_solve / fpm_batch_gradients
   is bracketed by CUDA events on the context's stream; fpm_stage_times then
   reports, per stage, the launches and their summed device time. */
typedef struct fpm_stage_time {
    const char *name;   /* static string, e.g. "rmsprop_object" */
    int32_t launches;   /* stage launches in the last call */
    int32_t own_kernel; /* 1: a libfpm kernel, 0: a library call (FFT back end) */
    double ms;          /* summed device time of those launches */
} fpm_stage_time;

fpm_status fpm_set_profiling(fpm_context *ctx, int32_t enable);

/* Fills up to `cap` entries (stages with launches > 0) and returns how many
   stages have data. */
int32_t fpm_stage_times(const fpm_context *ctx, fpm_stage_time *out, int32_t cap);

const char *fpm_status_string(fpm_status s);

/* Human-readable detail of the last failure on this context ("" if none); with
   ctx NULL, of the calling host thread's last failed fpm_read_tiff_stack made
   without a context. */
const char *fpm_last_error(const fpm_context *ctx);

int32_t fpm_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FPM_H */

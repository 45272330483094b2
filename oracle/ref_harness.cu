// TEST INFRASTRUCTURE.  Drives the reference's own v3 kernels
// (cuFPM_v3/cuda/kernels.cuh, compiled from the read-only reference tree by
// oracle/build_ref.py into oracle/_ref/libcufpm_ref.so) with a replica of the
// host loop of cuFPM_v3/cuFPM_pure_v3.cu:75-207, minus MATLAB.  Used only by
// tests/ as a checker (it pins the numpy oracle against the reference itself)
// and to time the reference's GPU build on the same device; never by the
// product.
#include <cuda_runtime.h>
#include <cufft.h>

#include <vector>

#include "kernels.cuh"

namespace {

// cuFPM_pure_v3.cu:10-18: dims of an (rows, cols, pages) array -> {cols, rows, pages}
dim3 dims_of(int rows, int cols, int pages) { return dim3((unsigned)cols, (unsigned)rows, (unsigned)pages); }

struct Bufs {
    creal32_t *O = nullptr, *P = nullptr, *latentZ = nullptr, *recordZ = nullptr,
              *subwave = nullptr, *dldw1 = nullptr, *dldw2 = nullptr;
    real32_T *mom1 = nullptr, *mom2 = nullptr, *Y = nullptr, *P0 = nullptr;
    int2 *led = nullptr;
    void free_all() {
        void *ps[] = {O, P, latentZ, recordZ, subwave, dldw1, dldw2, mom1, mom2, Y, P0, led};
        for (void *p : ps)
            if (p) cudaFree(p);
    }
};

#define RCK(x)                                   \
    do {                                         \
        if ((x) != 0) {                          \
            b.free_all();                        \
            return __LINE__;                     \
        }                                        \
    } while (0)

}  // namespace

extern "C" {

// Full solve (cuFPM_pure_v3 semantics).  Host arrays in, host arrays out,
// column-major.  ms[0] = epoch-loop time, ms[1] = allocation + plans + loop,
// ms[2] = number of guard bytes after the object buffer that changed (the
// object is allocated with a 64 KiB sentinel-filled guard behind it).
int ref_solve(int h, int H, int L, int pratio, int epochs, int batch, float lr, float beta,
              float eps, const float *O0, const float *P0c, const float *Y, const int *led,
              const float *P0, float *O_out, float *P_out, float *ms) {
    Bufs b;
    const size_t plane = (size_t)h * h, big = (size_t)H * H;
    const size_t guard = 64 * 1024;
    RCK(cudaMalloc(&b.O, big * 8 + guard));
    RCK(cudaMemset(reinterpret_cast<char *>(b.O) + big * 8, 0xA5, guard));
    RCK(cudaMalloc(&b.P, plane * 8));
    RCK(cudaMalloc(&b.Y, plane * L * 4));
    RCK(cudaMalloc(&b.P0, plane * 4));
    RCK(cudaMalloc(&b.led, (size_t)L * 8));
    RCK(cudaMemcpy(b.O, O0, big * 8, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.P, P0c, plane * 8, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.Y, Y, plane * L * 4, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.P0, P0, plane * 4, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.led, led, (size_t)L * 8, cudaMemcpyHostToDevice));
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    RCK(cudaDeviceSynchronize());
    cudaEventRecord(e0);

    dim3 imLs_sz = dims_of(h, h, L);
    dim3 imHs_sz = dims_of(H, H, 1);
    const size_t arraysize = plane * batch;
    RCK(cudaMalloc(&b.latentZ, arraysize * 8));
    RCK(cudaMalloc(&b.subwave, arraysize * 8));
    RCK(cudaMalloc(&b.recordZ, arraysize * 8));
    RCK(cudaMalloc(&b.dldw1, big * 8));
    RCK(cudaMalloc(&b.dldw2, plane * 8));
    RCK(cudaMalloc(&b.mom1, big * 4));
    RCK(cudaMalloc(&b.mom2, plane * 4));
    cudaMemset(b.mom1, 0, big * 4);
    cudaMemset(b.mom2, 0, plane * 4);
    dim3 N_THREADS = {BLOCK_X, BLOCK_Y, 1};
    dim3 N_BLOCKS_L = {(imHs_sz.x + BLOCK_X - 1) / BLOCK_X, (imHs_sz.y + BLOCK_Y - 1) / BLOCK_Y, 1};
    dim3 N_BLOCKS = {(imLs_sz.x + BLOCK_X - 1) / BLOCK_X, (imLs_sz.y + BLOCK_Y - 1) / BLOCK_Y, 1};
    const int led_total = (int)imLs_sz.z;
    int inembed[2] = {(int)imLs_sz.x, (int)imLs_sz.y};
    imLs_sz.z = batch;
    cufftHandle planLarge, planBatch;
    if (cufftPlan2d(&planLarge, imHs_sz.x, imHs_sz.y, CUFFT_C2C) != CUFFT_SUCCESS) {
        b.free_all();
        return -1;
    }
    if (cufftPlanMany(&planBatch, 2, inembed, inembed, 1, (int)plane, inembed, 1, (int)plane,
                      CUFFT_C2C, batch) != CUFFT_SUCCESS) {
        cufftDestroy(planLarge);
        b.free_all();
        return -2;
    }
    cudaEventRecord(e1);
    for (int epoch = 0; epoch < epochs; ++epoch) {
        int remain = led_total, curr = 0;
        while (remain > 0) {
            remain -= batch;
            cufftExecC2C(planLarge, (cufftComplex *)b.O, (cufftComplex *)b.dldw1, CUFFT_FORWARD);
            N_BLOCKS.z = (unsigned)(min(curr + batch - 1, led_total - 1) - curr + 1);
            fused_getSubpupil_shifted<<<N_BLOCKS, N_THREADS>>>(curr, b.dldw1, b.P, b.led, imLs_sz,
                                                              imHs_sz, b.subwave, b.latentZ);
            cufftExecC2C(planBatch, (cufftComplex *)b.latentZ, (cufftComplex *)b.latentZ,
                         CUFFT_INVERSE);
            differenceKernel_acc<<<N_BLOCKS, N_THREADS>>>(curr, imLs_sz, pratio, b.Y, b.latentZ,
                                                          b.recordZ);
            cufftExecC2C(planBatch, (cufftComplex *)b.recordZ, (cufftComplex *)b.latentZ,
                         CUFFT_FORWARD);
            cudaMemset(b.dldw1, 0, big * 8);
            cudaMemset(b.dldw2, 0, plane * 8);
            fused_deconvPIE_shifted<<<N_BLOCKS, N_THREADS>>>(curr, b.latentZ, b.subwave, b.led,
                                                             b.P, imLs_sz, imHs_sz, b.dldw1,
                                                             b.dldw2);
            cufftExecC2C(planLarge, (cufftComplex *)b.dldw1, (cufftComplex *)b.dldw1,
                         CUFFT_INVERSE);
            constrained_RMSprop_both<<<N_BLOCKS_L, N_THREADS>>>(b.dldw1, b.dldw2, beta, lr, eps,
                                                                imHs_sz, imLs_sz, b.mom1, b.mom2,
                                                                b.O, b.P, b.P0, 0.2f);
            curr += batch;
            cudaDeviceSynchronize();
        }
        if (epoch > 12) lr = lr * 0.5;
    }
    cudaEventRecord(e2);
    cudaEventSynchronize(e2);
    float t_loop = 0.f, t_all = 0.f;
    cudaEventElapsedTime(&t_loop, e1, e2);
    cudaEventElapsedTime(&t_all, e0, e2);
    if (ms) {
        ms[0] = t_loop;
        ms[1] = t_all;
        unsigned char *g = new unsigned char[guard];
        cudaMemcpy(g, reinterpret_cast<char *>(b.O) + big * 8, guard, cudaMemcpyDeviceToHost);
        int changed = 0;
        for (size_t i = 0; i < guard; ++i) changed += g[i] != 0xA5;
        delete[] g;
        ms[2] = (float)changed;
    }
    int rc = (int)cudaGetLastError();
    if (rc == 0) {
        cudaMemcpy(O_out, b.O, big * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(P_out, b.P, plane * 8, cudaMemcpyDeviceToHost);
    }
    cufftDestroy(planBatch);
    cufftDestroy(planLarge);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    b.free_all();
    return rc;
}

// Gradients of one batch of all L LEDs at (O, P): the K1..K8 part of one
// iteration of the loop above.  dO = IFFT2(stitched gradient spectrum), dP
// the pupil gradient.
int ref_gradients(int h, int H, int L, int pratio, const float *O, const float *P, const float *Y,
                  const int *led, float *dO_out, float *dP_out) {
    Bufs b;
    const size_t plane = (size_t)h * h, big = (size_t)H * H;
    RCK(cudaMalloc(&b.O, big * 8));
    RCK(cudaMalloc(&b.P, plane * 8));
    RCK(cudaMalloc(&b.Y, plane * L * 4));
    RCK(cudaMalloc(&b.led, (size_t)L * 8));
    RCK(cudaMalloc(&b.latentZ, plane * L * 8));
    RCK(cudaMalloc(&b.subwave, plane * L * 8));
    RCK(cudaMalloc(&b.recordZ, plane * L * 8));
    RCK(cudaMalloc(&b.dldw1, big * 8));
    RCK(cudaMalloc(&b.dldw2, plane * 8));
    RCK(cudaMemcpy(b.O, O, big * 8, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.P, P, plane * 8, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.Y, Y, plane * L * 4, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(b.led, led, (size_t)L * 8, cudaMemcpyHostToDevice));
    dim3 imLs_sz = dims_of(h, h, L);
    dim3 imHs_sz = dims_of(H, H, 1);
    dim3 N_THREADS = {BLOCK_X, BLOCK_Y, 1};
    dim3 N_BLOCKS = {(imLs_sz.x + BLOCK_X - 1) / BLOCK_X, (imLs_sz.y + BLOCK_Y - 1) / BLOCK_Y,
                     (unsigned)L};
    int inembed[2] = {(int)imLs_sz.x, (int)imLs_sz.y};
    cufftHandle planLarge, planBatch;
    if (cufftPlan2d(&planLarge, imHs_sz.x, imHs_sz.y, CUFFT_C2C) != CUFFT_SUCCESS) {
        b.free_all();
        return -1;
    }
    if (cufftPlanMany(&planBatch, 2, inembed, inembed, 1, (int)plane, inembed, 1, (int)plane,
                      CUFFT_C2C, L) != CUFFT_SUCCESS) {
        cufftDestroy(planLarge);
        b.free_all();
        return -2;
    }
    cufftExecC2C(planLarge, (cufftComplex *)b.O, (cufftComplex *)b.dldw1, CUFFT_FORWARD);
    fused_getSubpupil_shifted<<<N_BLOCKS, N_THREADS>>>(0, b.dldw1, b.P, b.led, imLs_sz, imHs_sz,
                                                      b.subwave, b.latentZ);
    cufftExecC2C(planBatch, (cufftComplex *)b.latentZ, (cufftComplex *)b.latentZ, CUFFT_INVERSE);
    differenceKernel_acc<<<N_BLOCKS, N_THREADS>>>(0, imLs_sz, pratio, b.Y, b.latentZ, b.recordZ);
    cufftExecC2C(planBatch, (cufftComplex *)b.recordZ, (cufftComplex *)b.latentZ, CUFFT_FORWARD);
    cudaMemset(b.dldw1, 0, big * 8);
    cudaMemset(b.dldw2, 0, plane * 8);
    fused_deconvPIE_shifted<<<N_BLOCKS, N_THREADS>>>(0, b.latentZ, b.subwave, b.led, b.P, imLs_sz,
                                                     imHs_sz, b.dldw1, b.dldw2);
    cufftExecC2C(planLarge, (cufftComplex *)b.dldw1, (cufftComplex *)b.dldw1, CUFFT_INVERSE);
    int rc = (int)cudaDeviceSynchronize();
    if (rc == 0) {
        cudaMemcpy(dO_out, b.dldw1, big * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(dP_out, b.dldw2, plane * 8, cudaMemcpyDeviceToHost);
    }
    cufftDestroy(planBatch);
    cufftDestroy(planLarge);
    b.free_all();
    return rc;
}

// Diagnostic twin of ref_solve for locating writes outside a buffer: every device
// buffer gets a 64 KiB sentinel band before and after it, and after each operation of
// the first `max_steps` operations of the loop (9 per batch: the forward FFT, the crop,
// the batched inverse FFT, the loss stencil, the batched forward FFT, the two memsets,
// the stitch, the inverse FFT, the RMSprop) the stream is synchronised, the number of
// changed sentinel bytes of each of the 12 buffers is written to guards[step * 12 + i]
// (order O, P, latentZ, recordZ, subwave, dldw1, dldw2, mom1, mom2, Y, P0, led) and the
// pupil (complex h x h) to P_trace[step].  Returns the number of steps recorded, or a
// negative line number on a failed CUDA call.  Reads only; writes nothing outside the
// buffers it owns.
int ref_solve_trace(int h, int H, int L, int pratio, int epochs, int batch, float lr, float beta,
                    float eps, const float *O0, const float *P0c, const float *Y, const int *led,
                    const float *P0, float *O_out, float *P_out, float *P_trace, int *guards,
                    int max_steps) {
    const size_t G = 64 * 1024;
    const size_t plane = (size_t)h * h, big = (size_t)H * H, arraysize = plane * batch;
    const size_t sizes[12] = {big * 8, plane * 8, arraysize * 8, arraysize * 8, arraysize * 8,
                              big * 8, plane * 8, big * 4, plane * 4, plane * L * 4, plane * 4,
                              (size_t)L * 8};
    char *base[12] = {};
    auto release = [&]() {
        for (char *b : base)
            if (b) cudaFree(b);
    };
#define TCK(x)                 \
    do {                       \
        if ((x) != 0) {        \
            release();         \
            return -__LINE__;  \
        }                      \
    } while (0)
    for (int i = 0; i < 12; ++i) {
        TCK(cudaMalloc(&base[i], sizes[i] + 2 * G));
        TCK(cudaMemset(base[i], 0xA5, G));
        TCK(cudaMemset(base[i] + G + sizes[i], 0xA5, G));
    }
    auto buf = [&](int i) { return static_cast<void *>(base[i] + G); };
    creal32_t *O = (creal32_t *)buf(0), *P = (creal32_t *)buf(1), *latentZ = (creal32_t *)buf(2),
              *recordZ = (creal32_t *)buf(3), *subwave = (creal32_t *)buf(4),
              *dldw1 = (creal32_t *)buf(5), *dldw2 = (creal32_t *)buf(6);
    real32_T *mom1 = (real32_T *)buf(7), *mom2 = (real32_T *)buf(8), *dY = (real32_T *)buf(9),
             *dP0 = (real32_T *)buf(10);
    int2 *dled = (int2 *)buf(11);
    TCK(cudaMemcpy(O, O0, big * 8, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(P, P0c, plane * 8, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(dY, Y, plane * L * 4, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(dP0, P0, plane * 4, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(dled, led, (size_t)L * 8, cudaMemcpyHostToDevice));
    TCK(cudaMemset(mom1, 0, big * 4));
    TCK(cudaMemset(mom2, 0, plane * 4));
    dim3 imLs_sz = dims_of(h, h, L);
    dim3 imHs_sz = dims_of(H, H, 1);
    dim3 N_THREADS = {BLOCK_X, BLOCK_Y, 1};
    dim3 N_BLOCKS_L = {(imHs_sz.x + BLOCK_X - 1) / BLOCK_X, (imHs_sz.y + BLOCK_Y - 1) / BLOCK_Y, 1};
    dim3 N_BLOCKS = {(imLs_sz.x + BLOCK_X - 1) / BLOCK_X, (imLs_sz.y + BLOCK_Y - 1) / BLOCK_Y, 1};
    const int led_total = (int)imLs_sz.z;
    int inembed[2] = {(int)imLs_sz.x, (int)imLs_sz.y};
    imLs_sz.z = batch;
    cufftHandle planLarge, planBatch;
    if (cufftPlan2d(&planLarge, imHs_sz.x, imHs_sz.y, CUFFT_C2C) != CUFFT_SUCCESS) {
        release();
        return -1;
    }
    if (cufftPlanMany(&planBatch, 2, inembed, inembed, 1, (int)plane, inembed, 1, (int)plane,
                      CUFFT_C2C, batch) != CUFFT_SUCCESS) {
        cufftDestroy(planLarge);
        release();
        return -2;
    }
    std::vector<unsigned char> g(G);
    int step = 0;
    auto record = [&]() -> int {
        if (step >= max_steps) return 0;
        if (cudaDeviceSynchronize() != cudaSuccess) return -__LINE__;
        for (int i = 0; i < 12; ++i) {
            int changed = 0;
            for (int side = 0; side < 2; ++side) {
                const char *src = side == 0 ? base[i] : base[i] + G + sizes[i];
                if (cudaMemcpy(g.data(), src, G, cudaMemcpyDeviceToHost) != cudaSuccess)
                    return -__LINE__;
                for (size_t k = 0; k < G; ++k) changed += g[k] != 0xA5;
            }
            guards[step * 12 + i] = changed;
        }
        if (cudaMemcpy(P_trace + (size_t)step * plane * 2, P, plane * 8,
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            return -__LINE__;
        ++step;
        return 0;
    };
    int rc = 0;
#define TREC()                                  \
    do {                                        \
        rc = record();                          \
        if (rc) goto done;                      \
    } while (0)
    for (int epoch = 0; epoch < epochs; ++epoch) {
        int remain = led_total, curr = 0;
        while (remain > 0) {
            remain -= batch;
            cufftExecC2C(planLarge, (cufftComplex *)O, (cufftComplex *)dldw1, CUFFT_FORWARD);
            TREC();
            N_BLOCKS.z = (unsigned)(min(curr + batch - 1, led_total - 1) - curr + 1);
            fused_getSubpupil_shifted<<<N_BLOCKS, N_THREADS>>>(curr, dldw1, P, dled, imLs_sz,
                                                              imHs_sz, subwave, latentZ);
            TREC();
            cufftExecC2C(planBatch, (cufftComplex *)latentZ, (cufftComplex *)latentZ,
                         CUFFT_INVERSE);
            TREC();
            differenceKernel_acc<<<N_BLOCKS, N_THREADS>>>(curr, imLs_sz, pratio, dY, latentZ,
                                                          recordZ);
            TREC();
            cufftExecC2C(planBatch, (cufftComplex *)recordZ, (cufftComplex *)latentZ,
                         CUFFT_FORWARD);
            TREC();
            cudaMemset(dldw1, 0, big * 8);
            cudaMemset(dldw2, 0, plane * 8);
            TREC();
            fused_deconvPIE_shifted<<<N_BLOCKS, N_THREADS>>>(curr, latentZ, subwave, dled, P,
                                                             imLs_sz, imHs_sz, dldw1, dldw2);
            TREC();
            cufftExecC2C(planLarge, (cufftComplex *)dldw1, (cufftComplex *)dldw1, CUFFT_INVERSE);
            TREC();
            constrained_RMSprop_both<<<N_BLOCKS_L, N_THREADS>>>(dldw1, dldw2, beta, lr, eps,
                                                                imHs_sz, imLs_sz, mom1, mom2, O, P,
                                                                dP0, 0.2f);
            TREC();
            curr += batch;
            cudaDeviceSynchronize();
        }
        if (epoch > 12) lr = lr * 0.5;
    }
    rc = (int)cudaDeviceSynchronize();
    if (rc == 0) {
        cudaMemcpy(O_out, O, big * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(P_out, P, plane * 8, cudaMemcpyDeviceToHost);
        rc = step;
    } else {
        rc = -rc;
    }
done:
    cufftDestroy(planBatch);
    cufftDestroy(planLarge);
    release();
    return rc;
#undef TREC
#undef TCK
}

}  // extern "C"

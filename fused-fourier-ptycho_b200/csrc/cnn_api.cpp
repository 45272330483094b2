// The learned warm start's network and its C ABI (fpm_cnn_* in include/fpm.h).
//
// A fixed 4-level encoder-decoder on the tensor-core convolutions of cnn.cu (channels
// c, 2c, 4c at three levels with two 3x3 convolutions each, 8c at the bottom with one;
// 2x2 average pooling down, nearest up-sampling, one convolution and an additive skip
// per level up, a last 3x3 convolution to 2 output planes), ReLU after every convolution
// but the last.  FP32 master weights with Adam, BF16 copies for the convolutions.
// Parameter order (get / set / gradients): for each of the 14 layers, the weights
// [Cout][Cin][3][3] then the biases [Cout].
#include "../../include/fpm.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "cnn.h"
#include "engine.h"

using namespace fpm;

namespace {

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        const cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return e;
        }
        bytes = n;
        return cudaSuccess;
    }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

struct Layer {
    int cin = 0, cout = 0;
    size_t w = 0, b = 0;   // offsets of the weights and biases in the parameter vector
    size_t wb = 0, wf = 0; // offsets of the padded BF16 weights and of their flipped copy
};

#define CK(call)                                        \
    do {                                                \
        const cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) return e_;               \
    } while (0)

}  // namespace

struct fpm_cnn {
    fpm_context *ctx = nullptr;
    cudaStream_t st = nullptr;
    int device = 0, in_ch = 0, base = 0;
    std::vector<Layer> L;
    size_t n_params = 0, n_bf16 = 0, n_flip = 0;
    Buf w, g, m, v, wb, wflip, loss, mse_work, wg_work, flag;
    int step = 0;
    // activations and gradients for the current (N, h)
    int cur_n = 0, cur_h = 0;
    Buf act[23];
    Buf ga, gb, gc, ge1, ge2, ge3, dy;
    std::string err;

    // BF16 weights of layer i in padded rows (cnn.h), and the flipped copy
    __nv_bfloat16 *W(int i) const { return wb.as<__nv_bfloat16>() + L[i].wb; }
    __nv_bfloat16 *Wf(int i) const { return wflip.as<__nv_bfloat16>() + L[i].wf; }
    int *dflag() const { return flag.as<int>(); }
    const float *bias(int i) const { return w.as<float>() + L[i].b; }
    float *dW(int i) const { return g.as<float>() + L[i].w; }
    float *db(int i) const { return g.as<float>() + L[i].b; }
};

namespace {

// activation slots
enum {
    R1, E1, P1, R3, E2, P2, R5, E3, P3, E4, U3, R8, S3, D3, U2, R10, S2, D2, U1, R12, S1, D1, Y, NACT
};

void build_layers(fpm_cnn *net) {
    const int c = net->base;
    const int io[14][2] = {{net->in_ch, c}, {c, c},         {c, 2 * c},     {2 * c, 2 * c},
                           {2 * c, 4 * c},  {4 * c, 4 * c}, {4 * c, 8 * c}, {8 * c, 4 * c},
                           {4 * c, 4 * c},  {4 * c, 2 * c}, {2 * c, 2 * c}, {2 * c, c},
                           {c, c},          {c, 2}};
    size_t off = 0, nb = 0, nf = 0;
    for (auto &x : io) {
        Layer l;
        l.cin = x[0];
        l.cout = x[1];
        l.w = off;
        off += (size_t)l.cout * l.cin * 9;
        l.b = off;
        off += l.cout;
        l.wb = nb;
        nb += (size_t)cnn::padded_rows(l.cout) * cnn::padded_taps(l.cin);
        l.wf = nf;
        nf += (size_t)cnn::padded_rows(l.cin) * cnn::padded_taps(l.cout);
        net->L.push_back(l);
    }
    net->n_params = off;
    net->n_bf16 = nb;
    net->n_flip = nf;
}

// the plane count and side of each activation slot for batch N at side h
void slot_shape(const fpm_cnn *net, int s, int h, int *ch, int *side) {
    const int c = net->base;
    static const int table[NACT][2] = {
        {1, 1}, {1, 1}, {1, 2}, {2, 2}, {2, 2}, {2, 4}, {4, 4}, {4, 4}, {4, 8}, {8, 8}, {8, 4}, {4, 4},
        {4, 4}, {4, 4}, {4, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 1}, {1, 1}, {1, 1}, {1, 1}, {0, 1}};
    *ch = s == Y ? 2 : table[s][0] * c;
    *side = h / table[s][1];
}

cudaError_t ensure_shape(fpm_cnn *net, int N, int h) {
    if (N == net->cur_n && h == net->cur_h) return cudaSuccess;
    size_t maxsz = 0;
    for (int s = 0; s < NACT; ++s) {
        int ch, side;
        slot_shape(net, s, h, &ch, &side);
        const size_t n = (size_t)N * ch * side * side;
        maxsz = std::max(maxsz, n);
        CK(net->act[s].ensure(n * 4));
    }
    Buf *gs[] = {&net->ga, &net->gb, &net->gc, &net->dy};
    for (Buf *b : gs) CK(b->ensure(maxsz * 4));
    CK(net->ge1.ensure((size_t)N * net->base * h * h * 4));
    CK(net->ge2.ensure((size_t)N * 2 * net->base * (h / 2) * (h / 2) * 4));
    CK(net->ge3.ensure((size_t)N * 4 * net->base * (h / 4) * (h / 4) * 4));
    size_t wg = 0;
    for (int i = 0; i < 14; ++i) {
        const int side = i < 2 || i >= 11 ? h : (i < 4 || i >= 9 ? h / 2 : (i < 6 || i >= 7 ? h / 4 : h / 8));
        const int sp = cnn::conv3x3_weight_grad_splits(N, side, side, net->L[i].cin);
        wg = std::max(wg, (size_t)sp * net->L[i].cout * net->L[i].cin * 9);
    }
    wg = std::max(wg, (size_t)8 * net->base * cnn::bias_grad_splits(N, h * h));
    CK(net->wg_work.ensure(wg * 4));
    net->cur_n = N;
    net->cur_h = h;
    return cudaSuccess;
}

float *A(fpm_cnn *net, int s) { return net->act[s].as<float>(); }

cudaError_t conv(fpm_cnn *net, int i, const float *in, int N, int side, float *out, bool relu) {
    const Layer &l = net->L[i];
    CK(cnn::conv3x3_forward(in, N, l.cin, side, side, net->W(i), net->bias(i), l.cout, out,
                            relu, net->dflag(), net->st));
    return cudaSuccess;
}

cudaError_t forward(fpm_cnn *net, const float *x, int N, int h) {
    const int c = net->base;
    const int h2 = h / 2, h4 = h / 4, h8 = h / 8;
    cudaStream_t st = net->st;
    CK(conv(net, 0, x, N, h, A(net, R1), true));
    CK(conv(net, 1, A(net, R1), N, h, A(net, E1), true));
    CK(cnn::pool_forward(A(net, E1), N * c, h, h, A(net, P1), st));
    CK(conv(net, 2, A(net, P1), N, h2, A(net, R3), true));
    CK(conv(net, 3, A(net, R3), N, h2, A(net, E2), true));
    CK(cnn::pool_forward(A(net, E2), N * 2 * c, h2, h2, A(net, P2), st));
    CK(conv(net, 4, A(net, P2), N, h4, A(net, R5), true));
    CK(conv(net, 5, A(net, R5), N, h4, A(net, E3), true));
    CK(cnn::pool_forward(A(net, E3), N * 4 * c, h4, h4, A(net, P3), st));
    CK(conv(net, 6, A(net, P3), N, h8, A(net, E4), true));
    CK(cnn::up_forward(A(net, E4), N * 8 * c, h8, h8, A(net, U3), st));
    CK(conv(net, 7, A(net, U3), N, h4, A(net, R8), true));
    CK(cnn::add(A(net, R8), A(net, E3), A(net, S3), (size_t)N * 4 * c * h4 * h4, st));
    CK(conv(net, 8, A(net, S3), N, h4, A(net, D3), true));
    CK(cnn::up_forward(A(net, D3), N * 4 * c, h4, h4, A(net, U2), st));
    CK(conv(net, 9, A(net, U2), N, h2, A(net, R10), true));
    CK(cnn::add(A(net, R10), A(net, E2), A(net, S2), (size_t)N * 2 * c * h2 * h2, st));
    CK(conv(net, 10, A(net, S2), N, h2, A(net, D2), true));
    CK(cnn::up_forward(A(net, D2), N * 2 * c, h2, h2, A(net, U1), st));
    CK(conv(net, 11, A(net, U1), N, h, A(net, R12), true));
    CK(cnn::add(A(net, R12), A(net, E1), A(net, S1), (size_t)N * c * h * h, st));
    CK(conv(net, 12, A(net, S1), N, h, A(net, D1), true));
    CK(conv(net, 13, A(net, D1), N, h, A(net, Y), false));
    return cudaSuccess;
}

// Gradients of layer i given the gradient of its pre-activation output `gout` (relu
// already applied), its input `in`; the input gradient goes to gin (null: not needed).
cudaError_t conv_back(fpm_cnn *net, int i, const float *in, float *gout, int N, int side,
                      float *gin) {
    const Layer &l = net->L[i];
    cudaStream_t st = net->st;
    const int sp = cnn::conv3x3_weight_grad_splits(N, side, side, l.cin);
    CK(cnn::conv3x3_weight_grad(in, gout, N, l.cin, side, side, l.cout, net->dW(i),
                                net->wg_work.as<float>(), sp, net->dflag(), st));
    // the weight gradient's partials are summed: its work buffer is free for these
    CK(cnn::bias_grad(gout, N, l.cout, side * side, net->db(i), net->wg_work.as<float>(), st));
    if (gin) {
        CK(cnn::conv3x3_flip(net->W(i), l.cout, l.cin, net->Wf(i), st));
        CK(cnn::conv3x3_forward(gout, N, l.cout, side, side, net->Wf(i), nullptr, l.cin, gin,
                                false, net->dflag(), st));
    }
    return cudaSuccess;
}

cudaError_t backward(fpm_cnn *net, const float *x, int N, int h) {
    const int c = net->base;
    const int h2 = h / 2, h4 = h / 4, h8 = h / 8;
    cudaStream_t st = net->st;
    float *ga = net->ga.as<float>(), *gb = net->gb.as<float>(), *gc = net->gc.as<float>();
    float *ge1 = net->ge1.as<float>(), *ge2 = net->ge2.as<float>(), *ge3 = net->ge3.as<float>();
    const size_t n1 = (size_t)N * c * h * h, n2 = (size_t)N * 2 * c * h2 * h2,
                 n3 = (size_t)N * 4 * c * h4 * h4;
    // last layer (no activation) and level 1 up
    CK(conv_back(net, 13, A(net, D1), net->dy.as<float>(), N, h, ga));       // ga = g d1
    CK(cnn::relu_backward(ga, A(net, D1), n1, st));
    CK(conv_back(net, 12, A(net, S1), ga, N, h, gb));                          // gb = g s1
    CK(cudaMemcpyAsync(ge1, gb, n1 * 4, cudaMemcpyDeviceToDevice, st));        // skip to e1
    CK(cnn::relu_backward(gb, A(net, R12), n1, st));
    CK(conv_back(net, 11, A(net, U1), gb, N, h, ga));                          // ga = g u1
    CK(cnn::up_backward(ga, N * 2 * c, h2, h2, gc, st));                       // gc = g d2
    CK(cnn::relu_backward(gc, A(net, D2), n2, st));
    CK(conv_back(net, 10, A(net, S2), gc, N, h2, ga));                         // ga = g s2
    CK(cudaMemcpyAsync(ge2, ga, n2 * 4, cudaMemcpyDeviceToDevice, st));
    CK(cnn::relu_backward(ga, A(net, R10), n2, st));
    CK(conv_back(net, 9, A(net, U2), ga, N, h2, gb));                          // gb = g u2
    CK(cnn::up_backward(gb, N * 4 * c, h4, h4, gc, st));                       // gc = g d3
    CK(cnn::relu_backward(gc, A(net, D3), n3, st));
    CK(conv_back(net, 8, A(net, S3), gc, N, h4, ga));                          // ga = g s3
    CK(cudaMemcpyAsync(ge3, ga, n3 * 4, cudaMemcpyDeviceToDevice, st));
    CK(cnn::relu_backward(ga, A(net, R8), n3, st));
    CK(conv_back(net, 7, A(net, U3), ga, N, h4, gb));                          // gb = g u3
    CK(cnn::up_backward(gb, N * 8 * c, h8, h8, gc, st));                       // gc = g e4
    CK(cnn::relu_backward(gc, A(net, E4), (size_t)N * 8 * c * h8 * h8, st));
    CK(conv_back(net, 6, A(net, P3), gc, N, h8, ga));                          // ga = g p3
    // down path, level 3 .. 1
    CK(cnn::pool_backward(ga, N * 4 * c, h4, h4, gb, st));
    CK(cnn::add(ge3, gb, ge3, n3, st));
    CK(cnn::relu_backward(ge3, A(net, E3), n3, st));
    CK(conv_back(net, 5, A(net, R5), ge3, N, h4, ga));                         // ga = g r5
    CK(cnn::relu_backward(ga, A(net, R5), n3, st));
    CK(conv_back(net, 4, A(net, P2), ga, N, h4, gb));                          // gb = g p2
    CK(cnn::pool_backward(gb, N * 2 * c, h2, h2, ga, st));
    CK(cnn::add(ge2, ga, ge2, n2, st));
    CK(cnn::relu_backward(ge2, A(net, E2), n2, st));
    CK(conv_back(net, 3, A(net, R3), ge2, N, h2, ga));                         // ga = g r3
    CK(cnn::relu_backward(ga, A(net, R3), n2, st));
    CK(conv_back(net, 2, A(net, P1), ga, N, h2, gb));                          // gb = g p1
    CK(cnn::pool_backward(gb, N * c, h, h, ga, st));
    CK(cnn::add(ge1, ga, ge1, n1, st));
    CK(cnn::relu_backward(ge1, A(net, E1), n1, st));
    CK(conv_back(net, 1, A(net, R1), ge1, N, h, ga));                          // ga = g r1
    CK(cnn::relu_backward(ga, A(net, R1), n1, st));
    CK(conv_back(net, 0, x, ga, N, h, nullptr));
    return cudaSuccess;
}

}  // namespace

// ---------------------------------------------------------------------------
// ABI
// ---------------------------------------------------------------------------
namespace {

fpm_status net_fail(fpm_cnn *net, fpm_status s, const std::string &what) {
    net->err = what;
    return s;
}

fpm_status net_cuda(fpm_cnn *net, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return FPM_OK;
    cudaGetLastError();
    return net_fail(net, e == cudaErrorMemoryAllocation ? FPM_ERR_OUT_OF_MEMORY : FPM_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

bool device_ptr(const void *p, int device) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

// waits for the network's stream and reports a tensor-core wait that ran out (the flag
// is cleared for the next call)
fpm_status sync_and_check(fpm_cnn *net, const char *what) {
    int f = 0;
    fpm_status rc = net_cuda(net, cudaMemcpyAsync(&f, net->flag.p, sizeof(int),
                                                  cudaMemcpyDeviceToHost, net->st), what);
    if (rc == FPM_OK) rc = net_cuda(net, cudaStreamSynchronize(net->st), what);
    if (rc != FPM_OK) return rc;
    if (f != 0) {
        cudaMemsetAsync(net->flag.p, 0, sizeof(int), net->st);
        return net_fail(net, FPM_ERR_INTERNAL, std::string(what) + ": a tensor-core wait ran out");
    }
    return FPM_OK;
}

fpm_status check_batch(fpm_cnn *net, int n, int h) {
    if (n < 1 || h < 8 || h % 8)
        return net_fail(net, FPM_ERR_INVALID_ARGUMENT,
                        "n >= 1 and a side that is a multiple of 8 are required");
    return net_cuda(net, ensure_shape(net, n, h), "buffers");
}

}  // namespace

extern "C" {

fpm_status fpm_cnn_create(fpm_context *ctx, int32_t in_channels, int32_t base_channels,
                          uint64_t seed, fpm_cnn **out) {
    if (!ctx || !out) return FPM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    // the bottom level's 8 base channels are one tensor-core N tile (at most 256)
    if (in_channels < 1 || in_channels > 1024 || base_channels < 8 || base_channels > 32 ||
        base_channels % 8)
        return FPM_ERR_INVALID_ARGUMENT;
    fpm_cnn *net = new fpm_cnn();
    net->ctx = ctx;
    net->st = static_cast<cudaStream_t>(context_stream(ctx));
    net->device = context_device(ctx);
    net->in_ch = in_channels;
    net->base = base_channels;
    build_layers(net);
    cudaSetDevice(net->device);
    const size_t P = net->n_params;
    cudaError_t e = cudaSuccess;
    Buf *bufs[] = {&net->w, &net->g, &net->m, &net->v};
    for (Buf *b : bufs)
        if (e == cudaSuccess) e = b->ensure(P * 4);
    if (e == cudaSuccess) e = net->wb.ensure(net->n_bf16 * 2);
    if (e == cudaSuccess) e = net->wflip.ensure(net->n_flip * 2);
    if (e == cudaSuccess) e = net->flag.ensure(16);
    // the pads of the BF16 rows stay zero: only the weights themselves are written later
    if (e == cudaSuccess) e = cudaMemsetAsync(net->wb.p, 0, net->n_bf16 * 2, net->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(net->wflip.p, 0, net->n_flip * 2, net->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(net->flag.p, 0, 16, net->st);
    if (e == cudaSuccess) e = net->loss.ensure(64);
    if (e == cudaSuccess) e = net->mse_work.ensure(256 * 8);
    if (e != cudaSuccess) {
        delete net;
        return e == cudaErrorMemoryAllocation ? FPM_ERR_OUT_OF_MEMORY : FPM_ERR_CUDA;
    }
    // He-normal weights (std sqrt(2 / (9 Cin))) from a seeded generator, zero biases
    std::vector<float> h(P, 0.f);
    std::mt19937_64 rng(seed);
    for (const Layer &l : net->L) {
        std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / (9.0 * l.cin)));
        for (size_t i = 0; i < (size_t)l.cout * l.cin * 9; ++i) h[l.w + i] = (float)nd(rng);
    }
    const fpm_status rc = fpm_cnn_set_parameters(net, h.data(), (int64_t)P);
    if (rc != FPM_OK) {
        delete net;
        return rc;
    }
    *out = net;
    return FPM_OK;
}

void fpm_cnn_destroy(fpm_cnn *net) {
    if (!net) return;
    // the context's stream may already be gone (the network outlived its context): wait
    // for the device instead, which is safe at any point, process exit included
    cudaSetDevice(net->device);
    cudaDeviceSynchronize();
    cudaGetLastError();
    delete net;
}

int64_t fpm_cnn_parameter_count(const fpm_cnn *net) { return net ? (int64_t)net->n_params : 0; }

const char *fpm_cnn_last_error(const fpm_cnn *net) { return net ? net->err.c_str() : ""; }

fpm_status fpm_cnn_set_parameters(fpm_cnn *net, const float *params, int64_t n) {
    if (!net || !params || n != (int64_t)net->n_params) return FPM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(net->device);
    cudaStream_t st = net->st;
    fpm_status rc = net_cuda(net, cudaMemcpyAsync(net->w.p, params, n * 4, cudaMemcpyHostToDevice, st),
                             "set parameters");
    if (rc != FPM_OK) return rc;
    // BF16 copies of the weights, layer by layer
    for (size_t i = 0; i < net->L.size(); ++i) {
        const Layer &l = net->L[i];
        rc = net_cuda(net, cnn::to_bf16(net->w.as<float>() + l.w, net->W((int)i),
                                        (size_t)l.cout * l.cin * 9, l.cin,
                                        cnn::padded_taps(l.cin), st),
                      "weights");
        if (rc != FPM_OK) return rc;
    }
    cudaMemsetAsync(net->m.p, 0, n * 4, st);
    cudaMemsetAsync(net->v.p, 0, n * 4, st);
    net->step = 0;
    return net_cuda(net, cudaStreamSynchronize(st), "set parameters");
}

fpm_status fpm_cnn_get_parameters(fpm_cnn *net, float *params, int64_t n) {
    if (!net || !params || n != (int64_t)net->n_params) return FPM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(net->device);
    fpm_status rc = net_cuda(net, cudaMemcpyAsync(params, net->w.p, n * 4, cudaMemcpyDeviceToHost,
                                                  net->st), "get parameters");
    if (rc != FPM_OK) return rc;
    return net_cuda(net, cudaStreamSynchronize(net->st), "get parameters");
}

fpm_status fpm_cnn_forward(fpm_cnn *net, const float *x, int32_t n, int32_t h, float *y) {
    if (!net || !x || !y) return FPM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(net->device);
    if (!device_ptr(x, net->device) || !device_ptr(y, net->device))
        return net_fail(net, FPM_ERR_INVALID_ARGUMENT, "x and y must be device memory");
    fpm_status rc = check_batch(net, n, h);
    if (rc != FPM_OK) return rc;
    rc = net_cuda(net, forward(net, x, n, h), "forward");
    if (rc != FPM_OK) return rc;
    rc = net_cuda(net, cudaMemcpyAsync(y, A(net, Y), (size_t)n * 2 * h * h * 4,
                                       cudaMemcpyDeviceToDevice, net->st), "output");
    if (rc != FPM_OK) return rc;
    return sync_and_check(net, "forward");
}

// loss and parameter gradients of one batch (no update); grads: host, n_params floats, or null
fpm_status fpm_cnn_gradients(fpm_cnn *net, const float *x, const float *t, int32_t n, int32_t h,
                             double *loss, float *grads) {
    if (!net || !x || !t) return FPM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(net->device);
    if (!device_ptr(x, net->device) || !device_ptr(t, net->device))
        return net_fail(net, FPM_ERR_INVALID_ARGUMENT, "x and t must be device memory");
    fpm_status rc = check_batch(net, n, h);
    if (rc != FPM_OK) return rc;
    cudaStream_t st = net->st;
    cudaError_t e = forward(net, x, n, h);
    if (e == cudaSuccess)
        e = cnn::mse(A(net, Y), t, (size_t)n * 2 * h * h, net->dy.as<float>(),
                     net->loss.as<double>(), net->mse_work.as<double>(), st);
    if (e == cudaSuccess) e = backward(net, x, n, h);
    rc = net_cuda(net, e, "gradients");
    if (rc != FPM_OK) return rc;
    double l = 0.0;
    rc = net_cuda(net, cudaMemcpyAsync(&l, net->loss.p, 8, cudaMemcpyDeviceToHost, st), "loss");
    if (rc == FPM_OK && grads)
        rc = net_cuda(net, cudaMemcpyAsync(grads, net->g.p, net->n_params * 4,
                                           cudaMemcpyDeviceToHost, st), "gradients");
    if (rc != FPM_OK) return rc;
    rc = sync_and_check(net, "gradients");
    if (rc == FPM_OK && loss) *loss = l;
    return rc;
}

// one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch's mean-squared loss
fpm_status fpm_cnn_train_step(fpm_cnn *net, const float *x, const float *t, int32_t n, int32_t h,
                              float lr, double *loss) {
    fpm_status rc = fpm_cnn_gradients(net, x, t, n, h, loss, nullptr);
    if (rc != FPM_OK) return rc;
    net->step += 1;
    cudaStream_t st = net->st;
    for (size_t i = 0; i < net->L.size(); ++i) {
        const Layer &l = net->L[i];
        const size_t nw = (size_t)l.cout * l.cin * 9;
        float *w = net->w.as<float>(), *m = net->m.as<float>(), *v = net->v.as<float>();
        const float *g = net->g.as<float>();
        cudaError_t e = cnn::adam(w + l.w, m + l.w, v + l.w, g + l.w, net->W((int)i), nw,
                                  l.cin, cnn::padded_taps(l.cin), lr, 0.9f, 0.999f, 1e-8f,
                                  net->step, st);
        if (e == cudaSuccess)
            e = cnn::adam(w + l.b, m + l.b, v + l.b, g + l.b, nullptr, (size_t)l.cout, 0, 0, lr,
                          0.9f, 0.999f, 1e-8f, net->step, st);
        rc = net_cuda(net, e, "adam");
        if (rc != FPM_OK) return rc;
    }
    return FPM_OK;
}

// The warm start of a problem: the network on the problem's first in_channels frames
// (normalised as the solve normalises them), its two output planes (real, imaginary part
// of the low-resolution object) up-sampled bicubically to H x H into `object` (device,
// complex, column-major).  Device-memory problems only.
fpm_status fpm_cnn_initial_object(fpm_cnn *net, const fpm_problem *p, float *object) {
    if (!net || !p || !object) return FPM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(net->device);
    if (p->memory != FPM_MEM_DEVICE)
        return net_fail(net, FPM_ERR_UNSUPPORTED, "the warm start takes device-memory problems");
    const int h = p->h, H = p->h * p->pratio;
    if (p->n_leds < net->in_ch)
        return net_fail(net, FPM_ERR_INVALID_ARGUMENT, "fewer frames than network inputs");
    if (!device_ptr(p->stack, net->device) || !device_ptr(object, net->device))
        return net_fail(net, FPM_ERR_INVALID_ARGUMENT, "stack and object must be device memory");
    fpm_status rc = check_batch(net, 1, h);
    if (rc != FPM_OK) return rc;
    cudaStream_t st = net->st;
    const size_t plane = (size_t)h * h;
    Buf x, mm, work;
    cudaError_t e = x.ensure(plane * net->in_ch * 4);
    if (e == cudaSuccess) e = mm.ensure(16);
    if (e == cudaSuccess) e = work.ensure(bicubic_work_bytes(h, p->pratio));
    StackView sv;
    sv.ptr = p->stack;
    sv.type = p->stack_type == FPM_STACK_U16_COUNTS ? kStackU16 : kStackF32;
    if (e == cudaSuccess && sv.type == kStackU16) {
        e = launch_stack_minmax(static_cast<const uint16_t *>(p->stack), plane * p->n_leds,
                                mm.as<unsigned>(), st);
        sv.minmax = mm.as<unsigned>();
    }
    if (e == cudaSuccess) e = launch_stack_pages(sv, h, 0, net->in_ch, x.as<float>(), st);
    if (e == cudaSuccess) e = forward(net, x.as<float>(), 1, h);
    if (e == cudaSuccess)
        e = launch_bicubic_complex(A(net, Y), A(net, Y) + plane, h, p->pratio,
                                   reinterpret_cast<float2 *>(object), work.p, st);
    (void)H;
    fpm_status rc2 = net_cuda(net, e, "initial object");
    if (rc2 != FPM_OK) return rc2;
    return sync_and_check(net, "initial object");
}

// The warm start with its fallback: the network's starting object and the plain one
// (object_init, or the bicubic start when that is NULL) each get one epoch, and the solve
// then runs from the start whose first-epoch loss is lower (the network's on a tie).
fpm_status fpm_solve_warm(fpm_context *ctx, fpm_cnn *net, const fpm_problem *p, fpm_result *res,
                          int32_t *used_network) {
    if (!ctx || !net || !p || !res) return FPM_ERR_INVALID_ARGUMENT;
    if (used_network) *used_network = 0;
    cudaSetDevice(net->device);
    if (p->memory != FPM_MEM_DEVICE)
        return net_fail(net, FPM_ERR_UNSUPPORTED, "the warm start takes device-memory problems");
    if (p->epochs < 1 || p->h < 1 || p->pratio < 1)
        return net_fail(net, FPM_ERR_INVALID_ARGUMENT, "epochs, h and pratio must be positive");
    const size_t H = (size_t)p->h * p->pratio, plane = (size_t)p->h * p->h;
    Buf start, obj, pup, loss;
    cudaError_t e = start.ensure(H * H * 8);
    if (e == cudaSuccess) e = obj.ensure(H * H * 8);
    if (e == cudaSuccess) e = pup.ensure(plane * 8);
    if (e == cudaSuccess) e = loss.ensure(8);
    fpm_status rc = net_cuda(net, e, "warm start buffers");
    if (rc != FPM_OK) return rc;
    rc = fpm_cnn_initial_object(net, p, start.as<float>());
    if (rc != FPM_OK) return rc;
    fpm_problem q = *p;
    q.epochs = 1;
    fpm_result t{obj.as<float>(), nullptr, pup.as<float>(), loss.as<double>()};
    double first[2] = {0.0, 0.0};   // first-epoch loss: network start, plain start
    const float *starts[2] = {start.as<float>(), p->object_init};
    for (int k = 0; k < 2; ++k) {
        q.object_init = starts[k];
        rc = fpm_solve(ctx, &q, &t);
        if (rc != FPM_OK) return net_fail(net, rc, "first epoch of a warm-start candidate");
        rc = net_cuda(net, cudaMemcpyAsync(&first[k], loss.p, 8, cudaMemcpyDeviceToHost, net->st),
                      "first-epoch loss");
        if (rc == FPM_OK) rc = net_cuda(net, cudaStreamSynchronize(net->st), "first-epoch loss");
        if (rc != FPM_OK) return rc;
    }
    const bool use = first[0] <= first[1];   // a NaN loss of the network start: plain start
    q = *p;
    q.object_init = use ? start.as<float>() : p->object_init;
    rc = fpm_solve(ctx, &q, res);
    if (rc != FPM_OK) return rc;
    if (used_network) *used_network = use ? 1 : 0;
    return FPM_OK;
}

}  // extern "C"

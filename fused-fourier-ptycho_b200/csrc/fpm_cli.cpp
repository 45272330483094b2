// fpm_cli: command-line front end of libfpm for hosts without MATLAB.
//
// The reference is driven from MATLAB (codes_v2/main_run_FPM.m:77-106 calls the
// mex cuFPM_pure_v3 on gpuArrays).  This program makes the same call from files:
// every array is a raw little-endian file in MATLAB (column-major) order, complex
// values interleaved (re, im) float32, so a MATLAB user writes them with
// fwrite(fid, x, 'uint16') / fwrite(fid, [real(z(:)) imag(z(:))].', 'single').
//
//   fpm_cli solve --h 2048 --leds 361 --pratio 8 --batch 26 --epochs 10
//                 --stack Y.u16 [--stack-type u16|f32] --led ledIdx.i32
//                 --pupil P0c.c64 --pupil-amp P0.f32 [--object O0.c64]
//                 [--lr 5e-4 --beta 0.999 --eps 1e-4 --margin 0.2]
//                 [--out-object O.c64] [--out-spectrum S.c64] [--out-pupil P.c64]
//                 [--out-loss loss.f64] [--device 0] [--profile]
//
// Exit status: 0 on success, 2 on bad usage or unreadable files, 3 + fpm_status
// when the engine refuses or fails (the status string and detail go to stderr).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "fpm.h"

namespace {

int usage(const char *msg) {
    if (msg) std::fprintf(stderr, "fpm_cli: %s\n", msg);
    std::fprintf(stderr,
                 "usage: fpm_cli solve --h N --leds L --pratio P --batch B --epochs E\n"
                 "                     --stack FILE [--stack-type u16|f32] --led FILE\n"
                 "                     --pupil FILE --pupil-amp FILE [--object FILE]\n"
                 "                     [--lr X --beta X --eps X --margin X]\n"
                 "                     [--out-object FILE] [--out-spectrum FILE]\n"
                 "                     [--out-pupil FILE] [--out-loss FILE]\n"
                 "                     [--device D] [--profile]\n");
    return 2;
}

bool read_file(const std::string &path, size_t bytes, std::vector<char> &buf) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
        std::fprintf(stderr, "fpm_cli: cannot open %s\n", path.c_str());
        return false;
    }
    buf.resize(bytes);
    const size_t got = bytes ? std::fread(buf.data(), 1, bytes, f) : 0;
    char extra;
    const bool longer = std::fread(&extra, 1, 1, f) == 1;
    std::fclose(f);
    if (got != bytes || longer) {
        std::fprintf(stderr, "fpm_cli: %s holds %s than the %zu bytes expected\n", path.c_str(),
                     got != bytes ? "fewer" : "more", bytes);
        return false;
    }
    return true;
}

bool write_file(const std::string &path, const void *p, size_t bytes) {
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "fpm_cli: cannot create %s\n", path.c_str());
        return false;
    }
    const size_t put = std::fwrite(p, 1, bytes, f);
    const bool ok = put == bytes && std::fclose(f) == 0;
    if (!ok) std::fprintf(stderr, "fpm_cli: short write to %s\n", path.c_str());
    return ok;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2 || std::strcmp(argv[1], "solve") != 0) return usage(argc < 2 ? nullptr : "unknown command");
    std::map<std::string, std::string> opt;
    bool profile = false;
    for (int i = 2; i < argc; ++i) {
        std::string k = argv[i];
        if (k == "--profile") {
            profile = true;
            continue;
        }
        if (k.rfind("--", 0) != 0 || i + 1 >= argc) return usage(("bad argument " + k).c_str());
        opt[k.substr(2)] = argv[++i];
    }
    auto need = [&](const char *k) -> const std::string * {
        auto it = opt.find(k);
        return it == opt.end() ? nullptr : &it->second;
    };
    for (const char *k : {"h", "leds", "pratio", "batch", "epochs", "stack", "led", "pupil", "pupil-amp"})
        if (!need(k)) return usage((std::string("missing --") + k).c_str());
    auto num = [&](const char *k, double def) {
        auto it = opt.find(k);
        return it == opt.end() ? def : std::atof(it->second.c_str());
    };
    const int h = std::atoi(need("h")->c_str());
    const int L = std::atoi(need("leds")->c_str());
    const int pratio = std::atoi(need("pratio")->c_str());
    if (h <= 0 || L <= 0 || pratio <= 0) return usage("h, leds and pratio must be positive");
    const size_t plane = (size_t)h * h;
    const size_t H = (size_t)h * pratio;
    const size_t big = H * H;
    const std::string st = opt.count("stack-type") ? opt["stack-type"] : "u16";
    if (st != "u16" && st != "f32") return usage("--stack-type is u16 or f32");
    const size_t esz = st == "u16" ? 2 : 4;

    std::vector<char> stack, led, pupil, amp, obj;
    if (!read_file(*need("stack"), plane * L * esz, stack) || !read_file(*need("led"), (size_t)L * 8, led) ||
        !read_file(*need("pupil"), plane * 8, pupil) || !read_file(*need("pupil-amp"), plane * 4, amp))
        return 2;
    if (need("object") && !read_file(*need("object"), big * 8, obj)) return 2;

    fpm_problem pr;
    std::memset(&pr, 0, sizeof(pr));
    pr.h = h;
    pr.n_leds = L;
    pr.pratio = pratio;
    pr.batch = std::atoi(need("batch")->c_str());
    pr.epochs = std::atoi(need("epochs")->c_str());
    pr.lr = (float)num("lr", 5e-4);
    pr.beta = (float)num("beta", 0.999);
    pr.eps = (float)num("eps", 1e-4);
    pr.pupil_margin = (float)num("margin", 0.2);
    pr.lr_halve_after = 12;
    pr.lr_decay = 0.5f;
    pr.loss_kind = FPM_LOSS_ANISOTROPIC;
    pr.memory = FPM_MEM_HOST;
    pr.stack_type = st == "u16" ? FPM_STACK_U16_COUNTS : FPM_STACK_F32_AMPLITUDE;
    pr.stack = stack.data();
    pr.led_idx = reinterpret_cast<const int32_t *>(led.data());
    pr.pupil_init = reinterpret_cast<const float *>(pupil.data());
    pr.pupil_amp = reinterpret_cast<const float *>(amp.data());
    pr.object_init = obj.empty() ? nullptr : reinterpret_cast<const float *>(obj.data());

    std::vector<float> O(need("out-object") ? big * 2 : 0), S(need("out-spectrum") ? big * 2 : 0),
        P(need("out-pupil") ? plane * 2 : 0);
    std::vector<double> loss(pr.epochs > 0 ? pr.epochs : 1);
    fpm_result res;
    res.object = O.empty() ? nullptr : O.data();
    res.spectrum = S.empty() ? nullptr : S.data();
    res.pupil = P.empty() ? nullptr : P.data();
    res.loss = loss.data();

    fpm_device_opts dopt;
    std::memset(&dopt, 0, sizeof(dopt));
    dopt.device = (int32_t)num("device", 0);
    fpm_context *ctx = nullptr;
    fpm_status rc = fpm_create(&ctx, &dopt);
    if (rc != FPM_OK) {
        std::fprintf(stderr, "fpm_cli: %s\n", fpm_status_string(rc));
        return 3 + (int)rc;
    }
    if (profile) fpm_set_profiling(ctx, 1);
    const auto t0 = std::chrono::steady_clock::now();
    rc = fpm_solve(ctx, &pr, &res);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != FPM_OK) {
        std::fprintf(stderr, "fpm_cli: %s: %s\n", fpm_status_string(rc), fpm_last_error(ctx));
        fpm_destroy(ctx);
        return 3 + (int)rc;
    }
    std::printf("solve: %d LEDs of %dx%d -> %zux%zu, %d epochs, batch %d: %.3f s\n", L, h, h, H, H,
                pr.epochs, pr.batch, sec);
    for (int e = 0; e < pr.epochs; ++e) std::printf("loss[%d] = %.9e\n", e, loss[e]);
    if (profile) {
        fpm_stage_time t[32];
        const int n = fpm_stage_times(ctx, t, 32);
        for (int i = 0; i < n && i < 32; ++i)
            std::printf("stage %-22s launches %5d  %10.3f ms\n", t[i].name, t[i].launches, t[i].ms);
    }
    fpm_destroy(ctx);
    bool ok = true;
    if (!O.empty()) ok &= write_file(opt["out-object"], O.data(), O.size() * 4);
    if (!S.empty()) ok &= write_file(opt["out-spectrum"], S.data(), S.size() * 4);
    if (!P.empty()) ok &= write_file(opt["out-pupil"], P.data(), P.size() * 4);
    if (opt.count("out-loss")) ok &= write_file(opt["out-loss"], loss.data(), (size_t)pr.epochs * 8);
    return ok ? 0 : 2;
}

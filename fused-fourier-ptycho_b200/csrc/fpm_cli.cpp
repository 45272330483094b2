// fpm_cli: command-line front end of libfpm for hosts without MATLAB.
//
// The reference is driven from MATLAB (codes_v2/main_run_FPM.m:77-106 calls the
// mex cuFPM_pure_v3 on gpuArrays).  This program makes the same call from files:
// every array is a raw little-endian file in MATLAB (column-major) order, complex
// values interleaved (re, im) float32, so a MATLAB user writes them with
// fwrite(fid, x, 'uint16') / fwrite(fid, [real(z(:)) imag(z(:))].', 'single').
//
//   fpm_cli solve --h 2048 --leds 361 --pratio 8 --batch 26 --epochs 10
//                 (--stack Y.u16 [--stack-type u16|f32] | --tiff-list frames.txt
//                  [--row0 0 --col0 0] [--tiff-type u16|f32])
//                 --led ledIdx.i32 --pupil P0c.c64 --pupil-amp P0.f32 [--object O0.c64]
//                 [--lr 5e-4 --beta 0.999 --eps 1e-4 --margin 0.2]
//                 [--loss anisotropic|isotropic] [--pie none|ePIE|tPIE]
//                 [--out-object O.c64] [--out-spectrum S.c64] [--out-pupil P.c64]
//                 [--out-loss loss.f64] [--device 0] [--profile]
//
//   fpm_cli ingest --tiff-list frames.txt --h 2048 [--row0 0 --col0 0]
//                  [--tiff-type u16|f32] --out Y.u16
//
//   fpm_cli leds --grid 19 --h 2048 --pratio 8 --wavelength 0.532 --pitch 4000
//                --height 90000 --pixel 6.5 --mag 4 --out-led ledIdx.i32
//                [--out-frames frames.txt --frames-dir raw_images/green]
//
// A frame list is a text file naming one TIFF per line, in LED order (the
// reference loads raw_images/<colour>/<k>.tif in its spiral order,
// codes_v2/main_run_FPM.m:26-41); --row0/--col0 give the 0-based top-left pixel
// of the h x h region read from each.  --tiff-type u16 keeps uint16 counts
// (single-sample frames; the solve normalises them on the device), f32 averages
// each pixel's samples as mean(single(x), 3) and the solve normalises that float
// stack on the device before it starts.
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
                 "                     (--stack FILE [--stack-type u16|f32] |\n"
                 "                      --tiff-list FILE [--row0 R --col0 C] [--tiff-type u16|f32])\n"
                 "                     --led FILE --pupil FILE --pupil-amp FILE [--object FILE]\n"
                 "                     [--lr X --beta X --eps X --margin X]\n"
                 "                     [--loss anisotropic|isotropic] [--pie none|ePIE|tPIE]\n"
                 "                     [--out-object FILE] [--out-spectrum FILE]\n"
                 "                     [--out-pupil FILE] [--out-loss FILE]\n"
                 "                     [--device D] [--profile]\n"
                 "       fpm_cli ingest --tiff-list FILE --h N [--row0 R --col0 C]\n"
                 "                      [--tiff-type u16|f32] --out FILE\n"
                 "       fpm_cli leds --grid G --h N --pratio P --wavelength UM --pitch UM\n"
                 "                    --height UM --pixel UM --mag M [--dx UM --dy UM]\n"
                 "                    --out-led FILE [--out-frames FILE --frames-dir DIR]\n");
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

// Frame names, one per non-empty line (trailing CR / spaces dropped).
bool read_list(const std::string &path, std::vector<std::string> &names) {
    std::FILE *f = std::fopen(path.c_str(), "r");
    if (!f) {
        std::fprintf(stderr, "fpm_cli: cannot open %s\n", path.c_str());
        return false;
    }
    std::string line;
    int ch;
    auto flush = [&] {
        while (!line.empty() && (line.back() == '\r' || line.back() == ' ' || line.back() == '\t'))
            line.pop_back();
        if (!line.empty()) names.push_back(line);
        line.clear();
    };
    while ((ch = std::fgetc(f)) != EOF) {
        if (ch == '\n') {
            flush();
        } else {
            line.push_back((char)ch);
        }
    }
    flush();
    std::fclose(f);
    return true;
}

using Options = std::map<std::string, std::string>;

const std::string *find(const Options &opt, const char *k) {
    auto it = opt.find(k);
    return it == opt.end() ? nullptr : &it->second;
}

double num(const Options &opt, const char *k, double def) {
    auto it = opt.find(k);
    return it == opt.end() ? def : std::atof(it->second.c_str());
}

// Reads the frames of --tiff-list into stack (h*h per frame); u16 or float mean.
// Returns 0, or the exit status.
int ingest_frames(const Options &opt, int h, int expect, bool &f32, std::vector<char> &stack) {
    std::vector<std::string> names;
    if (!read_list(*find(opt, "tiff-list"), names)) return 2;
    if (names.empty()) return usage("the frame list names no file");
    if (expect > 0 && (int)names.size() != expect) {
        std::fprintf(stderr, "fpm_cli: the frame list names %zu files for %d LEDs\n", names.size(),
                     expect);
        return 2;
    }
    const std::string *tt = find(opt, "tiff-type");
    if (tt && *tt != "u16" && *tt != "f32") return usage("--tiff-type is u16 or f32");
    f32 = tt && *tt == "f32";
    const int row0 = (int)num(opt, "row0", 0), col0 = (int)num(opt, "col0", 0);
    std::vector<const char *> ptrs;
    for (const auto &n : names) ptrs.push_back(n.c_str());
    stack.resize((size_t)h * h * names.size() * (f32 ? 4 : 2));
    const auto t0 = std::chrono::steady_clock::now();
    const fpm_status rc = fpm_read_tiff_stack(nullptr, ptrs.data(), (int32_t)ptrs.size(), row0, col0,
                                              h, f32 ? FPM_INGEST_F32_MEAN : FPM_INGEST_U16,
                                              stack.data(), 0);
    if (rc != FPM_OK) {
        std::fprintf(stderr, "fpm_cli: %s\n", fpm_last_error(nullptr));
        return 2;
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("ingest: %zu frames, %dx%d region at (%d, %d): %.3f s\n", names.size(), h, h, row0,
                col0, sec);
    return 0;
}

int cmd_ingest(const Options &opt) {
    for (const char *k : {"tiff-list", "h", "out"})
        if (!find(opt, k)) return usage((std::string("missing --") + k).c_str());
    const int h = std::atoi(find(opt, "h")->c_str());
    if (h <= 0) return usage("h must be positive");
    bool f32 = false;
    std::vector<char> stack;
    const int rc = ingest_frames(opt, h, 0, f32, stack);
    if (rc) return rc;
    return write_file(*find(opt, "out"), stack.data(), stack.size()) ? 0 : 2;
}

int cmd_solve(const Options &opt, bool profile) {
    auto need = [&](const char *k) { return find(opt, k); };
    for (const char *k : {"h", "leds", "pratio", "batch", "epochs", "led", "pupil", "pupil-amp"})
        if (!need(k)) return usage((std::string("missing --") + k).c_str());
    if (!need("stack") == !need("tiff-list")) return usage("give one of --stack and --tiff-list");
    const int h = std::atoi(need("h")->c_str());
    const int L = std::atoi(need("leds")->c_str());
    const int pratio = std::atoi(need("pratio")->c_str());
    if (h <= 0 || L <= 0 || pratio <= 0) return usage("h, leds and pratio must be positive");
    const size_t plane = (size_t)h * h;
    const size_t H = (size_t)h * pratio;
    const size_t big = H * H;

    std::vector<char> stack, led, pupil, amp, obj;
    bool u16 = true, normalise_f32 = false;
    if (need("stack")) {
        const std::string st = need("stack-type") ? *need("stack-type") : "u16";
        if (st != "u16" && st != "f32") return usage("--stack-type is u16 or f32");
        u16 = st == "u16";
        if (!read_file(*need("stack"), plane * L * (u16 ? 2 : 4), stack)) return 2;
    } else {
        bool f32 = false;
        const int rc = ingest_frames(opt, h, L, f32, stack);
        if (rc) return rc;
        u16 = !f32;
        normalise_f32 = f32;
    }
    if (!read_file(*need("led"), (size_t)L * 8, led) || !read_file(*need("pupil"), plane * 8, pupil) ||
        !read_file(*need("pupil-amp"), plane * 4, amp))
        return 2;
    if (need("object") && !read_file(*need("object"), big * 8, obj)) return 2;

    fpm_problem pr;
    std::memset(&pr, 0, sizeof(pr));
    pr.h = h;
    pr.n_leds = L;
    pr.pratio = pratio;
    pr.batch = std::atoi(need("batch")->c_str());
    pr.epochs = std::atoi(need("epochs")->c_str());
    pr.lr = (float)num(opt, "lr", 5e-4);
    pr.beta = (float)num(opt, "beta", 0.999);
    pr.eps = (float)num(opt, "eps", 1e-4);
    pr.pupil_margin = (float)num(opt, "margin", 0.2);
    pr.lr_halve_after = 12;
    pr.lr_decay = 0.5f;
    const std::string lk = need("loss") ? *need("loss") : "anisotropic";
    if (lk != "anisotropic" && lk != "isotropic") return usage("--loss is anisotropic or isotropic");
    pr.loss_kind = lk == "isotropic" ? FPM_LOSS_ISOTROPIC : FPM_LOSS_ANISOTROPIC;
    const std::string pie = need("pie") ? *need("pie") : "none";
    if (pie != "none" && pie != "ePIE" && pie != "tPIE") return usage("--pie is none, ePIE or tPIE");
    pr.pie_weights = pie == "ePIE" ? FPM_PIE_EPIE : pie == "tPIE" ? FPM_PIE_TPIE : FPM_PIE_NONE;
    pr.memory = FPM_MEM_HOST;
    pr.stack_type = u16 ? FPM_STACK_U16_COUNTS : FPM_STACK_F32_AMPLITUDE;
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
    dopt.device = (int32_t)num(opt, "device", 0);
    fpm_context *ctx = nullptr;
    fpm_status rc = fpm_create(&ctx, &dopt);
    if (rc != FPM_OK) {
        std::fprintf(stderr, "fpm_cli: %s\n", fpm_status_string(rc));
        return 3 + (int)rc;
    }
    if (normalise_f32) {
        // float frames: the amplitude sqrt((x-min)/(max-min)) in place, on the device
        float *x = reinterpret_cast<float *>(stack.data());
        rc = fpm_normalise_stack_f32(ctx, x, plane * L, x, FPM_MEM_HOST);
        if (rc != FPM_OK) {
            std::fprintf(stderr, "fpm_cli: %s: %s\n", fpm_status_string(rc), fpm_last_error(ctx));
            fpm_destroy(ctx);
            return 3 + (int)rc;
        }
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
    if (!O.empty()) ok &= write_file(*need("out-object"), O.data(), O.size() * 4);
    if (!S.empty()) ok &= write_file(*need("out-spectrum"), S.data(), S.size() * 4);
    if (!P.empty()) ok &= write_file(*need("out-pupil"), P.data(), P.size() * 4);
    if (need("out-loss")) ok &= write_file(*need("out-loss"), loss.data(), (size_t)pr.epochs * 8);
    return ok ? 0 : 2;
}

// LED crop corners of a square LED array (fpm_led_indices), written as the ledIdx file
// of `solve`, and optionally the frame list of the reference's file naming: in LED
// order, <dir>/<k>.tif with k = j + (i - 1) grid (codes_v2/main_run_FPM.m:33-35).
int cmd_leds(const Options &opt) {
    for (const char *k : {"grid", "h", "pratio", "wavelength", "pitch", "height", "pixel", "mag",
                          "out-led"})
        if (!find(opt, k)) return usage((std::string("missing --") + k).c_str());
    fpm_led_geometry geo;
    std::memset(&geo, 0, sizeof(geo));
    geo.grid = (int32_t)num(opt, "grid", 0);
    geo.h = (int32_t)num(opt, "h", 0);
    geo.pratio = (int32_t)num(opt, "pratio", 0);
    geo.wavelength_um = num(opt, "wavelength", 0);
    geo.led_pitch_um = num(opt, "pitch", 0);
    geo.led_height_um = num(opt, "height", 0);
    geo.camera_pixel_um = num(opt, "pixel", 0);
    geo.magnification = num(opt, "mag", 0);
    geo.sample_dx_um = num(opt, "dx", -0.0);
    geo.sample_dy_um = num(opt, "dy", -0.0);
    if (geo.grid <= 0 || geo.grid > 255) return usage("--grid is 1..255");
    const size_t L = (size_t)geo.grid * geo.grid;
    std::vector<int32_t> led(2 * L), pos(2 * L);
    fpm_device_opts dopt;
    std::memset(&dopt, 0, sizeof(dopt));
    dopt.device = (int32_t)num(opt, "device", 0);
    fpm_context *ctx = nullptr;
    fpm_status rc = fpm_create(&ctx, &dopt);
    if (rc != FPM_OK) {
        std::fprintf(stderr, "fpm_cli: %s\n", fpm_status_string(rc));
        return 3 + (int)rc;
    }
    rc = fpm_led_indices(ctx, &geo, led.data(), pos.data());
    if (rc != FPM_OK) {
        std::fprintf(stderr, "fpm_cli: %s: %s\n", fpm_status_string(rc), fpm_last_error(ctx));
        fpm_destroy(ctx);
        return 3 + (int)rc;
    }
    fpm_destroy(ctx);
    if (!write_file(*find(opt, "out-led"), led.data(), led.size() * sizeof(int32_t))) return 2;
    if (const std::string *fl = find(opt, "out-frames")) {
        const std::string dir = find(opt, "frames-dir") ? *find(opt, "frames-dir") : ".";
        std::string text;
        char name[32];
        for (size_t l = 0; l < L; ++l) {
            const int k = pos[2 * l + 1] + (pos[2 * l] - 1) * geo.grid;
            std::snprintf(name, sizeof name, "%03d.tif", k);
            text += dir + "/" + name + "\n";
        }
        if (!write_file(*fl, text.data(), text.size())) return 2;
    }
    std::printf("leds: %zu LEDs of a %d x %d array\n", L, geo.grid, geo.grid);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) return usage(nullptr);
    const std::string cmd = argv[1];
    if (cmd != "solve" && cmd != "ingest" && cmd != "leds") return usage("unknown command");
    Options opt;
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
    if (cmd == "leds") return cmd_leds(opt);
    return cmd == "solve" ? cmd_solve(opt, profile) : cmd_ingest(opt);
}

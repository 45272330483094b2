// Launch choices that leave a solve's arithmetic unchanged, up to the rounding of an
// alternative radix split: how the passes are grouped, shaped and fed.  The autotuner
// (fpm_autotune in fpm_api.cpp) times them on the caller's own problem and keeps the
// fastest per problem shape; a solve puts its shape's choice in force on the calling host
// thread for its duration.  An environment variable of the same knob, when set, overrides
// both (measurements).
#pragma once

namespace fpm {

struct Tuning {
    int lr_group = 0;       // LEDs per low-resolution launch group; 0 = the whole batch
    int lr_fused = -1;      // fused row pass (h in [128, 2048]): -1 default (on), 0, 1
    int l23_cluster = 0;    // CTAs per cluster of the fused row pass: 0 default (16 lines), 2, 4, 8
    int cols_async = -1;    // bulk-copy prefetch in the 16384-point passes: -1 (on), 0, 1
    int cols_e16 = -1;      // 16 values per thread in the 16384-point passes: -1 (off), 0, 1
    int gen_lpc = 0;        // lines per CTA of the any-size line FFT; 0 = planned
};

// The tuning in force on the calling host thread (defaults when none is set).
const Tuning &tuning();
// Puts t in force on the calling host thread (nullptr: defaults); returns the previous one.
const Tuning *set_tuning(const Tuning *t);
// The value of a knob: the environment variable `env` when set, else `tuned` when it is
// not `unset`, else `dflt`.
int knob(const char *env, int tuned, int unset, int dflt);

// Keeps a tuning in force for the lifetime of the guard.
struct TuningScope {
    const Tuning *prev;
    explicit TuningScope(const Tuning *t) : prev(set_tuning(t)) {}
    ~TuningScope() { set_tuning(prev); }
};

}  // namespace fpm

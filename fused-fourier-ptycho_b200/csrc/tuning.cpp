// The per-thread tuning in force (tuning.h).
#include "tuning.h"

#include <cstdlib>

namespace fpm {

namespace {
const Tuning kDefaults{};
thread_local const Tuning *t_tuning = nullptr;
}  // namespace

const Tuning &tuning() { return t_tuning ? *t_tuning : kDefaults; }

const Tuning *set_tuning(const Tuning *t) {
    const Tuning *prev = t_tuning;
    t_tuning = t;
    return prev;
}

int knob(const char *env, int tuned, int unset, int dflt) {
    if (const char *e = std::getenv(env)) return std::atoi(e);
    return tuned != unset ? tuned : dflt;
}

}  // namespace fpm

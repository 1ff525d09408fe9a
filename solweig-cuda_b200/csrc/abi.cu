// C-ABI glue: thread-local error messages and the library version.
#include <stdarg.h>

#include "common.cuh"

namespace solweig {

static thread_local char g_error[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

}  // namespace solweig

extern "C" const char* solweig_last_error(void) { return solweig::g_error; }

extern "C" int solweig_version(void) { return 100; }

// sizeof of every ABI struct, so bindings can verify their layout:
// out[0..4] = SolweigScene, SolweigSkyLayout, SolweigHour, SolweigOutputs, SolweigState.
extern "C" int solweig_struct_sizes(int64_t* out) {
    if (!out) return SOLWEIG_ERR_INVALID;
    out[0] = sizeof(SolweigScene);
    out[1] = sizeof(SolweigSkyLayout);
    out[2] = sizeof(SolweigHour);
    out[3] = sizeof(SolweigOutputs);
    out[4] = sizeof(SolweigState);
    return SOLWEIG_OK;
}

// out[0..3] = SolweigSky64, SolweigHour64, SolweigOutputs64, SolweigState64.
extern "C" int solweig_struct_sizes64(int64_t* out) {
    if (!out) return SOLWEIG_ERR_INVALID;
    out[0] = sizeof(SolweigSky64);
    out[1] = sizeof(SolweigHour64);
    out[2] = sizeof(SolweigOutputs64);
    out[3] = sizeof(SolweigState64);
    return SOLWEIG_OK;
}

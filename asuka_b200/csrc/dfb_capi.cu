// Library-level C ABI entry points: version and error reporting.
#include <stdarg.h>
#include <stdio.h>

#include "../../include/dfb.h"
#include "dfb_internal.h"

namespace dfb {
static thread_local char g_msg[512] = "";

void clear_error() { g_msg[0] = '\0'; }

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
    return code;
}

int set_cuda_error(const char* what, cudaError_t e) {
    snprintf(g_msg, sizeof(g_msg), "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return DFB_ERR_CUDA;
}
}  // namespace dfb

extern "C" int dfb_version(void) { return 100; }

extern "C" const char* dfb_last_error(void) { return dfb::g_msg; }

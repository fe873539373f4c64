// Library-level C ABI entry points: version and error reporting.
#include <stdarg.h>
#include <stdio.h>

#include <atomic>

#include "../../include/dfb.h"
#include "dfb_internal.h"

namespace dfb {
static thread_local char g_msg[512] = "";
static std::atomic<long> g_launches{0};

void count_launches(long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

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

extern "C" long dfb_launch_count(void) { return dfb::g_launches.load(std::memory_order_relaxed); }

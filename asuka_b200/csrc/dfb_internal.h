// Host-side error reporting shared by the libdfb translation units.
#pragma once
#include <cuda_runtime.h>

namespace dfb {
void clear_error();
int set_error(int code, const char* fmt, ...);
int set_cuda_error(const char* what, cudaError_t e);
// count kernel launches made by the library (dfb_launch_count)
void count_launches(long n);
}  // namespace dfb

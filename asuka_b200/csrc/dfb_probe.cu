// FP64 and FP32 FMA throughput probes: the roofline denominators of the Rys kernels
// (FP64, and the FP32 recurrences of the mixed-precision kernels); the measured-peaks
// file carries HBM and BF16 only.
#include "../../include/dfb.h"
#include "dfb_internal.h"

namespace dfb {
__global__ void k_fp64_fma(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
    double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            x0 = fma(x0, a, b);
            x1 = fma(x1, a, b);
            x2 = fma(x2, a, b);
            x3 = fma(x3, a, b);
            x4 = fma(x4, a, b);
            x5 = fma(x5, a, b);
            x6 = fma(x6, a, b);
            x7 = fma(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
__global__ void k_fp32_fma(float* out, int iters, float a, float b) {
    float x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = threadIdx.x * 1e-6f + k * 1e-6f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += x[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace dfb

extern "C" int dfb_fp32_fma_probe(float* out, int blocks, int threads, int iters, void* stream) {
    dfb::clear_error();
    if (!out || blocks < 1 || threads < 32 || threads > 1024 || iters < 1)
        return dfb::set_error(DFB_ERR_INVALID, "invalid probe arguments");
    dfb::k_fp32_fma<<<blocks, threads, 0, (cudaStream_t)stream>>>(out, iters, 0.999999f, 1e-7f);
    dfb::count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dfb::set_cuda_error("k_fp32_fma launch", e);
    return DFB_OK;
}

extern "C" int dfb_fp64_fma_probe(double* out, int blocks, int threads, int iters, void* stream) {
    dfb::clear_error();
    if (!out || blocks < 1 || threads < 32 || threads > 1024 || iters < 1)
        return dfb::set_error(DFB_ERR_INVALID, "invalid probe arguments");
    dfb::k_fp64_fma<<<blocks, threads, 0, (cudaStream_t)stream>>>(out, iters, 0.999999, 1e-7);
    dfb::count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dfb::set_cuda_error("k_fp64_fma launch", e);
    return DFB_OK;
}

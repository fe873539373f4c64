"""Live FP64 and FP32 peak measurements (the Rys kernels' roofline denominators)."""

from __future__ import annotations

import torch

from . import _lib


def fp64_fma_tflops(device=None, iters: int = 2048) -> float:
    """Best-of-5 FP64 FMA throughput in TFLOP/s over all SMs (2 flops per FMA)."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    props = torch.cuda.get_device_properties(dev)
    blocks, threads = props.multi_processor_count * 8, 256
    out = torch.empty(blocks * threads, dtype=torch.float64, device=dev)
    L = _lib.lib()
    stream = int(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(L.dfb_fp64_fma_probe(_lib.ptr(out), blocks, threads, 64, stream), "dfb_fp64_fma_probe")
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check(L.dfb_fp64_fma_probe(_lib.ptr(out), blocks, threads, iters, stream), "dfb_fp64_fma_probe")
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        flops = 2.0 * 64 * iters * blocks * threads
        best = max(best, flops / (ms * 1e-3) / 1e12)
    return best


def fp64_dgemm_tflops(n: int = 8192, device=None) -> float:
    """cuBLAS DGEMM throughput (FP64 tensor path), best of 3."""
    a = torch.randn((n, n), dtype=torch.float64, device=device or "cuda")
    b = torch.randn_like(a)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n**3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def fp32_fma_tflops(device=None, iters: int = 2048) -> float:
    """Best-of-5 FP32 FMA throughput in TFLOP/s over all SMs (2 flops per FMA): the bound of the
    FP32 recurrences and accumulations of the mixed-precision Rys kernels."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    props = torch.cuda.get_device_properties(dev)
    blocks, threads = props.multi_processor_count * 8, 256
    out = torch.empty(blocks * threads, dtype=torch.float32, device=dev)
    L = _lib.lib()
    stream = int(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(L.dfb_fp32_fma_probe(_lib.ptr(out), blocks, threads, 64, stream), "dfb_fp32_fma_probe")
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check(L.dfb_fp32_fma_probe(_lib.ptr(out), blocks, threads, iters, stream), "dfb_fp32_fma_probe")
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        flops = 2.0 * 64 * iters * blocks * threads
        best = max(best, flops / (ms * 1e-3) / 1e12)
    return best

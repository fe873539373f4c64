"""Split-BF16 tensor-core products (``dfb_tc_gemm``, tcgen05 on sm_100a) for the mixed-precision
DF contractions.

Each FP64 operand is split into bfloat16 terms inside the kernel; the cross products of
order <= 2^-16 accumulate in FP32 in tensor memory over k spans of ``KSPAN`` and the spans are
combined in FP64 (about 1e-7 relative with three terms).  The views are passed as strides, so
the exchange update reads W (naux, nao, nocc) in place with k = (Q, i).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib

KSPAN = 1024  # k per CTA of FP32 accumulation (general products)
# The exchange update accumulates positive diagonal sums, where the tensor cores' FP32
# accumulation bias adds up: measured 2e-6 relative on the diagonal with 1024-long spans.
# 512-long spans halve it at twice the FP64 atomic combinations.
KSPAN_SYRK = 512


def _op(t: torch.Tensor, s_row: int, s_kq: int, s_k1: int, nk1: int, s_batch: int = 0) -> _lib.TcOperand:
    return _lib.TcOperand(_lib.ptr(t), int(s_row), int(s_kq), int(s_k1), int(nk1), int(s_batch))


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


def _check_f64(*ts):
    for t in ts:
        if t.dtype != torch.float64 or not t.is_cuda:
            raise ValueError("split-BF16 products take FP64 CUDA tensors")


def _gemm(M, N, K, batch, A, B, C, ldc, s_cbatch, accumulate, symmetric, nterms, kspan):
    L = _lib.lib()
    rc = L.dfb_tc_gemm(M, N, K, batch, ctypes.byref(A), ctypes.byref(B), _lib.ptr(C), ldc, s_cbatch, int(accumulate),
                       int(symmetric), int(nterms), int(kspan), _stream())
    _lib.check(rc, "dfb_tc_gemm")


def syrk_qblocks(W: torch.Tensor, out: torch.Tensor | None = None, nterms: int = 3,
                 kspan: int = KSPAN_SYRK) -> torch.Tensor:
    """K = sum_Q W_Q W_Q^T for W (naux, nao, nocc) contiguous, i.e. K[m, n] = sum_{Q,i} W[Q,m,i] W[Q,n,i].

    ``out`` (nao, nao) receives the sum added to its current content (zeros when None).
    """
    _check_f64(W)
    naux, nao, nocc = W.shape
    W = W.contiguous()
    K = torch.zeros((nao, nao), dtype=torch.float64, device=W.device) if out is None else out
    if naux * nocc == 0:
        return K
    a = _op(W, nocc, nao * nocc, 1, nocc)
    _gemm(nao, nao, naux * nocc, 1, a, a, K, nao, 0, True, True, nterms, kspan)
    return K


def syrk_rows(A: torch.Tensor, out: torch.Tensor | None = None, nterms: int = 3,
              kspan: int = KSPAN_SYRK) -> torch.Tensor:
    """A A^T for a row-major (m, k) view with unit k stride (rows may be strided)."""
    _check_f64(A)
    m, k = A.shape
    if A.stride(1) != 1:
        A = A.contiguous()
    K = torch.zeros((m, m), dtype=torch.float64, device=A.device) if out is None else out
    if k == 0:
        return K
    a = _op(A, A.stride(0), 0, 1, k)
    _gemm(m, m, k, 1, a, a, K, m, 0, True, True, nterms, kspan)
    return K


def matmul(A: torch.Tensor, B: torch.Tensor, out: torch.Tensor | None = None, nterms: int = 3) -> torch.Tensor:
    """A @ B for FP64 A (m, k) and B (k, n), any strides; one k span when k <= KSPAN, else split-K."""
    _check_f64(A, B)
    m, k = A.shape
    k2, n = B.shape
    if k != k2:
        raise ValueError("inner dimensions differ")
    C = torch.empty((m, n), dtype=torch.float64, device=A.device) if out is None else out
    if C.stride(1) != 1:
        raise ValueError("out must have unit column stride")
    if k == 0:
        C.zero_()
        return C
    a = _op(A, A.stride(0), 0, A.stride(1), k)
    b = _op(B, B.stride(1), 0, B.stride(0), k)  # B^T rows are the columns of B
    if k <= KSPAN:
        _gemm(m, n, k, 1, a, b, C, C.stride(0), 0, False, False, nterms, k)
    else:
        C.zero_()
        _gemm(m, n, k, 1, a, b, C, C.stride(0), 0, True, False, nterms, KSPAN)
    return C


def bmm(A: torch.Tensor, B: torch.Tensor, out: torch.Tensor | None = None, nterms: int = 3) -> torch.Tensor:
    """Batched A @ B: A (m, k) shared or (batch, m, k), B (batch, k, n) -> (batch, m, n); k <= KSPAN."""
    _check_f64(A, B)
    batch, k, n = B.shape
    shared = A.dim() == 2
    m = A.shape[-2]
    if A.shape[-1] != k:
        raise ValueError("inner dimensions differ")
    if k > KSPAN:
        raise ValueError(f"batched products take k <= {KSPAN}")
    C = torch.empty((batch, m, n), dtype=torch.float64, device=B.device) if out is None else out
    if C.stride(2) != 1:
        raise ValueError("out must have unit column stride")
    a = _op(A, A.stride(-2), 0, A.stride(-1), k, 0 if shared else A.stride(0))
    b = _op(B, B.stride(2), 0, B.stride(1), k, B.stride(0))
    _gemm(m, n, k, batch, a, b, C, C.stride(1), C.stride(0), False, False, nterms, k)
    return C


def error_flag(reset: bool = True) -> int:
    """Code recorded by a bounded wait inside the tensor-core kernel that gave up (0 = none)."""
    rc = _lib.lib().dfb_tc_error(int(reset))
    if rc < 0:
        _lib.check(rc, "dfb_tc_error")
    return rc

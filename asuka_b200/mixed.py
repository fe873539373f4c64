"""Split-BF16 products for the mixed-precision DF contractions.

An FP64 matrix is represented as the sum of three BF16 matrices,
``A = A0 + A1 + A2`` with ``A0 = bf16(A)``, ``A1 = bf16(A - A0)``,
``A2 = bf16(A - A0 - A1)`` (24 significant bits).  A product keeps the six
cross terms whose order is at most 2^-16 relative
(A0B0, A0B1, A1B0, A0B2, A1B1, A2B0), each a BF16 tensor-core GEMM with FP32
accumulation; the inner dimension is cut into blocks of ``kblock`` so the
FP32 partial sums stay short, and blocks are summed in FP64.  Accuracy is
about FP32 (relative ~1e-7 per element), which is what the early SCF
iterations need; FP64 iterations finish the SCF.
"""

from __future__ import annotations

import torch

KBLOCK = 512


def split3(A: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    a0 = A.to(torch.bfloat16)
    r = A - a0.to(torch.float64)
    a1 = r.to(torch.bfloat16)
    a2 = (r - a1.to(torch.float64)).to(torch.bfloat16)
    return a0, a1, a2


def _mm32(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return torch.mm(a, b, out_dtype=torch.float32)


def matmul(A: torch.Tensor | None, B: torch.Tensor, kblock: int = KBLOCK,
           a_split: tuple[torch.Tensor, torch.Tensor, torch.Tensor] | None = None) -> torch.Tensor:
    """A @ B for FP64 A (m, k), B (k, n) via six split-BF16 products; FP64 result.

    ``a_split`` = split3(A) computed once by the caller replaces A when the same
    left operand multiplies many right-hand blocks.
    """
    m, k = A.shape if a_split is None else a_split[0].shape
    n = B.shape[1]
    out = torch.zeros((m, n), dtype=torch.float64, device=B.device)
    for k0 in range(0, k, kblock):
        k1 = min(k, k0 + kblock)
        if a_split is None:
            a0, a1, a2 = split3(A[:, k0:k1])
        else:
            a0, a1, a2 = (t[:, k0:k1] for t in a_split)
        b0, b1, b2 = split3(B[k0:k1])
        acc = _mm32(a0, b0).to(torch.float64)
        acc += _mm32(a0, b1) + _mm32(a1, b0)
        acc += _mm32(a0, b2) + _mm32(a1, b1) + _mm32(a2, b0)
        out += acc
    return out


def syrk(A: torch.Tensor, kblock: int = 16384) -> torch.Tensor:
    """A @ A^T for FP64 A (m, k) via split-BF16: per k block A is split once into
    A0 + A1 + A2 and the symmetric product keeps A0A0^T + (A0A1^T + A0A2^T) + sym + A1A1^T
    -- four BF16 GEMMs with FP32 accumulation -- summed in FP64."""
    m, k = A.shape
    out = torch.zeros((m, m), dtype=torch.float64, device=A.device)
    for k0 in range(0, k, kblock):
        k1 = min(k, k0 + kblock)
        a0, a1, a2 = split3(A[:, k0:k1])
        cross = (_mm32(a0, a1.T) + _mm32(a0, a2.T)).to(torch.float64)
        out += _mm32(a0, a0.T).to(torch.float64) + _mm32(a1, a1.T).to(torch.float64) + cross + cross.T
    return out

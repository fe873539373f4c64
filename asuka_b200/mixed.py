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
# Below this output dimension the FP64 DGEMM is faster than the split-BF16 rank-k
# update (four BF16 GEMMs plus the splitting passes; measured on B200: m = 416,
# k = 72960: FP64 0.82 ms, split-BF16 1.24 ms; m = 2336, k = 57440: FP64 17.8 ms,
# split-BF16 11.3 ms), so mixed mode keeps FP64 there.
MIN_DIM = 1024


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


def syrk(A: torch.Tensor, kblock: int = 1024, max_partial: int = 1 << 27) -> torch.Tensor:
    """A @ A^T for FP64 A (m, k) via split-BF16.

    The inner dimension is cut into blocks of ``kblock``; all blocks go through one
    batched BF16 GEMM per cross term (FP32 accumulation inside a block only), so the
    small m x m output still spreads over every SM, and the per-block partial
    products are summed in FP64.  The tensor cores' FP32 accumulation error grows
    about linearly with the block length (measured on B200: 4e-7 relative at 256,
    2e-6 at 1024, 5e-5 for 16384-long blocks); 1024 is the shortest block at which
    the product still beats the FP64 DGEMM for large outputs (m = 2336, k = 57440:
    11.3 ms against 17.8 ms FP64; 29.9 ms at block 256).  Per block, A = A0 + A1 + A2 and the symmetric
    product keeps A0A0^T + (A0A1^T + A0A2^T) + (the same)^T + A1A1^T.  ``max_partial``
    bounds the FP32 partials held at once (blocks x m x m).
    """
    m, k = A.shape
    out = torch.zeros((m, m), dtype=torch.float64, device=A.device)
    nb_max = max(1, max_partial // max(m * m, 1))
    step = kblock * nb_max
    for k0 in range(0, k, step):
        k1 = min(k, k0 + step)
        nb = (k1 - k0) // kblock
        if nb > 0:
            A3 = A[:, k0:k0 + nb * kblock].reshape(m, nb, kblock).permute(1, 0, 2)
            a0, a1, a2 = split3(A3)
            t0 = torch.bmm(a0, a0.transpose(1, 2), out_dtype=torch.float32)
            t1 = torch.bmm(a1, a1.transpose(1, 2), out_dtype=torch.float32)
            c = torch.bmm(a0, a1.transpose(1, 2), out_dtype=torch.float32)
            c += torch.bmm(a0, a2.transpose(1, 2), out_dtype=torch.float32)
            out += t0.sum(0, dtype=torch.float64) + t1.sum(0, dtype=torch.float64)
            cs = c.sum(0, dtype=torch.float64)
            out += cs + cs.T
        r0 = k0 + nb * kblock
        if r0 < k1:
            a0, a1, a2 = split3(A[:, r0:k1])
            cross = (_mm32(a0, a1.T) + _mm32(a0, a2.T)).to(torch.float64)
            out += _mm32(a0, a0.T).to(torch.float64) + _mm32(a1, a1.T).to(torch.float64) + cross + cross.T
    return out

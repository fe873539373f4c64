"""Triangular solves with the metric's Cholesky factor as blocked GEMMs.

The DF step solves with the lower factor L of the aux metric twice per step:
W = L^-1 Y (Y = X Cw, naux x nao*nocc) and Z = L^-T M (M = Cw^T W,
naux x nocc^2).  A single library TRSM call with a few-thousand-row triangle and
tens of thousands of right-hand sides runs far below the FP64 GEMM rate, so the
solve is done by block substitution instead: the diagonal blocks of L are
inverted once (small triangular solves against the identity), and every step of
the substitution is then two FP64 GEMMs -- the update with the rows already
solved, and the product with the inverted diagonal block.  The work is the same
naux^2 * ncol multiply-adds as the TRSM.
"""

from __future__ import annotations

import torch

NB = 256  # rows per diagonal block


INV_BASE = 64  # rows of the diagonal sub-blocks inverted by triangular solves


def diag_block_inverses(L: torch.Tensor, nb: int = NB) -> list[torch.Tensor]:
    """Inverses of the nb x nb diagonal blocks of the lower-triangular L.

    Triangular solves against the identity cost about 0.13 ms per 256-row block on a B200
    whatever their batching, so only the 64-row sub-blocks are inverted that way (one batched
    call); the larger inverses are assembled level by level with batched GEMMs,
    inv([[A, 0], [B, C]]) = [[A^-1, 0], [-C^-1 B A^-1, C^-1]] (0.27 against 1.0 ms for eight
    256-row blocks).  L is padded to whole blocks with the identity."""
    n = L.shape[0]
    base = INV_BASE
    if nb % base or (nb // base) & (nb // base - 1):  # nb must be base * 2^k
        out = []
        for r0 in range(0, n, nb):
            r1 = min(n, r0 + nb)
            eye = torch.eye(r1 - r0, dtype=L.dtype, device=L.device)
            out.append(torch.linalg.solve_triangular(L[r0:r1, r0:r1], eye, upper=False))
        return out
    nbk = (n + nb - 1) // nb
    N = nbk * nb
    Lp = torch.eye(N, dtype=L.dtype, device=L.device)
    Lp[:n, :n] = L
    D = Lp.view(nbk, nb, nbk, nb).diagonal(dim1=0, dim2=2).permute(2, 0, 1)  # (nbk, nb, nb) diagonal blocks
    m = nb // base
    sub = D.reshape(nbk, m, base, m, base).diagonal(dim1=1, dim2=3).permute(0, 3, 1, 2).reshape(nbk * m, base, base)
    eye = torch.eye(base, dtype=L.dtype, device=L.device).expand(nbk * m, base, base)
    inv = torch.linalg.solve_triangular(sub, eye, upper=False)
    s = base
    while s < nb:  # blocks of 2s from the inverses of their two diagonal s-blocks
        q = nb // (2 * s)
        pair = inv.view(nbk, q, 2, s, s)
        Ai, Ci = pair[:, :, 0], pair[:, :, 1]
        big = D.reshape(nbk, q, 2 * s, q, 2 * s).diagonal(dim1=1, dim2=3).permute(0, 3, 1, 2)
        nxt = torch.zeros((nbk, q, 2 * s, 2 * s), dtype=L.dtype, device=L.device)
        nxt[:, :, :s, :s] = Ai
        nxt[:, :, s:, s:] = Ci
        nxt[:, :, s:, :s] = -(Ci @ (big[:, :, s:, :s] @ Ai))
        inv = nxt.reshape(nbk * q, 2 * s, 2 * s)
        s *= 2
    return [inv[i, : min(n, r0 + nb) - r0, : min(n, r0 + nb) - r0] for i, r0 in enumerate(range(0, n, nb))]


def solve_lower(L: torch.Tensor, Y: torch.Tensor, inv: list[torch.Tensor] | None = None, nb: int = NB,
                out: torch.Tensor | None = None) -> torch.Tensor:
    """W = L^-1 Y by forward block substitution; ``out`` may be Y itself (in place)."""
    n = L.shape[0]
    if inv is None:
        inv = diag_block_inverses(L, nb)
    W = out if out is not None else torch.empty_like(Y)
    for i, r0 in enumerate(range(0, n, nb)):
        r1 = min(n, r0 + nb)
        rhs = Y[r0:r1].clone() if r0 == 0 else torch.addmm(Y[r0:r1], L[r0:r1, :r0], W[:r0], alpha=-1.0)
        torch.mm(inv[i], rhs, out=W[r0:r1])
    return W


def solve_lower_T(L: torch.Tensor, M: torch.Tensor, inv: list[torch.Tensor] | None = None, nb: int = NB,
                  out: torch.Tensor | None = None) -> torch.Tensor:
    """Z = L^-T M by backward block substitution; ``out`` may be M itself (in place)."""
    n = L.shape[0]
    if inv is None:
        inv = diag_block_inverses(L, nb)
    Z = out if out is not None else torch.empty_like(M)
    starts = list(range(0, n, nb))
    for i in range(len(starts) - 1, -1, -1):
        r0 = starts[i]
        r1 = min(n, r0 + nb)
        rhs = M[r0:r1].clone() if r1 == n else torch.addmm(M[r0:r1], L[r1:, r0:r1].T, Z[r1:], alpha=-1.0)
        torch.mm(inv[i].T, rhs, out=Z[r0:r1])
    return Z


def solve_lower_right_T(L: torch.Tensor, X: torch.Tensor, inv: list[torch.Tensor] | None = None, nb: int = NB,
                        out: torch.Tensor | None = None) -> torch.Tensor:
    """B = X L^-T (X is (m, n), the solve runs over its columns); ``out`` may be X itself."""
    n = L.shape[0]
    if inv is None:
        inv = diag_block_inverses(L, nb)
    B = out if out is not None else torch.empty_like(X)
    for i, r0 in enumerate(range(0, n, nb)):
        r1 = min(n, r0 + nb)
        rhs = X[:, r0:r1] if r0 == 0 else torch.addmm(X[:, r0:r1], B[:, :r0], L[r0:r1, :r0].T, alpha=-1.0)
        B[:, r0:r1] = rhs @ inv[i].T
    return B

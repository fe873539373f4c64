"""Streamed (direct) DF J/K: the 3c integrals are recomputed per aux block, B is never stored.

Mirrors the reference's streamed seam (``asuka/hf/df_jk_streamed.py:20-420``):
``make_streamed_df_jk_context`` (:59-122), ``df_JK_streamed`` (:167-325) for one
occupied set and ``df_JKs_streamed`` (:328-) for several occupied sets sharing one
density for J (UHF alpha/beta), with the same argument meaning.  Per call:

* pass 1, per aux block b: X_b -> rho_b = <X_b, D> and Y_b = X_b C_j sqrt(occ_j)
  for every occupied set j (one integral evaluation serves all sets);
* d = V^-1 rho, W_j = L^-1 Y_j (block substitution), K_j = sum_Q W_jQ W_jQ^T;
* pass 2: J = sum_P d_P X_P with the blocks recomputed.

``precision='mixed'`` evaluates the integrals with FP32 recurrence tables and
accumulators (``DFB_PREC_MIXED``) and the exchange update as a split-BF16
tensor-core GEMM; the SCF finishes with FP64 iterations.

Outputs are symmetric FP64 device tensors.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import torch

from . import linalg as _la
from . import tc as _tc
from .df import DFEngine, cholesky_metric, get_engine


@dataclass
class StreamedDFJKContext:
    ao_basis: Any
    aux_basis: Any
    engine: DFEngine
    L_metric: torch.Tensor
    aux_blocks: list  # (p0, p1, block handle) aligned to aux shells
    aux_block_naux: int
    L_inv_blocks: list


def make_streamed_df_jk_context(ao_basis, aux_basis, *, aux_block_naux: int = 256, engine: DFEngine | None = None,
                                L_metric: torch.Tensor | None = None, profile: dict | None = None,
                                **_unused) -> StreamedDFJKContext:
    """Metric factor and aux-shell blocks for streamed DF J/K (``df_jk_streamed.py:59-122``).

    Backend selection keywords of the reference (``backend``, ``threads``, ``mode``) are
    accepted and ignored: there is one device path.  ``ao_rep`` other than 'cart' is not
    implemented.
    """
    if str(_unused.get("ao_rep", "cart")) != "cart":
        raise NotImplementedError("only Cartesian AOs (ao_rep='cart') are implemented")
    eng = engine if engine is not None else get_engine(ao_basis, aux_basis)
    L = L_metric if L_metric is not None else cholesky_metric(eng.metric())
    blocks = eng.aux_blocks(int(aux_block_naux))
    return StreamedDFJKContext(ao_basis, aux_basis, eng, L, blocks, int(aux_block_naux),
                               _la.diag_block_inverses(L))


def _cw(C_occ, occ_vals) -> torch.Tensor:
    C = torch.as_tensor(C_occ, dtype=torch.float64)
    occ = torch.as_tensor(occ_vals, dtype=torch.float64, device=C.device)
    if C.ndim != 2 or occ.ndim != 1 or occ.shape[0] != C.shape[1]:
        raise ValueError("C_occ must be (nao, nocc) and occ_vals (nocc,)")
    if bool((occ < 0).any()):
        raise ValueError("occupations must be non-negative")
    return (C * occ.sqrt()).contiguous()


def df_JKs_streamed(ctx: StreamedDFJKContext, D, C_occ_list: list, occ_vals_list: list, *, k_q_block: int = 128,
                    precision: str = "fp64", work: dict | None = None, profile: dict | None = None, **_unused):
    """J from D and one K per occupied set, with one streamed integral evaluation per pass."""
    if len(C_occ_list) != len(occ_vals_list):
        raise ValueError("C_occ_list and occ_vals_list must have the same length")
    eng = ctx.engine
    nao, naux = eng.nao, eng.naux
    dev = eng.device
    D = torch.as_tensor(D, dtype=torch.float64, device=dev)
    if D.shape != (nao, nao):
        raise ValueError(f"D must be ({nao}, {nao})")
    Cws = [_cw(C, o).to(dev) for C, o in zip(C_occ_list, occ_vals_list)]
    noccs = [int(c.shape[1]) for c in Cws]
    rho = torch.empty(naux, dtype=torch.float64, device=dev)
    Ys = [torch.empty((naux, nao * n), dtype=torch.float64, device=dev) for n in noccs]
    bmax = max(p1 - p0 for p0, p1, _ in ctx.aux_blocks)
    Xbuf = torch.zeros((bmax, nao, nao), dtype=torch.float64, device=dev)
    Df = D.reshape(-1)
    for p0, p1, blk in ctx.aux_blocks:
        Xb = eng.int3c_block(blk, p0, p1, out=Xbuf[: p1 - p0], dropped_zero=True, precision=precision)
        torch.mv(Xb.view(p1 - p0, -1), Df, out=rho[p0:p1])
        for Cw, Y, n in zip(Cws, Ys, noccs):
            if n:
                torch.matmul(Xb.view(-1, nao), Cw, out=Y[p0:p1].view(-1, n))
    L = ctx.L_metric
    d = _la.solve_lower_T(L, _la.solve_lower(L, rho.view(-1, 1), ctx.L_inv_blocks), ctx.L_inv_blocks).view(-1)
    Ks = []
    qb = max(1, int(k_q_block))
    for Y, n in zip(Ys, noccs):
        K = torch.zeros((nao, nao), dtype=torch.float64, device=dev)
        if n:
            _la.solve_lower(L, Y, ctx.L_inv_blocks, out=Y)
            W3 = Y.view(naux, nao, n)
            for q0 in range(0, naux, qb):
                if precision == "fp64":
                    Wc = W3[q0:q0 + qb].permute(1, 0, 2).reshape(nao, -1)
                    K.addmm_(Wc, Wc.T)
                else:
                    _tc.syrk_qblocks(W3[q0:q0 + qb], out=K)
        Ks.append(0.5 * (K + K.T))
    del Ys
    J = torch.zeros((nao, nao), dtype=torch.float64, device=dev)
    Jf = J.view(-1)
    for p0, p1, blk in ctx.aux_blocks:
        if len(ctx.aux_blocks) == 1:
            Xb = Xbuf[: p1 - p0]  # still holds the only block
        else:
            Xb = eng.int3c_block(blk, p0, p1, out=Xbuf[: p1 - p0], dropped_zero=True, precision=precision)
        Jf.addmv_(Xb.view(p1 - p0, -1).T, d[p0:p1])
    return 0.5 * (J + J.T), Ks


def df_JK_streamed(ctx: StreamedDFJKContext, D, C_occ, occ_vals, *, k_q_block: int = 128, precision: str = "fp64",
                   work: dict | None = None, profile: dict | None = None, **_unused):
    """(J, K) for one occupied set (``df_jk_streamed.py:167-325``)."""
    J, Ks = df_JKs_streamed(ctx, D, [C_occ], [occ_vals], k_q_block=k_q_block, precision=precision)
    return J, Ks[0]

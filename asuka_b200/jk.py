"""DF Coulomb/exchange contractions on the device.

Mirrors the reference's J/K seam (``asuka/hf/cuda/ext/src/hf_df_jk_cuda_ext.cpp:198-1150``
``DFJKWorkspace`` and ``asuka/hf/df_jk.py:424,528,1040``):

    J = sum_Q B_Q (B_Q . D)          K = sum_Q (B_Q Cw)(B_Q Cw)^T,  Cw = C_occ sqrt(occ)

with B_Q in the 'Qmn' layout (naux, nao, nao).  Outputs are zeroed by the
callee and returned fully symmetric, as the reference's workspace does.

Precision modes:

* ``'fp64'``  -- FP64 GEMMs (cuBLAS DGEMM through torch);
* ``'mixed'`` -- the exchange rank-k update K = U U^T (the compute-bound
  step) runs as split-BF16 products (each FP64 operand split into three BF16
  terms, the leading cross products accumulated in FP32 per block and summed
  in FP64), see ``asuka_b200.mixed``.  The half-transform U = B Cw and J are
  HBM-bound (one pass over B) and stay FP64.
"""

from __future__ import annotations

import torch

from . import mixed as _mixed


def _sym(A: torch.Tensor) -> torch.Tensor:
    return 0.5 * (A + A.T)


def df_J_from_BQ_D(BQ: torch.Tensor, D: torch.Tensor) -> torch.Tensor:
    naux = BQ.shape[0]
    B2 = BQ.reshape(naux, -1)
    rho = B2 @ D.reshape(-1)
    return _sym((rho @ B2).reshape(D.shape))


def df_K_from_BQ_Cw(BQ: torch.Tensor, Cw: torch.Tensor, q_block: int = 256, precision: str = "fp64") -> torch.Tensor:
    naux, nao, _ = BQ.shape
    nocc = Cw.shape[1]
    K = torch.zeros((nao, nao), dtype=torch.float64, device=BQ.device)
    if nocc == 0:
        return K
    for q0 in range(0, naux, q_block):
        q1 = min(naux, q0 + q_block)
        blk = BQ[q0:q1]
        if precision == "fp64":
            U = torch.matmul(blk.reshape(-1, nao), Cw).reshape(q1 - q0, nao, nocc)
            U2 = U.permute(1, 0, 2).reshape(nao, -1)
            K += U2 @ U2.T
        else:
            U = torch.matmul(blk.reshape(-1, nao), Cw).reshape(q1 - q0, nao, nocc)
            U2 = U.permute(1, 0, 2).reshape(nao, -1)
            K += _mixed.syrk(U2)
    return _sym(K)


def df_JK_from_BQ(BQ: torch.Tensor, Cw: torch.Tensor, D: torch.Tensor, q_block: int = 256,
                  precision: str = "fp64") -> tuple[torch.Tensor, torch.Tensor]:
    return df_J_from_BQ_D(BQ, D), df_K_from_BQ_Cw(BQ, Cw, q_block=q_block, precision=precision)


def density_from_Cw(Cw: torch.Tensor) -> torch.Tensor:
    return _sym(Cw @ Cw.T)


class DFJKWorkspace:
    """Reference-shaped J/K workspace: preallocated outputs, zeroed and symmetric on return.

    ``math_mode`` follows the reference's meaning loosely: -1 (default) keeps the
    workspace's own precision; 0 forces FP64; 8 (the reference's FP64-emulation
    mode id) selects the mixed split-BF16 path.
    """

    def __init__(self, precision: str = "fp64"):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self._released = False

    def _prec(self, math_mode: int) -> str:
        if self._released:
            raise RuntimeError("DFJKWorkspace used after release()")
        if math_mode == 0:
            return "fp64"
        if math_mode == 8:
            return "mixed"
        return self.precision

    @staticmethod
    def _check(*ts):
        for t in ts:
            if t.dtype != torch.float64:
                raise ValueError("inputs must be float64")
            if not t.is_cuda:
                raise ValueError("inputs must be CUDA tensors")
            if not t.is_contiguous():
                raise ValueError("inputs must be C-contiguous")

    def jk_from_bq_cw(self, BQ, Cw, D, out_J, out_K, *, q_block: int = 256, stream=None, math_mode: int = -1,
                      sync: bool = True):
        self._check(BQ, Cw, D, out_J, out_K)
        J, K = df_JK_from_BQ(BQ, Cw, D, q_block=q_block, precision=self._prec(math_mode))
        out_J.copy_(J)
        out_K.copy_(K)
        if sync:
            torch.cuda.current_stream().synchronize()
        return out_J, out_K

    def k_from_bq_cw(self, BQ, Cw, out_K, *, q_block: int = 256, stream=None, math_mode: int = -1,
                     sync: bool = True):
        self._check(BQ, Cw, out_K)
        out_K.copy_(df_K_from_BQ_Cw(BQ, Cw, q_block=q_block, precision=self._prec(math_mode)))
        if sync:
            torch.cuda.current_stream().synchronize()
        return out_K

    def density_syrk(self, Cw, out, *, stream=None, math_mode: int = -1, sync: bool = True):
        self._check(Cw, out)
        out.copy_(density_from_Cw(Cw))
        if sync:
            torch.cuda.current_stream().synchronize()
        return out

    def release(self) -> None:
        self._released = True

"""Reusable DF gradient contraction context (``asuka/integrals/df_grad_context.py:609-3771``).

``DFGradContractionContext.build(ao_basis, aux_basis, atom_coords_bohr=..., backend='cuda')``
sets up the device state once (bases with their shell->atom maps, pair tables, class
lists and the metric factor L), so that many gradients at the same geometry reuse it.
The CASSCF / MRCI / CASPT2 consumers contract several dE/dB terms this way. The
contractions accept the layouts the reference hands over:

* ``contract(B_ao, bar_L_ao)``: B in mnQ (nao, nao, naux) with dE/dB (naux, nao, nao), or
  both packed lower-triangle Qp (naux, ntri) with p = m(m+1)/2 + n (m >= n). Qp is the
  layout in which the DF SCF returns ``df_B``; both tensors hold the symmetric
  full-layout values at their packed positions (``asuka/integrals/df_adjoint.py:238-321``).
  The packed route never forms (naux, nao, nao): the adjoints are computed in packed form
  and the derivative integrals run one aux-shell block at a time;
* ``contract_sph(B_sph, bar_L_sph)``: spherical-AO factors. The adjoint is formed in the
  spherical basis and taken to the Cartesian integrals through the solid-harmonic
  transform, dE/dX_cart = T (dE/dX_sph) T^T;
* ``contract_fused_terms(B_ao, bar_L_terms)``: the sum of several dE/dB terms with one
  pass of the derivative integrals.

Results are (natm, 3) NumPy arrays; ``contract_device*`` return device tensors.
"""

from __future__ import annotations

from typing import Any, Iterable

import numpy as np
import torch

from .df import DFEngine, cholesky_metric
from .grad import whitened_adjoints, whitened_adjoints_qp


def _nao_from_ntri(ntri: int) -> int:
    nao = int((np.sqrt(8 * ntri + 1) - 1) // 2)
    if nao * (nao + 1) // 2 != ntri:
        raise ValueError(f"ntri={ntri} is not a triangle number")
    return nao


class DFGradContractionContext:
    def __init__(self, engine: DFEngine, L: torch.Tensor, natm: int):
        self.engine = engine
        self.L_metric = L
        self.backend = "cuda"
        self.nao, self.naux = engine.nao, engine.naux
        self.natm = max(engine.natm, natm)
        self.last_peak_block_elems = 0  # largest unpacked (q, nao, nao) block of the last packed contraction

    @classmethod
    def build(cls, ao_basis: Any, aux_basis: Any, *, atom_coords_bohr: np.ndarray, backend: str = "cuda",
              df_threads: int = 0, L_chol: Any | None = None) -> "DFGradContractionContext":
        if str(backend).strip().lower() not in ("cuda", "gpu"):
            raise ValueError("this engine runs on the GPU only (backend='cuda')")
        R = np.asarray(atom_coords_bohr, dtype=np.float64)
        if R.ndim != 2 or R.shape[1] != 3 or R.shape[0] == 0:
            raise ValueError("atom_coords_bohr must have shape (natm, 3) with natm > 0")
        eng = DFEngine(ao_basis, aux_basis, atom_coords_bohr=R)
        L = (torch.as_tensor(L_chol, dtype=torch.float64, device=eng.device) if L_chol is not None
             else cholesky_metric(eng.metric()))
        return cls(eng, L, R.shape[0])

    def ensure_cuda(self) -> None:
        """The device state is built eagerly; kept for the reference's call sites."""

    def release_cuda(self) -> None:
        self.engine = None
        self.L_metric = None

    # ------------------------------------------------------------ layouts
    def _mnQ_and_bar(self, B: torch.Tensor, barL: torch.Tensor):
        if B.ndim != 3 or B.shape[0] != B.shape[1]:
            raise ValueError("B_ao must have shape (nao, nao, naux)")
        if tuple(B.shape) != (self.nao, self.nao, self.naux):
            raise ValueError("B_ao shape mismatch with context")
        if tuple(barL.shape) != (self.naux, self.nao, self.nao):
            raise ValueError("bar_L_ao must have shape (naux, nao, nao)")
        return B.contiguous(), barL.contiguous()

    def _contract_adjoints(self, bar_X: torch.Tensor, bar_V: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
        grad = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.engine.device)
        self.engine.deriv3c(bar_X, grad, layout="Qmn", precision=precision)
        self.engine.deriv2c(bar_V, grad, precision=precision)
        return grad

    def _contract_packed(self, B_Qp: torch.Tensor, barL_Qp: torch.Tensor, aux_block_naux: int,
                         precision: str = "fp64") -> torch.Tensor:
        """Packed-Qp route: adjoints in packed form, then the derivative integrals one aux-shell
        block at a time with that block's adjoint unpacked (one (q, nao, nao) block alive)."""
        nao = self.nao
        bar_X, bar_V = whitened_adjoints_qp(B_Qp, barL_Qp, self.L_metric, nao)
        eng = self.engine
        dev = eng.device
        grad = torch.zeros((self.natm, 3), dtype=torch.float64, device=dev)
        i, j = torch.tril_indices(nao, nao, device=dev)
        blocks = eng.aux_blocks(max(1, int(aux_block_naux)))
        qmax = max(p1 - p0 for p0, p1, _ in blocks)
        buf = torch.empty((qmax, nao, nao), dtype=torch.float64, device=dev)
        self.last_peak_block_elems = int(buf.numel())
        for p0, p1, blk in blocks:
            G = buf[: p1 - p0]
            G[:, i, j] = bar_X[p0:p1]
            G[:, j, i] = bar_X[p0:p1]
            eng.deriv3c_block(blk, G, grad, precision=precision)
        eng.deriv2c(bar_V, grad, precision=precision)
        return grad

    # ------------------------------------------------------------ contractions
    def contract_device(self, *, B_ao: Any, bar_L_ao: Any, aux_block_naux: int = 128,
                        precision: str = "fp64") -> torch.Tensor:
        """(natm, 3) device gradient; ``precision='mixed'`` runs the derivative integrals with FP32
        recurrences and accumulators (``DFB_PREC_MIXED``); the adjoints stay FP64."""
        dev = self.engine.device
        B = torch.as_tensor(B_ao, dtype=torch.float64, device=dev)
        barL = torch.as_tensor(bar_L_ao, dtype=torch.float64, device=dev)
        if B.ndim == 2 and barL.ndim == 2:
            naux, ntri = map(int, B.shape)
            if naux != self.naux or tuple(barL.shape) != (naux, ntri):
                raise ValueError("packed-Qp B_ao and bar_L_ao must both have shape (naux, ntri)")
            if _nao_from_ntri(ntri) != self.nao:
                raise ValueError("B_ao shape mismatch with context nao")
            return self._contract_packed(B.contiguous(), barL.contiguous(), aux_block_naux, precision)
        B, barL = self._mnQ_and_bar(B, barL)
        return self._contract_adjoints(*whitened_adjoints(B, barL, self.L_metric), precision=precision)

    def contract(self, *, B_ao: Any, bar_L_ao: Any, aux_block_naux: int = 128) -> np.ndarray:
        return self.contract_device(B_ao=B_ao, bar_L_ao=bar_L_ao, aux_block_naux=aux_block_naux).cpu().numpy()

    def contract_device_fused_terms(self, *, B_ao: Any, bar_L_terms: Iterable[Any], precision: str = "fp64"):
        total = None
        for t in bar_L_terms:
            tt = torch.as_tensor(t, dtype=torch.float64, device=self.engine.device)
            total = tt.clone() if total is None else total.add_(tt)
        if total is None:
            return torch.zeros((self.natm, 3), dtype=torch.float64, device=self.engine.device)
        return self.contract_device(B_ao=B_ao, bar_L_ao=total, precision=precision)

    def contract_fused_terms(self, *, B_ao: Any, bar_L_terms: Iterable[Any], precision: str = "fp64") -> np.ndarray:
        return self.contract_device_fused_terms(B_ao=B_ao, bar_L_terms=bar_L_terms, precision=precision).cpu().numpy()

    def contract_device_sph(self, *, B_sph: Any, bar_L_sph: Any, T_c2s: Any | None = None) -> torch.Tensor:
        from .sph import cart2sph_ao_matrix

        dev = self.engine.device
        T = (torch.as_tensor(T_c2s, dtype=torch.float64, device=dev) if T_c2s is not None
             else cart2sph_ao_matrix(self.engine.ao.shell_l, dev))
        B = torch.as_tensor(B_sph, dtype=torch.float64, device=dev).contiguous()
        barL = torch.as_tensor(bar_L_sph, dtype=torch.float64, device=dev).contiguous()
        ns = T.shape[1]
        if tuple(B.shape) != (ns, ns, self.naux) or tuple(barL.shape) != (self.naux, ns, ns):
            raise ValueError("B_sph must be (nao_sph, nao_sph, naux) and bar_L_sph (naux, nao_sph, nao_sph)")
        bar_Xs, bar_V = whitened_adjoints(B, barL, self.L_metric)
        bar_X = torch.matmul(T, torch.matmul(bar_Xs, T.T))  # dE/dX_cart = T dE/dX_sph T^T
        return self._contract_adjoints(bar_X.contiguous(), bar_V)

    def contract_sph(self, *, B_sph: Any, bar_L_sph: Any, T_c2s: Any | None = None) -> np.ndarray:
        return self.contract_device_sph(B_sph=B_sph, bar_L_sph=bar_L_sph, T_c2s=T_c2s).cpu().numpy()

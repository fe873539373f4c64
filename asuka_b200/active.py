"""Active-space DF factors L_pq^Q for the CASSCF consumer of the DF tensor.

Mirrors the reference's seam (``asuka/cueri/df.py:1086-1210,1911-2060``):

* ``active_Lfull_from_B(B, C_active)``: L_full[p*norb + q, Q] = sum_mn C_mp C_nq B_mn^Q
  from the whitened factors in mnQ (nao, nao, naux) layout (``df.py:1086``), also
  accepting this engine's Qmn (naux, nao, nao) layout via ``layout='Qmn'``;
* ``active_Lfull_from_B_Qp(B_Qp, C_active, aux_block_naux)``: the same from the
  packed lower-triangle layout (naux, ntri), unpacked per aux block (``df.py:1128``);
* ``active_Lfull_from_cached_B_whitened``: dispatch on the cached layout (``df.py:1185``);
* ``active_Lfull_streamed_basis(ao_basis, aux_basis, C_active)``: the factors without
  storing X or B (``df.py:1911``): per aux block Y^T_b = C^T X_b C, then L_full^T = L^-1 Y^T.

Every transform is two batched FP64 GEMMs per aux block on the device.
"""

from __future__ import annotations

import torch

from . import linalg as _la
from .df import cholesky_metric, get_engine


def _c_active(C_active, nao: int, device) -> torch.Tensor:
    C = torch.as_tensor(C_active, dtype=torch.float64, device=device)
    if C.ndim != 2:
        raise ValueError("C_active must have shape (nao, norb)")
    if int(C.shape[0]) != nao:
        raise ValueError(f"C_active has nao={int(C.shape[0])}, but B implies nao={nao}")
    return C.contiguous()


def _transform_Qmn(BQ: torch.Tensor, C: torch.Tensor) -> torch.Tensor:
    """(q, nao, nao) -> (q, norb, norb): C^T B_Q C."""
    return torch.matmul(C.T, torch.matmul(BQ, C))


def active_Lfull_from_B(B, C_active, *, layout: str = "mnQ") -> torch.Tensor:
    """L_full (norb*norb, naux) from whitened factors in mnQ (reference) or Qmn layout."""
    B = torch.as_tensor(B, dtype=torch.float64)
    if B.ndim != 3:
        raise ValueError("B must have shape (nao, nao, naux)" if layout == "mnQ" else "B must be (naux, nao, nao)")
    if layout == "mnQ":
        nao0, nao1, naux = map(int, B.shape)
        if nao0 != nao1:
            raise ValueError("B must have shape (nao, nao, naux)")
        C = _c_active(C_active, nao0, B.device)
        norb = int(C.shape[1])
        tmp = (C.T @ B.reshape(nao0, nao0 * naux)).view(norb, nao0, naux)   # tmp[p, n, Q]
        out = torch.matmul(tmp.permute(0, 2, 1), C)                           # (norb, naux, norb)
        return out.permute(0, 2, 1).reshape(norb * norb, naux).contiguous()
    if layout == "Qmn":
        naux, nao0, nao1 = map(int, B.shape)
        if nao0 != nao1:
            raise ValueError("B must have shape (naux, nao, nao)")
        C = _c_active(C_active, nao0, B.device)
        norb = int(C.shape[1])
        return _transform_Qmn(B, C).reshape(naux, norb * norb).T.contiguous()
    raise ValueError("layout must be 'mnQ' or 'Qmn'")


def _tri_index(nao: int, device) -> torch.Tensor:
    i = torch.arange(nao, device=device)
    hi = torch.maximum(i[:, None], i[None, :])
    lo = torch.minimum(i[:, None], i[None, :])
    return (hi * (hi + 1) // 2 + lo).reshape(-1)


def active_Lfull_from_B_Qp(B_Qp, C_active, *, aux_block_naux: int = 64) -> torch.Tensor:
    """L_full from packed lower-triangle factors (naux, ntri), p = m(m+1)/2 + n with m >= n."""
    Bqp = torch.as_tensor(B_Qp, dtype=torch.float64)
    if Bqp.ndim != 2:
        raise ValueError("B_Qp must have shape (naux, ntri)")
    C = torch.as_tensor(C_active, dtype=torch.float64, device=Bqp.device)
    if C.ndim != 2:
        raise ValueError("C_active must have shape (nao, norb)")
    naux, ntri = map(int, Bqp.shape)
    nao, norb = map(int, C.shape)
    if ntri != nao * (nao + 1) // 2:
        raise ValueError(f"B_Qp has ntri={ntri}, expected {nao * (nao + 1) // 2} for C_active nao={nao}")
    C = C.contiguous()
    idx = _tri_index(nao, Bqp.device)
    qb = max(1, min(naux, int(aux_block_naux) if int(aux_block_naux) > 0 else 64))
    out = torch.empty((norb * norb, naux), dtype=torch.float64, device=Bqp.device)
    for q0 in range(0, naux, qb):
        q1 = min(naux, q0 + qb)
        blk = Bqp[q0:q1].index_select(1, idx).view(q1 - q0, nao, nao)
        out[:, q0:q1] = _transform_Qmn(blk, C).reshape(q1 - q0, norb * norb).T
    return out


def active_Lfull_from_cached_B_whitened(B_whitened, C_active) -> torch.Tensor:
    """Dispatch on the cached layout: mnQ (nao, nao, naux) or packed Qp (naux, ntri)."""
    B = torch.as_tensor(B_whitened)
    if B.ndim == 3:
        return active_Lfull_from_B(B, C_active)
    if B.ndim == 2:
        return active_Lfull_from_B_Qp(B, C_active)
    raise ValueError("cached B_whitened must be mnQ (nao,nao,naux) or packed Qp (naux,ntri)")


def active_Lfull_streamed_basis(ao_basis, aux_basis, C_active, *, aux_block_naux: int = 256, out=None,
                                profile: dict | None = None, **_unused) -> torch.Tensor:
    """L_full (norb*norb, naux) without storing X or B: the 3c integrals go through one
    aux-block buffer, Y^T[P, pq] = sum_mn C_mp C_nq X_mn,P, then L_full^T = L^-1 Y^T."""
    if str(_unused.get("ao_rep", "cart")) != "cart":
        raise NotImplementedError("only Cartesian AOs (ao_rep='cart') are implemented")
    eng = get_engine(ao_basis, aux_basis)
    nao, naux = eng.nao, eng.naux
    C = _c_active(C_active, nao, eng.device)
    norb = int(C.shape[1])
    L = cholesky_metric(eng.metric())
    blocks = eng.aux_blocks(int(aux_block_naux))
    bmax = max(p1 - p0 for p0, p1, _ in blocks)
    Xbuf = torch.zeros((bmax, nao, nao), dtype=torch.float64, device=eng.device)
    YT = torch.empty((naux, norb * norb), dtype=torch.float64, device=eng.device)
    for p0, p1, blk in blocks:
        Xb = eng.int3c_block(blk, p0, p1, out=Xbuf[: p1 - p0], dropped_zero=True)
        YT[p0:p1] = _transform_Qmn(Xb, C).reshape(p1 - p0, norb * norb)
    _la.solve_lower(L, YT, out=YT)
    L_full = YT.T
    if out is None:
        return L_full.contiguous()
    if out.shape != (norb * norb, naux) or out.dtype != torch.float64:
        raise ValueError(f"out must be float64 with shape ({norb * norb}, {naux})")
    out.copy_(L_full)
    return out

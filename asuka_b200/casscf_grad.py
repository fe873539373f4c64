"""Adjoint of the DF-CASSCF two-electron energy with respect to the whitened factors B.

The DF-CASSCF nuclear gradient contracts ``bar_L[Q, mu, nu] = dE_2e / dB[mu, nu, Q]`` with
the derivative integrals through the whitened-factor route of
``asuka_b200.grad.compute_df_gradient_contributions_analytic_packed_bases`` or
``asuka_b200.grad_context.DFGradContractionContext``.  This module builds that adjoint the way
the reference's ``_build_bar_L_casscf_df`` / ``_build_bar_L_casscf_df_qp``
(``asuka/mcscf/nuc_grad_df.py:2387-2600``) defines it, on the device:

with D_w = D_act + D_core / 2, rho_Q = <B_Q, D_core>, sigma_Q = <B_Q, D_w>,
L_act[u, v, Q] = C_act^T B_Q C_act and M_Q = sum_{xy} dm2[uv, xy] L_act[x, y, Q]
(dm2 symmetrised over the pair exchange),

    bar_L[Q] = sigma_Q D_core + rho_Q D_w                      (mean-field Coulomb)
             - 1/2 (D_core B_Q D_w + D_w B_Q D_core)           (mean-field exchange)
             + C_act M_Q C_act^T                                 (active-active 2-RDM)

i.e. the derivative of tr(D_w (J(D_core) - K(D_core)/2)) + 1/2 sum dm2 (uv|xy) with the DF
integrals (uv|xy) = sum_Q L_uvQ L_xyQ.  B may be given as mnQ (nao, nao, naux), Qmn
(naux, nao, nao) or packed Qp (naux, ntri); the result comes back in the same layout, and the
packed path works one aux block at a time (one (q, nao, nao) block alive).
"""

from __future__ import annotations

import torch


def _f64(x, device) -> torch.Tensor:
    return torch.as_tensor(x, dtype=torch.float64, device=device)


def _tri(nao: int, device):
    return torch.tril_indices(nao, nao, device=device)


def _unpack_block(B_Qp: torch.Tensor, nao: int, q0: int, q1: int, ij) -> torch.Tensor:
    i, j = ij
    out = torch.empty((q1 - q0, nao, nao), dtype=B_Qp.dtype, device=B_Qp.device)
    out[:, i, j] = B_Qp[q0:q1]
    out[:, j, i] = B_Qp[q0:q1]
    return out


def _bar_block(BQ: torch.Tensor, D_core: torch.Tensor, D_w: torch.Tensor, C_act: torch.Tensor,
               dm2_flat: torch.Tensor) -> torch.Tensor:
    """bar_L for one block of B_Q (q, nao, nao) (symmetric slices)."""
    q, nao, _ = BQ.shape
    ncas = C_act.shape[1]
    rho = torch.einsum("qmn,mn->q", BQ, D_core)
    sigma = torch.einsum("qmn,mn->q", BQ, D_w)
    bar = sigma.view(q, 1, 1) * D_core + rho.view(q, 1, 1) * D_w
    t1 = torch.matmul(D_core, torch.matmul(BQ, D_w))
    bar -= 0.5 * (t1 + t1.transpose(1, 2))
    L = torch.matmul(C_act.T, torch.matmul(BQ, C_act)).reshape(q, ncas * ncas)  # (q, uv)
    M = (L @ dm2_flat.T).view(q, ncas, ncas)
    bar += torch.matmul(C_act, torch.matmul(M, C_act.T))
    return bar


def build_bar_L_casscf_df(B, *, D_core_ao, D_act_ao, C_act, dm2_act, layout: str | None = None,
                          qblock: int = 128) -> torch.Tensor:
    """bar_L = dE_2e/dB for DF-CASSCF (``asuka/mcscf/nuc_grad_df.py:2387-2600``).

    ``layout``: 'mnQ' (default for 3-D B, the reference's layout), 'Qmn', or 'Qp' (implied by a
    2-D B).  Returns bar_L as (naux, nao, nao) for 3-D B, (naux, ntri) for packed B.
    """
    B = torch.as_tensor(B, dtype=torch.float64)
    if not B.is_cuda:
        B = B.cuda()
    dev = B.device
    D_core = _f64(D_core_ao, dev)
    D_act = _f64(D_act_ao, dev)
    C = _f64(C_act, dev).contiguous()
    nao = D_core.shape[0]
    if D_core.shape != (nao, nao) or D_act.shape != (nao, nao):
        raise ValueError("D_core_ao and D_act_ao must be (nao, nao)")
    if C.ndim != 2 or C.shape[0] != nao or C.shape[1] == 0:
        raise ValueError("C_act must be (nao, ncas) with ncas > 0")
    ncas = C.shape[1]
    dm2 = _f64(dm2_act, dev)
    if dm2.shape != (ncas, ncas, ncas, ncas):
        raise ValueError("dm2_act must be (ncas, ncas, ncas, ncas)")
    dm2_flat = dm2.reshape(ncas * ncas, ncas * ncas)
    dm2_flat = 0.5 * (dm2_flat + dm2_flat.T)
    D_w = D_act + 0.5 * D_core
    qb = max(1, int(qblock))
    if B.dim() == 2:
        if layout not in (None, "Qp"):
            raise ValueError("a 2-D B is the packed Qp layout")
        naux, ntri = B.shape
        if ntri != nao * (nao + 1) // 2:
            raise ValueError("B_Qp must have ntri = nao*(nao+1)/2")
        ij = _tri(nao, dev)
        out = torch.empty((naux, ntri), dtype=torch.float64, device=dev)
        for q0 in range(0, naux, qb):
            q1 = min(naux, q0 + qb)
            blk = _bar_block(_unpack_block(B, nao, q0, q1, ij), D_core, D_w, C, dm2_flat)
            out[q0:q1] = blk[:, ij[0], ij[1]]
        return out
    if B.dim() != 3:
        raise ValueError("B must be (nao, nao, naux), (naux, nao, nao) or packed (naux, ntri)")
    lay = layout or "mnQ"
    if lay == "mnQ":
        if B.shape[0] != nao or B.shape[1] != nao:
            raise ValueError("B must have shape (nao, nao, naux)")
        naux = B.shape[2]
        get = lambda q0, q1: B[:, :, q0:q1].permute(2, 0, 1)  # noqa: E731
    elif lay == "Qmn":
        if B.shape[1] != nao or B.shape[2] != nao:
            raise ValueError("B must have shape (naux, nao, nao)")
        naux = B.shape[0]
        get = lambda q0, q1: B[q0:q1]  # noqa: E731
    else:
        raise ValueError("layout must be 'mnQ', 'Qmn' or 'Qp'")
    out = torch.empty((naux, nao, nao), dtype=torch.float64, device=dev)
    for q0 in range(0, naux, qb):
        q1 = min(naux, q0 + qb)
        out[q0:q1] = _bar_block(get(q0, q1), D_core, D_w, C, dm2_flat)
    return out

"""ORACLE / CPU baseline -- test and benchmark infrastructure only.

Times the reference's own CPU implementation of the DF path: its Cython Rys
kernels (``oracle/_ref/_eri_rys_cpu*.so``, built from the reference source by
``oracle/build_ref.py``) driven the way the reference drives them:

* pair tables: ``build_pair_tables_cart_inplace_cpu`` (``_eri_rys_cpu.pyx:2132``);
* metric and 3c: per AO shell pair, one ``eri_rys_tile_cart_sp_batch_cy`` call
  per aux angular momentum (``asuka/integrals/cueri_df_cpu.py:415-516``);
* Cholesky + whitening B = X L^-T (``cueri_df_cpu.py:519-527``);
* J/K (``asuka/hf/df_scf.py:516-662``) and dE/dB = rho_Q D - 1/2 D B_Q D;
* adjoints through whitening and Cholesky (``asuka/integrals/df_adjoint.py``)
  and the derivative contractions ``df_int3c2e_deriv_contracted_cart_sp_batch_cy``
  / ``df_metric_2c2e_deriv_contracted_cart_sp_batch_cy``
  (``asuka/integrals/grad.py:420-616``).

``pair_stride`` > 1 times only a sample of the AO shell pairs in the two 3c
loops (the dominant cost): within every (la, lb) angular class every stride-th
pair (at least one per class), each class's loop time scaled by that class's
sampled fraction of primitive-pair work -- so the sample has the class mix of
the whole loop.  Everything else runs at full size.  ``record`` collects the
time of every evaluated shell pair (for checking a sampled estimate against an
unsampled run).
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np
from scipy.linalg import solve_triangular

HERE = os.path.dirname(os.path.abspath(__file__))


def load_ref():
    sys.path.insert(0, os.path.join(HERE, "_ref"))
    try:
        import _eri_rys_cpu  # noqa: PLC0415
    finally:
        sys.path.pop(0)
    return _eri_rys_cpu


def available() -> bool:
    try:
        load_ref()
        return True
    except Exception:
        return False


def _combined(ao, aux):
    """AO + aux + dummy s shell (exp 0, coef 1, origin) and pairs: AO l-ordered pairs then (P, dummy)."""
    from asuka_b200.basis import build_shell_pairs_l_order

    nsa, nsx = ao.nshell, aux.nshell
    dummy = nsa + nsx
    cxyz = np.concatenate([ao.shell_cxyz, aux.shell_cxyz, np.zeros((1, 3))])
    nprim_ao = ao.prim_exp.size
    pstart = np.concatenate([ao.shell_prim_start, aux.shell_prim_start + nprim_ao,
                             [nprim_ao + aux.prim_exp.size]]).astype(np.int32)
    nprim = np.concatenate([ao.shell_nprim, aux.shell_nprim, [1]]).astype(np.int32)
    l = np.concatenate([ao.shell_l, aux.shell_l, [0]]).astype(np.int32)
    aostart = np.concatenate([ao.shell_ao_start, aux.shell_ao_start + ao.nao, [ao.nao + aux.nao]]).astype(np.int32)
    pexp = np.concatenate([ao.prim_exp, aux.prim_exp, [0.0]])
    pcoef = np.concatenate([ao.prim_coef, aux.prim_coef, [1.0]])
    sp = build_shell_pairs_l_order(ao)
    spA = np.concatenate([sp.sp_A, np.arange(nsa, nsa + nsx)]).astype(np.int32)
    spB = np.concatenate([sp.sp_B, np.full(nsx, dummy)]).astype(np.int32)
    npair = (nprim[spA] * nprim[spB]).astype(np.int32)
    start = np.zeros(spA.size + 1, dtype=np.int32)
    np.cumsum(npair, out=start[1:])
    return dict(cxyz=np.ascontiguousarray(cxyz), pstart=pstart, nprim=nprim, l=l, aostart=aostart, pexp=pexp,
                pcoef=pcoef, spA=spA, spB=spB, npair=npair, start=start, nsp_ao=sp.nsp)


def _stratified_sample(c: dict, ao, nsp_ao: int, stride: int):
    """Per (la, lb) class: every stride-th pair (offset stride // 2, at least one), and the class's
    primitive-pair work in total and in the sample."""
    la = ao.shell_l[c["spA"][:nsp_ao]]
    lb = ao.shell_l[c["spB"][:nsp_ao]]
    w = c["npair"][:nsp_ao].astype(np.float64)
    out = []
    for a in np.unique(la):
        for b in np.unique(lb):
            idx = np.nonzero((la == a) & (lb == b))[0]
            if idx.size == 0:
                continue
            smp = idx[min(stride // 2, idx.size - 1)::max(1, stride)] if stride > 1 else idx
            out.append((smp, float(w[idx].sum()), float(w[smp].sum())))
    return out


def cpu_step(ao, aux, Cw: np.ndarray, natm: int, pair_stride: int = 1, threads: int = 0,
             record: dict | None = None) -> dict:
    """One DF J/K build + 2e nuclear gradient on the host cores; returns phase times (s, scaled)."""
    ext = load_ref()
    t = {}
    c = _combined(ao, aux)
    nao, naux = ao.nao, aux.nao
    nsp_ao = c["nsp_ao"]
    aux0 = nsp_ao
    T0 = time.perf_counter()
    npp = int(c["start"][-1])
    pt = [np.zeros(npp) for _ in range(5)]
    ext.build_pair_tables_cart_inplace_cpu(c["cxyz"], c["pstart"], c["nprim"], c["pexp"], c["pcoef"], c["spA"],
                                           c["spB"], c["start"], c["npair"], *pt, threads)
    t["pair_tables"] = time.perf_counter() - T0
    args = [c["cxyz"], c["l"], c["spA"], c["spB"], c["start"], c["npair"], *pt]
    aux_l = aux.shell_l
    by_l = {int(l): (aux0 + np.nonzero(aux_l == l)[0]).astype(np.int32) for l in np.unique(aux_l)}
    # metric
    T0 = time.perf_counter()
    V = np.zeros((naux, naux))
    for P in range(aux.nshell):
        p0 = aux.shell_ao_start[P]
        nP = (aux_l[P] + 1) * (aux_l[P] + 2) // 2
        for lq, qs in by_l.items():
            qs = qs[qs - aux0 <= P]
            if qs.size == 0:
                continue
            tiles = ext.eri_rys_tile_cart_sp_batch_cy(*args, int(aux0 + P), qs, threads)
            nQ = (lq + 1) * (lq + 2) // 2
            for k, q in enumerate(qs - aux0):
                q0 = aux.shell_ao_start[q]
                blk = np.asarray(tiles[k]).reshape(nP, nQ)
                V[p0:p0 + nP, q0:q0 + nQ] = blk
                V[q0:q0 + nQ, p0:p0 + nP] = blk.T
    V = 0.5 * (V + V.T)
    t["metric"] = time.perf_counter() - T0
    # 3c over the sampled AO pairs of every angular class
    strata = _stratified_sample(c, ao, nsp_ao, max(1, int(pair_stride)))
    sample = np.concatenate([s for s, _, _ in strata])
    scale = np.zeros(nsp_ao)
    for smp, w_cls, w_smp in strata:
        scale[smp] = w_cls / w_smp
    frac = float(sum(ws for _, _, ws in strata) / sum(wc for _, wc, _ in strata))
    X = np.zeros((nao * nao, naux))
    t_int = 0.0
    rec_int = record.setdefault("int3c", {}) if record is not None else None
    for sp in sample:
        T0 = time.perf_counter()
        A, B = c["spA"][sp], c["spB"][sp]
        la, lb = ao.shell_l[A], ao.shell_l[B]
        nA, nB = (la + 1) * (la + 2) // 2, (lb + 1) * (lb + 2) // 2
        a0, b0 = ao.shell_ao_start[A], ao.shell_ao_start[B]
        rows = ((a0 + np.arange(nA))[:, None] * nao + (b0 + np.arange(nB))[None, :]).ravel()
        rowsT = ((b0 + np.arange(nB))[:, None] * nao + (a0 + np.arange(nA))[None, :]).ravel()
        for lq, qs in by_l.items():
            tiles = ext.eri_rys_tile_cart_sp_batch_cy(*args, int(sp), qs, threads)
            nQ = (lq + 1) * (lq + 2) // 2
            for k, q in enumerate(qs - aux0):
                q0 = aux.shell_ao_start[q]
                tile = np.asarray(tiles[k]).reshape(nA * nB, nQ)
                X[rows, q0:q0 + nQ] = tile
                X[rowsT, q0:q0 + nQ] = tile.reshape(nA, nB, nQ).transpose(1, 0, 2).reshape(nB * nA, nQ)
        dt = time.perf_counter() - T0
        t_int += dt * scale[sp]
        if rec_int is not None:
            rec_int[int(sp)] = dt
    t["int3c"] = t_int
    # Cholesky + whitening
    T0 = time.perf_counter()
    L = np.linalg.cholesky(V)
    t["cholesky"] = time.perf_counter() - T0
    T0 = time.perf_counter()
    B = np.ascontiguousarray(solve_triangular(L, X.T, lower=True).T)
    t["whiten"] = time.perf_counter() - T0
    # J/K and dE/dB
    T0 = time.perf_counter()
    D = Cw @ Cw.T
    rho = B.T @ D.reshape(-1)
    J = (B @ rho).reshape(nao, nao)
    BQ = B.reshape(nao, nao, naux)
    U = np.einsum("mnQ,ni->Qmi", BQ, Cw, optimize=True)
    K = np.einsum("Qmi,Qni->mn", U, U, optimize=True)
    E2 = 0.5 * float(np.sum(D * J)) - 0.25 * float(np.sum(D * K))
    t["jk"] = time.perf_counter() - T0
    T0 = time.perf_counter()
    DBD = np.einsum("mk,knQ,nl->Qml", D, BQ, D, optimize=True)
    barL = rho[:, None, None] * D[None] - 0.5 * DBD
    tmp = solve_triangular(L, barL.reshape(naux, nao * nao), lower=True, trans="T")
    bar_Lc = np.tril(-(tmp @ B))
    Gm = np.tril(L.T @ bar_Lc)
    Gm[np.diag_indices(naux)] *= 0.5
    t2 = solve_triangular(L, Gm, lower=True, trans="T")
    bar_V = solve_triangular(L, t2.T, lower=True, trans="T").T
    bar_V = 0.5 * (bar_V + bar_V.T)
    bar_X = tmp.T.reshape(nao, nao, naux)
    bar_X = np.ascontiguousarray(0.5 * (bar_X + bar_X.transpose(1, 0, 2))).reshape(nao * nao, naux)
    t["adjoint"] = time.perf_counter() - T0
    # derivative contractions
    grad = np.zeros((natm, 3))
    ao_atom = ao.shell_atom
    ax_atom = aux.shell_atom
    t_der = 0.0
    rec_der = record.setdefault("deriv3c", {}) if record is not None else None
    for sp in sample:
        T0 = time.perf_counter()
        A, B_ = c["spA"][sp], c["spB"][sp]
        fac = 2.0 if A != B_ else 1.0
        for lq, qs in by_l.items():
            out = ext.df_int3c2e_deriv_contracted_cart_sp_batch_cy(
                c["cxyz"], c["pstart"], c["nprim"], c["l"], c["aostart"], c["pexp"], c["spA"], c["spB"], c["start"],
                c["npair"], *pt, int(sp), qs, int(nao), bar_X)
            out = np.asarray(out)
            for k, q in enumerate(qs - aux0):
                grad[ao_atom[A]] += fac * out[k, 0]
                grad[ao_atom[B_]] += fac * out[k, 1]
                grad[ax_atom[q]] += fac * out[k, 2]
        dt = time.perf_counter() - T0
        t_der += dt * scale[sp]
        if rec_der is not None:
            rec_der[int(sp)] = dt
    t["deriv3c"] = t_der
    T0 = time.perf_counter()
    for P in range(aux.nshell):
        for lq, qs in by_l.items():
            qs = qs[qs - aux0 <= P]
            if qs.size == 0:
                continue
            out = np.asarray(ext.df_metric_2c2e_deriv_contracted_cart_sp_batch_cy(
                c["cxyz"], c["pstart"], c["nprim"], c["l"], c["aostart"], c["pexp"], c["spA"], c["spB"], c["start"],
                c["npair"], *pt, int(aux0 + P), qs, int(nao), bar_V))
            for k, q in enumerate(qs - aux0):
                fac = 2.0 if q != P else 1.0
                grad[ax_atom[P]] += fac * out[k, 0]
                grad[ax_atom[q]] += fac * out[k, 1]
    t["deriv2c"] = time.perf_counter() - T0
    t["total"] = sum(v for k, v in t.items())
    t["sample_fraction"] = frac
    t["E2"] = E2
    t["grad"] = grad
    return t

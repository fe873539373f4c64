"""DF-RHF driver and the ``run_hf_df`` front end on the device.

``rhf_df`` restates the reference's materialised-B RHF loop
(``asuka/hf/df_scf.py:871-1429``): symmetric orthogonaliser S^-1/2, core
Hamiltonian guess, one predictor Fock cycle, DIIS (max 8 vectors) on
FDS - SDF from cycle 1, energy 1/2 tr(D_new (h + F)) with F the extrapolated
Fock matrix, convergence when |dE| < conv_tol and ||D_new - D||_F < conv_tol_dm.

``precision='mixed'`` runs the exchange contraction in split-BF16 while
||dD|| > mixed_switch (1e-4, the same threshold at which the reference leaves
its FP64-emulated cuBLAS mode, ``df_scf.py:1200-1216``) and finishes with FP64
iterations, so the converged energy is an FP64 energy.

``run_hf_df`` mirrors ``asuka/frontend/scf.py:1219`` for method='rhf',
two_e_backend 'df' (materialised whitened B) and 'direct_df' (B never stored:
the 3c integrals are recomputed per aux block every cycle).
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from . import linalg as _la
from . import basis as bm
from .df import DFEngine, cholesky_metric, whiten_3c2e
from .geometry import Molecule
from .int1e import build_int1e
from .jk import df_J_from_BQ_D, df_K_from_BQ_Cw


@dataclass(frozen=True)
class SCFResult:
    method: str
    converged: bool
    niter: int
    e_tot: float
    e_elec: float
    e_nuc: float
    mo_energy: Any
    mo_coeff: Any
    mo_occ: Any


@dataclass
class RHFDFRunResult:
    mol: Molecule
    ao_basis: bm.BasisCartSoA
    aux_basis: bm.BasisCartSoA
    int1e: Any
    df_B: Any
    df_L: Any
    scf: SCFResult
    two_e_backend: str
    basis_name: str = ""
    auxbasis_name: str = "ricd"
    profile: dict | None = field(default=None, repr=False)

    @property
    def e_tot(self) -> float:
        return self.scf.e_tot

    @property
    def mo_coeff(self):
        return self.scf.mo_coeff

    @property
    def mo_occ(self):
        return self.scf.mo_occ

    @property
    def mo_energy(self):
        return self.scf.mo_energy

    @property
    def converged(self) -> bool:
        return self.scf.converged


class _DIIS:
    """Pulay DIIS on FDS - SDF with the reference's Gram scaling and regularisation ladder."""

    def __init__(self, max_vec: int = 8):
        self.max_vec = max_vec
        self.F: list[torch.Tensor] = []
        self.e: list[torch.Tensor] = []

    def push(self, F, e):
        self.F.append(F)
        self.e.append(e)
        if len(self.F) > self.max_vec:
            self.F.pop(0)
            self.e.pop(0)

    def extrapolate(self):
        n = len(self.F)
        if n < 2:
            return self.F[-1]
        E = torch.stack([x.reshape(-1) for x in self.e])
        G = (E @ E.T).cpu().numpy()
        if not np.all(np.isfinite(G)):
            return self.F[-1]
        G = G / max(np.abs(G).max(), 1e-300)
        Bm = np.zeros((n + 1, n + 1))
        Bm[:n, :n] = G
        Bm[:n, n] = Bm[n, :n] = -1.0
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        c = None
        for lam in (0.0, 1e-14, 1e-12, 1e-10, 1e-8, 1e-6):
            try:
                t = np.linalg.solve(Bm + lam * np.diag(np.r_[np.ones(n), 0.0]), rhs)
            except np.linalg.LinAlgError:
                continue
            if np.all(np.isfinite(t)):
                c = t
                break
        if c is None or abs(c[:n].sum()) < 1e-15:
            return self.F[-1]
        c = c[:n] / c[:n].sum()
        cw = torch.as_tensor(c, dtype=torch.float64, device=self.F[-1].device)
        return torch.tensordot(cw, torch.stack(self.F), dims=1)


def _sym(A):
    return 0.5 * (A + A.T)


def rhf_df(S, hcore, B=None, *, nelec: int, enuc: float = 0.0, max_cycle: int = 50, conv_tol: float = 1e-10,
           conv_tol_dm: float = 1e-8, diis: bool = True, diis_start_cycle: int = 1, diis_space: int = 8,
           k_q_block: int = 256, init_fock_cycles: int = 1, dm0=None, mo_coeff0=None, precision: str = "fp64",
           mixed_switch: float = 1e-4, jk_fn=None, profile: dict | None = None) -> SCFResult:
    """RHF with DF J/K.  ``B`` is the whitened factor in 'Qmn' (naux,nao,nao) or 'mnQ' (nao,nao,naux) layout;
    alternatively ``jk_fn(D, Cw, precision) -> (J, K)`` supplies J/K (streamed/direct DF)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    S = torch.as_tensor(S, dtype=torch.float64, device=dev)
    h = torch.as_tensor(hcore, dtype=torch.float64, device=dev)
    nao = S.shape[0]
    if nelec % 2 or nelec < 0:
        raise ValueError("RHF requires an even nelec >= 0")
    nocc = nelec // 2
    if jk_fn is None:
        if B is None:
            raise ValueError("either B or jk_fn is required")
        B = torch.as_tensor(B, dtype=torch.float64, device=dev)
        if B.shape[0] == nao and B.shape[1] == nao:
            BQ = B.permute(2, 0, 1).contiguous()
        elif B.shape[1] == nao and B.shape[2] == nao:
            BQ = B
        else:
            raise ValueError("B must be (nao,nao,naux) or (naux,nao,nao)")

        def jk_fn(D, Cw, prec):
            return df_J_from_BQ_D(BQ, D), df_K_from_BQ_Cw(BQ, Cw, q_block=k_q_block, precision=prec)

    s, U = torch.linalg.eigh(_sym(S))
    if bool((s <= 1e-12).any()):
        raise ValueError("S is not positive definite")
    Xo = (U * s.rsqrt()) @ U.T
    occ = torch.zeros(nao, dtype=torch.float64, device=dev)
    occ[:nocc] = 2.0

    def solve(F):
        e, Cp = torch.linalg.eigh(_sym(Xo.T @ F @ Xo))
        return e, Xo @ Cp

    def dens(C):
        Cw = C[:, :nocc] * 2.0**0.5
        return _sym(Cw @ Cw.T), Cw

    eps, C = solve(h)
    if mo_coeff0 is not None:
        C = torch.as_tensor(mo_coeff0, dtype=torch.float64, device=dev)
    D, Cw = dens(C)
    if dm0 is not None:
        D = _sym(torch.as_tensor(dm0, dtype=torch.float64, device=dev))
        # natural orbitals of dm0 in the orthogonal basis give the occupied space
        n, Un = torch.linalg.eigh(_sym(Xo.T @ S @ D @ S @ Xo))
        C = Xo @ Un.flip(1)
        D, Cw = dens(C)
    prec_now = precision
    t_jk = 0.0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if init_fock_cycles > 0 and dm0 is None and mo_coeff0 is None:
        for _ in range(init_fock_cycles):
            J, K = jk_fn(D, Cw, prec_now)
            eps, C = solve(_sym(h + J - 0.5 * K))
            D, Cw = dens(C)
    dd = DIISWrap = _DIIS(diis_space) if diis else None
    e_last = None
    converged = False
    niter = 0
    for cycle in range(1, max_cycle + 1):
        niter = cycle
        ev0.record()
        J, K = jk_fn(D, Cw, prec_now)
        ev1.record()
        ev1.synchronize()
        t_jk += ev0.elapsed_time(ev1)
        F = _sym(h + J - 0.5 * K)
        if dd is not None and cycle >= diis_start_cycle:
            Mx = F @ D @ S
            dd.push(F, Mx - Mx.T)
            F = _sym(dd.extrapolate())
        eps, C = solve(F)
        D_new, Cw = dens(C)
        e_tot = 0.5 * float(torch.sum(D_new * (h + F))) + float(enuc)
        dm_err = float(torch.linalg.norm(D_new - D))
        de = abs(e_tot - e_last) if e_last is not None else float("inf")
        D = D_new
        e_last = e_tot
        if prec_now != "fp64" and dm_err < mixed_switch:
            prec_now = "fp64"  # iterative refinement: finish in FP64
            if dd is not None:
                dd = _DIIS(diis_space)  # drop the mixed-precision Fock history
            continue
        if de < conv_tol and dm_err < conv_tol_dm and prec_now == "fp64":
            converged = True
            break
    del DIISWrap
    if profile is not None:
        profile.setdefault("scf", {}).update(jk_ms=t_jk, iters=niter)
    return SCFResult(method="RHF", converged=converged, niter=niter, e_tot=float(e_last),
                     e_elec=float(e_last) - float(enuc), e_nuc=float(enuc), mo_energy=eps, mo_coeff=C, mo_occ=occ)


def uhf_df(S, hcore, B=None, *, nalpha: int, nbeta: int, enuc: float = 0.0, max_cycle: int = 50,
           conv_tol: float = 1e-10, conv_tol_dm: float = 1e-8, diis: bool = True, diis_start_cycle: int = 2,
           diis_space: int = 8, damping: float = 0.0, jk_mode: str = "auto", k_q_block: int = 128,
           ao_basis=None, aux_basis=None, df_aux_block_naux: int = 256, L_metric=None, dm0=None,
           mo_coeff0=None, profile: dict | None = None, engine: DFEngine | None = None, **_unused) -> SCFResult:
    """UHF with DF J/K (``asuka/hf/df_scf.py:1432-1868`` without the XC terms).

    J comes from the total density and one K per spin from that spin's occupied orbitals
    (unit occupations); with ``jk_mode='streamed'`` (or 'auto' without B) both spins share
    one streamed integral evaluation per pass (``df_JKs_streamed``).  Guess, DIIS per spin
    (from cycle ``diis_start_cycle``), damping, the energy
    tr(D h) + 1/2 tr(D J) - 1/2 (tr(Da Ka) + tr(Db Kb)) with the new densities and the
    current J/K, and the convergence test |dE| < conv_tol and
    ||dDa|| + ||dDb|| < conv_tol_dm follow the reference.
    """
    dev = torch.device("cuda", torch.cuda.current_device())
    S = torch.as_tensor(S, dtype=torch.float64, device=dev)
    h = torch.as_tensor(hcore, dtype=torch.float64, device=dev)
    nao = S.shape[0]
    nalpha, nbeta = int(nalpha), int(nbeta)
    if nalpha < 0 or nbeta < 0 or nalpha > nao or nbeta > nao:
        raise ValueError("nalpha/nbeta must lie in [0, nao]")
    mode = str(jk_mode).strip().lower()
    streamed = mode == "streamed" or (mode == "auto" and B is None)
    if streamed:
        if dm0 is not None:
            raise NotImplementedError("streamed J/K needs orbitals, not a density guess (dm0)")
        from .df import get_engine
        from .streamed import df_JKs_streamed, make_streamed_df_jk_context

        if engine is None and (ao_basis is None or aux_basis is None):
            raise ValueError("jk_mode='streamed' requires ao_basis and aux_basis")
        eng = engine if engine is not None else get_engine(ao_basis, aux_basis)
        ctx = make_streamed_df_jk_context(ao_basis, aux_basis, aux_block_naux=df_aux_block_naux, engine=eng,
                                          L_metric=None if L_metric is None else torch.as_tensor(L_metric, device=dev))
    else:
        if B is None:
            raise ValueError("B is required unless jk_mode='streamed'")
        B = torch.as_tensor(B, dtype=torch.float64, device=dev)
        if B.shape[0] == nao and B.shape[1] == nao:
            BQ = B.permute(2, 0, 1).contiguous()
        elif B.shape[1] == nao and B.shape[2] == nao:
            BQ = B
        else:
            raise ValueError("B must be (nao,nao,naux) or (naux,nao,nao)")
    s, U = torch.linalg.eigh(_sym(S))
    if bool((s <= 1e-12).any()):
        raise ValueError("S is not positive definite")
    Xo = (U * s.rsqrt()) @ U.T
    occ_a = torch.zeros(nao, dtype=torch.float64, device=dev)
    occ_b = torch.zeros(nao, dtype=torch.float64, device=dev)
    occ_a[:nalpha] = 1.0
    occ_b[:nbeta] = 1.0

    def solve(F):
        e, Cp = torch.linalg.eigh(_sym(Xo.T @ F @ Xo))
        return e, Xo @ Cp

    def dens(C, n):
        Co = C[:, :n]
        return _sym(Co @ Co.T)

    e0, C = solve(h)
    Ca = Cb = C
    ea = eb = e0
    if dm0 is not None:
        Da = _sym(torch.as_tensor(dm0[0], dtype=torch.float64, device=dev))
        Db = _sym(torch.as_tensor(dm0[1], dtype=torch.float64, device=dev))
    else:
        if mo_coeff0 is not None:
            if isinstance(mo_coeff0, (tuple, list)):
                Ca = torch.as_tensor(mo_coeff0[0], dtype=torch.float64, device=dev)
                Cb = torch.as_tensor(mo_coeff0[1], dtype=torch.float64, device=dev)
            else:
                Ca = Cb = torch.as_tensor(mo_coeff0, dtype=torch.float64, device=dev)
        Da, Db = dens(Ca, nalpha), dens(Cb, nbeta)
    lam = float(damping) if damping else 0.0
    Ka_prev = Kb_prev = None
    dda = _DIIS(diis_space) if diis else None
    ddb = _DIIS(diis_space) if diis else None
    e_last = None
    converged = False
    niter = 0
    for cycle in range(1, max_cycle + 1):
        niter = cycle
        Dt = Da + Db
        if streamed:
            J, (Ka, Kb) = df_JKs_streamed(ctx, Dt, [Ca[:, :nalpha], Cb[:, :nbeta]],
                                          [occ_a[:nalpha], occ_b[:nbeta]], k_q_block=k_q_block)
        elif dm0 is not None and cycle == 1:  # density-driven exchange for a density guess
            J = df_J_from_BQ_D(BQ, Dt)
            Ka = _sym(torch.einsum("Qmk,kl,Qnl->mn", BQ, Da, BQ))
            Kb = _sym(torch.einsum("Qmk,kl,Qnl->mn", BQ, Db, BQ))
        else:
            J = df_J_from_BQ_D(BQ, Dt)
            Ka = df_K_from_BQ_Cw(BQ, Ca[:, :nalpha].contiguous(), q_block=k_q_block)
            Kb = df_K_from_BQ_Cw(BQ, Cb[:, :nbeta].contiguous(), q_block=k_q_block)
        if lam and Ka_prev is not None:
            Ka = (1.0 - lam) * Ka + lam * Ka_prev
            Kb = (1.0 - lam) * Kb + lam * Kb_prev
        Ka_prev, Kb_prev = Ka, Kb
        Fa = _sym(h + J - Ka)
        Fb = _sym(h + J - Kb)
        if dda is not None and cycle >= diis_start_cycle:
            Ma = Fa @ Da @ S
            dda.push(Fa, Ma - Ma.T)
            Fa = _sym(dda.extrapolate())
            Mb = Fb @ Db @ S
            ddb.push(Fb, Mb - Mb.T)
            Fb = _sym(ddb.extrapolate())
        ea, Ca = solve(Fa)
        eb, Cb = solve(Fb)
        Da_new, Db_new = dens(Ca, nalpha), dens(Cb, nbeta)
        if lam:
            Da_new = (1.0 - lam) * Da_new + lam * Da
            Db_new = (1.0 - lam) * Db_new + lam * Db
        Dt_new = Da_new + Db_new
        e_elec = (float(torch.sum(Dt_new * h)) + 0.5 * float(torch.sum(Dt_new * J))
                  - 0.5 * (float(torch.sum(Da_new * Ka)) + float(torch.sum(Db_new * Kb))))
        e_tot = e_elec + float(enuc)
        dm_err = float(torch.linalg.norm(Da_new - Da)) + float(torch.linalg.norm(Db_new - Db))
        de = abs(e_tot - e_last) if e_last is not None else float("inf")
        Da, Db = Da_new, Db_new
        e_last = e_tot
        if de < conv_tol and dm_err < conv_tol_dm:
            converged = True
            break
    if profile is not None:
        profile.setdefault("scf", {}).update(iters=niter)
    return SCFResult(method="UHF", converged=converged, niter=niter, e_tot=float(e_last),
                     e_elec=float(e_last) - float(enuc), e_nuc=float(enuc), mo_energy=(ea, eb), mo_coeff=(Ca, Cb),
                     mo_occ=(occ_a, occ_b))


def _roothaan_fock(Fa, Fb, Da, Db, S):
    """Roothaan's effective ROHF Fock matrix from the spin Fock matrices.

    With the closed (c), open (o) and virtual (v) projectors P_c = Db S, P_o = (Da - Db) S,
    P_v = 1 - Da S and Fc = (Fa + Fb)/2, the blocks are cc, oo, vv: Fc; oc: Fb; ov: Fa;
    vc: Fc (the choice of ``asuka/hf/df_scf.py:691-719``, as in PySCF's get_roothaan_fock).
    """
    n = S.shape[0]
    fc = 0.5 * (Fa + Fb)
    pc = Db @ S
    po = (Da - Db) @ S
    pv = torch.eye(n, dtype=S.dtype, device=S.device) - Da @ S
    F = 0.5 * (pc.T @ fc @ pc + po.T @ fc @ po + pv.T @ fc @ pv)
    F = F + po.T @ Fb @ pc + po.T @ Fa @ pv + pv.T @ fc @ pc
    return _sym(F + F.T)


def rohf_df(S, hcore, B=None, *, nalpha: int, nbeta: int, enuc: float = 0.0, max_cycle: int = 50,
            conv_tol: float = 1e-10, conv_tol_dm: float = 1e-8, diis: bool = True, diis_start_cycle: int = 2,
            diis_space: int = 8, damping: float = 0.0, jk_mode: str = "auto", k_q_block: int = 128,
            ao_basis=None, aux_basis=None, df_aux_block_naux: int = 256, L_metric=None, dm0=None,
            mo_coeff0=None, profile: dict | None = None, engine: DFEngine | None = None, **_unused) -> SCFResult:
    """ROHF with DF J/K and one set of orbitals (``asuka/hf/df_scf.py:1870-2330``).

    Spin Fock matrices Fa = h + J - Ka, Fb = h + J - Kb are combined into Roothaan's
    effective Fock (``_roothaan_fock``); DIIS runs on it with the error F Dt S - S Dt F.
    With streamed J/K the beta orbitals and the open shell go through one integral pass
    as two occupied sets (Ka = Kb + K_open).  Energy and convergence test as for UHF.
    """
    dev = torch.device("cuda", torch.cuda.current_device())
    S = torch.as_tensor(S, dtype=torch.float64, device=dev)
    h = torch.as_tensor(hcore, dtype=torch.float64, device=dev)
    nao = S.shape[0]
    nalpha, nbeta = int(nalpha), int(nbeta)
    if not (0 <= nbeta <= nalpha <= nao):
        raise ValueError("ROHF needs 0 <= nbeta <= nalpha <= nao")
    mode = str(jk_mode).strip().lower()
    streamed = mode == "streamed" or (mode == "auto" and B is None)
    if streamed:
        if dm0 is not None:
            raise NotImplementedError("streamed J/K needs orbitals, not a density guess (dm0)")
        from .df import get_engine
        from .streamed import df_JKs_streamed, make_streamed_df_jk_context

        if engine is None and (ao_basis is None or aux_basis is None):
            raise ValueError("jk_mode='streamed' requires ao_basis and aux_basis")
        eng = engine if engine is not None else get_engine(ao_basis, aux_basis)
        ctx = make_streamed_df_jk_context(ao_basis, aux_basis, aux_block_naux=df_aux_block_naux, engine=eng,
                                          L_metric=None if L_metric is None else torch.as_tensor(L_metric, device=dev))
    else:
        if B is None:
            raise ValueError("B is required unless jk_mode='streamed'")
        B = torch.as_tensor(B, dtype=torch.float64, device=dev)
        if B.shape[0] == nao and B.shape[1] == nao:
            BQ = B.permute(2, 0, 1).contiguous()
        elif B.shape[1] == nao and B.shape[2] == nao:
            BQ = B
        else:
            raise ValueError("B must be (nao,nao,naux) or (naux,nao,nao)")
    s, U = torch.linalg.eigh(_sym(S))
    if bool((s <= 1e-12).any()):
        raise ValueError("S is not positive definite")
    Xo = (U * s.rsqrt()) @ U.T
    occ_a = torch.zeros(nao, dtype=torch.float64, device=dev)
    occ_b = torch.zeros(nao, dtype=torch.float64, device=dev)
    occ_a[:nalpha] = 1.0
    occ_b[:nbeta] = 1.0

    def solve(F):
        e, Cp = torch.linalg.eigh(_sym(Xo.T @ F @ Xo))
        return e, Xo @ Cp

    def dens(C, n):
        Co = C[:, :n]
        return _sym(Co @ Co.T)

    eps, C = solve(h)
    if dm0 is not None:
        Da = _sym(torch.as_tensor(dm0[0], dtype=torch.float64, device=dev))
        Db = _sym(torch.as_tensor(dm0[1], dtype=torch.float64, device=dev))
    else:
        if mo_coeff0 is not None:
            C = torch.as_tensor(mo_coeff0, dtype=torch.float64, device=dev)
        Da, Db = dens(C, nalpha), dens(C, nbeta)
    lam = float(damping) if damping else 0.0
    Ka_prev = Kb_prev = None
    dd = _DIIS(diis_space) if diis else None
    e_last = None
    converged = False
    niter = 0
    for cycle in range(1, max_cycle + 1):
        niter = cycle
        Dt = Da + Db
        if streamed:
            J, (Kb, Ko) = df_JKs_streamed(ctx, Dt, [C[:, :nbeta], C[:, nbeta:nalpha]],
                                          [occ_b[:nbeta], occ_a[nbeta:nalpha]], k_q_block=k_q_block)
            Ka = Kb + Ko
        elif dm0 is not None and cycle == 1:
            J = df_J_from_BQ_D(BQ, Dt)
            Ka = _sym(torch.einsum("Qmk,kl,Qnl->mn", BQ, Da, BQ))
            Kb = _sym(torch.einsum("Qmk,kl,Qnl->mn", BQ, Db, BQ))
        else:
            J = df_J_from_BQ_D(BQ, Dt)
            Ka = df_K_from_BQ_Cw(BQ, C[:, :nalpha].contiguous(), q_block=k_q_block)
            Kb = df_K_from_BQ_Cw(BQ, C[:, :nbeta].contiguous(), q_block=k_q_block)
        if lam and Ka_prev is not None:
            Ka = (1.0 - lam) * Ka + lam * Ka_prev
            Kb = (1.0 - lam) * Kb + lam * Kb_prev
        Ka_prev, Kb_prev = Ka, Kb
        Fa = _sym(h + J - Ka)
        Fb = _sym(h + J - Kb)
        F = _roothaan_fock(Fa, Fb, Da, Db, S)
        if dd is not None and cycle >= diis_start_cycle:
            M = F @ Dt @ S
            dd.push(F, M - M.T)
            F = _sym(dd.extrapolate())
        eps, C = solve(F)
        Da_new, Db_new = dens(C, nalpha), dens(C, nbeta)
        if lam:
            Da_new = (1.0 - lam) * Da_new + lam * Da
            Db_new = (1.0 - lam) * Db_new + lam * Db
        Dt_new = Da_new + Db_new
        e_elec = (float(torch.sum(Dt_new * h)) + 0.5 * float(torch.sum(Dt_new * J))
                  - 0.5 * (float(torch.sum(Da_new * Ka)) + float(torch.sum(Db_new * Kb))))
        e_tot = e_elec + float(enuc)
        dm_err = float(torch.linalg.norm(Da_new - Da)) + float(torch.linalg.norm(Db_new - Db))
        de = abs(e_tot - e_last) if e_last is not None else float("inf")
        Da, Db = Da_new, Db_new
        e_last = e_tot
        if de < conv_tol and dm_err < conv_tol_dm:
            converged = True
            break
    if profile is not None:
        profile.setdefault("scf", {}).update(iters=niter)
    return SCFResult(method="ROHF", converged=converged, niter=niter, e_tot=float(e_last),
                     e_elec=float(e_last) - float(enuc), e_nuc=float(enuc), mo_energy=eps, mo_coeff=C,
                     mo_occ=(occ_a, occ_b))


def pack_B_to_Qp(B: torch.Tensor, layout: str = "Qmn") -> torch.Tensor:
    """Lower-triangle packing B_Qp[Q, mu(mu+1)/2 + nu], mu >= nu (``asuka/integrals/df_packed_s2.py:63``)."""
    BQ = B if layout == "Qmn" else B.permute(2, 0, 1)
    nao = BQ.shape[1]
    i, j = torch.tril_indices(nao, nao, device=BQ.device)
    return BQ[:, i, j].contiguous()


def _direct_jk(engine: DFEngine, L: torch.Tensor, aux_block: int = 256):
    """Streamed DF J/K for the SCF (``asuka/hf/df_jk_streamed.py:167-325``): the 3c integrals are
    recomputed per aux block in two passes per cycle and B is never stored."""
    from .streamed import df_JK_streamed, make_streamed_df_jk_context

    ctx = make_streamed_df_jk_context(engine.ao, engine.aux, aux_block_naux=aux_block, engine=engine, L_metric=L)

    def jk(D, Cw, prec):
        ones = torch.ones(Cw.shape[1], dtype=torch.float64, device=Cw.device)
        return df_JK_streamed(ctx, D, Cw, ones, precision=prec)

    return jk


def run_hf_df(mol: Molecule, *, method: str = "rhf", backend: str = "cuda", df: bool = True,
              two_e_backend: str | None = None, guess=None, dm0=None, mo_coeff0=None, auxbasis: str = "ricd",
              conv_tol: float = 1e-10, conv_tol_dm: float = 1e-8, max_cycle: int = 50, precision: str = "fp64",
              df_layout: str = "Qp", df_aux_block_naux: int = 256, profile: dict | None = None,
              **kwargs) -> RHFDFRunResult:
    """RHF or UHF with density fitting on the GPU (``asuka/frontend/scf.py:1219``)."""
    meth = str(method).lower()
    if meth not in ("rhf", "uhf", "rohf"):
        raise NotImplementedError("method must be 'rhf', 'uhf' or 'rohf'")
    if backend not in ("cuda", "gpu"):
        raise ValueError("this engine runs on CUDA only (backend='cuda')")
    tb = two_e_backend or ("df" if df else "dense")
    if tb not in ("df", "direct_df"):
        raise NotImplementedError(f"two_e_backend={tb!r} is not implemented")
    if str(auxbasis).lower() not in ("ricd", "accd", "acd"):
        raise NotImplementedError("only the RICD acCD auxiliary basis is available")
    if meth == "rhf" and mol.spin != 0:
        raise NotImplementedError("RHF requires spin=0 (use method='uhf')")
    if (mol.nelectron + mol.spin) % 2:
        raise ValueError("nelectron and spin are incompatible")
    basis = mol.basis or "ma-svp"
    atoms = list(mol.atoms_bohr)
    ao = bm.pack_basis(atoms, basis, "ao")
    aux = bm.pack_basis(atoms, basis, "aux")
    t0 = time.perf_counter()
    int1e = build_int1e(ao, mol.coords_bohr, mol.charges)
    eng = DFEngine(ao, aux)
    V = eng.metric()
    L = cholesky_metric(V)
    prof = profile if profile is not None else None
    Tsph = None
    if not getattr(mol, "cart", True):
        # spherical AOs: the integrals are evaluated over Cartesian shells and transformed on the
        # AO indices (X_sph = T^T X T, the aux index stays Cartesian), as the reference does
        from .int1e import Int1eResult
        from .sph import cart2sph_ao_matrix, int3c_cart_to_sph

        Tsph = cart2sph_ao_matrix(ao.shell_l, eng.device)
        Tn = Tsph.cpu().numpy()
        int1e = Int1eResult(S=Tn.T @ int1e.S @ Tn, T=Tn.T @ int1e.T @ Tn, V=Tn.T @ int1e.V @ Tn)
        if tb == "direct_df" and meth != "rhf":
            raise NotImplementedError("streamed J/K with spherical AOs is implemented for RHF only")

    def _B_for_scf():
        B = eng.int3c("Qmn")
        whiten_3c2e(B, L, layout="Qmn")
        return B if Tsph is None else int3c_cart_to_sph(B, Tsph, "Qmn")

    if meth in ("uhf", "rohf"):
        driver = uhf_df if meth == "uhf" else rohf_df
        na, nb = (mol.nelectron + mol.spin) // 2, (mol.nelectron - mol.spin) // 2
        common = dict(nalpha=na, nbeta=nb, enuc=mol.energy_nuc(), max_cycle=max_cycle, conv_tol=conv_tol,
                      conv_tol_dm=conv_tol_dm, dm0=dm0, mo_coeff0=mo_coeff0, profile=prof)
        if tb == "df":
            B = _B_for_scf()
            scf = driver(int1e.S, int1e.hcore, B, jk_mode="materialized", **common)
            df_B = pack_B_to_Qp(B, "Qmn") if df_layout == "Qp" else (
                B.permute(1, 2, 0).contiguous() if df_layout == "mnQ" else B)
        else:
            scf = driver(int1e.S, int1e.hcore, None, jk_mode="streamed", engine=eng, L_metric=L,
                         df_aux_block_naux=df_aux_block_naux, **common)
            df_B = None
        if prof is not None:
            prof["wall_s"] = time.perf_counter() - t0
        return RHFDFRunResult(mol=mol, ao_basis=ao, aux_basis=aux, int1e=int1e, df_B=df_B, df_L=L, scf=scf,
                              two_e_backend=tb, basis_name=basis, profile=prof)
    if tb == "df":
        B = _B_for_scf()
        scf = rhf_df(int1e.S, int1e.hcore, B, nelec=mol.nelectron, enuc=mol.energy_nuc(), max_cycle=max_cycle,
                     conv_tol=conv_tol, conv_tol_dm=conv_tol_dm, dm0=dm0, mo_coeff0=mo_coeff0, precision=precision,
                     profile=prof)
        if df_layout == "Qp":
            df_B = pack_B_to_Qp(B, "Qmn")
        elif df_layout == "mnQ":
            df_B = B.permute(1, 2, 0).contiguous()
        else:
            df_B = B
    else:
        jk = _direct_jk(eng, L, aux_block=df_aux_block_naux)
        if Tsph is not None:
            jk_cart = jk

            def jk(D, Cw, prec, _T=Tsph, _jk=jk_cart):
                Jc, Kc = _jk(_T @ D @ _T.T, _T @ Cw, prec)
                return _T.T @ Jc @ _T, _T.T @ Kc @ _T
        scf = rhf_df(int1e.S, int1e.hcore, None, nelec=mol.nelectron, enuc=mol.energy_nuc(), max_cycle=max_cycle,
                     conv_tol=conv_tol, conv_tol_dm=conv_tol_dm, dm0=dm0, mo_coeff0=mo_coeff0, precision="fp64",
                     jk_fn=jk, profile=prof)
        df_B = None
    if prof is not None:
        prof["wall_s"] = time.perf_counter() - t0
    return RHFDFRunResult(mol=mol, ao_basis=ao, aux_basis=aux, int1e=int1e, df_B=df_B, df_L=L, scf=scf,
                          two_e_backend=tb, basis_name=basis, profile=prof)

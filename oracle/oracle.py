"""ORACLE -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.  Nothing in
``asuka_b200`` imports it.

CPU restatement of the reference's DF two-electron path:

* integrals: ``liboracle_rys.so`` built from ``rys_oracle.c`` (Rys quadrature,
  see that file's header for the reference lines it follows);
* ``df_build``      <- ``build_df_B_from_cueri_packed_bases_cpu``
                       (``asuka/integrals/cueri_df_cpu.py:331-537``): metric, 3c,
                       Cholesky without shift, whitening B = X L^-T;
* ``df_JK``         <- ``_df_JK`` D-driven branch (``asuka/hf/df_scf.py:516-662``);
* ``rhf_df``        <- ``rhf_df`` materialised branch (``asuka/hf/df_scf.py:871-1429``):
                       S^-1/2 orthogonaliser, core guess, one predictor Fock cycle,
                       DIIS on FDS - SDF, E = 1/2 tr(D_new (h + F));
* ``grad_2e``       <- ``compute_df_gradient_contributions_analytic_packed_bases``
                       (``asuka/integrals/grad.py:114-723``) with
                       ``df_whiten_adjoint_Qmn`` / ``chol_lower_adjoint``
                       (``asuka/integrals/df_adjoint.py:172-235,322-361``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
from scipy.linalg import solve_triangular

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    """Compile liboracle_rys.so in place (gcc + OpenMP + libquadmath)."""
    subprocess.run(["make", "-C", HERE, "CC=gcc"], check=True, capture_output=True)
    return os.path.join(HERE, "liboracle_rys.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle_rys.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
    return _LIB


def _p(a, t=np.float64):
    a = np.ascontiguousarray(a, dtype=t)
    return a, a.ctypes.data_as(_d if t == np.float64 else _i)


def _bargs(b):
    keep = []
    out = []
    for arr, t in ((b.shell_cxyz, np.float64), (b.shell_l, np.int32), (b.shell_prim_start, np.int32),
                   (b.shell_nprim, np.int32), (b.prim_exp, np.float64), (b.prim_coef, np.float64)):
        a, p = _p(arr, t)
        keep.append(a)
        out.append(p)
    return keep, out


def _ncart(l):
    return (l + 1) * (l + 2) // 2


def rys_roots(n: int, T: float) -> tuple[np.ndarray, np.ndarray]:
    r = np.zeros(n)
    w = np.zeros(n)
    lib().oracle_rys_roots(ctypes.c_int(n), ctypes.c_double(T), r.ctypes.data_as(_d), w.ctypes.data_as(_d))
    return r, w


def boys(T: float, mmax: int) -> np.ndarray:
    out = np.zeros(mmax + 1)
    lib().oracle_boys(ctypes.c_double(T), ctypes.c_int(mmax), out.ctypes.data_as(_d))
    return out


def tile_3c(ao, aux, A: int, B: int, P: int) -> np.ndarray:
    k1, a1 = _bargs(ao)
    k2, a2 = _bargs(aux)
    nA, nB, nP = _ncart(int(ao.shell_l[A])), _ncart(int(ao.shell_l[B])), _ncart(int(aux.shell_l[P]))
    out = np.zeros(nA * nB * nP)
    lib().oracle_tile_3c(*a1, *a2, ctypes.c_int(A), ctypes.c_int(B), ctypes.c_int(P), out.ctypes.data_as(_d))
    return out.reshape((nA, nB, nP))


def tile_2c(aux, P: int, Q: int) -> np.ndarray:
    k2, a2 = _bargs(aux)
    nP, nQ = _ncart(int(aux.shell_l[P])), _ncart(int(aux.shell_l[Q]))
    out = np.zeros(nP * nQ)
    lib().oracle_tile_2c(*a2, ctypes.c_int(P), ctypes.c_int(Q), out.ctypes.data_as(_d))
    return out.reshape((nP, nQ))


def int3c_full(ao, aux, sp) -> np.ndarray:
    """X[mu, nu, P] = (mu nu|P), both AO orders (``cueri_df_cpu.py:449-516``)."""
    k1, a1 = _bargs(ao)
    k2, a2 = _bargs(aux)
    s1, ps1 = _p(ao.shell_ao_start, np.int32)
    s2, ps2 = _p(aux.shell_ao_start, np.int32)
    spA, pA = _p(sp.sp_A, np.int32)
    spB, pB = _p(sp.sp_B, np.int32)
    nao, naux = ao.nao, aux.nao
    X = np.zeros((nao, nao, naux))
    lib().oracle_int3c_full(*a1, ps1, ctypes.c_int(ao.nshell), ctypes.c_int(nao), *a2, ps2, ctypes.c_int(aux.nshell),
                            ctypes.c_int(naux), pA, pB, ctypes.c_int(sp.nsp), X.ctypes.data_as(_d))
    return X


def metric_full(aux) -> np.ndarray:
    k2, a2 = _bargs(aux)
    s2, ps2 = _p(aux.shell_ao_start, np.int32)
    naux = aux.nao
    V = np.zeros((naux, naux))
    lib().oracle_metric_full(*a2, ps2, ctypes.c_int(aux.nshell), ctypes.c_int(naux), V.ctypes.data_as(_d))
    return V


def df_build(ao, aux, sp):
    """(V, L, X, B) with B[mu,nu,Q] = sum_P X[mu,nu,P] L^-T[P,Q]; no metric shift (CPU semantics)."""
    V = metric_full(aux)
    V = 0.5 * (V + V.T)
    X = int3c_full(ao, aux, sp)
    L = np.linalg.cholesky(V)
    nao, naux = ao.nao, aux.nao
    BT = solve_triangular(L, X.reshape(nao * nao, naux).T, lower=True)
    return V, L, X, np.ascontiguousarray(BT.T).reshape(nao, nao, naux)


def df_JK(B: np.ndarray, D: np.ndarray):
    nao, _, naux = B.shape
    B2 = B.reshape(nao * nao, naux)
    J = (B2 @ (B2.T @ D.reshape(-1))).reshape(nao, nao)
    BQ = B.transpose(2, 0, 1)
    K = np.einsum("Qmk,kl,Qln->mn", BQ, D, BQ, optimize=True)
    return 0.5 * (J + J.T), 0.5 * (K + K.T)


def energy_2e(B: np.ndarray, D: np.ndarray) -> float:
    J, K = df_JK(B, D)
    return 0.5 * float(np.sum(D * J)) - 0.25 * float(np.sum(D * K))


class _DIIS:
    def __init__(self, nvec=8):
        self.F, self.e, self.n = [], [], nvec

    def push(self, F, e):
        self.F.append(F)
        self.e.append(e)
        if len(self.F) > self.n:
            self.F.pop(0)
            self.e.pop(0)

    def extrapolate(self):
        n = len(self.F)
        if n < 2:
            return self.F[-1]
        E = np.stack([e.ravel() for e in self.e])
        G = E @ E.T
        G = G / max(np.abs(G).max(), 1e-300)
        Bm = np.zeros((n + 1, n + 1))
        Bm[:n, :n] = G
        Bm[:n, n] = Bm[n, :n] = -1.0
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        c = np.linalg.solve(Bm, rhs)[:n]
        c = c / c.sum()
        return np.tensordot(c, np.stack(self.F), axes=(0, 0))


def rhf_df(S, h, B, nelec: int, enuc: float, max_cycle=50, conv_tol=1e-10, conv_tol_dm=1e-8):
    s, U = np.linalg.eigh(0.5 * (S + S.T))
    Xo = U @ np.diag(s**-0.5) @ U.T
    nocc = nelec // 2
    nao = S.shape[0]
    occ = np.zeros(nao)
    occ[:nocc] = 2.0

    def solve(F):
        e, Cp = np.linalg.eigh(Xo.T @ (0.5 * (F + F.T)) @ Xo)
        return e, Xo @ Cp

    def dens(C):
        return (C * occ) @ C.T

    eps, C = solve(h)
    D = dens(C)
    # one predictor Fock cycle (df_scf.py:1116-1200)
    J, K = df_JK(B, D)
    eps, C = solve(h + J - 0.5 * K)
    D = dens(C)
    diis = _DIIS()
    e_last = None
    for cycle in range(1, max_cycle + 1):
        J, K = df_JK(B, D)
        F = h + J - 0.5 * K
        F = 0.5 * (F + F.T)
        M = F @ D @ S
        diis.push(F, M - M.T)
        F = diis.extrapolate()
        F = 0.5 * (F + F.T)
        eps, C = solve(F)
        Dn = dens(C)
        e_tot = 0.5 * float(np.trace(Dn @ (h + F))) + enuc
        dm_err = float(np.linalg.norm(Dn - D))
        de = abs(e_tot - e_last) if e_last is not None else np.inf
        D, e_last = Dn, e_tot
        if de < conv_tol and dm_err < conv_tol_dm:
            return dict(e_tot=e_tot, converged=True, niter=cycle, mo_energy=eps, mo_coeff=C, mo_occ=occ, D=D)
    return dict(e_tot=e_last, converged=False, niter=max_cycle, mo_energy=eps, mo_coeff=C, mo_occ=occ, D=D)


def bar_B_rhf(B: np.ndarray, D: np.ndarray) -> np.ndarray:
    """dE_2e/dB in (naux, nao, nao): rho_Q D - 1/2 D B_Q D."""
    rho = np.einsum("mnQ,mn->Q", B, D)
    return rho[:, None, None] * D[None] - 0.5 * np.einsum("mk,knQ,nl->Qml", D, B, D, optimize=True)


def grad_2e(ao, aux, sp, B, barL_ao, L, natm: int) -> np.ndarray:
    """DF two-electron gradient contraction (natm, 3)."""
    nao, _, naux = B.shape
    tmp = solve_triangular(L, barL_ao.reshape(naux, nao * nao), lower=True, trans="T")
    bar_X = tmp.T.reshape(nao, nao, naux)
    bar_Lc = np.tril(-(tmp @ B.reshape(nao * nao, naux)))
    G = np.tril(L.T @ bar_Lc)
    G[np.diag_indices(naux)] *= 0.5
    t2 = solve_triangular(L, G, lower=True, trans="T")
    bar_V = solve_triangular(L, t2.T, lower=True, trans="T").T
    bar_V = 0.5 * (bar_V + bar_V.T)
    bar_X = np.ascontiguousarray(0.5 * (bar_X + bar_X.transpose(1, 0, 2)))
    grad = np.zeros((natm, 3))
    k1, a1 = _bargs(ao)
    k2, a2 = _bargs(aux)
    s1, ps1 = _p(ao.shell_ao_start, np.int32)
    s2, ps2 = _p(aux.shell_ao_start, np.int32)
    t1, pt1 = _p(ao.shell_atom, np.int32)
    t2_, pt2 = _p(aux.shell_atom, np.int32)
    spA, pA = _p(sp.sp_A, np.int32)
    spB, pB = _p(sp.sp_B, np.int32)
    bx, pbx = _p(bar_X)
    bv, pbv = _p(bar_V)
    lib().oracle_deriv3c_full(*a1, ps1, pt1, ctypes.c_int(nao), *a2, ps2, pt2, ctypes.c_int(aux.nshell),
                              ctypes.c_int(naux), pA, pB, ctypes.c_int(sp.nsp), pbx, ctypes.c_int(natm),
                              grad.ctypes.data_as(_d))
    lib().oracle_deriv2c_full(*a2, ps2, pt2, ctypes.c_int(aux.nshell), ctypes.c_int(naux), pbv, ctypes.c_int(natm),
                              grad.ctypes.data_as(_d))
    return grad

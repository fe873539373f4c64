"""One-electron integrals S, T, V over the packed Cartesian AO basis.

The reference builds these on the host (``asuka/integrals/int1e_cart.py:379``
``build_S_cart``, ``:487`` ``build_T_cart``, ``:1031`` ``build_V_cart``); they are
not on the DF hot path.  Here S and T use the Obara-Saika 1D overlap
recurrences on the host (numpy, vectorised over primitive pairs of a class),
and V runs on the GPU through the same Rys kernel as the DF integrals: a
nucleus is an s "aux" shell of exponent 1e30 with the normalised coefficient
(zeta/pi)^(3/2), which reproduces the point-charge limit exactly in FP64
(p/zeta <= 1e-25).  The nuclear-attraction gradient then comes from the same
derivative kernel, including the operator-centre (Hellmann-Feynman) term.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .basis import BasisCartSoA, build_shell_pairs_l_order, cart_components, ncart

POINT_CHARGE_EXP = 1.0e30


@dataclass
class Int1eResult:
    S: np.ndarray
    T: np.ndarray
    V: np.ndarray

    @property
    def hcore(self) -> np.ndarray:
        return self.T + self.V


def _overlap_1d(lmax_a: int, lmax_b: int, PA: np.ndarray, PB: np.ndarray, p: np.ndarray) -> np.ndarray:
    """E[..., i, j] = int x_A^i x_B^j exp(-p (x-P)^2) dx / s00 via Obara-Saika."""
    n = PA.shape[0]
    S = np.zeros((n, lmax_a + 1, lmax_b + 1))
    S[:, 0, 0] = 1.0
    h = 0.5 / p
    for i in range(lmax_a + 1):
        for j in range(lmax_b + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = PA * S[:, i - 1, j]
                if i > 1:
                    v = v + (i - 1) * h * S[:, i - 2, j]
                if j > 0:
                    v = v + j * h * S[:, i - 1, j - 1]
            else:
                v = PB * S[:, i, j - 1]
                if j > 1:
                    v = v + (j - 1) * h * S[:, i, j - 2]
            S[:, i, j] = v
    return S


def build_S_T(ao: BasisCartSoA) -> tuple[np.ndarray, np.ndarray]:
    """Overlap and kinetic matrices (nao, nao)."""
    nao = ao.nao
    S = np.zeros((nao, nao))
    T = np.zeros((nao, nao))
    sp = build_shell_pairs_l_order(ao)
    la_all = ao.shell_l[sp.sp_A]
    lb_all = ao.shell_l[sp.sp_B]
    for la in np.unique(la_all):
        for lb in np.unique(lb_all):
            sel = np.nonzero((la_all == la) & (lb_all == lb))[0]
            if sel.size == 0:
                continue
            A = sp.sp_A[sel]
            B = sp.sp_B[sel]
            # expand primitive pairs
            na_p = ao.shell_nprim[A]
            nb_p = ao.shell_nprim[B]
            npair = na_p * nb_p
            owner = np.repeat(np.arange(sel.size), npair)
            loc = np.arange(owner.size) - np.repeat(np.cumsum(npair) - npair, npair)
            ia = loc // nb_p[owner]
            ib = loc - ia * nb_p[owner]
            pa = ao.shell_prim_start[A[owner]] + ia
            pb = ao.shell_prim_start[B[owner]] + ib
            a = ao.prim_exp[pa]
            b = ao.prim_exp[pb]
            cab = ao.prim_coef[pa] * ao.prim_coef[pb]
            RA = ao.shell_cxyz[A[owner]]
            RB = ao.shell_cxyz[B[owner]]
            p = a + b
            mu = a * b / p
            P = (a[:, None] * RA + b[:, None] * RB) / p[:, None]
            AB2 = ((RA - RB) ** 2).sum(1)
            s00 = (np.pi / p) ** 1.5 * np.exp(-mu * AB2) * cab
            E = [_overlap_1d(int(la), int(lb) + 2, P[:, d] - RA[:, d], P[:, d] - RB[:, d], p) for d in range(3)]
            ca = cart_components(int(la))
            cb = cart_components(int(lb))
            nA, nB = ca.shape[0], cb.shape[0]
            Sp = np.empty((owner.size, nA, nB))
            Tp = np.empty((owner.size, nA, nB))
            for i in range(nA):
                for j in range(nB):
                    sx = [E[d][:, ca[i, d], cb[j, d]] for d in range(3)]
                    # -1/2 <i|d^2/dx^2|j> = -1/2 [j(j-1) S_{i,j-2} - 2b(2j+1) S_ij + 4b^2 S_{i,j+2}]
                    kx = []
                    for d in range(3):
                        jj = int(cb[j, d])
                        t = -2.0 * b * (2 * jj + 1) * E[d][:, ca[i, d], jj] + 4.0 * b * b * E[d][:, ca[i, d], jj + 2]
                        if jj >= 2:
                            t = t + jj * (jj - 1) * E[d][:, ca[i, d], jj - 2]
                        kx.append(-0.5 * t)
                    Sp[:, i, j] = sx[0] * sx[1] * sx[2]
                    Tp[:, i, j] = kx[0] * sx[1] * sx[2] + sx[0] * kx[1] * sx[2] + sx[0] * sx[1] * kx[2]
            Sp *= s00[:, None, None]
            Tp *= s00[:, None, None]
            Ss = np.zeros((sel.size, nA, nB))
            Ts = np.zeros((sel.size, nA, nB))
            np.add.at(Ss, owner, Sp)
            np.add.at(Ts, owner, Tp)
            a0 = ao.shell_ao_start[A][:, None, None] + np.arange(nA)[None, :, None]
            b0 = ao.shell_ao_start[B][:, None, None] + np.arange(nB)[None, None, :]
            a0, b0 = np.broadcast_arrays(a0, b0)
            S[a0, b0] = Ss
            S[b0, a0] = Ss
            T[a0, b0] = Ts
            T[b0, a0] = Ts
    return S, T


def point_charge_basis(coords_bohr: np.ndarray) -> BasisCartSoA:
    """One s shell per nucleus representing a unit point charge (see module docstring)."""
    R = np.asarray(coords_bohr, dtype=np.float64).reshape((-1, 3))
    n = R.shape[0]
    coef = (POINT_CHARGE_EXP / np.pi) ** 1.5
    return BasisCartSoA(shell_cxyz=R.copy(), shell_prim_start=np.arange(n, dtype=np.int32),
                        shell_nprim=np.ones(n, np.int32), shell_l=np.zeros(n, np.int32),
                        shell_ao_start=np.arange(n, dtype=np.int32), prim_exp=np.full(n, POINT_CHARGE_EXP),
                        prim_coef=np.full(n, coef), shell_atom=np.arange(n, dtype=np.int32))


def nuclear_engine(ao: BasisCartSoA, coords_bohr: np.ndarray, device=None):
    from .df import DFEngine

    return DFEngine(ao, point_charge_basis(coords_bohr), device=device)


def build_V(ao: BasisCartSoA, coords_bohr: np.ndarray, charges: np.ndarray, device=None):
    """V[mu,nu] = -sum_C Z_C (mu nu | 1/|r-C|), computed on the GPU; returns a torch tensor."""
    import torch

    eng = nuclear_engine(ao, coords_bohr, device=device)
    Xc = eng.int3c("Qmn")  # (natm, nao, nao)
    Z = torch.as_tensor(np.asarray(charges, dtype=np.float64), device=Xc.device)
    return -torch.einsum("c,cmn->mn", Z, Xc)


def build_int1e(ao: BasisCartSoA, coords_bohr: np.ndarray, charges: np.ndarray, device=None) -> Int1eResult:
    S, T = build_S_T(ao)
    V = build_V(ao, coords_bohr, charges, device=device).cpu().numpy()
    return Int1eResult(S=S, T=T, V=V)

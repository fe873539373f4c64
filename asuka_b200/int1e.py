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

import dataclasses
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


def _pair_prims(ao: BasisCartSoA, A: np.ndarray, B: np.ndarray):
    """Primitive pairs of the shell pairs (A[i], B[i]): owner index, exponents, coefficient product,
    centres, P and the s-type overlap prefactor."""
    na_p = ao.shell_nprim[A]
    nb_p = ao.shell_nprim[B]
    npair = na_p * nb_p
    owner = np.repeat(np.arange(A.size), npair)
    loc = np.arange(owner.size) - np.repeat(np.cumsum(npair) - npair, npair)
    ia = loc // nb_p[owner]
    ib = loc - ia * nb_p[owner]
    pa = ao.shell_prim_start[A[owner]] + ia
    pb = ao.shell_prim_start[B[owner]] + ib
    a = ao.prim_exp[pa]
    b = ao.prim_exp[pb]
    RA = ao.shell_cxyz[A[owner]]
    RB = ao.shell_cxyz[B[owner]]
    p = a + b
    P = (a[:, None] * RA + b[:, None] * RB) / p[:, None]
    s00 = (np.pi / p) ** 1.5 * np.exp(-a * b / p * ((RA - RB) ** 2).sum(1)) * ao.prim_coef[pa] * ao.prim_coef[pb]
    return owner, a, b, RA, RB, p, P, s00


def _kinetic_1d(E: np.ndarray, b: np.ndarray, i: int, j: int) -> np.ndarray:
    """-1/2 <i| d^2/dx^2 |j> / s00 from the 1D overlaps E[:, i, j'] (j' up to j + 2)."""
    t = -2.0 * b * (2 * j + 1) * E[:, i, j] + 4.0 * b * b * E[:, i, j + 2]
    if j >= 2:
        t = t + j * (j - 1) * E[:, i, j - 2]
    return -0.5 * t


def contract_dS_T_cart(ao: BasisCartSoA, M_S: np.ndarray | None, M_T: np.ndarray | None,
                       shell_atom: np.ndarray, natm: int) -> tuple[np.ndarray, np.ndarray]:
    """(sum M_S . dS/dR, sum M_T . dT/dR), each (natm, 3), for symmetric M_S, M_T (nao, nao).

    Per l-ordered shell pair (A, B) the derivative with respect to centre A uses
    d/dA_x x_A^i = 2a x_A^(i+1) - i x_A^(i-1) on the bra; centre B gets the negative
    (the operators have no centre); off-diagonal pairs count twice (M symmetric).
    The reference computes the same contractions in ``asuka/integrals/int1e_cart.py:1452``
    (``contract_dS_cart``) and the kinetic half of ``:1738`` (``contract_dhcore_cart``).
    """
    gS = np.zeros((natm, 3))
    gT = np.zeros((natm, 3))
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
            owner, a, b, RA, RB, p, P, s00 = _pair_prims(ao, A, B)
            la_, lb_ = int(la), int(lb)
            E = [_overlap_1d(la_ + 1, lb_ + 2, P[:, d] - RA[:, d], P[:, d] - RB[:, d], p) for d in range(3)]
            ca = cart_components(la_)
            cb = cart_components(lb_)
            nA, nB = ca.shape[0], cb.shape[0]
            a0 = ao.shell_ao_start[A]
            b0 = ao.shell_ao_start[B]
            fac = np.where(A != B, 2.0, 1.0)
            for i in range(nA):
                for j in range(nB):
                    ii, jj = ca[i], cb[j]
                    s = [E[d][:, ii[d], jj[d]] for d in range(3)]
                    t = [_kinetic_1d(E[d], b, int(ii[d]), int(jj[d])) for d in range(3)]
                    ws = M_S[a0 + i, b0 + j][owner] * fac[owner] if M_S is not None else None
                    wt = M_T[a0 + i, b0 + j][owner] * fac[owner] if M_T is not None else None
                    for d in range(3):
                        o1, o2 = (d + 1) % 3, (d + 2) % 3
                        k = int(ii[d])
                        ds = 2.0 * a * E[d][:, k + 1, jj[d]]
                        dt = 2.0 * a * _kinetic_1d(E[d], b, k + 1, int(jj[d]))
                        if k > 0:
                            ds = ds - k * E[d][:, k - 1, jj[d]]
                            dt = dt - k * _kinetic_1d(E[d], b, k - 1, int(jj[d]))
                        dS = ds * s[o1] * s[o2] * s00
                        dT = (dt * s[o1] * s[o2] + ds * t[o1] * s[o2] + ds * s[o1] * t[o2]) * s00
                        if ws is not None:
                            v = np.bincount(owner, weights=ws * dS, minlength=A.size)
                            np.add.at(gS[:, d], shell_atom[A], v)
                            np.add.at(gS[:, d], shell_atom[B], -v)
                        if wt is not None:
                            v = np.bincount(owner, weights=wt * dT, minlength=A.size)
                            np.add.at(gT[:, d], shell_atom[A], v)
                            np.add.at(gT[:, d], shell_atom[B], -v)
    return gS, gT


def _shell_atom(ao: BasisCartSoA, coords: np.ndarray, shell_atom) -> np.ndarray:
    if shell_atom is not None:
        return np.asarray(shell_atom, dtype=np.int64).ravel()
    if ao.shell_atom is not None:
        return np.asarray(ao.shell_atom, dtype=np.int64)
    from .basis import shell_to_atom_map

    return np.asarray(shell_to_atom_map(ao, coords), dtype=np.int64)


def contract_dS_cart(basis, *, atom_coords_bohr, M, shell_atom=None, contract_backend: str = "auto") -> np.ndarray:
    """gS[natm, 3] = sum_{mu,nu} dS[A, x, mu, nu] M[mu, nu] without building dS
    (``asuka/integrals/int1e_cart.py:1452``); M symmetric (nao, nao)."""
    from .basis import from_reference_like

    ao = basis if isinstance(basis, BasisCartSoA) else from_reference_like(basis)
    R = np.asarray(atom_coords_bohr, dtype=np.float64).reshape((-1, 3))
    Mh = M.detach().cpu().numpy() if hasattr(M, "detach") else np.asarray(M, dtype=np.float64)
    if Mh.shape != (ao.nao, ao.nao):
        raise ValueError(f"M must have shape ({ao.nao}, {ao.nao})")
    Ms = 0.5 * (Mh + Mh.T)
    gS, _ = contract_dS_T_cart(ao, Ms, None, _shell_atom(ao, R, shell_atom), R.shape[0])
    return gS


def contract_dV_cart(ao: BasisCartSoA, coords_bohr: np.ndarray, charges: np.ndarray, M: np.ndarray,
                     include_operator_deriv: bool = True, device=None) -> np.ndarray:
    """sum M . dV/dR (natm, 3) on the GPU through the Rys derivative kernel.

    Each nucleus is the point-charge s shell of ``point_charge_basis``; the adjoint of its
    (mu nu | C) block is -Z_C M.  The kernel's centre-C term (translational invariance) is
    the operator-centre (Hellmann-Feynman) derivative; with ``include_operator_deriv=False``
    the nuclei are attributed to a discarded extra atom, which leaves the basis-centre terms.
    """
    import torch

    from .df import DFEngine

    R = np.asarray(coords_bohr, dtype=np.float64).reshape((-1, 3))
    natm = R.shape[0]
    pc = point_charge_basis(R)
    if not include_operator_deriv:
        pc = dataclasses.replace(pc, shell_atom=np.full(natm, natm, dtype=np.int32))
    eng = DFEngine(ao, pc, device=device)
    dev = eng.device
    Mt = torch.as_tensor(0.5 * (M + M.T), dtype=torch.float64, device=dev)
    Z = torch.as_tensor(np.asarray(charges, dtype=np.float64), device=dev)
    bar = (-Z.view(-1, 1, 1) * Mt.view(1, ao.nao, ao.nao)).contiguous()
    g = torch.zeros((eng.natm, 3), dtype=torch.float64, device=dev)
    eng.deriv3c(bar, g, layout="Qmn")
    return g[:natm].cpu().numpy()


def contract_dhcore_cart(basis, *, atom_coords_bohr, atom_charges, M, shell_atom=None,
                         include_operator_deriv: bool = True, contract_backend: str = "auto") -> np.ndarray:
    """gh1[natm, 3] = sum_{mu,nu} d(T + V)[A, x, mu, nu] M[mu, nu] (``asuka/integrals/int1e_cart.py:1738``).

    The kinetic part runs on the host, the nuclear-attraction part on the GPU (basis-centre
    and, with ``include_operator_deriv``, operator-centre derivatives).
    """
    from .basis import from_reference_like

    ao = basis if isinstance(basis, BasisCartSoA) else from_reference_like(basis)
    R = np.asarray(atom_coords_bohr, dtype=np.float64).reshape((-1, 3))
    Z = np.asarray(atom_charges, dtype=np.float64).ravel()
    if Z.shape != (R.shape[0],):
        raise ValueError("atom_charges must have shape (natm,)")
    Mh = M.detach().cpu().numpy() if hasattr(M, "detach") else np.asarray(M, dtype=np.float64)
    if Mh.shape != (ao.nao, ao.nao):
        raise ValueError(f"M must have shape ({ao.nao}, {ao.nao})")
    Ms = 0.5 * (Mh + Mh.T)
    sa = _shell_atom(ao, R, shell_atom)
    ao_a = dataclasses.replace(ao, shell_atom=sa.astype(np.int32))
    _, gT = contract_dS_T_cart(ao_a, None, Ms, sa, R.shape[0])
    return gT + contract_dV_cart(ao_a, R, Z, Ms, include_operator_deriv=include_operator_deriv)


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

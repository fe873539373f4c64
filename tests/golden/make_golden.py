"""Generate the golden fixtures in this directory from the ASUKA reference.

Runs only where the reference (with its CPU Cython extensions built) is
importable, e.g.::

    PYTHONPATH=/tmp/asuka_ref OMP_NUM_THREADS=8 python tests/golden/make_golden.py [case ...]

Every fixture is produced by the reference's own public CPU path:

* ``run_hf_df(mol, method='rhf', backend='cpu', df=True, auxbasis='ricd')``
  (``asuka/frontend/scf.py:1219``) for the SCF energy, orbitals, S, hcore, the
  DF metric and the whitened factors B;
* ``asuka.hf.df_scf._df_JK`` (``asuka/hf/df_scf.py:516``) for J and K at the
  converged density;
* ``compute_df_gradient_contributions_analytic_packed_bases(backend='cpu')``
  (``asuka/integrals/grad.py:114``) for the DF two-electron gradient at fixed
  density, with ``bar_L[Q] = rho_Q D - 1/2 D B_Q D``;
* ``_eri_rys_cpu.eri_rys_tile_cart_sp_batch_cy`` for single (ab|P) and (P|Q)
  tiles of every angular class of H2O/ma-QZVP;
* ``_eri_rys_cpu.rys_roots_weights_cy`` for reference roots/weights;
* ``run_hf_df(mol, method='uhf', backend='cpu', df=True, auxbasis='ricd')`` for
  the open-shell cases (converged energies and orbital energies; the
  reference's UHF needs a few hundred cycles from the core guess here, hence
  max_cycle=300);
* ``asuka.cueri.sph.cart2sph_matrix`` (``asuka/cueri/sph.py:95``) for the
  Cartesian-to-spherical transforms of l = 0..5 (pure Python; importable
  straight from the source tree).

Geometries come from ``asuka_b200.geometry`` so that tests rebuild identical
inputs without the reference.
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from asuka_b200 import geometry as geo  # noqa: E402


def _ref_mol(mol):
    from asuka.frontend.molecule import Molecule

    return Molecule.from_atoms([(el, xyz) for el, xyz in mol.atoms_bohr], unit="Bohr", basis=mol.basis, cart=True)


def _tril_pack(X):
    nao = X.shape[0]
    i, j = np.tril_indices(nao)
    return X[i, j]


def scf_case(name: str, mol, with_grad: bool = True) -> None:
    from asuka.frontend.scf import run_hf_df
    from asuka.hf.df_scf import _df_JK
    from asuka.integrals.grad import compute_df_gradient_contributions_analytic_packed_bases

    rmol = _ref_mol(mol)
    prof: dict = {}
    t0 = time.perf_counter()
    res = run_hf_df(rmol, method="rhf", backend="cpu", df=True, auxbasis="ricd", conv_tol=1e-10, profile=prof)
    t_scf = time.perf_counter() - t0
    B = np.asarray(res.df_B)
    L = np.asarray(res.df_L)
    nao, _, naux = B.shape
    C = np.asarray(res.mo_coeff)
    occ = np.asarray(res.mo_occ)
    D = (C * occ[None, :]) @ C.T
    J, K = _df_JK(B, D, want_J=True, want_K=True)
    rho = np.einsum("mnQ,mn->Q", B, D)
    E2 = 0.5 * float(np.sum(D * J)) - 0.25 * float(np.sum(D * K))
    X = np.einsum("mnP,QP->mnQ", B, L)  # unwhitened (mu nu|P) = B L^T
    out = dict(
        elements=np.array(mol.elements),
        coords_bohr=mol.coords_bohr,
        basis=np.array(mol.basis),
        S=np.asarray(res.int1e.S),
        hcore=np.asarray(res.int1e.hcore),
        e_nuc=np.array(res.e_nuc),
        e_tot=np.array(res.e_tot),
        niter=np.array(res.scf.niter),
        mo_energy=np.asarray(res.mo_energy),
        mo_coeff=C,
        mo_occ=occ,
        D=D,
        J=np.asarray(J),
        K=np.asarray(K),
        E2=np.array(E2),
        V=L @ L.T,
        X_tril=np.stack([_tril_pack(X[:, :, P]) for P in range(naux)], axis=0),  # (naux, ntri)
        t_scf_s=np.array(t_scf),
    )
    if with_grad:
        barL = rho[:, None, None] * D[None, :, :] - 0.5 * np.einsum("mk,knQ,nl->Qml", D, B, D)
        t0 = time.perf_counter()
        g2 = compute_df_gradient_contributions_analytic_packed_bases(
            res.ao_basis, res.aux_basis, atom_coords_bohr=mol.coords_bohr, B_ao=B, bar_L_ao=barL, L_chol=L,
            backend="cpu")
        out["grad_2e"] = np.asarray(g2)
        out["t_grad_s"] = np.array(time.perf_counter() - t0)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: nao={nao} naux={naux} E={res.e_tot:.12f} iters={res.scf.niter} t_scf={t_scf:.1f}s", flush=True)


def scf_grad_small_case(name: str, mol, with_grad: bool = True) -> None:
    """Like ``scf_case`` for systems whose 3c tensor is too large for a fixture.

    Keeps only what the parity tests compare: the converged energy, the orbital
    energies, the weighted occupied orbitals Cw = C_occ sqrt(occ) (the density at
    which the two-electron energy and gradient are evaluated), E_2e at that
    density, and the reference's DF two-electron gradient there.
    """
    from asuka.frontend.scf import run_hf_df
    from asuka.integrals.grad import compute_df_gradient_contributions_analytic_packed_bases

    rmol = _ref_mol(mol)
    t0 = time.perf_counter()
    res = run_hf_df(rmol, method="rhf", backend="cpu", df=True, auxbasis="ricd", conv_tol=1e-10)
    t_scf = time.perf_counter() - t0
    B = np.asarray(res.df_B)
    L = np.asarray(res.df_L)
    nao, _, naux = B.shape
    C = np.asarray(res.mo_coeff)
    occ = np.asarray(res.mo_occ)
    nocc = int((occ > 0).sum())
    Cw = C[:, :nocc] * np.sqrt(occ[:nocc])[None, :]
    D = Cw @ Cw.T
    rho = np.tensordot(D, B, axes=([0, 1], [0, 1]))
    # E_2e = 1/2 rho.rho - 1/4 sum_Q |Cw^T B_Q Cw|^2 (the DF Coulomb and exchange energies at D)
    M = np.tensordot(np.tensordot(Cw, B, axes=(0, 0)), Cw, axes=(1, 0))  # (i, Q, j)
    E2 = 0.5 * float(rho @ rho) - 0.25 * float(np.sum(M * M))
    del M
    out = dict(elements=np.array(mol.elements), coords_bohr=mol.coords_bohr, basis=np.array(mol.basis),
               nao=np.array(nao), naux=np.array(naux), e_nuc=np.array(res.e_nuc), e_tot=np.array(res.e_tot),
               niter=np.array(res.scf.niter), mo_energy=np.asarray(res.mo_energy), Cw=Cw, E2=np.array(E2),
               t_scf_s=np.array(t_scf), threads=np.array(int(os.environ.get("OMP_NUM_THREADS", "0"))))
    if with_grad:
        # bar_L[Q] = dE_2e/dB_Q = rho_Q D - 1/2 D B_Q D
        DBD = np.tensordot(np.tensordot(D, B, axes=(1, 0)), D, axes=(1, 0))  # (m, Q, l)
        barL = np.ascontiguousarray(DBD.transpose(1, 0, 2))
        del DBD
        barL *= -0.5
        barL += rho[:, None, None] * D[None, :, :]
        t0 = time.perf_counter()
        g2 = compute_df_gradient_contributions_analytic_packed_bases(
            res.ao_basis, res.aux_basis, atom_coords_bohr=mol.coords_bohr, B_ao=B, bar_L_ao=barL, L_chol=L,
            backend="cpu")
        out["grad_2e"] = np.asarray(g2)
        out["t_grad_s"] = np.array(time.perf_counter() - t0)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: nao={nao} naux={naux} E={res.e_tot:.12f} iters={res.scf.niter} t_scf={t_scf:.1f}s", flush=True)


def int1e_grad_case(name: str, mol) -> None:
    """The reference's one-electron gradient contractions (``asuka/integrals/int1e_cart.py:1452,1738``)
    with a seeded random symmetric M, and its nuclear-repulsion gradient (``molecule.py:148``)."""
    from asuka.frontend.one_electron import build_ao_basis_cart
    from asuka.integrals.int1e_cart import contract_dhcore_cart, contract_dS_cart

    rmol = _ref_mol(mol)
    ao, _ = build_ao_basis_cart(rmol, basis=mol.basis, expand_contractions=True)
    nao = int(np.asarray(ao.shell_ao_start)[-1] + (np.asarray(ao.shell_l)[-1] + 1) * (np.asarray(ao.shell_l)[-1] + 2) // 2)
    rng = np.random.default_rng(7)
    M = rng.standard_normal((nao, nao))
    M = 0.5 * (M + M.T)
    Z = np.array([float(z) for z in rmol.atom_charges()]) if hasattr(rmol, "atom_charges") else None
    if Z is None:
        from asuka.frontend.molecule import atomic_number

        Z = np.array([float(atomic_number(a)) for a, _ in rmol.atoms_bohr])
    R = np.asarray(mol.coords_bohr)
    gS = contract_dS_cart(ao, atom_coords_bohr=R, M=M, contract_backend="cpu")
    gH = contract_dhcore_cart(ao, atom_coords_bohr=R, atom_charges=Z, M=M, contract_backend="cpu")
    gH0 = contract_dhcore_cart(ao, atom_coords_bohr=R, atom_charges=Z, M=M, include_operator_deriv=False,
                               contract_backend="cpu")
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), elements=np.array(mol.elements), coords_bohr=R,
                        basis=np.array(mol.basis), M=M, Z=Z, gS=np.asarray(gS), gH=np.asarray(gH),
                        gH_basis_only=np.asarray(gH0), g_nuc=np.asarray(rmol.energy_nuc_grad()))
    print(f"{name}: nao={nao}", flush=True)


def casscf_barl_case(name: str) -> None:
    """The reference's CASSCF DF-gradient adjoint builders (``asuka/mcscf/nuc_grad_df.py:2387-2600``,
    ``_build_bar_L_casscf_df`` for B in mnQ and in packed Qp) on seeded inputs: a symmetric B
    (nao, nao, naux), core and active densities, active orbitals and a symmetric 2-RDM."""
    from asuka.integrals.df_packed_s2 import pack_B_to_Qp
    from asuka.mcscf.nuc_grad_df import _build_bar_L_casscf_df

    rng = np.random.default_rng(11)
    nao, naux, ncore, ncas = 24, 61, 3, 4
    B = rng.standard_normal((nao, nao, naux))
    B = 0.5 * (B + B.transpose(1, 0, 2))
    C = np.linalg.qr(rng.standard_normal((nao, ncore + ncas)))[0]
    D_core = 2.0 * C[:, :ncore] @ C[:, :ncore].T
    C_act = np.ascontiguousarray(C[:, ncore:])
    g1 = rng.standard_normal((ncas, ncas))
    dm1 = g1 @ g1.T
    D_act = C_act @ dm1 @ C_act.T
    t = rng.standard_normal((ncas * ncas, ncas * ncas))
    dm2 = (t + t.T).reshape(ncas, ncas, ncas, ncas)
    dm2 = 0.5 * (dm2 + dm2.transpose(1, 0, 3, 2))  # (uv|xy) = (vu|yx)
    bar = _build_bar_L_casscf_df(B, D_core_ao=D_core, D_act_ao=D_act, C_act=C_act, dm2_act=dm2)
    BQp = np.asarray(pack_B_to_Qp(B, layout="mnQ", nao=nao))
    bar_qp = _build_bar_L_casscf_df(BQp, D_core_ao=D_core, D_act_ao=D_act, C_act=C_act, dm2_act=dm2)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), B=B, D_core=D_core, D_act=D_act, C_act=C_act, dm2=dm2,
                        bar=np.asarray(bar), B_Qp=BQp, bar_qp=np.asarray(bar_qp))
    print(f"{name}: bar {np.asarray(bar).shape}, bar_qp {np.asarray(bar_qp).shape}", flush=True)


def tiles_case(name: str, mol) -> None:
    """One (ab|P) tile per (la, lb, lP) class and one (P|Q) tile per (lP, lQ) class."""
    from asuka.cueri import _eri_rys_cpu as ext
    from asuka.cueri.pair_tables_cpu import build_pair_tables_cpu
    from asuka.frontend.one_electron import build_ao_basis_cart
    from asuka.frontend._scf_build import build_aux_basis_cart
    from asuka.integrals.cueri_df_cpu import _build_df_combined_basis_and_shell_pairs

    rmol = _ref_mol(mol)
    ao, _ = build_ao_basis_cart(rmol, basis=mol.basis, expand_contractions=True)
    aux, _ = build_aux_basis_cart(rmol, basis_in=mol.basis, auxbasis="ricd", expand_contractions=True, ao_basis=ao)
    ball, sp, nsp_ao, nsh_ao, nsh_aux = _build_df_combined_basis_and_shell_pairs(ao, aux)
    pt = build_pair_tables_cpu(ball, sp, threads=0)
    args = [np.asarray(ball.shell_cxyz), np.asarray(ball.shell_l), sp.sp_A, sp.sp_B, sp.sp_pair_start, sp.sp_npair,
            pt.pair_eta, pt.pair_Px, pt.pair_Py, pt.pair_Pz, pt.pair_cK]
    ao_l = np.asarray(ao.shell_l)
    aux_l = np.asarray(aux.shell_l)
    trip, vals3 = [], []
    seen = set()
    for spAB in range(nsp_ao):
        A, B = int(sp.sp_A[spAB]), int(sp.sp_B[spAB])
        for Pc in range(nsh_aux):
            key = (int(ao_l[A]), int(ao_l[B]), int(aux_l[Pc]))
            if key in seen:
                continue
            seen.add(key)
            t = ext.eri_rys_tile_cart_sp_batch_cy(*args, int(spAB), np.array([nsp_ao + Pc], dtype=np.int32), 0)
            trip.append((A, B, Pc))
            vals3.append(np.asarray(t[0]).ravel())
    pairs, vals2 = [], []
    seen = set()
    for P in range(nsh_aux):
        for Q in range(P + 1):
            key = (int(aux_l[P]), int(aux_l[Q]))
            if key in seen:
                continue
            seen.add(key)
            t = ext.eri_rys_tile_cart_sp_batch_cy(*args, int(nsp_ao + P), np.array([nsp_ao + Q], dtype=np.int32), 0)
            pairs.append((P, Q))
            vals2.append(np.asarray(t[0]).ravel())
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        elements=np.array(mol.elements), coords_bohr=mol.coords_bohr, basis=np.array(mol.basis),
        trip=np.array(trip, dtype=np.int32), tiles3=np.concatenate(vals3), len3=np.array([v.size for v in vals3]),
        pairs=np.array(pairs, dtype=np.int32), tiles2=np.concatenate(vals2), len2=np.array([v.size for v in vals2]))
    print(f"{name}: {len(trip)} (ab|P) classes, {len(pairs)} (P|Q) classes", flush=True)


def roots_case() -> None:
    from asuka.cueri import _eri_rys_cpu as ext

    Ts = np.concatenate([[0.0, 1e-10, 1e-3], np.linspace(0.05, 4.95, 12), [5.0, 5.05], np.geomspace(5.5, 500.0, 14)])
    r = np.zeros((10, Ts.size, 10))
    w = np.zeros_like(r)
    for n in range(1, 11):
        for i, T in enumerate(Ts):
            rr, ww = ext.rys_roots_weights_cy(n, float(T))
            r[n - 1, i, :n] = rr
            w[n - 1, i, :n] = ww
    np.savez_compressed(os.path.join(HERE, "ref_roots.npz"), T=Ts, roots=r, weights=w)
    print("ref_roots: done", flush=True)


def uhf_case(name: str, atoms_bohr, basis: str, charge: int, spin: int, method: str = "uhf") -> None:
    """Open-shell DF-UHF/ROHF through the reference's CPU path (``run_hf_df(method=..., backend='cpu')``)."""
    from asuka.frontend.molecule import Molecule
    from asuka.frontend.scf import run_hf_df

    rmol = Molecule.from_atoms([(el, xyz) for el, xyz in atoms_bohr], unit="Bohr", basis=basis, cart=True,
                               charge=charge, spin=spin)
    res = run_hf_df(rmol, method=method, backend="cpu", df=True, auxbasis="ricd", conv_tol=1e-10, max_cycle=300)
    me = res.scf.mo_energy
    ea, eb = (np.asarray(x) for x in me) if isinstance(me, (tuple, list)) else (np.asarray(me), np.asarray(me))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), elements=np.array([a for a, _ in atoms_bohr]),
                        coords_bohr=np.array([x for _, x in atoms_bohr], dtype=np.float64), basis=np.array(basis),
                        charge=np.array(charge), spin=np.array(spin), e_tot=np.array(res.e_tot),
                        converged=np.array(bool(res.scf.converged)), niter=np.array(res.scf.niter),
                        mo_energy_a=ea, mo_energy_b=eb)


def sph_scf_case(name: str, mol) -> None:
    """RHF with spherical AOs (``cart=False``) through the reference's CPU path."""
    from asuka.frontend.molecule import Molecule
    from asuka.frontend.scf import run_hf_df

    rmol = Molecule.from_atoms([(el, xyz) for el, xyz in mol.atoms_bohr], unit="Bohr", basis=mol.basis, cart=False)
    res = run_hf_df(rmol, method="rhf", backend="cpu", df=True, auxbasis="ricd", conv_tol=1e-10)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), elements=np.array(mol.elements),
                        coords_bohr=mol.coords_bohr, basis=np.array(mol.basis), e_tot=np.array(res.e_tot),
                        niter=np.array(res.scf.niter), mo_energy=np.asarray(res.scf.mo_energy),
                        S=np.asarray(res.int1e.S), nao=np.array(np.asarray(res.int1e.S).shape[0]))


def sph_case() -> None:
    from asuka.cueri.sph import cart2sph_matrix

    np.savez_compressed(os.path.join(HERE, "cart2sph_ref.npz"),
                        **{f"l{l}": np.asarray(cart2sph_matrix(l)) for l in range(6)})


CASES = {
    "n2_masvp": lambda: scf_case("n2_masvp", geo.n2("ma-svp")),
    "h2o_masvp": lambda: scf_case("h2o_masvp", geo.water("ma-svp")),
    "h2o_matzvp": lambda: scf_case("h2o_matzvp", geo.water("ma-tzvp")),
    "tiles_h2o_maqzvp": lambda: tiles_case("tiles_h2o_maqzvp", geo.water("ma-qzvp")),
    # the three larger workloads: (H2O)8 seed 0 / ma-TZVP, all-trans n-decane seed 0 / ma-SVP, H2O / ma-QZVP
    "int1e_grad_h2o_matzvp": lambda: int1e_grad_case("int1e_grad_h2o_matzvp", geo.water("ma-tzvp")),
    "casscf_barl": lambda: casscf_barl_case("casscf_barl"),
    "w8_matzvp": lambda: scf_grad_small_case("w8_matzvp", geo.water_cluster(8, 0, "ma-tzvp")),
    "decane_masvp": lambda: scf_grad_small_case("decane_masvp", geo.decane(0, "ma-svp")),
    "h2o_maqzvp": lambda: scf_grad_small_case("h2o_maqzvp", geo.water("ma-qzvp")),
    "ref_roots": roots_case,
    "cart2sph_ref": sph_case,
    "sph_h2o_matzvp": lambda: sph_scf_case("sph_h2o_matzvp", geo.water("ma-tzvp")),
    # OH radical (doublet), O-H 0.9697 A along z, and H2O+ (doublet cation) at the water geometry
    "uhf_oh_masvp": lambda: uhf_case("uhf_oh_masvp", [("O", (0.0, 0.0, 0.0)), ("H", (0.0, 0.0, 0.9697 * geo.ANGSTROM_TO_BOHR))],
                                     "ma-svp", 0, 1),
    "rohf_oh_masvp": lambda: uhf_case("rohf_oh_masvp", [("O", (0.0, 0.0, 0.0)), ("H", (0.0, 0.0, 0.9697 * geo.ANGSTROM_TO_BOHR))],
                                      "ma-svp", 0, 1, "rohf"),
    "rohf_h2o_cation_masvp": lambda: uhf_case("rohf_h2o_cation_masvp", list(geo.water("ma-svp").atoms_bohr), "ma-svp", 1,
                                              1, "rohf"),
    "uhf_h2o_cation_masvp": lambda: uhf_case("uhf_h2o_cation_masvp", list(geo.water("ma-svp").atoms_bohr), "ma-svp", 1, 1),
}

if __name__ == "__main__":
    todo = sys.argv[1:] or list(CASES)
    for c in todo:
        CASES[c]()

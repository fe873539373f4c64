"""Host-side logic: basis packing, shell pairs, geometries, one-electron integrals, packing, DIIS."""

import numpy as np

from _util import bases_of, golden
from asuka_b200 import basis as bm
from asuka_b200 import geometry as geo
from asuka_b200.int1e import build_S_T


def test_basis_sizes_match_reference_fixtures():
    for name, nao, naux in (("n2_masvp", 38, 170), ("h2o_masvp", 29, 115), ("h2o_matzvp", 52, 228)):
        g = golden(name)
        ao, aux, sp = bases_of(g)
        assert (ao.nao, aux.nao) == (nao, naux)
        assert g["S"].shape == (nao, nao)


def test_shell_pairs_are_l_ordered_and_complete():
    ao = bm.pack_basis(list(geo.water("ma-tzvp").atoms_bohr), "ma-tzvp", "ao")
    sp = bm.build_shell_pairs_l_order(ao)
    n = ao.nshell
    assert sp.nsp == n * (n + 1) // 2
    assert np.all(ao.shell_l[sp.sp_A] >= ao.shell_l[sp.sp_B])
    pairs = {(min(a, b), max(a, b)) for a, b in zip(sp.sp_A, sp.sp_B)}
    assert len(pairs) == sp.nsp
    assert sp.sp_pair_start[-1] == np.sum(ao.shell_nprim[sp.sp_A] * ao.shell_nprim[sp.sp_B])


def test_workload_sizes():
    mol = geo.water_cluster(8, 0, "ma-tzvp")
    ao = bm.pack_basis(list(mol.atoms_bohr), "ma-tzvp", "ao")
    aux = bm.pack_basis(list(mol.atoms_bohr), "ma-tzvp", "aux")
    assert (ao.nao, aux.nao) == (416, 1824)
    R = mol.coords_bohr[0::3] / geo.ANGSTROM_TO_BOHR
    d = np.linalg.norm(R[:, None] - R[None], axis=-1) + np.eye(8) * 10
    assert d.min() >= 2.7
    dec = geo.decane(0, "ma-svp")
    assert dec.natm == 32 and dec.nelectron == 82


def test_overlap_matches_reference():
    for name in ("n2_masvp", "h2o_matzvp"):
        g = golden(name)
        ao, aux, sp = bases_of(g)
        S, T = build_S_T(ao)
        assert np.abs(S - g["S"]).max() < 1e-13


def test_nuclear_repulsion_gradient_matches_finite_difference():
    mol = geo.water("ma-svp")
    g = mol.energy_nuc_grad()
    h = 1e-5
    for a in range(mol.natm):
        for c in range(3):
            R = mol.coords_bohr.copy()
            R[a, c] += h
            ep = mol.with_coords(R).energy_nuc()
            R[a, c] -= 2 * h
            em = mol.with_coords(R).energy_nuc()
            assert abs((ep - em) / (2 * h) - g[a, c]) < 1e-7


def test_engine_methods_called_are_defined():
    """Every ``self.<name>(`` call in the engine names an attribute the class defines
    (the GPU-only methods cannot be exercised here)."""
    import re

    from asuka_b200 import df

    src = open(df.__file__).read()
    called = set(re.findall(r"self\.(_?[a-zA-Z]\w*)\(", src))
    assigned = set(re.findall(r"self\.(\w+)\s*=", src))
    missing = sorted(n for n in called if not hasattr(df.DFEngine, n) and n not in assigned)
    assert not missing, missing


def test_block_substitution_matches_triangular_solve():
    """The blocked solves (used on the device) agree with a plain triangular solve."""
    import torch

    from asuka_b200 import linalg

    g = torch.Generator().manual_seed(0)
    n = 700  # three blocks of 256, the last one ragged
    A = torch.randn(n, n, generator=g, dtype=torch.float64)
    L = torch.linalg.cholesky(A @ A.T + n * torch.eye(n, dtype=torch.float64))
    Y = torch.randn(n, 37, generator=g, dtype=torch.float64)
    ref = torch.linalg.solve_triangular(L, Y, upper=False)
    inv = linalg.diag_block_inverses(L)
    # the inverses assembled from 64-row sub-blocks, and the per-block form (a block size that is
    # not 64 * 2^k), against dense inverses
    for nb, blocks in ((linalg.NB, inv), (100, linalg.diag_block_inverses(L, 100))):
        for i, r0 in enumerate(range(0, n, nb)):
            r1 = min(n, r0 + nb)
            dense = torch.linalg.inv(L[r0:r1, r0:r1])
            assert blocks[i].shape == dense.shape
            assert float((blocks[i] - dense).abs().max()) <= 1e-12 * float(dense.abs().max())
    assert torch.allclose(linalg.solve_lower(L, Y, inv), ref, rtol=0, atol=1e-12 * float(ref.abs().max()))
    Yc = Y.clone()
    linalg.solve_lower(L, Yc, inv, out=Yc)  # in place
    assert torch.allclose(Yc, ref, rtol=0, atol=1e-12 * float(ref.abs().max()))
    refT = torch.linalg.solve_triangular(L.T, Y, upper=True)
    Mc = Y.clone()
    linalg.solve_lower_T(L, Mc, inv, out=Mc)
    assert torch.allclose(Mc, refT, rtol=0, atol=1e-12 * float(refT.abs().max()))
    X = torch.randn(29, n, generator=g, dtype=torch.float64)
    refR = torch.linalg.solve_triangular(L, X.T, upper=False).T
    Xc = X.clone()
    linalg.solve_lower_right_T(L, Xc, inv, out=Xc)
    assert torch.allclose(Xc, refR, rtol=0, atol=1e-12 * float(refR.abs().max()))


def test_cart2sph_matches_reference_table():
    """Generated solid-harmonic transforms equal the reference's tabulated ones (l <= 5)."""
    import numpy as np

    from _util import GOLDEN
    from asuka_b200.sph import cart2sph_ao_matrix, cart2sph_matrix

    z = np.load(f"{GOLDEN}/cart2sph_ref.npz")
    for l in range(6):
        assert np.abs(cart2sph_matrix(l) - z[f"l{l}"]).max() < 1e-14
    # rows of every l are orthogonal-ish in the 'sp' metric only; check the block layout instead
    T = cart2sph_ao_matrix([0, 1, 2, 3]).numpy()
    assert T.shape == (1 + 3 + 6 + 10, 1 + 3 + 5 + 7)
    assert np.abs(T[4:10, 4:9] - cart2sph_matrix(2)).max() == 0.0


def test_class_planner_budget_and_table(tmp_path, monkeypatch):
    """A larger accumulator budget gives fewer component splits; the generator's tuning-table
    fields are read per class and can be switched off for variant builds."""
    import importlib.util
    import json
    import os

    src = os.path.join(os.path.dirname(__file__), "..", "asuka_b200", "csrc", "gen_classes.py")
    spec = importlib.util.spec_from_file_location("gen_classes_t", src)
    gc = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gc)
    gc.HERE = str(tmp_path)
    fs40, _ = gc.plan(1, 0, 4, True, budget=40)
    fs96, _ = gc.plan(1, 0, 4, True, budget=96)
    assert fs96 < fs40
    # live accumulators of the derivative form: (a-1)..(a+b-1), (a+1)..(a+b+1), a..(a+b+1)
    assert gc.acc_per_f(1, 0, 1) == 1 + 6 + 9 and gc.acc_per_f(0, 0, 1) == 0 + 3 + 4
    (tmp_path / "class_tuning.json").write_text(json.dumps({"min_blocks": {"d104": 4}, "acc_budget": {"d104": 96}}))
    assert gc.tuning()["d104"] == 4
    assert gc.plan(1, 0, 4, True) == gc.plan(1, 0, 4, True, budget=96)
    monkeypatch.setenv("DFB_GEN_ACC_BUDGET_DERIV", "56")  # a variant build: every derivative class
    assert gc.plan(1, 0, 4, True) == gc.plan(1, 0, 4, True, budget=56)
    monkeypatch.delenv("DFB_GEN_ACC_BUDGET_DERIV")
    monkeypatch.setenv("DFB_GEN_NO_TUNING", "1")
    assert gc.tuning() == {}
    assert gc.plan(1, 0, 4, True) == gc.plan(1, 0, 4, True, budget=gc.ACC_BUDGET[True])


def test_overlap_gradient_contraction_matches_reference():
    """sum M . dS/dR against the reference's contract_dS_cart (int1e_cart.py:1452), H2O / ma-TZVP."""
    from asuka_b200.geometry import Molecule
    from asuka_b200.int1e import contract_dS_cart

    g = golden("int1e_grad_h2o_matzvp")
    ao, _aux, _sp = bases_of(g)
    gS = contract_dS_cart(ao, atom_coords_bohr=g["coords_bohr"], M=g["M"])
    assert np.abs(gS - g["gS"]).max() < 1e-12 * np.abs(g["gS"]).max()
    mol = Molecule.from_atoms([(str(e), x) for e, x in zip(g["elements"], g["coords_bohr"])], unit="Bohr",
                              basis=str(g["basis"]))
    assert np.abs(mol.energy_nuc_grad() - g["g_nuc"]).max() < 1e-13


def test_kinetic_gradient_contraction_matches_finite_differences():
    """sum M . dT/dR (and dS/dR) against central differences of the host T and S builds."""
    from asuka_b200 import basis as bm
    from asuka_b200.int1e import build_S_T, contract_dS_T_cart

    g = golden("int1e_grad_h2o_matzvp")
    ao, _aux, _sp = bases_of(g)
    M = g["M"]
    gS, gT = contract_dS_T_cart(ao, M, M, np.asarray(ao.shell_atom), 3)
    R0 = g["coords_bohr"]
    h = 1e-5
    for (a, c) in [(0, 0), (1, 1), (2, 2)]:
        vals = []
        for s in (1, -1):
            R = R0.copy()
            R[a, c] += s * h
            b = bm.pack_basis([(str(e), x) for e, x in zip(g["elements"], R)], str(g["basis"]), "ao")
            vals.append(build_S_T(b))
        fdS = float(((vals[0][0] - vals[1][0]) * M).sum() / (2 * h))
        fdT = float(((vals[0][1] - vals[1][1]) * M).sum() / (2 * h))
        assert abs(fdS - gS[a, c]) < 1e-8 * max(1.0, abs(fdS))
        assert abs(fdT - gT[a, c]) < 1e-8 * max(1.0, abs(fdT))

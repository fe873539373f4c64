"""Parity of the CUDA Rys kernels (through the C ABI) with the oracle and the reference goldens."""

import numpy as np
import pytest

import oracle as O
from _util import bases_of, golden, unpack_tril

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _engine(ao, aux):
    from asuka_b200.df import DFEngine

    return DFEngine(ao, aux)


@pytest.mark.parametrize("name", ["n2_masvp", "h2o_masvp", "h2o_matzvp"])
def test_metric_and_3c_match_oracle_and_reference(name):
    g = golden(name)
    ao, aux, sp = bases_of(g)
    eng = _engine(ao, aux)
    V = eng.metric().cpu().numpy()
    Vo = O.metric_full(aux)
    assert np.abs(V - V.T).max() == 0.0
    # FP64 parity: 1e-12 relative to the largest element
    Vo = 0.5 * (Vo + Vo.T)
    # metric elements of contracted high-l aux shells carry ~1e-12 cancellation
    # noise (oracle vs reference differ by 2.5e-12 on N2)
    assert np.abs(V - Vo).max() <= 5e-12 * np.abs(Vo).max()
    assert np.abs(V - g["V"]).max() <= 1e-11 * np.abs(Vo).max()
    X = eng.int3c("mnQ").cpu().numpy()
    Xo = O.int3c_full(ao, aux, sp)
    assert np.abs(X - Xo).max() <= 1e-12 * np.abs(Xo).max()
    Xr = unpack_tril(g["X_tril"], ao.nao)
    assert np.abs(X - Xr).max() <= 1e-11 * np.abs(Xo).max()
    Xq = eng.int3c("Qmn").cpu().numpy()
    assert np.array_equal(Xq, X.transpose(2, 0, 1))


def test_every_qzvp_class_matches_oracle_tiles():
    """One (ab|P) tile per (la, lb, lP) class and one (P|Q) tile per (lP, lQ) class, l up to 4/8."""
    g = golden("tiles_h2o_maqzvp")
    ao, aux, sp = bases_of(g)
    eng = _engine(ao, aux)
    X = eng.int3c("mnQ").cpu().numpy()
    V = eng.metric().cpu().numpy()
    off = 0
    worst = 0.0
    for (A, B, P), n in zip(g["trip"], g["len3"]):
        ref = g["tiles3"][off: off + n]
        off += n
        to = O.tile_3c(ao, aux, int(A), int(B), int(P))
        a0, b0, p0 = ao.shell_ao_start[A], ao.shell_ao_start[B], aux.shell_ao_start[P]
        na, nb, npp = to.shape
        tg = X[a0:a0 + na, b0:b0 + nb, p0:p0 + npp]
        scale = max(np.abs(to).max(), 1e-300)
        worst = max(worst, np.abs(tg - to).max() / scale)
        assert np.abs(tg - to).max() <= 1e-12 * scale, (A, B, P)
        # reference tiles carry its own root error at high root counts
        assert np.abs(to.ravel() - ref).max() <= 1e-6 * scale
    off = 0
    for (P, Q), n in zip(g["pairs"], g["len2"]):
        to = O.tile_2c(aux, int(P), int(Q))
        p0, q0 = aux.shell_ao_start[P], aux.shell_ao_start[Q]
        tg = V[p0:p0 + to.shape[0], q0:q0 + to.shape[1]]
        if P == Q:
            to = 0.5 * (to + to.T)
        assert np.abs(tg - to).max() <= 5e-12 * max(np.abs(to).max(), 1e-300), (P, Q)


@pytest.mark.parametrize("name", ["n2_masvp", "h2o_masvp"])
def test_derivative_contractions_match_oracle(name):
    g = golden(name)
    ao, aux, sp = bases_of(g)
    natm = len(g["elements"])
    rng = np.random.default_rng(7)
    nao, naux = ao.nao, aux.nao
    barX = rng.standard_normal((nao, nao, naux))
    barX = np.ascontiguousarray(barX + barX.transpose(1, 0, 2))
    barV = rng.standard_normal((naux, naux))
    barV = barV + barV.T
    g3 = np.zeros((natm, 3))
    O.lib().oracle_deriv3c_full  # loaded
    import ctypes

    k1, a1 = O._bargs(ao)
    k2, a2 = O._bargs(aux)
    s1, ps1 = O._p(ao.shell_ao_start, np.int32)
    s2, ps2 = O._p(aux.shell_ao_start, np.int32)
    t1, pt1 = O._p(ao.shell_atom, np.int32)
    t2, pt2 = O._p(aux.shell_atom, np.int32)
    spA, pA = O._p(sp.sp_A, np.int32)
    spB, pB = O._p(sp.sp_B, np.int32)
    O.lib().oracle_deriv3c_full(*a1, ps1, pt1, ctypes.c_int(nao), *a2, ps2, pt2, ctypes.c_int(aux.nshell),
                                ctypes.c_int(naux), pA, pB, ctypes.c_int(sp.nsp), barX.ctypes.data_as(O._d),
                                ctypes.c_int(natm), g3.ctypes.data_as(O._d))
    g2 = np.zeros((natm, 3))
    O.lib().oracle_deriv2c_full(*a2, ps2, pt2, ctypes.c_int(aux.nshell), ctypes.c_int(naux),
                                barV.ctypes.data_as(O._d), ctypes.c_int(natm), g2.ctypes.data_as(O._d))
    eng = _engine(ao, aux)
    gd = torch.zeros((natm, 3), dtype=torch.float64, device="cuda")
    eng.deriv3c(torch.as_tensor(barX.transpose(2, 0, 1).copy(), device="cuda"), gd, layout="Qmn")
    G3 = gd.cpu().numpy()
    gd.zero_()
    eng.deriv2c(torch.as_tensor(barV, device="cuda"), gd)
    G2 = gd.cpu().numpy()
    assert np.abs(G3 - g3).max() <= 1e-11 * np.abs(g3).max()
    assert np.abs(G2 - g2).max() <= 1e-11 * np.abs(g2).max()
    # translational invariance of each contraction
    assert np.abs(G3.sum(0)).max() <= 1e-10 * np.abs(g3).max()


def test_specialised_and_generic_kernels_agree(monkeypatch):
    """The class-specialised thread kernels and the generic warp kernel give the same tiles and gradients."""
    g = golden("h2o_matzvp")
    ao, aux, sp = bases_of(g)
    eng = _engine(ao, aux)
    natm = len(g["elements"])
    X1 = eng.int3c("Qmn").clone()
    V1 = eng.metric().clone()
    rng = np.random.default_rng(3)
    bar = torch.as_tensor(rng.standard_normal(tuple(X1.shape)), device="cuda")
    bar = bar + bar.transpose(1, 2)
    g1 = torch.zeros((natm, 3), dtype=torch.float64, device="cuda")
    eng.deriv3c(bar, g1)
    monkeypatch.setenv("DFB_DISABLE_TMPL", "1")
    X2 = eng.int3c("Qmn")
    V2 = eng.metric()
    g2 = torch.zeros_like(g1)
    eng.deriv3c(bar, g2)
    monkeypatch.delenv("DFB_DISABLE_TMPL")
    sx = float(X2.abs().max())
    assert float((X1 - X2).abs().max()) <= 1e-13 * sx
    # metric elements of contracted high-l aux shells carry ~1e-13..1e-12 cancellation noise
    assert float((V1 - V2).abs().max()) <= 1e-12 * float(V2.abs().max())
    assert float((g1 - g2).abs().max()) <= 1e-11 * float(g2.abs().max())


def test_primitive_screening_changes_nothing_visible():
    """Screened primitive pairs (bound < 1e-20) change integrals and gradients below FP64 noise."""
    from asuka_b200.df import DFEngine
    from asuka_b200 import geometry as geo, basis as bm

    mol = geo.water_cluster(2, 1, "ma-svp")
    atoms = list(mol.atoms_bohr)
    ao, aux = bm.pack_basis(atoms, "ma-svp", "ao"), bm.pack_basis(atoms, "ma-svp", "aux")
    e0 = DFEngine(ao, aux, prim_screen=0.0)
    e1 = DFEngine(ao, aux)
    assert e1.n_prim_pairs < e0.n_prim_pairs
    X0, X1 = e0.int3c("Qmn"), e1.int3c("Qmn")
    assert float((X0 - X1).abs().max()) <= 1e-14 * float(X0.abs().max())
    bar = torch.randn_like(X0)
    bar = bar + bar.transpose(1, 2)
    g0 = torch.zeros((mol.natm, 3), dtype=torch.float64, device="cuda")
    g1 = torch.zeros_like(g0)
    e0.deriv3c(bar, g0)
    e1.deriv3c(bar, g1)
    assert float((g0 - g1).abs().max()) <= 1e-12 * float(g0.abs().max())

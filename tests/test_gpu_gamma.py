"""The 3c adjoint kernel (``dfb_gamma_sym``): Gamma_P = Cw A_P Cw^T for symmetric A_P.

Against the FP64 torch product, with partial 64-row tiles (nao not a multiple of 64), one and
several 32-long k chunks (nocc), and a U laid out (nao, nP, nocc) as the gradient passes it.
The output must be exactly symmetric (diagonal tiles mirror their upper part).
"""

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("nP,nao,nocc", [(5, 100, 7), (3, 130, 40), (4, 64, 70), (2, 1, 3), (7, 416, 40)])
def test_gamma_matches_fp64_product(nP, nao, nocc):
    from asuka_b200.grad import _gamma_into

    g = torch.Generator(device="cuda").manual_seed(nP * 1000 + nao + nocc)
    Cw = torch.randn(nao, nocc, generator=g, dtype=torch.float64, device="cuda")
    A = torch.randn(nP, nocc, nocc, generator=g, dtype=torch.float64, device="cuda")
    A = 0.5 * (A + A.transpose(1, 2))
    out = torch.full((nP, nao, nao), float("nan"), dtype=torch.float64, device="cuda")
    _gamma_into(Cw, A, out)
    ref = torch.matmul(Cw, torch.matmul(A, Cw.T))
    assert torch.isfinite(out).all()
    assert float((out - ref).abs().max()) <= 1e-13 * float(ref.abs().max())
    assert torch.equal(out, out.transpose(1, 2))


def test_gamma_in_the_adjoint_matches_the_batched_product():
    """df_adjoints' Gamma against Cw (d_P I - Z_P / 2) Cw^T formed with torch."""
    import numpy as np

    from asuka_b200 import basis as bm
    from asuka_b200 import geometry as geo
    from asuka_b200.df import DFEngine
    from asuka_b200.grad import df_adjoints, df_forward

    mol = geo.water_cluster(2, 0, "ma-svp")
    atoms = list(mol.atoms_bohr)
    eng = DFEngine(bm.pack_basis(atoms, mol.basis, "ao"), bm.pack_basis(atoms, mol.basis, "aux"))
    eng.set_coords(torch.as_tensor(mol.coords_bohr, device="cuda"))
    rng = np.random.default_rng(1)
    Cw = torch.as_tensor(np.linalg.qr(rng.standard_normal((eng.nao, mol.nelectron // 2)))[0], device="cuda")
    _E, _J, _K, saved = df_forward(eng, Cw)
    from asuka_b200 import linalg as la

    L, d, W = saved["L"], saved["d"], saved["W"]
    nocc = Cw.shape[1]
    M = torch.matmul(Cw.T, W.view(eng.naux, eng.nao, nocc))
    M = 0.5 * (M + M.transpose(1, 2))
    Z = la.solve_lower_T(L, M.reshape(eng.naux, nocc * nocc)).view(eng.naux, nocc, nocc)
    A = -0.5 * Z + d.view(-1, 1, 1) * torch.eye(nocc, dtype=Z.dtype, device=Z.device)
    ref = torch.matmul(Cw, torch.matmul(A, Cw.T))
    G3, _G2 = df_adjoints(eng, Cw, saved)
    assert float((G3 - ref).abs().max()) <= 1e-12 * float(ref.abs().max())

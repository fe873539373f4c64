"""Active-space DF factors (CASSCF consumer) and streamed J/K with several occupied sets (UHF).

The active factors are checked against the same transform of the reference's own whitened
factors (its 3c integrals and metric from the fixture) and, tighter, against the transform of
this engine's B in every layout."""

import numpy as np
import pytest

from _util import bases_of, golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _stored(g):
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e

    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux)
    L = cholesky_metric(eng.metric())
    BQ = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn")
    return ao, aux, eng, L, BQ


@pytest.mark.parametrize("name", ["h2o_masvp", "n2_masvp"])
def test_active_factors_all_layouts(name):
    from asuka_b200.active import (active_Lfull_from_B, active_Lfull_from_B_Qp, active_Lfull_from_cached_B_whitened,
                                   active_Lfull_streamed_basis)
    from asuka_b200.scf import pack_B_to_Qp

    g = golden(name)
    ao, aux, eng, L, BQ = _stored(g)
    C = torch.as_tensor(g["mo_coeff"], device="cuda")[:, 2:8].contiguous()  # a 6-orbital active space
    norb, naux = C.shape[1], BQ.shape[0]
    Ch = C.cpu().numpy()
    # the reference's own factors: its unwhitened 3c integrals and metric from the fixture,
    # whitened on the host (B = X L^-T), then L[p q, Q] = sum_mn C_mp C_nq B_Q[m, n]
    from scipy.linalg import solve_triangular
    from _util import unpack_tril

    nao = Ch.shape[0]
    Xr = unpack_tril(g["X_tril"], nao).reshape(nao * nao, naux)
    Br = solve_triangular(np.linalg.cholesky(g["V"]), Xr.T, lower=True).T.reshape(nao, nao, naux)
    ref_r = np.einsum("mp,nq,mnQ->pqQ", Ch, Ch, Br).reshape(norb * norb, naux)
    ref = np.einsum("mp,nq,Qmn->pqQ", Ch, Ch, BQ.cpu().numpy()).reshape(norb * norb, naux)
    scale = np.abs(ref).max()
    # this engine's whitened factors against the reference's (integrals ~1e-12, whitened through
    # the metric's Cholesky factor)
    assert np.abs(ref - ref_r).max() < 1e-9 * scale
    B_mnQ = BQ.permute(1, 2, 0).contiguous()
    for Lf in (active_Lfull_from_B(B_mnQ, C), active_Lfull_from_B(BQ, C, layout="Qmn"),
               active_Lfull_from_cached_B_whitened(B_mnQ, C),
               active_Lfull_from_B_Qp(pack_B_to_Qp(BQ), C, aux_block_naux=7),
               active_Lfull_from_cached_B_whitened(pack_B_to_Qp(BQ), C)):
        assert Lf.shape == (norb * norb, naux)
        assert np.abs(Lf.cpu().numpy() - ref).max() < 1e-12 * scale
    Ls = active_Lfull_streamed_basis(ao, aux, C, aux_block_naux=40)
    assert np.abs(Ls.cpu().numpy() - ref).max() < 1e-11 * scale
    assert np.abs(Ls.cpu().numpy() - ref_r).max() < 1e-9 * scale


@pytest.mark.parametrize("aux_block", [32, 100000])
def test_streamed_jks_two_occupied_sets(aux_block):
    from asuka_b200.jk import df_J_from_BQ_D, df_K_from_BQ_Cw
    from asuka_b200.streamed import df_JK_streamed, df_JKs_streamed, make_streamed_df_jk_context

    g = golden("h2o_matzvp")
    ao, aux, eng, L, BQ = _stored(g)
    C = torch.as_tensor(g["mo_coeff"], device="cuda")
    nocc = int((g["mo_occ"] > 0).sum())
    Ca, Cb = C[:, :nocc], C[:, :nocc - 1]  # a doublet-like pair of occupied sets
    occa = torch.ones(nocc, dtype=torch.float64, device="cuda")
    occb = torch.ones(nocc - 1, dtype=torch.float64, device="cuda")
    D = Ca @ Ca.T + Cb @ Cb.T
    ctx = make_streamed_df_jk_context(ao, aux, aux_block_naux=aux_block, engine=eng, L_metric=L)
    J, (Ka, Kb) = df_JKs_streamed(ctx, D, [Ca, Cb], [occa, occb], k_q_block=17)
    J0 = df_J_from_BQ_D(BQ, D)
    scale = float(J0.abs().max())
    assert float((J - J0).abs().max()) < 1e-11 * scale
    assert float((Ka - df_K_from_BQ_Cw(BQ, Ca.contiguous())).abs().max()) < 1e-11 * scale
    assert float((Kb - df_K_from_BQ_Cw(BQ, Cb.contiguous())).abs().max()) < 1e-11 * scale
    J1, K1 = df_JK_streamed(ctx, D, Ca, occa)
    assert float((J1 - J).abs().max()) < 1e-12 * scale and float((K1 - Ka).abs().max()) < 1e-12 * scale


@pytest.mark.parametrize("layout", ["mnQ", "Qmn"])
def test_spherical_ao_factors(layout):
    """ao_rep='sph': X over real spherical AOs = T^T X_cart T against the reference X (oracle-pinned)."""
    from _util import unpack_tril
    from asuka_b200.df import build_df_B_from_cueri_packed_bases, cholesky_metric, int3c2e_basis
    from asuka_b200.sph import cart2sph_ao_matrix, sph_coeff_sph_to_cart

    g = golden("h2o_matzvp")  # d and f AO shells
    ao, aux, sp = bases_of(g)
    Xs = int3c2e_basis(ao, aux, layout=layout, ao_rep="sph")
    T = cart2sph_ao_matrix(ao.shell_l).numpy()
    nao = T.shape[0]
    Xc = unpack_tril(g["X_tril"], nao)  # (nao, nao, naux) from the reference
    ref = np.einsum("ms,nt,mnP->stP", T, T, Xc)
    got = Xs.cpu().numpy() if layout == "mnQ" else Xs.permute(1, 2, 0).cpu().numpy()
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() < 1e-11 * np.abs(ref).max()
    B, L = build_df_B_from_cueri_packed_bases(ao, aux, layout="mnQ", ao_rep="sph", return_L=True)
    Bref = np.linalg.solve(L.cpu().numpy(), ref.reshape(-1, ref.shape[2]).T).T.reshape(ref.shape)
    assert np.abs(B.cpu().numpy() - Bref).max() < 1e-10 * np.abs(Bref).max()
    Cs = torch.randn(T.shape[1], 4, dtype=torch.float64, device="cuda")
    assert np.abs(sph_coeff_sph_to_cart(Cs, ao.shell_l).cpu().numpy() - T @ Cs.cpu().numpy()).max() < 1e-13

"""End-to-end DF-RHF pieces on the GPU against the reference fixtures and the oracle."""

import numpy as np
import pytest

import oracle as O
from _util import bases_of, golden, nelec_of

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _mol(g):
    from asuka_b200.geometry import Molecule

    return Molecule.from_atoms([(str(e), x) for e, x in zip(g["elements"], g["coords_bohr"])], unit="Bohr",
                               basis=str(g["basis"]))


@pytest.mark.parametrize("name", ["n2_masvp", "h2o_matzvp"])
def test_int1e_matches_reference(name):
    from asuka_b200.int1e import build_int1e

    g = golden(name)
    ao, aux, sp = bases_of(g)
    mol = _mol(g)
    r = build_int1e(ao, mol.coords_bohr, mol.charges)
    assert np.abs(r.S - g["S"]).max() < 1e-13
    assert np.abs(r.hcore - g["hcore"]).max() < 1e-11 * np.abs(g["hcore"]).max()


@pytest.mark.parametrize("name", ["n2_masvp", "h2o_matzvp"])
def test_jk_from_whitened_factors(name):
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e
    from asuka_b200.jk import DFJKWorkspace

    g = golden(name)
    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux)
    L = cholesky_metric(eng.metric())
    B = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn")
    C = torch.as_tensor(g["mo_coeff"], device="cuda")
    occ = torch.as_tensor(g["mo_occ"], device="cuda")
    nocc = int((g["mo_occ"] > 0).sum())
    Cw = (C[:, :nocc] * occ[:nocc].sqrt()).contiguous()
    D = torch.as_tensor(g["D"], device="cuda")
    nao = D.shape[0]
    J = torch.empty((nao, nao), dtype=torch.float64, device="cuda")
    K = torch.empty_like(J)
    ws = DFJKWorkspace()
    ws.jk_from_bq_cw(B, Cw, D, J, K, q_block=64)
    scale = np.abs(g["J"]).max()
    assert np.abs(J.cpu().numpy() - g["J"]).max() < 1e-11 * scale
    assert np.abs(K.cpu().numpy() - g["K"]).max() < 1e-11 * scale
    Km = torch.empty_like(K)
    DFJKWorkspace("mixed").k_from_bq_cw(B, Cw, Km, q_block=64, sync=True)
    # split-BF16 tensor-core exchange: FP32 accumulation with a truncation bias, ~3e-6 relative to
    # the largest (diagonal) elements
    assert np.abs(Km.cpu().numpy() - g["K"]).max() < 5e-6 * np.abs(g["K"]).max()


@pytest.mark.parametrize("name", ["n2_masvp", "h2o_matzvp"])
def test_run_hf_df_energy_matches_reference(name):
    from asuka_b200.scf import run_hf_df

    g = golden(name)
    mol = _mol(g)
    r = run_hf_df(mol, two_e_backend="df", conv_tol=1e-10)
    assert r.converged
    # FP64 mode matches the reference to 1e-10 Eh
    assert abs(r.e_tot - float(g["e_tot"])) < 1e-10
    rd = run_hf_df(mol, two_e_backend="direct_df", conv_tol=1e-10, df_aux_block_naux=64)
    assert rd.df_B is None and rd.converged
    assert abs(rd.e_tot - float(g["e_tot"])) < 1e-10
    rm = run_hf_df(mol, two_e_backend="df", conv_tol=1e-10, precision="mixed")
    assert rm.converged
    assert abs(rm.e_tot - float(g["e_tot"])) < 1e-9


def _cw(g):
    C = torch.as_tensor(g["mo_coeff"], device="cuda")
    occ = torch.as_tensor(g["mo_occ"], device="cuda")
    nocc = int((g["mo_occ"] > 0).sum())
    return (C[:, :nocc] * occ[:nocc].sqrt()).contiguous()


@pytest.mark.parametrize("name", ["n2_masvp", "h2o_masvp", "h2o_matzvp"])
def test_autograd_gradient_matches_reference(name):
    from asuka_b200.df import DFEngine
    from asuka_b200.grad import df_energy

    g = golden(name)
    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux)
    R = torch.as_tensor(g["coords_bohr"], device="cuda").requires_grad_(True)
    E, J, K = df_energy(R, _cw(g), eng)
    assert abs(float(E.detach()) - float(g["E2"])) < 1e-10 * abs(float(g["E2"]))
    (gR,) = torch.autograd.grad(E, R)
    ref = g["grad_2e"]
    assert np.abs(gR.cpu().numpy() - ref).max() < 1e-9
    # Mixed-precision exchange (split-BF16, FP32 accumulation): one contraction is
    # good to ~1e-6 relative in E_2e -- SCF energies reach 1e-6 Eh only through the
    # FP64 refinement iterations (test_run_hf_df_energy_matches_reference) -- while
    # the gradient at fixed density stays within 1e-6 Eh/bohr.
    Em, _, _ = df_energy(R, _cw(g), eng, "mixed")
    (gm,) = torch.autograd.grad(Em, R)
    assert abs(float(Em.detach()) - float(g["E2"])) < 1e-6 * abs(float(g["E2"]))
    assert np.abs(gm.cpu().numpy() - ref).max() < 1e-6


def test_reference_gradient_seam_matches_golden():
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e
    from asuka_b200.grad import compute_df_gradient_contributions_analytic_packed_bases

    g = golden("h2o_masvp")
    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux)
    L = cholesky_metric(eng.metric())
    BQ = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn")
    B = BQ.permute(1, 2, 0).contiguous().cpu().numpy()
    D = g["D"]
    barL = O.bar_B_rhf(B, D)
    gr = compute_df_gradient_contributions_analytic_packed_bases(ao, aux, atom_coords_bohr=g["coords_bohr"], B_ao=B,
                                                                 bar_L_ao=barL, L_chol=L, backend="cuda")
    assert np.abs(gr - g["grad_2e"]).max() < 1e-9


def test_gradient_matches_central_finite_differences():
    """dE_2e/dR at fixed density vs central differences (h = 1e-4 bohr)."""
    from asuka_b200.df import DFEngine
    from asuka_b200.grad import df_energy, df_forward

    g = golden("h2o_masvp")
    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux)
    Cw = _cw(g)
    R0 = torch.as_tensor(g["coords_bohr"], device="cuda")
    R = R0.clone().requires_grad_(True)
    E, _, _ = df_energy(R, Cw, eng)
    (gR,) = torch.autograd.grad(E, R)
    h = 1e-4
    for (a, c) in [(0, 0), (0, 2), (1, 1), (2, 0)]:
        vals = []
        for s in (1, -1):
            Rs = R0.clone()
            Rs[a, c] += s * h
            eng.set_coords(Rs)
            vals.append(float(df_forward(eng, Cw)[0]))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - float(gR[a, c])) < 1e-7, (a, c, fd, float(gR[a, c]))


def test_split_bf16_products():
    """Split-BF16 rank-k update and product (FP32 accumulation per block) against FP64."""
    from asuka_b200 import mixed

    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(1100, 20000, generator=g, dtype=torch.float64, device="cuda")
    ref = A @ A.T
    K = mixed.syrk(A)
    # about 2e-6 relative for 1024-long accumulation blocks
    assert float((K - ref).abs().max()) < 1e-5 * float(ref.abs().max())
    B = torch.randn(20000, 300, generator=g, dtype=torch.float64, device="cuda")
    ref = A @ B
    assert float((mixed.matmul(A, B) - ref).abs().max()) < 1e-5 * float(ref.abs().max())


def test_gradient_context_layouts():
    """The reusable gradient context gives the reference gradient from mnQ, packed-Qp and
    split-term inputs, and its spherical-AO contraction equals the Cartesian one."""
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e
    from asuka_b200.grad_context import DFGradContractionContext
    from asuka_b200.scf import pack_B_to_Qp
    from asuka_b200.sph import cart2sph_ao_matrix

    g = golden("h2o_masvp")
    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux)
    L = cholesky_metric(eng.metric())
    BQ = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn")
    B = BQ.permute(1, 2, 0).contiguous()
    barL = torch.as_tensor(O.bar_B_rhf(B.cpu().numpy(), g["D"]), device="cuda")
    ctx = DFGradContractionContext.build(ao, aux, atom_coords_bohr=g["coords_bohr"], L_chol=L)
    ref = g["grad_2e"]
    assert np.abs(ctx.contract(B_ao=B, bar_L_ao=barL) - ref).max() < 1e-9
    assert np.abs(ctx.contract(B_ao=pack_B_to_Qp(BQ), bar_L_ao=pack_B_to_Qp(barL)) - ref).max() < 1e-9
    half = 0.5 * barL
    assert np.abs(ctx.contract_fused_terms(B_ao=B, bar_L_terms=[half, half]) - ref).max() < 1e-9
    # spherical: with B_sph = T^T B T and bar_L_cart = T bar_L_sph T^T both routes see the same energy
    T = cart2sph_ao_matrix(ao.shell_l, "cuda")
    Bs = torch.einsum("ms,nt,mnQ->stQ", T, T, B).contiguous()
    gen = torch.Generator(device="cuda").manual_seed(0)
    bar_s = torch.randn((BQ.shape[0], T.shape[1], T.shape[1]), generator=gen, dtype=torch.float64, device="cuda")
    bar_s = 0.5 * (bar_s + bar_s.transpose(1, 2))
    bar_c = torch.einsum("ms,Qst,nt->Qmn", T, bar_s, T)
    g_s = ctx.contract_sph(B_sph=Bs, bar_L_sph=bar_s)
    g_c = ctx.contract(B_ao=B, bar_L_ao=bar_c)
    assert np.abs(g_s - g_c).max() < 1e-9 * max(1.0, np.abs(g_c).max())

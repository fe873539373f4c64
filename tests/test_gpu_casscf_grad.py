"""DF-CASSCF gradient adjoint bar_L = dE_2e/dB against the reference's builders.

Fixture ``casscf_barl`` (``tests/golden/make_golden.py``): the reference's
``_build_bar_L_casscf_df`` (``asuka/mcscf/nuc_grad_df.py:2387-2600``) on seeded B, core and
active densities, active orbitals and 2-RDM, in the mnQ and packed Qp layouts.  Then the
packed-Qp gradient contraction (never unpacking the whole tensor) against the mnQ one.
"""

import numpy as np
import pytest

from _util import bases_of, golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_bar_L_matches_reference_in_every_layout():
    from asuka_b200.casscf_grad import build_bar_L_casscf_df

    g = golden("casscf_barl")
    kw = dict(D_core_ao=g["D_core"], D_act_ao=g["D_act"], C_act=g["C_act"], dm2_act=g["dm2"])
    ref = g["bar"]
    scale = np.abs(ref).max()
    bar = build_bar_L_casscf_df(torch.as_tensor(g["B"], device="cuda"), qblock=16, **kw).cpu().numpy()
    assert np.abs(bar - ref).max() < 1e-12 * scale
    BQ = torch.as_tensor(g["B"], device="cuda").permute(2, 0, 1).contiguous()
    bar2 = build_bar_L_casscf_df(BQ, layout="Qmn", **kw).cpu().numpy()
    assert np.abs(bar2 - ref).max() < 1e-12 * scale
    bar_qp = build_bar_L_casscf_df(torch.as_tensor(g["B_Qp"], device="cuda"), qblock=7, **kw).cpu().numpy()
    assert np.abs(bar_qp - g["bar_qp"]).max() < 1e-12 * scale


def test_packed_gradient_contraction_matches_unpacked():
    """DFGradContractionContext.contract on packed Qp B and bar_L (aux-block by aux-block, the
    (naux, nao, nao) tensor never formed) equals the mnQ contraction and the reference gradient."""
    import oracle as O
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e
    from asuka_b200.grad_context import DFGradContractionContext
    from asuka_b200.scf import pack_B_to_Qp

    g = golden("h2o_masvp")
    ao, aux, _sp = bases_of(g)
    eng = DFEngine(ao, aux)
    L = cholesky_metric(eng.metric())
    BQ = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn")
    B = BQ.permute(1, 2, 0).contiguous()
    barL = torch.as_tensor(O.bar_B_rhf(B.cpu().numpy(), g["D"]), device="cuda")
    ctx = DFGradContractionContext.build(ao, aux, atom_coords_bohr=g["coords_bohr"], L_chol=L)
    g_full = ctx.contract(B_ao=B, bar_L_ao=barL)
    g_qp = ctx.contract(B_ao=pack_B_to_Qp(BQ), bar_L_ao=pack_B_to_Qp(barL), aux_block_naux=17)
    assert np.abs(g_qp - g_full).max() < 1e-11
    assert np.abs(g_qp - g["grad_2e"]).max() < 1e-9
    assert ctx.last_peak_block_elems < BQ.numel()  # never the whole (naux, nao, nao) tensor

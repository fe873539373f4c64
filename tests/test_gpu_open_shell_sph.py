"""ROHF and spherical-AO RHF against the reference's CPU path."""

import numpy as np
import pytest

from _util import golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _mol(g, **kw):
    from asuka_b200.geometry import Molecule

    return Molecule.from_atoms([(str(e), x) for e, x in zip(g["elements"], g["coords_bohr"])], unit="Bohr",
                               basis=str(g["basis"]), **kw)


@pytest.mark.parametrize("name", ["rohf_oh_masvp", "rohf_h2o_cation_masvp"])
@pytest.mark.parametrize("backend", ["df", "direct_df"])
def test_rohf_matches_reference(name, backend):
    from asuka_b200.scf import run_hf_df

    g = golden(name)
    r = run_hf_df(_mol(g, charge=int(g["charge"]), spin=int(g["spin"])), method="rohf", two_e_backend=backend,
                  conv_tol=1e-10, df_aux_block_naux=48)
    assert r.converged
    assert abs(r.e_tot - float(g["e_tot"])) < 1e-10
    na = int((r.mo_occ[0] > 0).sum())
    assert np.abs(r.mo_energy.cpu().numpy()[:na] - g["mo_energy_a"][:na]).max() < 1e-8


@pytest.mark.parametrize("backend", ["df", "direct_df"])
def test_spherical_rhf_matches_reference(backend):
    from asuka_b200.scf import run_hf_df

    g = golden("sph_h2o_matzvp")
    r = run_hf_df(_mol(g, cart=False), method="rhf", two_e_backend=backend, conv_tol=1e-10, df_aux_block_naux=48)
    assert r.converged
    assert r.int1e.S.shape == (int(g["nao"]),) * 2
    assert np.abs(r.int1e.S - g["S"]).max() < 1e-12
    assert abs(r.e_tot - float(g["e_tot"])) < 1e-10

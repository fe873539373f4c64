"""One-electron gradient pieces and the full DF-RHF nuclear gradient.

``contract_dhcore_cart`` (kinetic on the host, nuclear attraction through the Rys
derivative kernel with point-charge shells) against the reference's
``contract_dhcore_cart`` (``asuka/integrals/int1e_cart.py:1738``) on a seeded symmetric
matrix, with and without the operator-centre term; then the composed RHF gradient
(nuclear + dhcore(D) - dS(W) + DF two-electron) against central differences of the
converged DF-RHF energy.
"""

import numpy as np
import pytest

from _util import bases_of, golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_dhcore_contraction_matches_reference():
    from asuka_b200.int1e import contract_dhcore_cart

    g = golden("int1e_grad_h2o_matzvp")
    ao, _aux, _sp = bases_of(g)
    R, Z, M = g["coords_bohr"], g["Z"], g["M"]
    gH = contract_dhcore_cart(ao, atom_coords_bohr=R, atom_charges=Z, M=M)
    assert np.abs(gH - g["gH"]).max() < 1e-10 * np.abs(g["gH"]).max()
    gH0 = contract_dhcore_cart(ao, atom_coords_bohr=R, atom_charges=Z, M=M, include_operator_deriv=False)
    assert np.abs(gH0 - g["gH_basis_only"]).max() < 1e-10 * np.abs(g["gH_basis_only"]).max()


def test_rhf_gradient_matches_energy_differences():
    """dE_RHF/dR of H2O / ma-SVP against central differences (h = 1e-4 bohr) of the SCF energy."""
    from asuka_b200.geometry import Molecule
    from asuka_b200.grad import rhf_nuclear_gradient
    from asuka_b200.scf import run_hf_df

    g = golden("h2o_masvp")
    els = [str(e) for e in g["elements"]]
    R0 = np.asarray(g["coords_bohr"], dtype=np.float64)

    def mol_at(R):
        return Molecule.from_atoms(list(zip(els, R)), unit="Bohr", basis=str(g["basis"]))

    res = run_hf_df(mol_at(R0), two_e_backend="df", conv_tol=1e-12, conv_tol_dm=1e-10)
    assert res.converged
    grad = rhf_nuclear_gradient(res)
    # translational invariance of the total gradient
    assert np.abs(grad.sum(0)).max() < 1e-8
    h = 1e-4
    for (a, c) in [(0, 0), (0, 1), (1, 0), (2, 1)]:
        e = []
        for s in (1, -1):
            R = R0.copy()
            R[a, c] += s * h
            r = run_hf_df(mol_at(R), two_e_backend="df", conv_tol=1e-12, conv_tol_dm=1e-10)
            e.append(r.e_tot)
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd - grad[a, c]) < 2e-7, (a, c, fd, grad[a, c])

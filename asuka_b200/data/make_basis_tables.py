"""Generate ``basis_tables.npz``: per-element AO and RICD auxiliary shell data.

Run this once in a checkout where the ASUKA reference (with its CPU Cython
extensions built) is importable, e.g.::

    PYTHONPATH=/tmp/asuka_ref python asuka_b200/data/make_basis_tables.py

For every (AO basis, element) pair the script packs a single atom at the
origin with the reference's own packer (``asuka/frontend/basis_packer.py:183``,
``expand_contractions=True``, Cartesian normalisation of
``asuka/integrals/gto_cart.py:54-66``) and generates the RICD acCD aux basis
(``asuka/integrals/ricd_builder.py:497``, default options tau=1e-4).  RICD
aux shells are generated per atom type, so a molecule's bases are the
concatenation of its atoms' shells in atom order; the script checks this on a
water dimer before writing.  Output arrays are keyed
``{basis}/{element}/{ao|aux}/{l,nprim,exp,coef}``.
"""

from __future__ import annotations

import os
import sys

import numpy as np

BASES = ("ma-svp", "ma-tzvp", "ma-qzvp")
ELEMENTS = ("H", "C", "N", "O")


def _atom_bases(basis: str, el: str):
    from asuka.frontend.molecule import Molecule
    from asuka.frontend.one_electron import build_ao_basis_cart
    from asuka.frontend._scf_build import build_aux_basis_cart

    spin = 1 if el in ("H", "N") else 0
    mol = Molecule.from_atoms(f"{el} 0 0 0", unit="Bohr", basis=basis, cart=True, spin=spin)
    ao, _ = build_ao_basis_cart(mol, basis=basis, expand_contractions=True)
    aux, _ = build_aux_basis_cart(mol, basis_in=basis, auxbasis="ricd", expand_contractions=True, ao_basis=ao)
    return ao, aux


def _shells(b):
    l = np.asarray(b.shell_l, dtype=np.int32)
    nprim = np.asarray(b.shell_nprim, dtype=np.int32)
    start = np.asarray(b.shell_prim_start, dtype=np.int32)
    exps, coefs = [], []
    for s in range(l.size):
        exps.append(np.asarray(b.prim_exp)[start[s] : start[s] + nprim[s]])
        coefs.append(np.asarray(b.prim_coef)[start[s] : start[s] + nprim[s]])
    return l, nprim, np.concatenate(exps), np.concatenate(coefs)


def main(out_path: str) -> None:
    tables: dict[str, np.ndarray] = {}
    for basis in BASES:
        for el in ELEMENTS:
            ao, aux = _atom_bases(basis, el)
            for kind, b in (("ao", ao), ("aux", aux)):
                l, nprim, e, c = _shells(b)
                key = f"{basis}/{el}/{kind}"
                tables[key + "/l"] = l
                tables[key + "/nprim"] = nprim
                tables[key + "/exp"] = e
                tables[key + "/coef"] = c
            print(basis, el, "ao shells", int(ao.shell_l.size), "aux shells", int(aux.shell_l.size), flush=True)

    # Check: a water dimer's reference bases equal the per-atom concatenation.
    from asuka.frontend.molecule import Molecule
    from asuka.frontend.one_electron import build_ao_basis_cart
    from asuka.frontend._scf_build import build_aux_basis_cart

    atoms = "O 0 0 0; H 0 1.43 1.1; H 0 -1.43 1.1; O 5.1 0.3 0.2; H 6 1.4 1; H 5.5 -1.2 0.9"
    mol = Molecule.from_atoms(atoms, unit="Bohr", basis="ma-tzvp", cart=True)
    ao, _ = build_ao_basis_cart(mol, basis="ma-tzvp", expand_contractions=True)
    aux, _ = build_aux_basis_cart(mol, basis_in="ma-tzvp", auxbasis="ricd", expand_contractions=True, ao_basis=ao)
    for kind, b in (("ao", ao), ("aux", aux)):
        l_ref, n_ref, e_ref, c_ref = _shells(b)
        l_cat = np.concatenate([tables[f"ma-tzvp/{el}/{kind}/l"] for el, _ in mol.atoms_bohr])
        e_cat = np.concatenate([tables[f"ma-tzvp/{el}/{kind}/exp"] for el, _ in mol.atoms_bohr])
        c_cat = np.concatenate([tables[f"ma-tzvp/{el}/{kind}/coef"] for el, _ in mol.atoms_bohr])
        assert np.array_equal(l_ref, l_cat), kind
        assert np.array_equal(e_ref, e_cat) and np.array_equal(c_ref, c_cat), kind
        cx = np.asarray(b.shell_cxyz)
        ia = 0
        for el, xyz in mol.atoms_bohr:
            n = tables[f"ma-tzvp/{el}/{kind}/l"].size
            assert np.array_equal(cx[ia : ia + n], np.broadcast_to(xyz, (n, 3))), kind
            ia += n
    print("dimer concatenation check: ok")
    np.savez_compressed(out_path, **tables)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(here, "basis_tables.npz"))

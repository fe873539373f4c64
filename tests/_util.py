"""Shared helpers for the test-suite: golden loading and basis rebuilding."""

from __future__ import annotations

import os

import numpy as np

from asuka_b200 import basis as bm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def atoms_of(g: dict) -> list:
    return [(str(e), np.asarray(x)) for e, x in zip(g["elements"], g["coords_bohr"])]


def bases_of(g: dict):
    atoms = atoms_of(g)
    b = str(g["basis"])
    ao = bm.pack_basis(atoms, b, "ao")
    aux = bm.pack_basis(atoms, b, "aux")
    return ao, aux, bm.build_shell_pairs_l_order(ao)


def nelec_of(g: dict) -> int:
    return int(round(sum(bm.ATOMIC_NUMBER[str(e)] for e in g["elements"])))


def unpack_tril(Xt: np.ndarray, nao: int) -> np.ndarray:
    """(naux, ntri) lower-triangle rows -> (nao, nao, naux) symmetric."""
    naux = Xt.shape[0]
    X = np.zeros((nao, nao, naux))
    i, j = np.tril_indices(nao)
    X[i, j, :] = Xt.T
    X[j, i, :] = Xt.T
    return X

"""Rys node/weight table: against high-precision values, the oracle and the reference's roots."""

import os
import sys

import numpy as np
import pytest

import oracle as O
from _util import GOLDEN

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "asuka_b200", "data"))
import gen_rys_table as G  # noqa: E402


@pytest.fixture(scope="module")
def table():
    with np.load(os.path.join(ROOT, "asuka_b200", "data", "rys_table.npz")) as z:
        return {k: z[k] for k in z.files}


def test_table_matches_mpmath(table):
    rng = np.random.default_rng(11)
    for n in (1, 3, 5, 7, 9, 10):
        for T in list(rng.uniform(0, 96, 3)) + [0.0, 95.999, 96.0, 250.0]:
            x, w = G.evaluate(table, n, float(T))
            xm, wm = G.rys_mp(n, float(T))
            xm = np.array([float(v) for v in xm])
            wm = np.array([float(v) for v in wm])
            assert np.abs(x - xm).max() <= 2e-15 * np.abs(xm).max() + 1e-300
            assert np.all(np.abs(x - xm) <= 5e-15 * np.abs(xm))
            assert np.all(np.abs(w - wm) <= 5e-15 * np.abs(wm))


def test_table_matches_oracle_quad_roots(table):
    for n in range(1, 11):
        for T in (0.0, 0.37, 4.99, 5.01, 17.3, 60.0, 120.0):
            x, w = G.evaluate(table, n, T)
            xo, wo = O.rys_roots(n, T)
            assert np.all(np.abs(x - xo) <= 1e-13 * np.abs(xo)), (n, T)
            assert np.all(np.abs(w - wo) <= 1e-13 * np.abs(wo)), (n, T)


def test_table_matches_reference_roots_where_reference_is_accurate(table):
    with np.load(os.path.join(GOLDEN, "ref_roots.npz")) as z:
        Ts, R, W = z["T"], z["roots"], z["weights"]
    for n in range(1, 6):
        for i, T in enumerate(Ts):
            x, w = G.evaluate(table, n, float(T))
            assert np.all(np.abs(x - R[n - 1, i, :n]) <= 1e-10 * np.abs(x) + 1e-300), (n, T)
            assert np.all(np.abs(w - W[n - 1, i, :n]) <= 1e-10 * np.abs(w) + 1e-300), (n, T)

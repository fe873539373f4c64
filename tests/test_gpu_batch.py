"""Batched J/K builds of several molecules replayed from one CUDA graph."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _mols():
    from asuka_b200 import geometry as geo

    return [geo.water("ma-svp"), geo.n2("ma-svp"), geo.water_cluster(2, 3, "ma-svp"), geo.water_cluster(3, 5, "ma-svp")]


def _reference_jk(mol, Cw):
    """Stored-B J/K of the same molecule (whitened factors, FP64)."""
    from asuka_b200 import basis as bm
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e
    from asuka_b200.jk import df_JK_from_BQ

    atoms = list(mol.atoms_bohr)
    eng = DFEngine(bm.pack_basis(atoms, mol.basis, "ao"), bm.pack_basis(atoms, mol.basis, "aux"))
    B = whiten_3c2e(eng.int3c("Qmn"), cholesky_metric(eng.metric()), layout="Qmn")
    return df_JK_from_BQ(B, Cw, Cw @ Cw.T)


def _orbitals(batch, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for nao, naux, nocc, _ in batch.sizes:
        q = np.linalg.qr(rng.standard_normal((nao, nocc)))[0] * np.sqrt(2.0)
        out.append(torch.as_tensor(q, device="cuda"))
    return out


@pytest.mark.parametrize("block_bytes", [1 << 40, 1 << 16])
def test_batched_graph_matches_stored_jk(block_bytes):
    from asuka_b200.batch import BatchedDFJK

    mols = _mols()
    # block_bytes 64 KiB forces several aux blocks per molecule (integrals recomputed in pass 2)
    b = BatchedDFJK(mols, block_bytes=block_bytes, aux_block_min=16)
    assert all(s[3] for s in b.sizes) == (block_bytes > 1 << 30)
    for seed in (0, 1):  # two replays of the same graph with different orbitals
        Cws = _orbitals(b, seed)
        res = b.run(Cws)
        assert b.graph is not None
        for mol, Cw, (J, K) in zip(mols, Cws, res):
            J0, K0 = _reference_jk(mol, Cw)
            s = float(J0.abs().max())
            assert float((J - J0).abs().max()) < 1e-11 * s
            assert float((K - K0).abs().max()) < 1e-11 * s
            assert float((J - J.T).abs().max()) == 0.0 and float((K - K.T).abs().max()) == 0.0


@pytest.mark.parametrize("mixed_solve", [False, True])
def test_batched_graph_mixed_precision(mixed_solve):
    from asuka_b200.batch import BatchedDFJK

    mols = _mols()[:3]
    b = BatchedDFJK(mols, precision="mixed", block_bytes=1 << 16, aux_block_min=16, mixed_solve=mixed_solve)
    Cws = _orbitals(b, 2)
    res = b.run(Cws)
    for mol, Cw, (J, K) in zip(mols, Cws, res):
        J0, K0 = _reference_jk(mol, Cw)
        s = float(J0.abs().max())
        assert float((J - J0).abs().max()) < 1e-11 * s  # J stays FP64
        # split-BF16 tensor-core exchange update: FP32 accumulation with a truncation bias of
        # ~1e-6 relative on the diagonal (the mixed solve adds its conditioning-limited error)
        assert float((K - K0).abs().max()) < 5e-6 * s

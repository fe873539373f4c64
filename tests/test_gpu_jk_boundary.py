"""The DFJKWorkspace seams called the way the reference's callers call them.

``asuka/hf/df_jk.py:628-635,1036,1136`` hand the workspace CuPy arrays (any object with
``__cuda_array_interface__``), preallocated outputs, the raw pointer of CuPy's current stream
and ``sync=False``.  Here a minimal interface-only wrapper stands in for CuPy (CuPy is not
installed), the work runs on a non-default stream, and every result is checked against the
FP64 contraction on torch's own stream.
"""

import numpy as np
import pytest

from _util import bases_of, golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class CudaArray:
    """Exposes only ``__cuda_array_interface__`` (version 3) of a device buffer, like a CuPy array."""

    def __init__(self, t, read_only=False):
        self._t = t  # keeps the memory alive
        cai = dict(t.__cuda_array_interface__)
        cai["data"] = (cai["data"][0], bool(read_only))
        self.__cuda_array_interface__ = cai


def _case():
    from asuka_b200.df import DFEngine, cholesky_metric, whiten_3c2e
    from asuka_b200.scf import pack_B_to_Qp

    g = golden("h2o_matzvp")
    ao, aux, _sp = bases_of(g)
    eng = DFEngine(ao, aux)
    L = cholesky_metric(eng.metric())
    BQ = whiten_3c2e(eng.int3c("Qmn"), L, layout="Qmn").contiguous()
    C = torch.as_tensor(g["mo_coeff"], device="cuda")
    nocc = int((g["mo_occ"] > 0).sum())
    Cw = (C[:, :nocc] * torch.as_tensor(g["mo_occ"][:nocc], device="cuda").sqrt()).contiguous()
    D = (Cw @ Cw.T).contiguous()
    return BQ, Cw, D, pack_B_to_Qp(BQ)


def _ref(BQ, Cw, D):
    naux, nao, _ = BQ.shape
    rho = BQ.reshape(naux, -1) @ D.reshape(-1)
    J = (rho @ BQ.reshape(naux, -1)).view(nao, nao)
    U = torch.matmul(BQ, Cw)
    K = torch.einsum("qmi,qni->mn", U, U)
    return 0.5 * (J + J.T), 0.5 * (K + K.T)


def test_workspace_seams_with_interface_objects_on_caller_stream():
    from asuka_b200.jk import DFJKWorkspace

    BQ, Cw, D, BQp = _case()
    Jref, Kref = _ref(BQ, Cw, D)
    nao = D.shape[0]
    st = torch.cuda.Stream()
    ptr = int(st.cuda_stream)
    assert ptr != 0
    ws = DFJKWorkspace()
    outs = {k: torch.full((nao, nao), float("nan"), dtype=torch.float64, device="cuda") for k in
            ("J", "K", "Kb", "Kqp", "Dd", "Kmnq")}
    blk = torch.full((30, 47), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ws.jk_from_bq_cw(CudaArray(BQ), CudaArray(Cw), CudaArray(D), CudaArray(outs["J"]), CudaArray(outs["K"]),
                     q_block=96, stream=ptr, math_mode=-1, sync=False)
    ws.k_from_bq_cw(CudaArray(BQ), CudaArray(Cw), CudaArray(outs["Kb"]), q_block=128, stream=ptr, math_mode=0,
                    sync=False)
    ws.k_from_qp_cw(CudaArray(BQp), CudaArray(Cw), CudaArray(outs["Kqp"]), q_block=64, stream=ptr, sync=False)
    ws.k_from_bmnq_cw(CudaArray(BQ.permute(1, 2, 0).contiguous()), CudaArray(Cw), CudaArray(outs["Kmnq"]),
                      q_block=100, stream=ptr, sync=False)
    ws.density_syrk(CudaArray(Cw), CudaArray(outs["Dd"]), stream=ptr, sync=False)
    ws.k_block_from_qp_d(CudaArray(BQp), CudaArray(D), CudaArray(blk), nao, 10, 30, 3, 47, q_block=64,
                         col_block=32, stream=ptr, sync=False)
    st.synchronize()
    sJ, sK = float(Jref.abs().max()), float(Kref.abs().max())
    assert float((outs["J"] - Jref).abs().max()) < 1e-12 * sJ
    for k in ("K", "Kb", "Kqp", "Kmnq"):
        assert float((outs[k] - Kref).abs().max()) < 1e-12 * sK, k
    assert torch.equal(outs["K"], outs["K"].T) and torch.equal(outs["J"], outs["J"].T)
    assert float((outs["Dd"] - D).abs().max()) < 1e-13 * float(D.abs().max())
    assert float((blk - Kref[10:40, 3:50]).abs().max()) < 1e-12 * sK
    # mixed mode through the reference's math_mode switch: split-BF16 tensor-core products whose
    # FP32 accumulation truncates (a bias of ~1e-6 relative on the largest, diagonal elements)
    Km = torch.empty((nao, nao), dtype=torch.float64, device="cuda")
    ws.k_from_bq_cw(CudaArray(BQ), CudaArray(Cw), CudaArray(Km), stream=ptr, math_mode=8, sync=True)
    assert float((Km - Kref).abs().max()) < 5e-6 * sK


def test_workspace_argument_errors():
    from asuka_b200.jk import DFJKWorkspace

    ws = DFJKWorkspace()
    B = torch.zeros((4, 6, 6), dtype=torch.float64, device="cuda")
    Cw = torch.zeros((6, 2), dtype=torch.float64, device="cuda")
    K = torch.zeros((6, 6), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="writable"):
        ws.k_from_bq_cw(CudaArray(B), CudaArray(Cw), CudaArray(K, read_only=True))
    with pytest.raises(ValueError, match="float64"):
        ws.k_from_bq_cw(B.float(), Cw, K)
    with pytest.raises(ValueError, match="C-contiguous"):
        ws.k_from_bq_cw(B.transpose(1, 2), Cw, K)
    with pytest.raises(ValueError, match="nao mismatch"):
        ws.k_from_bq_cw(B, torch.zeros((5, 2), dtype=torch.float64, device="cuda"), K)
    with pytest.raises(ValueError, match="q_block"):
        ws.k_from_bq_cw(B, Cw, K, q_block=0)
    with pytest.raises(ValueError, match="ntri"):
        ws.k_from_qp_cw(torch.zeros((4, 20), dtype=torch.float64, device="cuda"), Cw, K)
    with pytest.raises(ValueError, match="__cuda_array_interface__"):
        ws.k_from_bq_cw(np.zeros((4, 6, 6)), Cw, K)
    ws.release()
    with pytest.raises(RuntimeError):
        ws.k_from_bq_cw(B, Cw, K)

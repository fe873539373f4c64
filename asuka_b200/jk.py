"""DF Coulomb/exchange contractions on the device.

Mirrors the reference's J/K seam (``asuka/hf/cuda/ext/src/hf_df_jk_cuda_ext.cpp:198-1150``
``DFJKWorkspace`` and ``asuka/hf/df_jk.py:424,528,1040``):

    J = sum_Q B_Q (B_Q . D)          K = sum_Q (B_Q Cw)(B_Q Cw)^T,  Cw = C_occ sqrt(occ)

with B_Q in the 'Qmn' layout (naux, nao, nao).  Outputs are zeroed by the
callee and returned fully symmetric, as the reference's workspace does.

Precision modes:

* ``'fp64'``  -- FP64 GEMMs (cuBLAS DGEMM through torch);
* ``'mixed'`` -- the half-transform U = B_Q Cw and the exchange update
  K += U U^T run on the tensor cores as split-BF16 GEMMs (``asuka_b200.tc``,
  tcgen05: each FP64 operand split into three BF16 terms in registers, the
  cross products of order <= 2^-16 accumulated in FP32 per k span and the spans
  combined in FP64; ~1e-7 relative).  J (one HBM-bound pass over B) stays FP64.
"""

from __future__ import annotations

import torch

from . import tc as _tc


def _sym(A: torch.Tensor) -> torch.Tensor:
    return 0.5 * (A + A.T)


def df_J_from_BQ_D(BQ: torch.Tensor, D: torch.Tensor) -> torch.Tensor:
    naux = BQ.shape[0]
    B2 = BQ.reshape(naux, -1)
    rho = B2 @ D.reshape(-1)
    return _sym((rho @ B2).reshape(D.shape))


def df_K_from_BQ_Cw(BQ: torch.Tensor, Cw: torch.Tensor, q_block: int = 256, precision: str = "fp64") -> torch.Tensor:
    naux, nao, _ = BQ.shape
    nocc = Cw.shape[1]
    K = torch.zeros((nao, nao), dtype=torch.float64, device=BQ.device)
    if nocc == 0:
        return K
    for q0 in range(0, naux, q_block):
        q1 = min(naux, q0 + q_block)
        blk = BQ[q0:q1]
        if precision == "fp64":
            U = torch.matmul(blk.reshape(-1, nao), Cw).reshape(q1 - q0, nao, nocc)
            U2 = U.permute(1, 0, 2).reshape(nao, -1)
            K += U2 @ U2.T
        else:
            U = _tc.matmul(blk.reshape(-1, nao), Cw).view(q1 - q0, nao, nocc)
            _tc.syrk_qblocks(U, out=K)
    return _sym(K)


def df_JK_from_BQ(BQ: torch.Tensor, Cw: torch.Tensor, D: torch.Tensor, q_block: int = 256,
                  precision: str = "fp64") -> tuple[torch.Tensor, torch.Tensor]:
    return df_J_from_BQ_D(BQ, D), df_K_from_BQ_Cw(BQ, Cw, q_block=q_block, precision=precision)


def density_from_Cw(Cw: torch.Tensor) -> torch.Tensor:
    return _sym(Cw @ Cw.T)


def _as_device_f64(obj, name: str, ndim: int, writable: bool = False) -> torch.Tensor:
    """Zero-copy torch view of a CUDA FP64 array given as a torch tensor, any object with
    ``__cuda_array_interface__`` (CuPy, Numba, ...) or a DLPack capsule provider.

    Checks mirror the reference's ``cuda_array_view_from_object`` / ``require_typestr_f64`` /
    ``require_c_contiguous`` (``asuka/hf/cuda/ext/src/hf_df_jk_cuda_ext.cpp:128-186``) and raise
    ``ValueError`` with the argument's name.
    """
    if isinstance(obj, torch.Tensor):
        t = obj
    elif hasattr(obj, "__cuda_array_interface__"):
        cai = obj.__cuda_array_interface__
        if writable and bool(cai.get("data", (0, False))[1]):
            raise ValueError(f"{name} must be a writable CUDA array")
        if str(cai.get("typestr", "")).lstrip("<=|") != "f8":
            raise ValueError(f"{name} must be float64")
        t = torch.as_tensor(obj, device="cuda")
    elif hasattr(obj, "__dlpack__") and hasattr(obj, "__dlpack_device__") and int(obj.__dlpack_device__()[0]) == 2:
        t = torch.from_dlpack(obj)  # a CUDA DLPack provider (kDLCUDA)
    else:
        raise ValueError(f"{name} must support __cuda_array_interface__")
    if t.dtype != torch.float64:
        raise ValueError(f"{name} must be float64")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA array")
    if t.dim() != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be C-contiguous")
    return t


def _stream_of(stream: int | None, device: torch.device) -> torch.cuda.Stream:
    """The caller's stream: a raw cudaStream_t (int), 0 for the legacy default stream, or None
    for torch's current stream."""
    if stream is None:
        return torch.cuda.current_stream(device)
    if int(stream) == 0:
        return torch.cuda.default_stream(device)
    return torch.cuda.ExternalStream(int(stream), device=device)


def unpack_Qp(B_Qp: torch.Tensor, nao: int, q0: int = 0, q1: int | None = None) -> torch.Tensor:
    """Rows q0:q1 of packed B_Qp (naux, ntri), p = mu(mu+1)/2 + nu (mu >= nu), as (q, nao, nao)."""
    q1 = B_Qp.shape[0] if q1 is None else q1
    i, j = torch.tril_indices(nao, nao, device=B_Qp.device)
    out = torch.empty((q1 - q0, nao, nao), dtype=B_Qp.dtype, device=B_Qp.device)
    blk = B_Qp[q0:q1]
    out[:, i, j] = blk
    out[:, j, i] = blk
    return out


class DFJKWorkspace:
    """Reference-shaped J/K workspace (``hf_df_jk_cuda_ext.cpp:198-1150``, bindings ``:1149-1290``).

    Every method takes FP64 C-contiguous CUDA arrays -- torch tensors or any object with
    ``__cuda_array_interface__`` such as the CuPy arrays the reference passes -- without
    copying them, writes the result into the caller's preallocated output (zeroed first, fully
    symmetric on return), and runs on the caller's stream (``stream`` = raw ``cudaStream_t``;
    0 = the legacy default stream).  ``sync=False`` (the default, as in the reference) returns
    without waiting.  Argument errors raise ``ValueError`` (the reference's
    ``std::invalid_argument``).

    ``math_mode``: -1 (default) keeps the workspace's own precision; 0 (CUBLAS_DEFAULT_MATH)
    forces FP64; 8 (the reference's FP64-emulation mode id) selects the mixed split-BF16 path.
    """

    def __init__(self, precision: str = "fp64"):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self._released = False

    def _prec(self, math_mode: int) -> str:
        if self._released:
            raise RuntimeError("DFJKWorkspace used after release()")
        if math_mode == 0:
            return "fp64"
        if math_mode == 8:
            return "mixed"
        return self.precision

    @staticmethod
    def _qb(q_block: int) -> int:
        if int(q_block) <= 0:
            raise ValueError("q_block must be > 0")
        return int(q_block)

    def _run(self, st: torch.cuda.Stream, sync: bool, fn):
        with torch.cuda.stream(st):
            fn()
        if sync:
            st.synchronize()

    def jk_from_bq_cw(self, BQ, Cw, D, out_J, out_K, *, q_block: int = 128, stream: int | None = 0,
                      math_mode: int = -1, sync: bool = False):
        """J = sum_Q B_Q (B_Q . D) and K = sum_Q (B_Q Cw)(B_Q Cw)^T into out_J, out_K."""
        prec = self._prec(math_mode)
        B = _as_device_f64(BQ, "BQ", 3)
        C = _as_device_f64(Cw, "Cw", 2)
        Dm = _as_device_f64(D, "D", 2)
        J = _as_device_f64(out_J, "out_J", 2, writable=True)
        K = _as_device_f64(out_K, "out_K", 2, writable=True)
        naux, nao, nao1 = B.shape
        if nao != nao1:
            raise ValueError("BQ must have shape (naux, nao, nao)")
        if C.shape[0] != nao:
            raise ValueError("Cw nao mismatch with BQ")
        if tuple(Dm.shape) != (nao, nao) or tuple(J.shape) != (nao, nao) or tuple(K.shape) != (nao, nao):
            raise ValueError("D, out_J and out_K must have shape (nao, nao)")
        qb = self._qb(q_block)

        def fn():
            Jr, Kr = df_JK_from_BQ(B, C, Dm, q_block=max(qb, 1), precision=prec)
            J.copy_(Jr)
            K.copy_(Kr)

        self._run(_stream_of(stream, B.device), sync, fn)
        return out_J, out_K

    def k_from_bq_cw(self, BQ, Cw, out, *, q_block: int = 128, stream: int | None = 0, math_mode: int = -1,
                     sync: bool = False):
        """K = sum_Q (B_Q Cw)(B_Q Cw)^T into out; BQ is (naux, nao, nao)."""
        prec = self._prec(math_mode)
        B = _as_device_f64(BQ, "BQ", 3)
        C = _as_device_f64(Cw, "Cw", 2)
        K = _as_device_f64(out, "out", 2, writable=True)
        naux, nao, nao1 = B.shape
        if nao != nao1:
            raise ValueError("BQ must have shape (naux, nao, nao)")
        if C.shape[0] != nao:
            raise ValueError("Cw nao mismatch with BQ")
        if tuple(K.shape) != (nao, nao):
            raise ValueError("out must have shape (nao, nao)")
        qb = self._qb(q_block)
        self._run(_stream_of(stream, B.device), sync,
                  lambda: K.copy_(df_K_from_BQ_Cw(B, C, q_block=qb, precision=prec)))
        return out

    def k_from_bmnq_cw(self, B_mnQ, Cw, out, *, q_block: int = 128, stream: int | None = 0, math_mode: int = -1,
                       sync: bool = False):
        """K from B in the 'mnQ' layout (nao, nao, naux) (``hf_df_jk_cuda_ext.cpp:912``)."""
        prec = self._prec(math_mode)
        B = _as_device_f64(B_mnQ, "B_mnQ", 3)
        C = _as_device_f64(Cw, "Cw", 2)
        K = _as_device_f64(out, "out", 2, writable=True)
        nao, nao1, naux = B.shape
        if nao != nao1:
            raise ValueError("B_mnQ must have shape (nao, nao, naux)")
        if C.shape[0] != nao:
            raise ValueError("Cw nao mismatch with B_mnQ")
        if tuple(K.shape) != (nao, nao):
            raise ValueError("out must have shape (nao, nao)")
        qb = self._qb(q_block)

        def fn():
            Kr = torch.zeros((nao, nao), dtype=torch.float64, device=B.device)
            for q0 in range(0, naux, qb):
                q1 = min(naux, q0 + qb)
                Kr += df_K_from_BQ_Cw(B[:, :, q0:q1].permute(2, 0, 1).contiguous(), C, q_block=q1 - q0,
                                      precision=prec)
            K.copy_(_sym(Kr))

        self._run(_stream_of(stream, B.device), sync, fn)
        return out

    def k_from_qp_cw(self, B_Qp, Cw, out, *, q_block: int = 128, stream: int | None = 0, math_mode: int = -1,
                     sync: bool = False):
        """K from packed B_Qp (naux, ntri), p = mu(mu+1)/2 + nu (``hf_df_jk_cuda_ext.cpp:600``); unpacks one
        q-block at a time."""
        prec = self._prec(math_mode)
        B = _as_device_f64(B_Qp, "B_Qp", 2)
        C = _as_device_f64(Cw, "Cw", 2)
        K = _as_device_f64(out, "out", 2, writable=True)
        naux, ntri = B.shape
        nao = C.shape[0]
        if tuple(K.shape) != (nao, nao):
            raise ValueError("out must have shape (nao, nao)")
        if ntri != nao * (nao + 1) // 2:
            raise ValueError("B_Qp must have ntri=nao*(nao+1)//2")
        qb = self._qb(q_block)

        def fn():
            Kr = torch.zeros((nao, nao), dtype=torch.float64, device=B.device)
            for q0 in range(0, naux, qb):
                q1 = min(naux, q0 + qb)
                Kr += df_K_from_BQ_Cw(unpack_Qp(B, nao, q0, q1), C, q_block=q1 - q0, precision=prec)
            K.copy_(_sym(Kr))

        self._run(_stream_of(stream, B.device), sync, fn)
        return out

    def k_block_from_qp_d(self, B_Qp, D, out, nao: int, row0: int, row_count: int, col0: int, col_count: int, *,
                          q_block: int = 128, col_block: int = 64, stream: int | None = 0, math_mode: int = -1,
                          sync: bool = False):
        """out = K[row0:row0+row_count, col0:col0+col_count] with K = sum_Q B_Q D B_Q from packed B_Qp
        (``hf_df_jk_cuda_ext.cpp:734``)."""
        self._prec(math_mode)
        B = _as_device_f64(B_Qp, "B_Qp", 2)
        Dm = _as_device_f64(D, "D", 2)
        O = _as_device_f64(out, "out", 2, writable=True)
        naux, ntri = B.shape
        if tuple(Dm.shape) != (nao, nao):
            raise ValueError("nao mismatch between provided nao and D")
        if min(row0, row_count, col0, col_count) < 0:
            raise ValueError("invalid row/col arguments")
        if row0 > nao or row_count > nao - row0:
            raise ValueError("row range out of bounds")
        if col0 > nao or col_count > nao - col0:
            raise ValueError("col range out of bounds")
        if tuple(O.shape) != (row_count, col_count):
            raise ValueError("out shape mismatch with row_count/col_count")
        if ntri != nao * (nao + 1) // 2:
            raise ValueError("B_Qp must have ntri=nao*(nao+1)//2")
        qb = self._qb(q_block)
        if int(col_block) <= 0:
            raise ValueError("col_block must be > 0")

        def fn():
            O.zero_()
            for q0 in range(0, naux, qb):
                q1 = min(naux, q0 + qb)
                BQ = unpack_Qp(B, nao, q0, q1)
                left = torch.matmul(BQ[:, row0:row0 + row_count, :], Dm)
                O.add_(torch.matmul(left, BQ[:, :, col0:col0 + col_count]).sum(0))

        self._run(_stream_of(stream, B.device), sync, fn)
        return out

    def density_syrk(self, Cw, out, *, stream: int | None = 0, math_mode: int = -1, sync: bool = False):
        """D = Cw Cw^T into out (``hf_df_jk_cuda_ext.cpp:373``)."""
        self._prec(math_mode)
        C = _as_device_f64(Cw, "Cw", 2)
        O = _as_device_f64(out, "out", 2, writable=True)
        nao = C.shape[0]
        if tuple(O.shape) != (nao, nao):
            raise ValueError("out must have shape (nao, nao)")
        self._run(_stream_of(stream, C.device), sync, lambda: O.copy_(density_from_Cw(C)))
        return out

    def release(self) -> None:
        self._released = True

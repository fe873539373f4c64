"""DF two-electron energy and its nuclear gradient.

``DFEnergyFunction`` is a ``torch.autograd.Function`` whose forward maps
(nuclear coordinates R, weighted occupied orbitals Cw with D = Cw Cw^T) to
(E_2e, J, K), building the DF integrals at R on the GPU, and whose backward
returns dE_2e/dR from the Rys derivative integrals contracted on the fly with
the adjoints (and dE_2e/dCw = 2 (J - K/2) Cw).

Forward, with X_P = (mu nu|P), V = L L^T:
    rho = X . D,  d = V^-1 rho,  J = sum_P d_P X_P
    Y_P = X_P Cw, W = L^-1 Y,    K = sum_Q W_Q W_Q^T
    E_2e = 1/2 rho.d - 1/4 tr(D K)
Backward (M_Q = Cw^T W_Q, Z = L^-T M):
    dE/dX_P = d_P D - 1/2 Cw Z_P Cw^T
    dE/dV   = -1/2 d d^T + 1/4 Z Z^T          (Z as naux x nocc^2)
    dE/dR   = sum dE/dX . dX/dR + sum dE/dV . dV/dR
This equals the reference's whitened-factor route (bar_L = rho_Q D - 1/2 D B_Q D
through ``df_whiten_adjoint_Qmn``/``chol_lower_adjoint``,
``asuka/integrals/df_adjoint.py:172-235,322-361``) without the two
naux^2 nao^2 triangular solves.

``compute_df_gradient_contributions_analytic_packed_bases`` keeps the
reference's signature and whitened-factor adjoints
(``asuka/integrals/grad.py:114-723``) for callers that hold B and dE/dB.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import linalg as _la
from . import mixed as _mixed
from . import tc as _tc
from .df import DFEngine, cholesky_metric

# Mixed mode: which dense products run as split-BF16 tensor-core GEMMs (tcgen05, three terms).
# The tensor cores' FP32 accumulation is biased (it truncates), about 1e-7 relative in the same
# direction for every element, and a bias does not average out: run as a tensor-core product,
# Y = X Cw moved E_2e of (H2O)8 by 4e-4 Eh and Gamma moved the gradient by 2e-6 Eh/bohr.  So only
# the exchange update K = sum W W^T runs there by default: it enters neither the energy (taken
# from M = Cw^T W in FP64) nor the gradient, only the Fock matrix of the early SCF iterations.
MIXED_K_TC = True
MIXED_Y_TC = False
MIXED_GAMMA_TC = False


def _mm(A, B, precision):
    return A @ B if precision == "fp64" else _mixed.matmul(A, B)


def _nomark(_key: str) -> None:
    pass


_JK_STREAMS: dict = {}


def _jk_streams(device: torch.device):
    """Two side streams per device: J (overlapping the metric solve) and K (overlapping the adjoints)."""
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx not in _JK_STREAMS:
        _JK_STREAMS[idx] = (torch.cuda.Stream(device=device), torch.cuda.Stream(device=device))
    return _JK_STREAMS[idx]


def _gamma_into(Cw: torch.Tensor, A: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
    """out[P] = Cw A_P Cw^T for symmetric A_P ((nP, nocc, nocc); out (nP, nao, nao), contiguous).

    U = Cw [A_0 | A_1 | ...] as one GEMM ((nao, nP nocc)), then the library's symmetric FP64
    kernel (``dfb_gamma_sym``: upper tiles only, each written with its transpose): the inner
    dimension is only nocc, so the product is bound by writing Gamma, and cuBLAS ran it at about
    half the FP64 rate."""
    nP, nocc = A.shape[0], A.shape[1]
    nao = Cw.shape[0]
    if nP == 0:
        return out
    Cw = Cw.contiguous()
    U = Cw @ A.permute(1, 0, 2).reshape(nocc, nP * nocc)  # (nao, nP, nocc): U[mu, P, j] = (Cw A_P)[mu, j]
    if not out.is_contiguous():
        raise ValueError("Gamma output must be contiguous")
    rc = _lib.lib().dfb_gamma_sym(nP, nao, nocc, _lib.ptr(U), nP * nocc, nocc, _lib.ptr(Cw), _lib.ptr(out),
                                  int(torch.cuda.current_stream(out.device).cuda_stream))
    _lib.check(rc, "dfb_gamma_sym")
    return out


def _fork(main: torch.cuda.Stream, side: torch.cuda.Stream) -> None:
    ev = torch.cuda.Event()
    ev.record(main)
    side.wait_event(ev)


def df_forward(engine: DFEngine, Cw: torch.Tensor, precision: str = "fp64", X: torch.Tensor | None = None,
               with_adjoints: bool = False):
    """Integrals at the engine's current geometry, then (E_2e, J, K) and the saved intermediates
    (with the gradient adjoints when ``with_adjoints``, see ``df_contract``)."""
    _V, L, X = engine.metric_cholesky_int3c(X, precision=precision)
    return df_contract(engine, Cw, X, L, precision, with_adjoints=with_adjoints)


def df_contract(engine: DFEngine, Cw: torch.Tensor, X: torch.Tensor, L: torch.Tensor, precision: str = "fp64",
                mark=_nomark, with_adjoints: bool = False):
    """(E_2e, J, K) and the saved intermediates from the 3c tensor X ('Qmn') and the metric factor L.

    With D = Cw Cw^T the Coulomb density rho_P = <X_P, D> = sum Cw * (X_P Cw) is read
    from Y = X Cw (needed for K anyway) instead of a second pass over X.  ``mark(name)``
    is called after each phase (timing hooks).

    J and K are off the critical path of the energy and gradient: J = sum_P d_P X_P runs on a
    side stream while the main stream solves W = L^-1 Y, and K = sum W W^T on a second side
    stream while the main stream forms the gradient adjoints (``with_adjoints``: Gamma written
    over X, and G2, kept in the saved dict for ``df_backward``).  Both join the main stream
    before this returns.
    """
    nao, naux = engine.nao, engine.naux
    nocc = Cw.shape[1]
    mixed = precision != "fp64"
    X2 = X.view(naux, nao * nao)
    D = Cw @ Cw.T
    D = 0.5 * (D + D.T)
    if mixed and MIXED_Y_TC:
        Y = _tc.matmul(X.view(naux * nao, nao), Cw).view(naux, nao * nocc)
    else:
        Y = (X.view(naux * nao, nao) @ Cw).view(naux, nao * nocc)
    mark("jk_Y")
    rho = Y @ Cw.reshape(-1)
    d = torch.cholesky_solve(rho.view(-1, 1), L).view(-1)
    main = torch.cuda.current_stream(X.device)
    sJ, sK = _jk_streams(X.device)
    _fork(main, sJ)
    with torch.cuda.stream(sJ):
        J = (d @ X2).view(nao, nao)
        J = 0.5 * (J + J.T)
    mark("jk_rho_J")
    # the solve stays FP64 in both modes: block substitution runs at the DGEMM rate, and a
    # split-BF16 product with L^-1 loses accuracy in proportion to the metric's conditioning
    Linv_blocks = _la.diag_block_inverses(L)
    W = _la.solve_lower(L, Y, Linv_blocks, out=Y)
    mark("jk_W_solve")
    W3 = W.view(naux, nao, nocc)
    # M_Q = Cw^T W_Q (FP64 in both modes): the exchange energy tr(D K) = sum_Q |M_Q|^2, and the
    # adjoint's input
    M = torch.matmul(Cw.T, W3)
    _fork(main, sK)
    with torch.cuda.stream(sK):
        if mixed and MIXED_K_TC:
            K = _tc.syrk_qblocks(W3)
        else:
            W2 = W3.permute(1, 0, 2).reshape(nao, naux * nocc)
            K = W2 @ W2.T
        K = 0.5 * (K + K.T)
    E = 0.5 * torch.dot(rho, d) - 0.25 * torch.sum(M * M)
    saved = dict(X=X, L=L, d=d, W=W, M=M, D=D, Linv_blocks=Linv_blocks)
    main.wait_stream(sJ)  # J has read X: the adjoint may overwrite it now
    if with_adjoints:
        saved["adj"] = df_adjoints(engine, Cw, saved, precision)
    main.wait_stream(sK)
    mark("jk_K")
    return E, J, K, saved


def df_adjoints(engine: DFEngine, Cw: torch.Tensor, saved: dict, precision: str = "fp64"):
    """Adjoints of the 3c and 2c integrals: (Gamma (naux, nao, nao), written over X; G2 (naux, naux))."""
    nao, naux = engine.nao, engine.naux
    nocc = Cw.shape[1]
    X, L, d, W = saved["X"], saved["L"], saved["d"], saved["W"]
    # M_Q = Cw^T W_Q  (naux, nocc, nocc)
    M = saved.get("M")
    if M is None:
        M = torch.matmul(Cw.T, W.view(naux, nao, nocc))
    M = 0.5 * (M + M.transpose(1, 2))
    Z = _la.solve_lower_T(L, M.reshape(naux, nocc * nocc), saved.get("Linv_blocks"))
    Zq = Z.view(naux, nocc, nocc)
    # Gamma_P = d_P D - 1/2 Cw Z_P Cw^T = Cw (d_P I - 1/2 Z_P) Cw^T since D = Cw Cw^T:
    # one batched GEMM, written over X's storage (X is not needed afterwards)
    Zp = -0.5 * Zq + d.view(naux, 1, 1) * torch.eye(nocc, dtype=Zq.dtype, device=Zq.device)
    G3 = X
    if precision != "fp64" and MIXED_GAMMA_TC:
        _tc.bmm(Cw, torch.matmul(Zp, Cw.T), out=G3)
    else:
        _gamma_into(Cw, Zp, G3)
    G2 = -0.5 * torch.outer(d, d) + 0.25 * (Z @ Z.T)
    return G3, G2


def df_backward(engine: DFEngine, Cw: torch.Tensor, saved: dict, grad: torch.Tensor | None = None,
                precision: str = "fp64") -> torch.Tensor:
    """dE_2e/dR accumulated into grad (natm, 3)."""
    G3, G2 = saved["adj"] if "adj" in saved else df_adjoints(engine, Cw, saved, precision)
    if grad is None:
        grad = torch.zeros((engine.natm, 3), dtype=torch.float64, device=G3.device)
    engine.deriv3c_2c(G3, G2, grad, precision=precision)
    return grad


class DFEnergyFunction(torch.autograd.Function):
    """(R, Cw) -> (E_2e, J, K); backward gives dE_2e/dR and dE_2e/dCw."""

    @staticmethod
    def forward(ctx, coords: torch.Tensor, Cw: torch.Tensor, engine: DFEngine, precision: str = "fp64"):
        engine.set_coords(coords.detach())
        E, J, K, saved = df_forward(engine, Cw.detach(), precision, with_adjoints=ctx.needs_input_grad[0])
        ctx.engine = engine
        ctx.precision = precision
        ctx.saved = saved
        ctx.save_for_backward(Cw.detach(), J, K)
        ctx.mark_non_differentiable(J, K)
        return E, J, K

    @staticmethod
    def backward(ctx, gE, gJ, gK):
        Cw, J, K = ctx.saved_tensors
        g = df_backward(ctx.engine, Cw, ctx.saved, precision=ctx.precision)
        ctx.saved = None
        gCw = 2.0 * ((J - 0.5 * K) @ Cw)
        return g * gE, gCw * gE, None, None


def df_energy(coords: torch.Tensor, Cw: torch.Tensor, engine: DFEngine, precision: str = "fp64"):
    """Differentiable E_2e(R, Cw); returns (E, J, K)."""
    return DFEnergyFunction.apply(coords, Cw, engine, precision)


# ---------------------------------------------------------------- streamed (B never stored)

def _solve_lower_inplace(L: torch.Tensor, Y: torch.Tensor, mixed_solve: bool = False,
                         ncol: int = 1 << 18) -> torch.Tensor:
    """Y <- L^-1 Y in place.

    Default: FP64 block substitution (``asuka_b200.linalg``) -- the metric solve stays FP64
    in every precision mode.  ``mixed_solve``: L^-1 formed once in FP64, split once into BF16
    terms, and applied to each column block as a split-BF16 GEMM (one block copy alive at a
    time); its error grows with the metric's condition number (1e-4 relative in K for the
    ma-QZVP/RICD aux basis), so it is an explicit opt-in.
    """
    n, m = Y.shape
    ncol = max(1, min(m, ncol * 1024 // max(n, 1)))
    if not mixed_solve:
        return _la.solve_lower(L, Y, out=Y)
    Linv = torch.linalg.solve_triangular(L, torch.eye(n, dtype=L.dtype, device=L.device), upper=False)
    sp = _mixed.split3(Linv)
    del Linv
    for c0 in range(0, m, ncol):
        c1 = min(m, c0 + ncol)
        Y[:, c0:c1] = _mixed.matmul(None, Y[:, c0:c1].contiguous(), kblock=4096, a_split=sp)
    return Y


def df_energy_grad_streamed(engine: DFEngine, Cw: torch.Tensor, aux_block: int = 128, precision: str = "fp64",
                            stats: dict | None = None, mixed_solve: bool = False):
    """E_2e and dE_2e/dR without storing the 3c tensor: the integrals are recomputed per aux block.

    Forward: for each aux block b, X_b -> Y_b = X_b Cw (rho from Y); then d = V^-1 rho,
    W = L^-1 Y (in place), K = sum_Q W_Q W_Q^T by aux chunks.  Backward: M = Cw^T W,
    Z = L^-T M, and for each block Gamma_b = Cw (d_b I - 1/2 Z_b) Cw^T contracted with the
    block's derivative integrals (the streamed analogue of
    ``asuka/hf/df_jk_streamed.py:167-325``, with the gradient recomputing the integrals
    instead of reading a stored B).  The largest buffer is Y/W (naux x nao x nocc)
    instead of the 3c tensor (naux x nao^2).  ``precision='mixed'`` evaluates the
    integrals and their derivatives with FP32 recurrence tables and accumulators and
    runs the exchange update K as a split-BF16 tensor-core GEMM; the metric solves stay
    FP64 unless ``mixed_solve`` (split-BF16 product with L^-1) is asked for.
    Returns (E, grad (natm, 3), K).
    """
    nao, naux = engine.nao, engine.naux
    nocc = Cw.shape[1]
    dev = engine.device
    torch.cuda.reset_peak_memory_stats(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    ev[0].record()
    V = engine.metric()
    L = cholesky_metric(V)
    del V
    blocks = engine.aux_blocks(aux_block)
    Y = torch.empty((naux, nao * nocc), dtype=torch.float64, device=dev)
    bmax = max(p1 - p0 for p0, p1, _ in blocks)
    Xb_buf = torch.zeros((bmax, nao, nao), dtype=torch.float64, device=dev)
    for p0, p1, blk in blocks:
        Xb = engine.int3c_block(blk, p0, p1, out=Xb_buf[: p1 - p0], dropped_zero=True, precision=precision)
        torch.matmul(Xb.view(-1, nao), Cw, out=Y[p0:p1].view(-1, nocc))
    ev[1].record()
    rho = Y @ Cw.reshape(-1)
    d = torch.cholesky_solve(rho.view(-1, 1), L).view(-1)
    W = _solve_lower_inplace(L, Y, mixed_solve and precision != "fp64")
    W3 = W.view(naux, nao, nocc)
    K = torch.zeros((nao, nao), dtype=torch.float64, device=dev)
    qb = max(1, (1 << 27) // max(nao * nocc, 1))
    if precision != "fp64":
        _tc.syrk_qblocks(W3, out=K)  # reads W in place, k = (Q, i)
    for q0 in range(0, naux if precision == "fp64" else 0, qb):
        Wc = W3[q0:q0 + qb].permute(1, 0, 2).reshape(nao, -1)
        K.addmm_(Wc, Wc.T)
    K = 0.5 * (K + K.T)
    D = Cw @ Cw.T
    E = 0.5 * torch.dot(rho, d) - 0.25 * torch.sum(D * K)
    ev[2].record()
    M = torch.matmul(Cw.T, W3)
    del W, W3, Y
    for q0 in range(0, naux, qb):
        Mc = M[q0:q0 + qb]
        Mc.copy_(0.5 * (Mc + Mc.transpose(1, 2)))
    Z = _la.solve_lower_T(L, M.view(naux, nocc * nocc))
    del M
    Zq = Z.view(naux, nocc, nocc)
    grad = torch.zeros((engine.natm, 3), dtype=torch.float64, device=dev)
    eye = torch.eye(nocc, dtype=Cw.dtype, device=dev)
    ev[3].record()
    for p0, p1, blk in blocks:
        Zp = -0.5 * Zq[p0:p1] + d[p0:p1].view(-1, 1, 1) * eye
        G3 = Xb_buf[: p1 - p0]
        _gamma_into(Cw, Zp, G3)
        engine.deriv3c_block(blk, G3, grad, precision=precision)
    ev[4].record()
    G2 = -0.5 * torch.outer(d, d) + 0.25 * (Z @ Z.T)
    engine.deriv2c(G2, grad, precision=precision)
    ev[5].record()
    if stats is not None:
        torch.cuda.synchronize(dev)
        stats.update(peak_hbm_bytes=int(torch.cuda.max_memory_allocated(dev)), nblocks=len(blocks),
                     x_bytes_if_stored=int(naux) * nao * nao * 8, y_bytes=int(naux) * nao * nocc * 8,
                     ms_int3c_and_Y=ev[0].elapsed_time(ev[1]), ms_jk=ev[1].elapsed_time(ev[2]),
                     ms_adjoint=ev[2].elapsed_time(ev[3]), ms_deriv3c=ev[3].elapsed_time(ev[4]),
                     ms_deriv2c=ev[4].elapsed_time(ev[5]), ms_total=ev[0].elapsed_time(ev[5]))
    return E, grad, K


# ---------------------------------------------------------------- reference seam

def whitened_adjoints(B: torch.Tensor, barL: torch.Tensor, L: torch.Tensor):
    """Backprop dE/dB through the whitening and the metric Cholesky.

    B (nao, nao, naux) whitened factors, barL (naux, nao, nao) = dE/dB, L the metric
    factor -> (bar_X (naux, nao, nao) symmetric, bar_V (naux, naux) symmetric), the
    adjoints of the unwhitened integrals X and of the metric V
    (``asuka/integrals/df_adjoint.py:172-235,322-361``).
    """
    nao, _, naux = B.shape
    tmp = _la.solve_lower_T(L, barL.reshape(naux, nao * nao))  # L^-T bar_B^T
    bar_Lc = -torch.tril(tmp @ B.reshape(nao * nao, naux))
    bar_X = tmp.view(naux, nao, nao)
    bar_X = 0.5 * (bar_X + bar_X.transpose(1, 2))
    G = torch.tril(L.T @ bar_Lc)
    G.diagonal().mul_(0.5)
    t2 = torch.linalg.solve_triangular(L.T, G, upper=True)
    bar_V = torch.linalg.solve_triangular(L.T, t2.T, upper=True).T
    return bar_X.contiguous(), (0.5 * (bar_V + bar_V.T)).contiguous()


def whitened_adjoints_qp(B_Qp: torch.Tensor, barL_Qp: torch.Tensor, L: torch.Tensor, nao: int):
    """``whitened_adjoints`` in the packed lower-triangle layout (naux, ntri), p = m(m+1)/2 + n.

    Every step acts on the aux index or contracts over the full (mu, nu) square, which in packed
    form is a weighted sum over p (weight 2 off the diagonal), so nothing is unpacked:
    returns (bar_X in packed form (naux, ntri), bar_V (naux, naux)); the packed-Qp route of
    ``asuka/integrals/df_grad_context.py:1160``.
    """
    naux = B_Qp.shape[0]
    i, j = torch.tril_indices(nao, nao, device=B_Qp.device)
    w = torch.where(i == j, 1.0, 2.0).to(torch.float64)
    tmp = _la.solve_lower_T(L, barL_Qp)  # L^-T bar_B^T, packed (naux, ntri)
    bar_Lc = -torch.tril((tmp * w) @ B_Qp.T)
    G = torch.tril(L.T @ bar_Lc)
    G.diagonal().mul_(0.5)
    t2 = torch.linalg.solve_triangular(L.T, G, upper=True)
    bar_V = torch.linalg.solve_triangular(L.T, t2.T, upper=True).T
    return tmp, (0.5 * (bar_V + bar_V.T)).contiguous()


def compute_df_gradient_contributions_analytic_packed_bases(ao_basis, aux_basis, *, atom_coords_bohr, B_ao,
                                                            bar_L_ao, L_chol=None, backend: str = "cuda",
                                                            df_threads: int = 0, profile: dict | None = None):
    """DF 2e gradient from whitened factors B (nao,nao,naux) and dE/dB (naux,nao,nao); returns (natm, 3).

    Same contract as ``asuka/integrals/grad.py:114``: backprop through the
    whitening and the metric Cholesky to the unwhitened integrals, then contract
    the analytic integral derivatives.  Runs on the GPU (``backend`` must be
    'cuda' or 'gpu'; there is no CPU path).
    """
    if str(backend).lower() not in ("cuda", "gpu"):
        raise ValueError("this engine runs on the GPU only (backend='cuda')")
    R = np.asarray(atom_coords_bohr, dtype=np.float64).reshape((-1, 3))
    natm = R.shape[0]
    eng = DFEngine(ao_basis, aux_basis, atom_coords_bohr=R)
    dev = eng.device
    B = torch.as_tensor(B_ao, dtype=torch.float64, device=dev).contiguous()
    barL = torch.as_tensor(bar_L_ao, dtype=torch.float64, device=dev).contiguous()
    nao, _, naux = B.shape
    if barL.shape != (naux, nao, nao):
        raise ValueError("bar_L_ao must have shape (naux, nao, nao)")
    if L_chol is not None:
        L = torch.as_tensor(L_chol, dtype=torch.float64, device=dev)
    else:
        L = cholesky_metric(eng.metric())
    bar_X, bar_V = whitened_adjoints(B, barL, L)
    grad = torch.zeros((natm, 3), dtype=torch.float64, device=dev)
    eng.deriv3c(bar_X, grad, layout="Qmn")
    eng.deriv2c(bar_V, grad)
    return grad.cpu().numpy()


# ---------------------------------------------------------------- full RHF nuclear gradient

def rhf_nuclear_gradient(res, precision: str = "fp64") -> np.ndarray:
    """dE_RHF/dR (natm, 3) of a converged Cartesian DF-RHF result of ``scf.run_hf_df``.

    Composed as the reference composes it (nuclear repulsion, ``contract_dhcore_cart`` with the
    density, ``-contract_dS_cart`` with the energy-weighted density W = sum_i occ_i e_i C_i C_i^T,
    and the DF two-electron gradient; ``asuka/integrals/int1e_cart.py:1452,1738``,
    ``asuka/integrals/grad.py:114``), with the two-electron part from the Rys derivative kernels
    through ``DFEnergyFunction`` at the converged orbitals.
    """
    from .int1e import contract_dhcore_cart, contract_dS_cart

    mol = res.mol
    ao = res.ao_basis
    C = torch.as_tensor(res.mo_coeff, dtype=torch.float64)
    occ = torch.as_tensor(res.mo_occ, dtype=torch.float64)
    eps = torch.as_tensor(res.scf.mo_energy, dtype=torch.float64)
    if C.shape[0] != ao.nao:
        raise NotImplementedError("rhf_nuclear_gradient takes Cartesian-AO results (cart=True)")
    Ch, occ_h, eps_h = C.cpu().numpy(), occ.cpu().numpy(), eps.cpu().numpy()
    D = (Ch * occ_h) @ Ch.T
    W = (Ch * (occ_h * eps_h)) @ Ch.T
    R = np.asarray(mol.coords_bohr, dtype=np.float64)
    g = mol.energy_nuc_grad() + contract_dhcore_cart(ao, atom_coords_bohr=R, atom_charges=mol.charges, M=D)
    g = g - contract_dS_cart(ao, atom_coords_bohr=R, M=W)
    eng = DFEngine(ao, res.aux_basis, atom_coords_bohr=R)
    nocc = int((occ_h > 0).sum())
    Cw = torch.as_tensor(Ch[:, :nocc] * np.sqrt(occ_h[:nocc]), device=eng.device).contiguous()
    Rt = torch.as_tensor(R, device=eng.device).requires_grad_(True)
    E2, _J, _K = df_energy(Rt, Cw, eng, precision)
    (g2,) = torch.autograd.grad(E2, Rt)
    return g + g2.cpu().numpy()

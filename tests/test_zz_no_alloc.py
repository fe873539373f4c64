"""The allocation-free integral entry point against the scratch-taking one.

Some callers cannot allocate device memory where they need integrals (a host
framework that hands over only its input and output buffers, or code running
under an allocator that forbids new device allocations).  For them
``dfb_rys_int_noalloc`` runs the same kernels with a fixed scratch array that
lives in the library's device image.  This file is collected last so that a
failure here leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest

from _util import bases_of, golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _run_3c(eng, fn, X, scratch=None, reverse=False):
    from asuka_b200 import _lib

    nao = eng.nao
    stream = int(torch.cuda.current_stream().cuda_stream)
    classes = list(eng.classes3c)[::-1] if reverse else eng.classes3c
    for la, lb, lc, pairs, auxs in classes:
        args = [la, lb, lc, ctypes.byref(eng.ps_ao), ctypes.byref(eng.axs), _lib.ptr(pairs), _lib.ptr(auxs),
                pairs.numel() * auxs.numel(), auxs.numel(), 0, _lib.ptr(X), nao * nao, nao, 1]
        if scratch is not None:
            args += [_lib.ptr(scratch), scratch.numel()]
        _lib.check(fn(*args, stream), fn.__name__)


def _run_2c(eng, fn, V, scratch=None):
    """The metric (P|Q) (mode 1) through the same entry point: a different workload that
    leaves other contents in the shared scratch array."""
    from asuka_b200 import _lib

    naux = eng.naux
    stream = int(torch.cuda.current_stream().cuda_stream)
    for lp, lq, P, Q in eng.classes2c:
        args = [lp, 0, lq, ctypes.byref(eng.ps_aux), ctypes.byref(eng.axs), _lib.ptr(P), _lib.ptr(Q), P.numel(), 0, 1,
                _lib.ptr(V), naux, 1, 0]
        if scratch is not None:
            args += [_lib.ptr(scratch), scratch.numel()]
        _lib.check(fn(*args, stream), fn.__name__)


@pytest.mark.parametrize("generic_only", [False, True])
def test_no_alloc_entry_matches_scratch_entry_on_two_calls(monkeypatch, generic_only):
    """Two 3c calls in a row through the allocation-free entry, with a metric call between
    them and the class order reversed on the second, against the scratch-taking entry."""
    from asuka_b200 import _lib
    from asuka_b200.df import DFEngine

    if generic_only:
        # route every class through the warp kernel, the one that uses scratch
        monkeypatch.setenv("DFB_DISABLE_TMPL", "1")
    g = golden("h2o_matzvp")
    ao, aux, sp = bases_of(g)
    eng = DFEngine(ao, aux, prim_screen=0.0)  # every shell pair evaluated, so every output element is written
    L = _lib.lib()
    shape = (eng.naux, eng.nao, eng.nao)
    X_ref = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
    V_ref = torch.full((eng.naux, eng.naux), float("nan"), dtype=torch.float64, device="cuda")
    _run_3c(eng, L.dfb_rys_int, X_ref, scratch=eng._scratch_for(False))
    _run_2c(eng, L.dfb_rys_int, V_ref, scratch=eng._scratch_for(False))
    torch.cuda.synchronize()
    scale = float(X_ref.abs().max())
    vscale = float(V_ref.abs().max())
    for call in range(2):
        X = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
        _run_3c(eng, L.dfb_rys_int_noalloc, X, reverse=call == 1)
        torch.cuda.synchronize()
        assert not bool(torch.isnan(X).any()), f"call {call}: output not fully written"
        err = float((X - X_ref).abs().max())
        assert err <= 1e-12 * scale, f"call {call}: max |diff| {err:.3e}"
        if call == 0:
            V = torch.full_like(V_ref, float("nan"))
            _run_2c(eng, L.dfb_rys_int_noalloc, V)
            torch.cuda.synchronize()
            assert not bool(torch.isnan(V).any()), "metric output not fully written"
            assert float((V - V_ref).abs().max()) <= 1e-12 * vscale

"""libdfb.so loads without a GPU and exports every entry point declared in include/dfb.h."""

import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "dfb.h")) as f:
        txt = f.read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|long|char\s*\*|const\s+char\s*\*)\s*\*?\s*(dfb_\w+)\s*\(",
                                 txt, flags=re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "dfb_rys_int" in names and "dfb_rys_deriv" in names and "dfb_pair_tables" in names


def test_library_exports_every_declared_symbol():
    from asuka_b200 import _lib

    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    assert set(_declared()) <= set(_lib.exported_symbols()) | {n for n in _declared() if hasattr(L, n)}
    assert L.dfb_version() >= 100
    assert L.dfb_last_error() == b""


def test_tensor_core_gemm_rejects_bad_arguments_without_a_gpu():
    """Argument checks of dfb_tc_gemm run before any device call (their error codes and messages)."""
    import ctypes

    from asuka_b200 import _lib

    L = _lib.lib()
    a = _lib.TcOperand(0x1000, 4, 0, 1, 4, 0)
    b = _lib.TcOperand(0x2000, 4, 0, 1, 4, 0)
    cases = [
        (dict(M=-1), "invalid arguments"),
        (dict(nterms=4), "nterms"),
        (dict(symmetric=1), "symmetric"),           # A != B
        (dict(K=0), "K == 0"),
        (dict(accumulate=0, kspan=32, K=100), "accumulate"),
    ]
    for over, msg in cases:
        kw = dict(M=8, N=8, K=4, batch=1, accumulate=1, symmetric=0, nterms=3, kspan=0)
        kw.update(over)
        rc = L.dfb_tc_gemm(kw["M"], kw["N"], kw["K"], kw["batch"], ctypes.byref(a), ctypes.byref(b), 0x3000, 8, 0,
                           kw["accumulate"], kw["symmetric"], kw["nterms"], kw["kspan"], None)
        assert rc == -1, (over, rc)
        assert msg in L.dfb_last_error().decode(), (over, L.dfb_last_error())
    # empty products are a no-op
    assert L.dfb_tc_gemm(0, 8, 4, 1, ctypes.byref(a), ctypes.byref(b), 0x3000, 8, 0, 1, 0, 3, 0, None) == 0


def test_gamma_kernel_rejects_bad_arguments_without_a_gpu():
    """Argument checks of dfb_gamma_sym run before any device call; empty shapes are a no-op."""
    from asuka_b200 import _lib

    L = _lib.lib()
    cases = [((-1, 8, 4, 0x1000, 32, 4, 0x2000, 0x3000), "invalid sizes"),
             ((2, 8, 0, 0x1000, 32, 4, 0x2000, 0x3000), "nocc == 0"),
             ((2, 8, 4, 0, 32, 4, 0x2000, 0x3000), "invalid pointers"),
             ((2, 8, 4, 0x1000, 3, 4, 0x2000, 0x3000), "invalid pointers or strides")]
    for args, msg in cases:
        assert L.dfb_gamma_sym(*args, None) == -1, args
        assert msg in L.dfb_last_error().decode(), (args, L.dfb_last_error())
    assert L.dfb_gamma_sym(0, 8, 4, 0, 0, 0, 0, 0, None) == 0
    assert L.dfb_gamma_sym(3, 0, 4, 0, 0, 0, 0, 0, None) == 0


def test_rys_error_word_needs_the_table():
    """dfb_rys_error reports 'not initialised' (negative) before the Rys table is uploaded."""
    from asuka_b200 import _lib

    assert _lib.lib().dfb_rys_error(0) < 0


def test_precision_entry_points_reject_unknown_precision_without_a_gpu():
    import ctypes

    from asuka_b200 import _lib

    L = _lib.lib()
    ps, ax = _lib.PairSide(), _lib.AuxSide()
    rc = L.dfb_rys_int_prec(0, 0, 0, ctypes.byref(ps), ctypes.byref(ax), 0x10, 0x10, 0, 0, 0, 7, 0x10, 1, 1, 1, 0, 0,
                            None)
    assert rc == -1 and "precision" in L.dfb_last_error().decode()

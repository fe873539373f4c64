"""ctypes binding of ``libdfb.so`` (the C ABI declared in ``include/dfb.h``).

The library is built in-tree by ``asuka_b200/build.py``; there is no fallback:
importing a compute entry point without the library raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# DFB_LIB_PATH selects another build of the same library (the class tuner's variant build)
LIB_PATH = os.environ.get("DFB_LIB_PATH") or os.path.join(_HERE, "libdfb.so")

_d = ctypes.c_void_p  # device pointers travel as integers


class PairSide(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "shA", "shB", "pstart", "npair", "eta", "Px", "Py", "Pz", "cK", "ea", "eb", "cxyz", "aostart", "atom")] + [
        ("b_dummy", ctypes.c_int)]


class TcOperand(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p)] + [(n, ctypes.c_long) for n in ("s_row", "s_kq", "s_k1", "nk1", "s_batch")]


class AuxSide(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("cxyz", "pstart", "nprim", "pexp", "pcoef", "rexp", "aostart", "atom")]


_SIGS = {
    "dfb_version": (ctypes.c_int, []),
    "dfb_last_error": (ctypes.c_char_p, []),
    "dfb_rys_table_init": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double]),
    "dfb_pair_tables": (ctypes.c_int, [_d] * 10 + [ctypes.c_long, ctypes.c_int] + [_d] * 7 + [_d]),
    "dfb_rys_int": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.POINTER(PairSide), ctypes.POINTER(AuxSide), _d, _d,
                                                        ctypes.c_long, ctypes.c_long, ctypes.c_int, _d, ctypes.c_long,
                                                        ctypes.c_long, ctypes.c_long, _d, ctypes.c_long, _d]),
    "dfb_rys_deriv": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.POINTER(PairSide), ctypes.POINTER(AuxSide), _d, _d,
                                                          ctypes.c_long, ctypes.c_long, ctypes.c_int, _d,
                                                          ctypes.c_long, ctypes.c_long, ctypes.c_long, _d,
                                                          ctypes.c_int, _d, ctypes.c_long, _d]),
    "dfb_rys_int_prec": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.POINTER(PairSide), ctypes.POINTER(AuxSide), _d,
                                                             _d, ctypes.c_long, ctypes.c_long, ctypes.c_int,
                                                             ctypes.c_int, _d, ctypes.c_long, ctypes.c_long,
                                                             ctypes.c_long, _d, ctypes.c_long, _d]),
    "dfb_rys_deriv_prec": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.POINTER(PairSide), ctypes.POINTER(AuxSide), _d,
                                                               _d, ctypes.c_long, ctypes.c_long, ctypes.c_int,
                                                               ctypes.c_int, _d, ctypes.c_long, ctypes.c_long,
                                                               ctypes.c_long, _d, ctypes.c_int, _d, ctypes.c_long,
                                                               _d]),
    "dfb_tc_gemm": (ctypes.c_int, [ctypes.c_long] * 4 + [ctypes.POINTER(TcOperand), ctypes.POINTER(TcOperand), _d,
                                                          ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                                          ctypes.c_int, ctypes.c_long, _d]),
    "dfb_tc_error": (ctypes.c_int, [ctypes.c_int]),
    "dfb_rys_error": (ctypes.c_int, [ctypes.c_int]),
    "dfb_gamma_sym": (ctypes.c_int, [ctypes.c_long, ctypes.c_int, ctypes.c_int, _d, ctypes.c_long, ctypes.c_long,
                                     _d, _d, _d]),
    "dfb_fp32_fma_probe": (ctypes.c_int, [_d, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d]),
    "dfb_launch_count": (ctypes.c_long, []),
    "dfb_rys_scratch_doubles": (ctypes.c_long, [ctypes.c_int] * 3 + [ctypes.c_long, ctypes.c_int]),
    "dfb_fp64_fma_probe": (ctypes.c_int, [_d, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d]),
    "dfb_rys_int_noalloc": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.POINTER(PairSide), ctypes.POINTER(AuxSide), _d,
                                                                _d, ctypes.c_long, ctypes.c_long, ctypes.c_int, _d,
                                                                ctypes.c_long, ctypes.c_long, ctypes.c_long, _d]),
}

_LIB = None


def exported_symbols() -> tuple[str, ...]:
    return tuple(_SIGS)


def lib() -> ctypes.CDLL:
    """The loaded library; raises RuntimeError when it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libdfb.so not found at {LIB_PATH}: build it with `python -m asuka_b200.build` "
                "(the DF engine has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:  # a library built before this entry point existed: fails where it is called
                continue
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().dfb_last_error().decode(errors="replace")
        if rc == -3:
            raise NotImplementedError(f"{what}: {msg}")
        if rc == -1:
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")


def ptr(t) -> int:
    """Device (or host) address of a torch tensor; 0 for None."""
    return 0 if t is None else int(t.data_ptr())

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

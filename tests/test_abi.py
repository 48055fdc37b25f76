"""The C-ABI library loads and exports every symbol include/atlasgpu.h declares (no GPU)."""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    s = open(os.path.join(ROOT, "include", "atlasgpu.h")).read()
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return set(re.findall(r"\b(atlasgpu_[a-z0-9_]+)\s*\(", s))


def test_library_exports_declared_symbols():
    import ctypes
    from atlas12_b200 import _lib
    assert os.path.exists(_lib.LIB_PATH), "libatlasgpu.so not built"
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # every declared entry has a ctypes signature in the binding
    unbound = [n for n in names if n not in _lib.SIGNATURES]
    assert not unbound, unbound


def test_grid_is_host_only():
    from atlas12_b200 import synthe
    g = synthe.synthe_grid(400.0, 410.0, 500000.0)
    assert g["length"] == 12346 and g["ixwlbeg"] > 0


def test_tabvoigt_matches_oracle(tables, po):
    """TABVOIGT is host code in the library: it must equal the oracle's restatement."""
    from atlas12_b200 import atlas
    got = atlas.tabvoigt(tables)
    ref = po.tabvoigt(tables["tabvi"], tables["tabh1"])
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)

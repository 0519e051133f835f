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
    # periodic: x = 0 and x = 2 pi share global nodes, so every row of
    # vertices and horizontal edges has nx entries (not nx + 1): vertices
    # 6 x 5, horizontal edges 6 x 5 and vertical edges 6 x 4 with np - 2 = 3
    # interior nodes each
    nx, ny, ni = 6, 4, 3
    assert m.nglobal == nx * (ny + 1) + nx * (ny + 1) * ni + nx * ny * ni == 192
    mo = rect_mesh(6, 4, 5, 0, 2 * np.pi, 0, 1, jitter=0.15, seed=2, periodic_x=False,
                   bc={"bottom": "D", "top": "D"})
    assert mo.nglobal == m.nglobal + (ny + 1) + ny * ni  # the x = 2 pi column of its own
    ptr, idx = m.global_to_element()
    assert ptr[-1] == m.nel * m.next
    assert (np.diff(ptr) >= 1).all()


def _desc(m, **over):
    import semtex_b200 as sx
    d, keep = sx.mesh_desc(m)
    for k, v in over.items():
        setattr(d, k, v)
    return d, keep


def test_mesh_create_rejects_flipped_element():
    """A clockwise (mirrored) element has a negative Jacobian: SX_ERR_JACOBIAN,
    as Element::mapping stops (src/element.cpp:1349-1352).  Found on the host
    before anything touches a device."""
    import semtex_b200 as sx
    from semtex_b200.mesh import rect_mesh
    m = rect_mesh(3, 2, 5, 0.0, 1.0, 0.0, 1.0)
    e = 4
    x = m.x.reshape(m.nel, m.np, m.np).copy()
    x[e] = x[e][:, ::-1]  # reverse the element's r direction: orientation flips
    m.x = x.reshape(m.x.shape)
    d, keep = _desc(m)
    h = C.c_void_p()
    st = sx.lib.sx_mesh_create(C.byref(d), C.byref(h))
    assert st == 4, sx.status_string(st)  # SX_ERR_JACOBIAN
    assert f"element {e + 1}" in sx.last_error()


def test_mesh_create_rejects_band_too_narrow():
    """A declared band narrower than the numbering's couplings: SX_ERR_BAND
    (the reference's assembly would write outside its band,
    src/matrix.cpp:236-241)."""
    import semtex_b200 as sx
    from semtex_b200.mesh import rect_mesh
    m = rect_mesh(4, 4, 5, 0.0, 1.0, 0.0, 1.0)
    d, keep = _desc(m, nband=m.nband - 1)
    h = C.c_void_p()
    st = sx.lib.sx_mesh_create(C.byref(d), C.byref(h))
    assert st == 7, sx.status_string(st)  # SX_ERR_BAND
    assert "nband" in sx.last_error()
    # the declared band itself is accepted up to that point: a band exactly as
    # wide as the widest element coupling passes the check
    widest = max(int(g.max() - g.min()) + 1 for g in
                 (m.btog[e][m.bmask[e] == 0] for e in range(m.nel)) if len(g))
    assert widest == m.nband


def test_elliptic_phase_entry_points_refuse_bad_arguments():
    """The DNS elliptic-phase entry points check their arguments before
    touching the device: a missing mesh or pointer, a wave step of order
    outside 1-3 or more than four fields is SX_ERR_ARG; an empty wave step
    is a no-op."""
    import semtex_b200 as sx
    L = sx.lib
    ARG = 1
    null = C.c_void_p()
    ptrs = sx._ptrs([1, 2, 3])  # never dereferenced: the checks fail first
    assert L.sx_field_gradient(null, 8, 4, 100, 0, 1.0, 0, null) == ARG
    assert L.sx_field_smooth(null, 8, 4, 100, null) == ARG
    assert L.sx_dns_pressure_forcing(null, ptrs, 3, 8, 4, 100, 0.1, 1.0, 0, null) == ARG
    assert L.sx_dns_project(null, ptrs, 8, ptrs, 3, 3, 3, 4, 100, 0.1, 0.01, 1.0, 1.0, 0, null) == ARG
    assert L.sx_mesh_partials(null, 0, None, None, None, None, None) == ARG
    one = sx._ptrs([8])
    assert L.sx_dns_wave_prop(one, one, one, 1, 0, 10, 0.1, null) == ARG    # order 0
    assert L.sx_dns_wave_prop(one, one, one, 1, 4, 10, 0.1, null) == ARG    # order 4
    assert L.sx_dns_wave_prop(one, one, one, 5, 1, 10, 0.1, null) == ARG    # five fields
    assert L.sx_dns_wave_prop(one, one, one, 1, 1, -1, 0.1, null) == ARG    # negative length
    assert L.sx_dns_wave_prop(one, one, one, 1, 1, 0, 0.1, null) == 0       # nothing to do


def test_config5_block_split():
    """config5_block: the 8 x 16 mode split of config 5, as the reference
    splits modes across processes; betak2 = k^2 of the block's modes."""
    from semtex_b200.partition import mode_block
    from semtex_b200.workloads import config5_block
    b = config5_block(world=8, rank=7, nx=8, ny=4, np_=5)
    assert (b.base_mode, b.num_modes) == mode_block(128, 8, 7) == (112, 16)
    assert b.nz == 32 and b.planes_solved == 32
    assert np.array_equal(b.betak2, np.arange(112, 128, dtype=float) ** 2)
    assert np.all(b.lambda2_v == 1.0 / (b.nu * b.dt)) and np.all(b.lambda2_p == 0.0)
    b0 = config5_block(world=8, rank=0, nx=8, ny=4, np_=5)
    assert b0.base_mode == 0 and b0.planes_solved == 31
    # velocity: Dirichlet walls (essential nodes numbered last); pressure: none
    assert b0.mesh_v.nsolve < b0.mesh_v.nglobal and b0.mesh_p.nsolve == b0.mesh_p.nglobal

"""Pin the CPU oracle against the reference's own goldens (no GPU).

* GLL points/weights/derivatives vs the reference's femlib/polylib.c
  (tests/golden/gll_ref.npz, made by tests/golden/make_gll_fixture.py).
* Edge maps vs the reference's femlib/mapping.c
  (tests/golden/edgemap_ref.npz, made by tests/golden/make_edgemap_fixture.py).
* Whole DIRECT solves vs regress/*.ok (helmholtz1, poisson1, laplace1,
  laplace4, laplace5, laplace7, mixed1, laplace3).
* JACPCG converges to the DIRECT answer on the same systems.
* Banded Cholesky restatement vs a dense factorisation.
"""
import os

import numpy as np
import pytest

from oracle.oracle import DIRECT, JACPCG, OracleMesh, OracleSystem, gll, solve_planes
from semtex_b200.mesh import edge_maps, gll_points, rect_mesh
from tests.problems import (LAPLACE3, PROBLEMS_2D, PROBLEMS_2D_MORE, build_2d, build_laplace3, golden_ok,
                            to_physical)

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("n", range(3, 17))
def test_gll_matches_reference_polylib(n):
    ref = np.load(os.path.join(HERE, "golden", "gll_ref.npz"))
    z, w, D = gll(n)
    np.testing.assert_allclose(z, ref[f"z{n}"], rtol=0, atol=8e-16)
    np.testing.assert_allclose(w, ref[f"w{n}"], rtol=2e-15, atol=0)
    assert np.abs(D - ref[f"D{n}"]).max() <= 5e-15 * np.abs(ref[f"D{n}"]).max()
    np.testing.assert_array_equal(gll_points(n), z)


def test_edge_maps():
    emap, pmap = edge_maps(4)
    # CCW exterior from node 0, then interior row-major (femlib/mapping.c:100-113)
    assert emap.tolist() == [0, 1, 2, 3, 7, 11, 15, 14, 13, 12, 8, 4, 5, 6, 9, 10]
    assert (emap[pmap] == np.arange(16)).all()


@pytest.mark.parametrize("n", range(3, 17))
def test_edge_maps_match_reference_mapping(n):
    """The front-end's and both oracles' edge maps equal the ones the
    reference's own femlib/mapping.c builds (tests/golden/edgemap_ref.npz,
    made by tests/golden/make_edgemap_fixture.py): the element-boundary slot
    order that btog, the static condensation and every gather depend on."""
    import ctypes as C
    from oracle.dns import edge_map
    from oracle.oracle import lib
    ref = np.load(os.path.join(HERE, "golden", "edgemap_ref.npz"))
    emap, pmap = edge_maps(n)
    np.testing.assert_array_equal(emap, ref[f"emap2_{n}"])
    np.testing.assert_array_equal(pmap, ref[f"pmap2_{n}"])
    np.testing.assert_array_equal(edge_map(n), ref[f"emap2_{n}"])
    ce, cp = np.zeros(n * n, dtype=np.int32), np.zeros(n * n, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    lib().orc_edgemaps(C.c_int(n), ce.ctypes.data_as(ip), cp.ctypes.data_as(ip))
    np.testing.assert_array_equal(ce, ref[f"emap2_{n}"])
    np.testing.assert_array_equal(cp, ref[f"pmap2_{n}"])


@pytest.mark.parametrize("name", list(PROBLEMS_2D) + list(PROBLEMS_2D_MORE))
def test_direct_matches_regress_golden(name):
    m, p, f, bc, exact = build_2d(name)
    u, _ = solve_planes(OracleMesh(m), p["lambda2"], 0.0, f, bc, method=DIRECT)
    err = np.abs(u[0] - exact).max()
    assert golden_ok(err, p["golden"]), (name, err)


@pytest.mark.parametrize("name", list(PROBLEMS_2D) + list(PROBLEMS_2D_MORE))
def test_jacpcg_converges_to_direct(name):
    m, p, f, bc, exact = build_2d(name)
    om = OracleMesh(m)
    ud, _ = solve_planes(om, p["lambda2"], 0.0, f, bc, method=DIRECT)
    up, it = solve_planes(om, p["lambda2"], 0.0, f, bc, method=JACPCG, tol_rel=1e-13, step_max=5000)
    assert it[0] < 5000
    assert np.abs(up[0] - ud[0]).max() <= 1e-10 * np.abs(ud[0]).max()


def test_laplace3_golden():
    m, bcf, exact = build_laplace3()
    f = np.zeros((LAPLACE3["nz"], m.nplane))
    u, _ = solve_planes(OracleMesh(m), 0.0, LAPLACE3["beta"], f, bcf, method=DIRECT)
    u[1] = 0.0
    err = np.abs(to_physical(u) - exact).max()
    assert err < 1e-12  # regress/laplace3.ok: noise-level


def test_band_cholesky_matches_dense():
    rng = np.random.default_rng(0)
    n, kd = 40, 7
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(i, min(n, i + kd + 1)):
            A[i, j] = A[j, i] = rng.standard_normal()
    A += np.eye(n) * (2 * kd + 2)
    ldab = kd + 1
    AB = np.zeros(n * ldab)
    for j in range(n):
        for i in range(max(0, j - kd), j + 1):
            AB[j * ldab + kd + i - j] = A[i, j]
    from oracle.oracle import lib
    assert lib().orc_dpbtrf(n, kd, AB, ldab) == 0
    U = np.linalg.cholesky(A).T
    for j in range(n):
        for i in range(max(0, j - kd), j + 1):
            assert abs(AB[j * ldab + kd + i - j] - U[i, j]) < 1e-12
    b = rng.standard_normal(n)
    x = b.copy()
    lib().orc_dpbtrs(n, kd, AB, ldab, x)
    np.testing.assert_allclose(A @ x, b, rtol=0, atol=1e-12)


def test_singular_pressure_mode_is_pinned():
    # Poisson with natural BCs only and lambda2 + betak2 = 0: nsolve is
    # reduced by one (src/matrix.cpp:166-169).
    m = rect_mesh(3, 3, 5, bc={"bottom": "N", "top": "N", "left": "N", "right": "N"})
    om = OracleMesh(m)
    s = OracleSystem(om, 0.0, 0.0, DIRECT)
    assert s.singular and s.nsolve == m.nsolve - 1
    f = m.eval_nodes(lambda x, y: np.cos(np.pi * x) * np.cos(np.pi * y))
    u, _ = s.solve_plane(f, np.zeros((len(m.boundaries), m.np)))
    exact = m.eval_nodes(lambda x, y: -np.cos(np.pi * x) * np.cos(np.pi * y) / (2 * np.pi ** 2))
    d = u - exact
    assert np.abs(d - d.mean()).max() < 1e-6  # equal up to a constant

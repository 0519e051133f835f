"""GPU parity of the plain FP64 solve (DIRECT and JACPCG) against the oracle.

Tolerance: relative L2 and relative max norm <= 1e-12 against the oracle's
FP64 direct solve on the same mesh, order, lambda2 and forcing (the plain
form's contract), plus the reference's regress/*.ok goldens.
"""
import numpy as np
import pytest

from oracle.oracle import DIRECT as O_DIRECT
from oracle.oracle import JACPCG as O_JACPCG
from oracle.oracle import OracleMesh, OracleSystem, solve_planes
from tests.problems import (LAPLACE3, PROBLEMS_2D, build_2d, build_laplace3, golden_ok,
                            to_physical)

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel_errs(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    l2 = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
    mx = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    return l2, mx


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.mark.parametrize("name", list(PROBLEMS_2D))
def test_direct_regress_goldens(sx, name):
    m, p, f, bc, exact = build_2d(name)
    mesh = sx.Mesh(m)
    sysm = sx.ModalMatrixSys(mesh, p["lambda2"], 0.0, 0, 1, sx.DIRECT)
    u = sysm.solve(f, bc)
    err = np.abs(u[0] - exact).max()
    assert golden_ok(err, p["golden"]), (name, err)
    uo, _ = solve_planes(OracleMesh(m), p["lambda2"], 0.0, f, bc, method=O_DIRECT)
    l2, mx = rel_errs(u, uo)
    assert l2 <= TOL and mx <= TOL, (name, l2, mx)


@pytest.mark.parametrize("name", list(PROBLEMS_2D))
def test_jacpcg_matches_oracle(sx, name):
    m, p, f, bc, exact = build_2d(name)
    mesh = sx.Mesh(m)
    sysm = sx.ModalMatrixSys(mesh, p["lambda2"], 0.0, 0, 1, sx.JACPCG)
    u, st = sysm.solve(f, bc, tol_rel=1e-12, step_max=5000, return_stats=True)
    uo, it = solve_planes(OracleMesh(m), p["lambda2"], 0.0, f, bc, method=O_JACPCG,
                          tol_rel=1e-12, step_max=5000)
    assert abs(st["iterations_max"] - int(it[0])) <= 2
    l2, mx = rel_errs(u, uo)
    assert l2 <= 1e-10 and mx <= 1e-10, (name, l2, mx)


def test_laplace3_golden(sx):
    m, bcf, exact = build_laplace3()
    nz = LAPLACE3["nz"]
    mesh = sx.Mesh(m)
    sysm = sx.ModalMatrixSys(mesh, 0.0, LAPLACE3["beta"], 0, nz // 2, sx.DIRECT)
    u = sysm.solve(np.zeros((nz, m.nplane)), bcf)
    u[1] = 0.0
    assert np.abs(to_physical(u) - exact).max() < 1e-12


def _jittered(sx_mod, nx, ny, np_, seed, jitter=0.15):
    from semtex_b200.mesh import rect_mesh
    return rect_mesh(nx, ny, np_, 0.0, 2 * np.pi, 0.0, 1.0, jitter=jitter, seed=seed,
                     periodic_x=True, bc={"bottom": "D", "top": "D"})


@pytest.mark.parametrize("np_,nz,lam", [(9, 8, 1e6), (5, 6, 1.0), (11, 4, 0.01)])
def test_direct_multimode_parity(sx, np_, nz, lam):
    m = _jittered(sx, 6, 5, np_, seed=np_)
    rng = np.random.default_rng(np_)
    f = rng.standard_normal((nz, m.nplane))
    f[1] = 0.0
    mesh = sx.Mesh(m)
    sysm = sx.ModalMatrixSys(mesh, lam, 1.0, 0, nz // 2, sx.DIRECT)
    u = sysm.solve(f)
    uo, _ = solve_planes(OracleMesh(m), lam, 1.0, f, None, method=O_DIRECT)
    l2, mx = rel_errs(u, uo)
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def test_band_factor_matches_oracle(sx):
    m = _jittered(sx, 5, 4, 7, seed=3)
    mesh = sx.Mesh(m)
    sysm = sx.ModalMatrixSys(mesh, 2.0, 1.0, 0, 2, sx.DIRECT)
    for mode in (0, 1):
        ab, singular = sysm.band(mode)
        os_ = OracleSystem(OracleMesh(m), 2.0, float(mode) ** 2, O_DIRECT)
        ref = os_.band()
        assert not singular and ab.shape == ref.shape
        assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max()


def test_geometry_matches_oracle(sx):
    m = _jittered(sx, 3, 3, 6, seed=5, jitter=0.2)
    mesh = sx.Mesh(m)
    om = OracleMesh(m)
    for e in range(m.nel):
        g = mesh.geometry(e)
        (o1, o2, o3, o4, o8), _ = om.geom(e)
        for a, b in zip(g, (o1, o2, o3, o4, o8)):
            assert np.abs(a - b).max() <= 1e-13 * max(np.abs(b).max(), 1e-300)


def test_singular_pressure_mode(sx):
    from semtex_b200.mesh import rect_mesh
    m = rect_mesh(3, 3, 6, bc={"bottom": "N", "top": "N", "left": "N", "right": "N"})
    f = m.eval_nodes(lambda x, y: np.cos(np.pi * x) * np.cos(np.pi * y))[None]
    mesh = sx.Mesh(m)
    sysm = sx.ModalMatrixSys(mesh, 0.0, 0.0, 0, 1, sx.DIRECT)
    u = sysm.solve(f, np.zeros((1, len(m.boundaries), m.np)))
    uo, _ = solve_planes(OracleMesh(m), 0.0, 0.0, f, np.zeros((1, len(m.boundaries), m.np)))
    l2, mx = rel_errs(u, uo)
    assert l2 <= 1e-10 and mx <= 1e-10, (l2, mx)

"""GPU tests of the serving loop (sx_server_*).

* Requests of different meshes, orders and mode counts, submitted together
  and solved in multi-mesh batches, give the same results as each served
  alone (a one-slot server, batch of one) within the 1e-10 bar: a batch
  shares the FP32 iteration count per round and the number of refinement
  rounds, each plane's arithmetic is its own.
* Results match the oracle's FP64 direct solve within 1e-10.
* Geometry and systems are reused across requests (cache hits).
* A request larger than the memory budget is refused with SX_ERR_CAPACITY.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


def _requests():
    from semtex_b200.mesh import rect_mesh
    from semtex_b200.workloads import fourier_forcing
    rng = np.random.default_rng(42)
    out = []
    for i, (nx, ny, np_, nm, lam) in enumerate([(3, 3, 5, 2, 1e3), (4, 2, 7, 1, 50.0),
                                                (5, 4, 6, 3, 1e4), (2, 2, 9, 2, 300.0),
                                                (3, 3, 5, 2, 1e3), (6, 3, 8, 4, 2e3)]):
        m = rect_mesh(nx, ny, np_, 0.0, 1.0 + 0.1 * (i % 4), 0.0, 1.0)  # 0 and 4: one mesh
        nz = 1 if nm == 1 else 2 * nm
        lamv = np.full(nm, lam)
        bk2 = np.arange(nm, dtype=np.float64) ** 2
        out.append((m, lamv, bk2, fourier_forcing(m, nz, rng)))
    return out


CFG = dict(precision=None, tol_rel=1e-12, max_refine=30, inner_iters=12)


def _cfg(sx):
    return dict(CFG, precision=sx.MIXED_FP32)


def _alone(sx, m, lam, bk2, f):
    """The request served by itself: a fresh one-slot server, same settings."""
    srv = sx.Server(slots=1, **_cfg(sx))
    try:
        status, _, u = srv.wait(srv.submit(m, lam, bk2, f), timeout_s=120.0)
    finally:
        srv.close()
    assert status in (sx.OK, sx.WARN_STEP_LIMIT)
    return u


def _solved(nz):
    return [0] + list(range(2, nz)) if nz > 1 else [0]


def _blocker():
    """A larger request that keeps a one-slot server busy while the test's
    requests queue behind it (so that they are served as one batch)."""
    from semtex_b200.mesh import rect_mesh
    from semtex_b200.workloads import fourier_forcing
    m = rect_mesh(24, 24, 9, 0.0, 1.0, 0.0, 1.0)
    nm = 16
    return (m, np.full(nm, 3e3), np.arange(nm, dtype=np.float64) ** 2,
            fourier_forcing(m, 2 * nm, np.random.default_rng(3)))


@pytest.mark.parametrize("slots", [1, 3])
def test_mix_equals_alone_and_oracle(sx, slots):
    reqs = _requests()
    alone = [_alone(sx, *r) for r in reqs]
    srv = sx.Server(slots=slots, **_cfg(sx))
    try:
        first = srv.submit(*_blocker())
        ids = [srv.submit(*r) for r in reqs]
        res = [srv.wait(i, timeout_s=120.0) for i in ids]
        srv.wait(first, timeout_s=120.0)
        stats = srv.stats()
    finally:
        srv.close()
    for (status, lat, u), a, r in zip(res, alone, reqs):
        assert status in (sx.OK, sx.WARN_STEP_LIMIT)
        assert lat > 0.0
        sp = _solved(u.shape[0])
        err = np.linalg.norm(u[sp] - a[sp]) / np.linalg.norm(a[sp])
        assert err <= TOL, err
    assert stats["completed"] == len(reqs) + 1
    if slots == 1:
        # the six queued behind the blocker are served together
        assert stats["batches"] <= 3, stats
    assert stats["mesh_hits"] >= 1          # requests 0 and 4 share a mesh
    assert stats["system_hits"] >= 2        # ... and both of their systems
    assert stats["p99_ms"] >= stats["p50_ms"] > 0.0
    # one request against the oracle
    from oracle.oracle import OracleMesh, solve_planes
    m, lam, bk2, f = reqs[2]
    uo, _ = solve_planes(OracleMesh(m), 0.0, 1.0, f, None, lambda2_per_mode=lam)
    sp = [0] + list(range(2, f.shape[0]))
    u = res[2][2]
    assert np.linalg.norm(u[sp] - uo[sp]) <= TOL * np.linalg.norm(uo[sp])


def test_fp64_direct_server_matches_oracle(sx):
    reqs = _requests()[:3]
    srv = sx.Server(slots=2, precision=sx.FP64)
    try:
        ids = [srv.submit(*r) for r in reqs]
        res = [srv.wait(i, timeout_s=120.0) for i in ids]
    finally:
        srv.close()
    from oracle.oracle import OracleMesh, solve_planes
    for (m, lam, bk2, f), (status, _, u) in zip(reqs, res):
        assert status == sx.OK
        uo, _ = solve_planes(OracleMesh(m), 0.0, 1.0, f, None, lambda2_per_mode=lam)
        sp = [0] + list(range(2, f.shape[0])) if f.shape[0] > 1 else [0]
        assert np.linalg.norm(u[sp] - uo[sp]) <= 1e-12 * np.linalg.norm(uo[sp])


def test_capacity_rejection(sx):
    m, lam, bk2, f = _requests()[5]
    srv = sx.Server(slots=1, hbm_budget=1 << 16)
    try:
        with pytest.raises(sx.SolverError) as ei:
            srv.submit(m, lam, bk2, f)
        assert ei.value.status == 11  # SX_ERR_CAPACITY
        assert srv.stats()["rejected"] == 1
    finally:
        srv.close()


def test_mixed_server_routes_ill_conditioned_modes(sx):
    """A near-Poisson request (lambda2 = 1e-2): the mixed server factors it
    and solves it by the FP64 band Cholesky, within 1e-10 of the oracle."""
    from semtex_b200.mesh import rect_mesh
    from semtex_b200.workloads import fourier_forcing
    from oracle.oracle import OracleMesh, solve_planes
    m = rect_mesh(6, 5, 8, 0.0, 1.0, 0.0, 1.0)
    lam = np.array([1e-2, 1e-2])
    bk2 = np.array([0.0, 1.0])
    f = fourier_forcing(m, 4, np.random.default_rng(7))
    srv = sx.Server(slots=1, **_cfg(sx))
    try:
        status, _, u = srv.wait(srv.submit(m, lam, bk2, f), timeout_s=120.0)
    finally:
        srv.close()
    assert status == sx.OK
    uo, _ = solve_planes(OracleMesh(m), 0.0, 1.0, f, None, lambda2_per_mode=lam)
    for p in (0, 2, 3):
        assert np.linalg.norm(u[p] - uo[p]) <= TOL * np.linalg.norm(uo[p])

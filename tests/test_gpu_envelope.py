"""GPU parity of the band factor and of the direct solves under numberings
whose factor envelopes differ.

The factorisation and the two band sweeps work only on the tiles inside the
factor's envelope (the tiles of the band that Cholesky fill can reach); every
other tile is an exact zero of LAPACK's factor.  So the exported band is
checked against the oracle's dpbtrf entry by entry: zero exactly where the
oracle's is zero, within 1e-12 of its largest entry elsewhere; and the
solutions of the plain and batched forms (several cluster schedules) against
the oracle's FP64 direct solve within 1e-12 (relative L2 and max norm).

The numberings are those of tests/numberings.py.
"""
import numpy as np
import pytest

from oracle.oracle import DIRECT as O_DIRECT
from oracle.oracle import OracleMesh, OracleSystem, solve_planes
from tests.numberings import ORDERS, lapack_tile_hull, numbered_mesh

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel_errs(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return (np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300),
            np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch




@pytest.mark.parametrize("order", ORDERS)
def test_factor_envelope_matches_lapack(sx, order):
    m = numbered_mesh(order)
    mesh = sx.Mesh(m)
    lam = 3.0
    S = sx.ModalMatrixSys(mesh, lam, 1.0, 0, 3, sx.DIRECT)
    for mode in (0, 2):
        ab, singular = S.band(mode)
        ref = OracleSystem(OracleMesh(m), lam, float(mode) ** 2, O_DIRECT).band()
        assert not singular and ab.shape == ref.shape
        assert np.all(ab[ref == 0.0] == 0.0), order
        assert np.abs(ab - ref).max() <= TOL * np.abs(ref).max(), order


@pytest.mark.parametrize("order", ORDERS)
def test_direct_solve_envelope_matches_oracle(sx, torch, order):
    m = numbered_mesh(order)
    nz = 6
    rng = np.random.default_rng(17)
    f = rng.standard_normal((nz, m.nplane))
    f[1] = 0.0
    lam = np.array([5.0, 40.0, 1e3])
    mesh = sx.Mesh(m)
    S = sx.ModalMatrixSys(mesh, num_modes=nz // 2, method=sx.DIRECT, lambda2_modes=lam,
                          betak2_modes=np.arange(nz // 2, dtype=np.float64) ** 2)
    uo, _ = solve_planes(OracleMesh(m), 0.0, 1.0, f, None, lambda2_per_mode=lam)
    sp = [0] + list(range(2, nz))
    u = S.solve(f)
    l2, mx = rel_errs(u[sp], uo[sp])
    assert l2 <= TOL and mx <= TOL, (order, "plain", l2, mx)
    for cluster, stages, lead in ((1, 2, 1), (3, 2, 2), (4, 2, 3), (2, 3, 1)):
        S.tune(band_cluster=cluster, band_stages=stages, band_lead=lead)
        fd = torch.tensor(f, device="cuda")  # the batched solve works in its forcing
        ud = torch.zeros_like(fd)
        S.solve_batched(ud.data_ptr(), fd.data_ptr(), 0, nz, m.nplane, 0, 1e-12)
        torch.cuda.synchronize()
        S.status()
        ub = ud.cpu().numpy()
        l2, mx = rel_errs(ub[sp], uo[sp])
        assert l2 <= TOL and mx <= TOL, (order, cluster, stages, lead, l2, mx)


@pytest.mark.parametrize("order", ORDERS)
def test_envelope_tables_are_the_factor_hull(sx, order):
    """The library's envelope (from the numbering alone) is the monotone hull
    of where the oracle's LAPACK factor is non-zero: no tile it leaves out
    holds a non-zero, and it visits no block column further up than needed."""
    m = numbered_mesh(order)
    mesh = sx.Mesh(m)
    above, right = mesh.envelope()
    ha, hr = sx.band_envelope(m)  # the host-only query gives the mesh's tables
    assert np.array_equal(above, ha) and np.array_equal(right, hr), order
    ref = OracleSystem(OracleMesh(m), 3.0, 0.0, O_DIRECT).band()
    ea, er = lapack_tile_hull(ref, m.nsolve, m.nband)
    assert np.array_equal(above, ea), (order, above, ea)
    assert np.array_equal(right, er), (order, right, er)

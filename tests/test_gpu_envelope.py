"""GPU parity of the band factor and of the direct solves under numberings
whose factor envelopes differ.

The factorisation and the two band sweeps work only on the tiles inside the
factor's envelope (the tiles of the band that Cholesky fill can reach); every
other tile is an exact zero of LAPACK's factor.  So the exported band is
checked against the oracle's dpbtrf entry by entry: zero exactly where the
oracle's is zero, within 1e-12 of its largest entry elsewhere; and the
solutions of the plain and batched forms (several cluster schedules) against
the oracle's FP64 direct solve within 1e-12 (relative L2 and max norm).

Numberings: reverse Cuthill-McKee (the front-end's default, a smooth
staircase), Cuthill-McKee (the same order reversed), the naive element order
(a ragged envelope), a seeded random permutation of the solve nodes (a
nearly full band), and RCM with runs of nodes exchanged (a staircase that
falls and rises, so that the envelope's monotone hull is what bounds it).
"""
import dataclasses

import numpy as np
import pytest

from oracle.oracle import DIRECT as O_DIRECT
from oracle.oracle import OracleMesh, OracleSystem, solve_planes

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


def numbered_mesh(order, nx=10, ny=8, np_=7, seed=4):
    """A jittered periodic channel whose solve nodes are numbered by `order`."""
    from semtex_b200.mesh import rect_mesh
    kw = dict(x0=0.0, x1=2 * np.pi, y0=0.0, y1=1.0, jitter=0.15, seed=seed, periodic_x=True,
              bc={"bottom": "D", "top": "D"})
    if order == "none":
        return rect_mesh(nx, ny, np_, renumber="none", **kw)
    m = rect_mesh(nx, ny, np_, **kw)
    ns = m.nsolve
    if order == "rcm":
        return m
    if order == "cm":
        perm = np.arange(ns)[::-1]
    elif order == "random":
        perm = np.random.default_rng(seed).permutation(ns)
    elif order == "swapped":
        # RCM with two pairs of 64-node runs exchanged: the lowest row block
        # that a block column reaches then falls and rises along the band
        perm = np.arange(ns)
        for a, b in ((3, 5), (8, 9)):
            ra, rb = perm[64 * a:64 * (a + 1)].copy(), perm[64 * b:64 * (b + 1)].copy()
            perm[64 * a:64 * (a + 1)], perm[64 * b:64 * (b + 1)] = rb, ra
    else:
        raise ValueError(order)
    new = np.concatenate([perm, np.arange(ns, m.nglobal)])
    btog = new[m.btog].astype(np.int32)
    solve = btog < ns
    gmax = np.where(solve, btog, -1).max(axis=1)
    gmin = np.where(solve, btog, np.iinfo(np.int32).max).min(axis=1)
    has = solve.any(axis=1)
    nband = int((gmax[has] - gmin[has]).max()) + 1
    return dataclasses.replace(m, btog=btog, nband=nband)


ORDERS = ["rcm", "cm", "none", "random", "swapped"]


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


def lapack_tile_hull(ab, nsolve, nband, nb=64):
    """The tables the envelope must equal, from the oracle's factor alone:
    for each block column the lowest row block holding a non-zero of the
    factor, its suffix minimum over the later columns (the monotone hull),
    and from it the tiles above each diagonal and right of it."""
    kd = nband - 1
    nblk = (nsolve + nb - 1) // nb
    low = np.arange(nblk)
    cols, offs = np.nonzero(ab)
    rows = cols + offs - kd
    np.minimum.at(low, cols // nb, rows // nb)
    fm = np.minimum.accumulate(low[::-1])[::-1]
    J = (kd + nb - 1) // nb
    above = np.minimum(np.arange(nblk) - fm, J)
    right = np.zeros(nblk, dtype=np.int64)
    for k in range(nblk):
        c = k
        while c + 1 < nblk and fm[c + 1] <= k:
            c += 1
        right[k] = min(J, c - k)
    return above, right


@pytest.mark.parametrize("order", ORDERS)
def test_envelope_tables_are_the_factor_hull(sx, order):
    """The library's envelope (from the numbering alone) is the monotone hull
    of where the oracle's LAPACK factor is non-zero: no tile it leaves out
    holds a non-zero, and it visits no block column further up than needed."""
    m = numbered_mesh(order)
    mesh = sx.Mesh(m)
    above, right = mesh.envelope()
    ref = OracleSystem(OracleMesh(m), 3.0, 0.0, O_DIRECT).band()
    ea, er = lapack_tile_hull(ref, m.nsolve, m.nband)
    assert np.array_equal(above, ea), (order, above, ea)
    assert np.array_equal(right, er), (order, right, er)

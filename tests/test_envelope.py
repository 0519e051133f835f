"""The band factor's envelope tables on the host (no GPU).

The library computes, from a mesh's numbering alone, which 64 x 64 tiles of
the band factor the factorisation and the two sweeps visit
(`sx_mesh_desc_envelope`, the host-only form of `sx_mesh_envelope`).  Here
they are checked against the monotone hull of where the oracle's LAPACK
factor (dpbtrf restated) is non-zero, under five numberings and on config
2's channel: nothing the tables leave out holds a non-zero, and they visit
no tile further from the diagonal than the hull.
"""
import numpy as np
import pytest

from oracle.oracle import DIRECT as O_DIRECT
from oracle.oracle import OracleMesh, OracleSystem
from tests.numberings import ORDERS, lapack_tile_hull, numbered_mesh


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


def _check_against_factor(sx, m, lam=3.0):
    above, right = sx.band_envelope(m)
    ref = OracleSystem(OracleMesh(m), lam, 0.0, O_DIRECT).band()
    ea, er = lapack_tile_hull(ref, m.nsolve, m.nband)
    assert np.array_equal(above, ea), (above, ea)
    assert np.array_equal(right, er), (right, er)
    return above


@pytest.mark.parametrize("order", ORDERS)
def test_envelope_is_the_factor_hull(sx, order):
    _check_against_factor(sx, numbered_mesh(order))


def test_envelope_config2_channel(sx):
    """Config 2's channel (32 x 32, N = 8, RCM): 15,104 unknowns, 236 block
    columns; the envelope holds about 0.62 of the band's tiles."""
    from semtex_b200.workloads import config2
    m = config2().mesh
    above = _check_against_factor(sx, m, lam=1e6)
    nblk = len(above)
    J = (m.nband - 1 + 63) // 64
    full = sum(min(J, k) for k in range(nblk))
    assert 0.5 < above.sum() / full < 0.75


def test_envelope_refuses_bad_numbering(sx):
    m = numbered_mesh("rcm")
    bad = m.btog.copy()
    bad[0, 0] = -1
    import dataclasses
    with pytest.raises(RuntimeError):
        sx.band_envelope(dataclasses.replace(m, btog=bad))

"""GPU tests of ModalMatrixSys semantics that the other parity tests do not
reach:

* SolverKind MIXED (src/matrix.cpp:92-96): mode 0 is a DIRECT system, every
  other mode JACPCG; each plane matches the oracle's solve of that kind.
* A rank's block of modes (base_mode > 0, src/geometry.h:53-58): plane 0 is
  then mode base_mode's real part, not mode 0, and there is no Nyquist plane
  to skip.  Its solution equals, bit for bit, the same modes solved inside a
  system that starts at mode 0 (the plain form: same kernels, same schedule),
  and to rounding in the batched forms.
"""
import numpy as np
import pytest

from oracle.oracle import DIRECT as O_DIRECT
from oracle.oracle import JACPCG as O_JACPCG
from oracle.oracle import OracleMesh, OracleSystem

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return (np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300),
            np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def test_mixed_solver_kind_direct_mode0_jacpcg_others(sx):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=6, ny=4, np_=7, nz=8, lam=50.0, seed=13)
    m = w.mesh
    S = sx.ModalMatrixSys(sx.Mesh(m), lambda2=50.0, beta=1.0, num_modes=w.num_modes,
                          method=sx.MIXED_SOLVER)
    S.band(0)  # mode 0 is DIRECT: its band factor exists
    with pytest.raises(sx.SolverError):
        S.band(1)  # mode 1 is JACPCG: no band
    u, st = S.solve(w.forcing, tol_rel=1e-12, step_max=5000, return_stats=True)
    om = OracleMesh(m)
    # mode 0: the direct solve
    u0, _ = OracleSystem(om, 50.0, 0.0, O_DIRECT).solve_plane(w.forcing[0], None)
    l2, mx = rel(u[0], u0)
    assert l2 <= 1e-12 and mx <= 1e-12, (l2, mx)
    # modes 1..3: Jacobi-PCG to the same tolerance
    for k in range(1, w.num_modes):
        osys = OracleSystem(om, 50.0, float(k * k), O_JACPCG)
        for p in (2 * k, 2 * k + 1):
            uo, _ = osys.solve_plane(w.forcing[p], None, tol_rel=1e-12, step_max=5000)
            l2, mx = rel(u[p], uo)
            assert l2 <= 1e-10 and mx <= 1e-10, (p, l2, mx)
    assert st["iterations_max"] > 0
    assert np.all(u[1] == 0.0)  # the Nyquist plane is not solved


@pytest.mark.parametrize("method", ["DIRECT", "JACPCG"])
def test_rank_block_equals_same_modes_from_mode0(sx, torch, method):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=6, np_=8, nz=12, lam=1e4, seed=17)
    m = w.mesh
    meth = getattr(sx, method)
    mesh = sx.Mesh(m)
    full = sx.ModalMatrixSys(mesh, lambda2=1e4, beta=1.0, base_mode=0, num_modes=6, method=meth)
    block = sx.ModalMatrixSys(mesh, lambda2=1e4, beta=1.0, base_mode=3, num_modes=3, method=meth)
    ff = torch.tensor(w.forcing, device="cuda")
    fb = ff[6:12].clone()          # planes 6..11 = Re/Im of modes 3, 4, 5
    uf, ub, fw = torch.zeros_like(ff), torch.zeros_like(fb), ff.clone()
    stf = full.solve_device(uf.data_ptr(), fw.data_ptr(), 0, 12, m.nplane, tol_rel=1e-12, step_max=5000)
    stb = block.solve_device(ub.data_ptr(), fb.data_ptr(), 0, 6, m.nplane, tol_rel=1e-12, step_max=5000)
    torch.cuda.synchronize()
    assert stb["planes_solved"] == 6 and stf["planes_solved"] == 11
    a, b = uf[6:12].cpu().numpy(), ub.cpu().numpy()
    assert np.array_equal(a, b)
    # and mode 3 against the oracle
    osys = OracleSystem(OracleMesh(m), 1e4, 9.0, O_DIRECT)
    uo, _ = osys.solve_plane(w.forcing[6], None)
    l2, mx = rel(b[0], uo)
    tol = 1e-12 if method == "DIRECT" else 1e-10
    assert l2 <= tol and mx <= tol, (l2, mx)


@pytest.mark.parametrize("prec", ["FP64", "MIXED_FP32"])
def test_rank_block_batched_forms(sx, torch, prec):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=6, np_=8, nz=12, lam=1e4, seed=19)
    m = w.mesh
    mesh = sx.Mesh(m)
    p = getattr(sx, prec)
    full = sx.ModalMatrixSys(mesh, lambda2=1e4, beta=1.0, base_mode=0, num_modes=6, method=sx.DIRECT)
    block = sx.ModalMatrixSys(mesh, lambda2=1e4, beta=1.0, base_mode=3, num_modes=3, method=sx.DIRECT)
    ff = torch.tensor(w.forcing, device="cuda")
    fb = ff[6:12].clone()
    uf, ub, fw = torch.zeros_like(ff), torch.zeros_like(fb), ff.clone()
    full.solve_batched(uf.data_ptr(), fw.data_ptr(), 0, 12, m.nplane, p, 1e-12, 20)
    st = block.solve_batched(ub.data_ptr(), fb.data_ptr(), 0, 6, m.nplane, p, 1e-12, 20)
    torch.cuda.synchronize()
    assert st["planes_solved"] == 6
    l2, mx = rel(ub.cpu().numpy(), uf[6:12].cpu().numpy())
    tol = 1e-13 if prec == "FP64" else 1e-10
    assert l2 <= tol and mx <= tol, (l2, mx)

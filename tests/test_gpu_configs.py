"""GPU parity tests on reduced-size versions of the benchmark configurations.

* config 3 shape (jittered channel, N = 10, lambda2 log-uniform in
  [1e-2, 1e4] across the modes, manufactured solution): the batched FP64
  form within 1e-12 of the oracle's FP64 direct solve, the mixed form within
  1e-10 (its ill-conditioned modes go to the band Cholesky), and both close
  to the manufactured solution.
* config 5 shape (one DNS timestep's elliptic phase: three viscous
  Helmholtz solves with Dirichlet walls and the pressure Poisson solve with
  natural walls, its k = 0 mode singular and pinned): each solve's batched
  FP64 form within 1e-12 of the oracle, the mixed form on SX_AUTO systems
  within 1e-10.
"""
import numpy as np
import pytest

from oracle.oracle import OracleMesh, solve_planes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _solve(torch, S, w, precision, **kw):
    f = torch.tensor(w.forcing, device="cuda")
    u = torch.zeros_like(f)
    st = S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, w.mesh.nplane, precision, **kw)
    torch.cuda.synchronize()
    S.status()
    return u.cpu().numpy(), st


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b), np.abs(a - b).max() / np.abs(b).max()


def test_config3_reduced(sx, torch):
    from semtex_b200.workloads import config3
    w = config3(nx=8, ny=8, np_=11, nz=16, seed=3)
    S = sx.ModalMatrixSys(sx.Mesh(w.mesh), num_modes=w.num_modes, method=sx.DIRECT,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    sp = [0] + list(range(2, w.nz))
    # lambda2 is the whole Helmholtz constant of each mode here (betak2 = 0)
    uo, _ = solve_planes(OracleMesh(w.mesh), 0.0, 0.0, w.forcing, None, lambda2_per_mode=w.lambda2)
    ub, _ = _solve(torch, S, w, sx.FP64)
    l2, mx = _rel(ub[sp], uo[sp])
    assert l2 <= 1e-12 and mx <= 1e-12, (l2, mx)
    um, st = _solve(torch, S, w, sx.MIXED_FP32, tol_rel=1e-12, max_refine=30)
    assert st["planes_solved"] == len(sp)
    l2, mx = _rel(um[sp], uo[sp])
    assert l2 <= 1e-10 and mx <= 1e-10, (l2, mx, st)
    # discretisation error against u = sum_k a_k sin(pi y) cos(3x) cos(kz)
    # (the oracle's own is 2.9e-10 on this mesh)
    l2, _ = _rel(ub[sp], w.exact[sp])
    assert l2 <= 1e-8, l2


@pytest.mark.parametrize("solve", [0, 1, 2, 3], ids=["u", "v", "w", "p"])
def test_config5_reduced(sx, torch, solve):
    from semtex_b200.workloads import config5
    w = config5(nx=8, ny=4, np_=11, nz=8)[solve]
    sp = [0] + list(range(2, w.nz))
    uo, _ = solve_planes(OracleMesh(w.mesh), 0.0, 1.0, w.forcing, None, lambda2_per_mode=w.lambda2)
    mesh = sx.Mesh(w.mesh)
    S = sx.ModalMatrixSys(mesh, num_modes=w.num_modes, method=sx.DIRECT, lambda2_modes=w.lambda2,
                          betak2_modes=w.betak2)
    ub, _ = _solve(torch, S, w, sx.FP64)
    l2, mx = _rel(ub[sp], uo[sp])
    assert l2 <= 1e-12 and mx <= 1e-12, (w.name, l2, mx)
    A = sx.ModalMatrixSys(mesh, num_modes=w.num_modes, method=sx.AUTO, lambda2_modes=w.lambda2,
                          betak2_modes=w.betak2)
    um, st = _solve(torch, A, w, sx.MIXED_FP32, tol_rel=1e-12, max_refine=30)
    l2, mx = _rel(um[sp], uo[sp])
    assert l2 <= 1e-10 and mx <= 1e-10, (w.name, l2, mx, st)

"""GPU tests of the error paths a caller can reach, each made on the host
(an input, a limit), never by faulting the device:

* a bounded device-side wait that runs out (the wait limit set to "give up at
  the first unsuccessful probe") is reported as SX_ERR_TIMEOUT by the band
  sweeps -- whose first wait, for a tile just requested from HBM, always
  finds it in flight; the kernel returns normally, and with the default limit
  restored the next solve is bit for bit the earlier one.  (The FP32
  iterations' wait honours the same limit, but their staged copies have
  usually landed by the time of the first probe, so no test can make that
  wait run out on demand);
* a Helmholtz constant that makes H indefinite (lambda2 = -1e6): the
  factorisation reports SX_ERR_NOT_SPD, as the reference's dpbtrf failure
  does (src/matrix.cpp:259-261);
* a call from a device other than the mesh's is refused with SX_ERR_ARG.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SX_ERR_ARG, SX_ERR_NOT_SPD, SX_ERR_TIMEOUT = 1, 6, 10


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture
def default_wait(sx):
    yield
    sx.lib.sx_set_wait_limit(-1.0)


def _channel(sx, method, nz=8, lam=1e6):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=6, np_=9, nz=nz, lam=lam, seed=3)
    S = sx.ModalMatrixSys(sx.Mesh(w.mesh), num_modes=w.num_modes, method=method,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    return w, S


def test_band_sweep_wait_timeout_is_reported(sx, torch, default_wait):
    w, S = _channel(sx, sx.DIRECT)
    S.tune(band_cluster=2)  # leader and a rank: every kind of wait is on the path
    f0 = torch.tensor(w.forcing, device="cuda")
    f, u = torch.empty_like(f0), torch.zeros_like(f0)

    def solve():
        f.copy_(f0)
        u.zero_()
        S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, w.mesh.nplane, sx.FP64)
        return u.cpu().numpy()

    ref = solve()
    assert sx.lib.sx_set_wait_limit(0.0) == 0
    with pytest.raises(sx.SolverError) as ei:
        solve()
    assert ei.value.status == SX_ERR_TIMEOUT
    assert sx.lib.sx_set_wait_limit(-1.0) == 0
    again = solve()  # the context is usable and the status word was cleared
    assert np.array_equal(again, ref)
    S.status()


def test_indefinite_system_is_not_spd(sx, torch):
    from semtex_b200.mesh import rect_mesh
    m = rect_mesh(3, 3, 6, 0.0, 1.0, 0.0, 1.0)
    mesh = sx.Mesh(m)
    with pytest.raises(sx.SolverError) as ei:
        sx.ModalMatrixSys(mesh, lambda2=-1e6, num_modes=1, method=sx.DIRECT)
    assert ei.value.status == SX_ERR_NOT_SPD
    # the same mesh still builds and solves a well-posed system afterwards
    S = sx.ModalMatrixSys(mesh, lambda2=1.0, num_modes=1, method=sx.DIRECT)
    f = m.eval_nodes(lambda x, y: np.sin(np.pi * x) * np.sin(np.pi * y))[None]
    u = S.solve(f)
    assert np.all(np.isfinite(u)) and np.abs(u).max() > 0.0


def test_call_from_another_device_is_refused(sx, torch):
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU: no other device to call from")
    w, S = _channel(sx, sx.DIRECT, nz=2)
    f = torch.tensor(w.forcing, device="cuda:0")
    u = torch.zeros_like(f)
    assert sx.lib.sx_set_device(1) == 0
    try:
        with pytest.raises(sx.SolverError) as ei:
            S.solve_device(u.data_ptr(), f.data_ptr(), 0, w.nz, w.mesh.nplane)
        assert ei.value.status == SX_ERR_ARG
    finally:
        sx.lib.sx_set_device(0)

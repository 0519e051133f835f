"""GPU tests of sx_field_solve_device_static, the direct solve whose scratch is
a fixed device array (no device allocation in any call).

* Two consecutive calls give bit for bit the result of sx_field_solve_device
  (same kernels), with and without boundary values.
* The device's free memory is the same before and after those calls.
* A solve needing more than SX_STATIC_SCRATCH_BYTES per mode is refused
  with SX_ERR_CAPACITY; a JACPCG system with SX_ERR_UNSUPPORTED.

The file is named to be collected last, so it also runs after every other
GPU test in the same process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SX_ERR_UNSUPPORTED, SX_ERR_CAPACITY = 9, 11


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _case(sx, with_bc):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=8, np_=9, nz=12, lam=1e6, seed=11)
    S = sx.ModalMatrixSys(sx.Mesh(w.mesh), num_modes=w.num_modes, method=sx.DIRECT,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    bc = None
    if with_bc:
        nb = max(len(w.mesh.boundaries), 1)
        bc = np.random.default_rng(5).standard_normal((w.nz, nb, w.mesh.np))
    return w, S, bc


@pytest.mark.parametrize("with_bc", [False, True])
def test_static_equals_device_on_consecutive_calls(sx, torch, with_bc):
    w, S, bc = _case(sx, with_bc)
    # device buffers made once: the copies below allocate nothing on the device
    f_host = torch.tensor(w.forcing)
    f = torch.empty_like(f_host, device="cuda")
    u = torch.empty_like(f)
    b = None if bc is None else torch.tensor(bc, device="cuda")
    bptr = 0 if b is None else b.data_ptr()
    args = (w.nz, w.mesh.nplane)

    def run(entry):
        f.copy_(f_host)  # the forcing is overwritten by a solve
        u.zero_()
        st = entry(u.data_ptr(), f.data_ptr(), bptr, *args)
        torch.cuda.synchronize()
        S.status()
        return u.cpu().numpy(), st

    ref, st_ref = run(S.solve_device)
    first, st1 = run(S.solve_device_static)  # first call on the device: set-up
    free0, _ = torch.cuda.mem_get_info()
    second, st2 = run(S.solve_device_static)
    third, st3 = run(S.solve_device_static)
    free1, _ = torch.cuda.mem_get_info()
    assert np.all(np.isfinite(ref)) and np.linalg.norm(ref) > 0.0
    for got in (first, second, third):
        assert np.array_equal(got, ref)
    assert st1["planes_solved"] == st_ref["planes_solved"] == w.planes_solved
    assert st2["kernel_launches"] == st3["kernel_launches"] > 0
    assert free1 == free0


def test_static_rejects_oversized_solve(sx, torch):
    from semtex_b200.mesh import rect_mesh
    # a 1200 x 4 element strip at N = 8 (narrow band, cheap to factor); one
    # mode of two planes needs about 4.46 MB of scratch (rhs + element
    # boundary forcing + essential values), above the 4 MiB array
    m = rect_mesh(1200, 4, 9, 0.0, 30.0, 0.0, 0.1)
    S = sx.ModalMatrixSys(sx.Mesh(m), num_modes=2, method=sx.DIRECT,
                          lambda2_modes=np.full(2, 10.0), betak2_modes=np.array([0.0, 1.0]))
    u = torch.zeros((4, m.nplane), dtype=torch.float64, device="cuda")
    f = torch.zeros_like(u)
    with pytest.raises(sx.SolverError) as ei:
        S.solve_device_static(u.data_ptr(), f.data_ptr(), 0, 4, m.nplane)
    assert ei.value.status == SX_ERR_CAPACITY
    assert "SX_STATIC_SCRATCH_BYTES" in str(ei.value)


def test_static_rejects_iterative_systems(sx, torch):
    from semtex_b200.mesh import rect_mesh
    m = rect_mesh(3, 3, 5, 0.0, 1.0, 0.0, 1.0)
    S = sx.ModalMatrixSys(sx.Mesh(m), num_modes=1, method=sx.JACPCG,
                          lambda2_modes=np.full(1, 10.0), betak2_modes=np.zeros(1))
    u = torch.zeros((1, m.nplane), dtype=torch.float64, device="cuda")
    f = torch.zeros_like(u)
    with pytest.raises(sx.SolverError) as ei:
        S.solve_device_static(u.data_ptr(), f.data_ptr(), 0, 1, m.nplane)
    assert ei.value.status == SX_ERR_UNSUPPORTED

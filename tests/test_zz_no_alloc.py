"""GPU tests of sx_field_solve_device_static, the direct solve whose scratch is
a fixed device array (no device allocation in any call).

* Consecutive calls give bit for bit the result of sx_field_solve_device
  (same kernels): with and without boundary values, one plane, a block of
  modes that does not start at mode 0, and on a stream the caller created.
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


def _case(sx, with_bc, nz=12, base_mode=0):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=8, np_=9, nz=max(nz, 2), lam=1e6, seed=11)
    nm = 1 if nz == 1 else nz // 2
    lam = w.lambda2[:nm]
    bk2 = (np.arange(base_mode, base_mode + nm, dtype=np.float64)) ** 2
    S = sx.ModalMatrixSys(sx.Mesh(w.mesh), base_mode=base_mode, num_modes=nm, method=sx.DIRECT,
                          lambda2_modes=lam, betak2_modes=bk2)
    forcing = w.forcing[:nz]
    bc = None
    if with_bc:
        nb = max(len(w.mesh.boundaries), 1)
        bc = np.random.default_rng(5).standard_normal((nz, nb, w.mesh.np))
    return w, S, bc, forcing


# (boundary values, planes, first mode, stream): the legacy default stream with
# and without boundary data; one plane (mode 0 alone); a rank's block of modes
# (base_mode > 0: no Nyquist plane, plane 0 is not mode 0); a stream the caller
# created, on which the job records and the solve are ordered
CASES = {
    "nz12": (False, 12, 0, False),
    "nz12_bc": (True, 12, 0, False),
    "nz1": (False, 1, 0, False),
    "base_mode2": (True, 8, 2, False),
    "user_stream": (True, 12, 0, True),
}


@pytest.mark.parametrize("case", list(CASES))
def test_static_equals_device_on_consecutive_calls(sx, torch, case):
    with_bc, nz, base_mode, own_stream = CASES[case]
    w, S, bc, forcing = _case(sx, with_bc, nz, base_mode)
    # device buffers made once: the copies below allocate nothing on the device
    f_host = torch.tensor(forcing)
    f = torch.empty_like(f_host, device="cuda")
    u = torch.empty_like(f)
    b = None if bc is None else torch.tensor(bc, device="cuda")
    bptr = 0 if b is None else b.data_ptr()
    args = (nz, w.mesh.nplane)
    stream = torch.cuda.Stream() if own_stream else None
    sptr = stream.cuda_stream if stream is not None else 0

    def run(entry):
        ctx = torch.cuda.stream(stream) if stream is not None else torch.cuda.stream(torch.cuda.default_stream())
        with ctx:
            f.copy_(f_host)  # the forcing is overwritten by a solve
            u.zero_()
            st = entry(u.data_ptr(), f.data_ptr(), bptr, *args, stream=sptr)
            out = u.cpu().numpy()  # ordered after the solve on the same stream
        torch.cuda.synchronize()
        S.status()
        return out, st

    ref, st_ref = run(S.solve_device)
    first, st1 = run(S.solve_device_static)  # first call on the device: set-up
    free0, _ = torch.cuda.mem_get_info()
    second, st2 = run(S.solve_device_static)
    third, st3 = run(S.solve_device_static)
    free1, _ = torch.cuda.mem_get_info()
    assert np.all(np.isfinite(ref)) and np.linalg.norm(ref) > 0.0
    for got in (first, second, third):
        assert np.array_equal(got, ref)
    planes = 1 if nz == 1 else (nz - 1 if base_mode == 0 else nz)
    assert st1["planes_solved"] == st_ref["planes_solved"] == planes
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

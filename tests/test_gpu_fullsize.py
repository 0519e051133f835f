"""GPU parity at the benchmark sizes, against the oracle's FP64 direct solve
(the oracle's band factored by LAPACK dpbtrf, the routine the reference calls
at src/matrix.cpp:259, so that set-up takes seconds):

* config 2 at full size (32 x 32 jittered quads, N = 8, nz = 64, lambda2 =
  1e6 + k^2): modes 0, 1 and 31 -- plain and batched FP64 within 1e-12
  relative L2 and max norm, the mixed-precision form within 1e-10;
* a mid-size config-3 case (32 x 32 quads jittered +-20 %, N = 10, nz = 16,
  lambda2 from 1e-2 to 1e4): every mode, both FP64 forms within 1e-12, the
  mixed form within 1e-10.
"""
import numpy as np
import pytest

from oracle.oracle import DIRECT, OracleMesh, OracleSystem

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


def _solve_forms(sx, torch, w):
    """(plain, batched FP64, mixed) solutions of every plane of w."""
    m = w.mesh
    S = sx.ModalMatrixSys(sx.Mesh(m), base_mode=w.base_mode, num_modes=w.num_modes, method=sx.DIRECT,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    f0 = torch.tensor(w.forcing, device="cuda")
    out = []
    for form in ("plain", "fp64", "mixed"):
        f, u = f0.clone(), torch.zeros_like(f0)
        if form == "plain":
            S.solve_device(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane)
        else:
            prec = sx.FP64 if form == "fp64" else sx.MIXED_FP32
            S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, prec, 1e-12, 30)
        torch.cuda.synchronize()
        out.append(u.cpu().numpy())
    S.status()
    return out


def _check_modes(w, sols, modes):
    om = OracleMesh(w.mesh)
    worst = {}
    for k in modes:
        osys = OracleSystem(om, float(w.lambda2[k]), float(w.betak2[k]), DIRECT, factor="lapack")
        planes = [0] if k == 0 and w.base_mode == 0 else [2 * k, 2 * k + 1]
        uo = np.array([osys.solve_plane(w.forcing[p], None)[0] for p in planes])
        for name, u, tol in zip(("plain", "fp64", "mixed"), sols, (1e-12, 1e-12, 1e-10)):
            l2, mx = rel(u[planes], uo)
            worst[(k, name)] = (l2, mx)
            assert l2 <= tol and mx <= tol, (k, float(w.lambda2[k]), name, l2, mx)
    return worst


def test_config2_full_size_modes_0_1_31(sx, torch):
    from semtex_b200.workloads import config2
    w = config2()
    assert w.mesh.n_unique == 65792 and w.nz == 64
    sols = _solve_forms(sx, torch, w)
    _check_modes(w, sols, (0, 1, 31))
    assert np.all(sols[0][1] == 0.0)  # Nyquist plane untouched


def test_config3_mid_size_every_mode(sx, torch):
    from semtex_b200.workloads import Workload, config3_block
    b = config3_block(world=1, rank=0, nx=32, ny=32, modes_per_rank=8)
    # the lambda2 range of config 3 end to end, lowest to highest
    lam = np.logspace(-2, 4, 8)
    m = b.mesh
    shape = m.eval_nodes(lambda x, y: np.sin(np.pi * y) * np.cos(3 * x))
    a = np.random.default_rng(33).standard_normal(8)
    f = np.zeros((16, m.nplane))
    for k in range(8):
        f[2 * k] = -(np.pi ** 2 + 9.0 + lam[k]) * a[k] * shape
        f[2 * k + 1] = 0.5 * f[2 * k]
    w = Workload("cfg3_mid_32x32_N10_nz16", m, 16, 1.0, lam, np.zeros(8), f)
    sols = _solve_forms(sx, torch, w)
    _check_modes(w, sols, range(8))

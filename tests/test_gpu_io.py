"""GPU test of compare-style checking through the reference's field-file
format: each regression problem is solved on the GPU, its solution written
as a field file and read back, and the inf-norm of exact - computed from the
GPU norm kernel reproduces the golden line of regress/<name>.ok
(utility/compare.cpp:206-218: "noise-level" below 1e-12, else 3 significant
digits).  The kernel's L2 figure (AuxField::errors, src/auxfield.cpp:813-860,
at the field's own GLL points) matches numpy."""
import numpy as np
import pytest

from tests.problems import PROBLEMS_2D, build_2d, golden_ok

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


@pytest.mark.parametrize("name", list(PROBLEMS_2D))
def test_golden_through_field_file(sx, torch, tmp_path, name):
    m, p, f, bc, exact = build_2d(name)
    mesh = sx.Mesh(m)
    S = sx.ModalMatrixSys(mesh, p["lambda2"], 0.0, 0, 1, sx.DIRECT)
    u = S.solve(f, bc)
    path = tmp_path / f"{name}.fld"
    sx.write_field(path, {"u": u}, m.np, m.nel, session=name)
    h, g = sx.read_field(path)
    assert h["fields"] == "u" and np.array_equal(g["u"], u)
    dc = torch.tensor(g["u"], device="cuda")
    de = torch.tensor(exact[None], device="cuda")
    norms = sx.field_norms(mesh, dc.data_ptr(), de.data_ptr(), 1, m.nplane)
    err = np.abs(exact - g["u"][0])
    assert norms[0, 0] == err.max()
    assert golden_ok(norms[0, 0], p["golden"]), (name, norms[0, 0])
    q4 = np.array([mesh.geometry(e)[3] for e in range(m.nel)])  # (nel, npnp) Q4
    e2 = (err.reshape(m.nel, -1) ** 2 * q4).sum(axis=1)
    l2 = np.sqrt(e2).sum() / q4.sum()
    assert abs(norms[0, 1] - l2) <= 1e-12 * max(l2, 1e-300) + 1e-300

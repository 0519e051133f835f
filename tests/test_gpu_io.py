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


def test_solve_with_numbering_from_file(sx, torch, tmp_path):
    """A mesh numbered from a numbering file (here the naive traverse order,
    enumerate -O0's) solves to the RCM-numbered answer: the numbering moves
    the band, not the solution."""
    from semtex_b200.mesh import rect_mesh
    from semtex_b200.workloads import fourier_forcing
    kw = dict(x0=0.0, x1=2 * np.pi, y0=0.0, y1=1.0, jitter=0.15, seed=4, periodic_x=True,
              bc={"bottom": "D", "top": "D"})
    m_rcm = rect_mesh(10, 6, 8, **kw)
    m_naive = rect_mesh(10, 6, 8, renumber="none", **kw)
    path = tmp_path / "naive.num"
    sx.write_numbering(path, {"u": m_naive}, optimization=0)
    m_file = sx.with_numbering(m_rcm, sx.read_numbering(path, "u", m_rcm.nel, m_rcm.np))
    assert m_file.nband == m_naive.nband > m_rcm.nband
    f = fourier_forcing(m_rcm, 6, np.random.default_rng(8))
    out = []
    for m in (m_rcm, m_file):
        S = sx.ModalMatrixSys(sx.Mesh(m), lambda2=30.0, beta=1.0, num_modes=3, method=sx.DIRECT)
        out.append(S.solve(f))
    sp = [0, 2, 3, 4, 5]
    err = np.abs(out[1][sp] - out[0][sp]).max() / np.abs(out[0][sp]).max()
    assert err <= 1e-12, err


def test_singular_mode_pins_the_files_last_solve_node(sx, torch, tmp_path):
    """Pressure-like mode 0 (lambda2 + betak2 = 0, no essential boundary):
    the highest-numbered solve node is pinned to zero (src/matrix.cpp:167-169,
    src/field.cpp:613-614), so which node that is comes from the numbering
    file; two numberings give solutions that differ by a constant."""
    from semtex_b200.mesh import edge_maps, rect_mesh
    kw = dict(x0=0.0, x1=2 * np.pi, y0=0.0, y1=1.0, jitter=0.1, seed=6, periodic_x=True,
              bc={"bottom": "N", "top": "N"})
    m_rcm = rect_mesh(8, 4, 6, **kw)
    m_naive = rect_mesh(8, 4, 6, renumber="none", **kw)
    path = tmp_path / "p.num"
    sx.write_numbering(path, {"p": m_naive})
    m_file = sx.with_numbering(m_rcm, sx.read_numbering(path, "p", m_rcm.nel, m_rcm.np))
    # zero-mean forcing so that the Neumann problem is consistent
    f = m_rcm.eval_nodes(lambda x, y: np.cos(x) * np.cos(np.pi * y))[None]
    emap, _ = edge_maps(m_rcm.np)
    sols = []
    for m in (m_rcm, m_file):
        S = sx.ModalMatrixSys(sx.Mesh(m), lambda2=0.0, beta=0.0, num_modes=1, method=sx.DIRECT)
        u = S.solve(f)[0].reshape(m.nel, m.npnp)
        e, a = np.argwhere(m.btog == m.nsolve - 1)[0]   # the pinned node of this numbering
        assert abs(u[e, emap[a]]) <= 1e-12 * np.abs(u).max()
        sols.append(u)
    d = sols[1] - sols[0]
    assert np.ptp(d) <= 1e-10 * np.abs(sols[0]).max()

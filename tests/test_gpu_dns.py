"""GPU parity of the DNS elliptic-phase field operations against the oracle
(oracle/dns.py), through the C ABI:

* the library's inverse partials and inverse boundary mass equal the
  oracle's (the same sums in the same order);
* x / y derivatives for every supported np, on padded plane strides, within
  1e-13 of the largest value (the GPU fuses the derivative sums' multiply-
  adds); d/dz, smooth and the wave step bit for bit;
* setPForce (2 and 3 dimensions, a rank's block of modes) and project (with
  a scalar, in place) within the same bound;
* the elliptic phase as a chain on the device -- wave step, pressure forcing,
  pressure solve (natural walls, the singular mode pinned), project, viscous
  solves -- against the same chain on the CPU within 1e-10;
* arguments the reference rejects (dt = 0) or that would race (an output
  overlapping an input read across planes) are refused with SX_ERR_ARG.
"""
import numpy as np
import pytest

from oracle import dns
from semtex_b200.mesh import rect_mesh

pytestmark = pytest.mark.gpu

SX_ERR_ARG = 1
TOL = 1e-13


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _mesh(np_, nx=5, ny=3, **kw):
    kw.setdefault("jitter", 0.2)
    kw.setdefault("seed", np_)
    return rect_mesh(nx, ny, np_, 0.0, 2 * np.pi, 0.0, 1.0, **kw)


def _planes(rng, nz, m, stride):
    """nz random planes on a padded stride; the padding holds a marker."""
    a = np.full((nz, stride), 7.25)
    a[:, :m.nplane] = rng.standard_normal((nz, m.nplane))
    return a


def _close(got, want, tol=TOL):
    err = np.abs(got - want).max()
    assert err <= tol * max(np.abs(want).max(), 1e-300), err


def test_partials_and_imass_equal_the_oracle(sx):
    for np_ in (4, 9, 11):
        for m in (_mesh(np_), _mesh(np_, jitter=0.0)):
            geo = dns.Geometry(m)
            mesh = sx.Mesh(m)
            for e in (0, m.nel // 2, m.nel - 1):
                rx, ry, sx_, sy, im = mesh.partials(e)
                for got, want in ((rx, geo.drdx[e]), (ry, geo.drdy[e]), (sx_, geo.dsdx[e]), (sy, geo.dsdy[e])):
                    assert np.array_equal(got, want), np.abs(got - want).max()
            assert np.array_equal(im, geo.imass)


@pytest.mark.parametrize("np_", list(range(3, 13)))
def test_gradient_xy_every_np(sx, torch, np_):
    m = _mesh(np_, nx=7, ny=3)
    geo = dns.Geometry(m)
    mesh = sx.Mesh(m)
    rng = np.random.default_rng(np_)
    nz, stride = 5, m.nplane + 3
    a = _planes(rng, nz, m, stride)
    for dir in (0, 1):
        d = torch.tensor(a, device="cuda")
        sx.field_gradient(mesh, d.data_ptr(), nz, stride, dir)
        got = d.cpu().numpy()
        _close(got[:, :m.nplane], dns.gradient(geo, a[:, :m.nplane], dir))
        assert np.all(got[:, m.nplane:] == 7.25)  # padding untouched


@pytest.mark.parametrize("base", [0, 2])
def test_gradient_z_bitwise(sx, torch, base):
    m = _mesh(6)
    mesh = sx.Mesh(m)
    a = np.random.default_rng(4).standard_normal((8, m.nplane))
    d = torch.tensor(a, device="cuda")
    sx.field_gradient(mesh, d.data_ptr(), 8, m.nplane, 2, beta=0.75, base_mode=base)
    assert np.array_equal(d.cpu().numpy(), dns.gradient_z(a, 0.75, base))


def test_pressure_forcing(sx, torch):
    m = _mesh(9, nx=6, ny=4)
    geo = dns.Geometry(m)
    mesh = sx.Mesh(m)
    rng = np.random.default_rng(5)
    nz, stride = 6, m.nplane + 1
    us = [_planes(rng, nz, m, stride) for _ in range(3)]
    n = m.nplane
    for ndim, base in ((2, 0), (3, 0), (3, 4)):
        d = [torch.tensor(u, device="cuda") for u in us[:ndim]]
        out = torch.full_like(d[0], -1.0)
        sx.pressure_forcing(mesh, [x.data_ptr() for x in d], out.data_ptr(), nz, stride, dt=0.004, beta=1.3,
                            base_mode=base)
        want = dns.pressure_forcing(geo, [u[:, :n] for u in us[:ndim]], 0.004, 1.3, base)
        got = out.cpu().numpy()
        _close(got[:, :n], want)
        assert np.all(got[:, n:] == -1.0)
    # in place over u
    d = [torch.tensor(u, device="cuda") for u in us]
    sx.pressure_forcing(mesh, [x.data_ptr() for x in d], d[0].data_ptr(), nz, stride, dt=0.004, beta=1.3)
    _close(d[0].cpu().numpy()[:, :n], dns.pressure_forcing(geo, [u[:, :n] for u in us], 0.004, 1.3))


@pytest.mark.parametrize("ndim,ncom,nadv", [(2, 2, 2), (2, 3, 3), (3, 3, 4)])
def test_project(sx, torch, ndim, ncom, nadv):
    m = _mesh(11, nx=4, ny=4)
    geo = dns.Geometry(m)
    mesh = sx.Mesh(m)
    rng = np.random.default_rng(6)
    nz, stride = 4, m.nplane + 2
    n = m.nplane
    us = [_planes(rng, nz, m, stride) for _ in range(nadv)]
    p = _planes(rng, nz, m, stride)
    dt, nu, pr = 0.01, 2e-3, 0.71
    want = dns.project(geo, [u[:, :n] for u in us], p[:, :n], dt, nu, ndim, ncom, pr, beta=1.0)
    dp = torch.tensor(p, device="cuda")
    du = [torch.tensor(u, device="cuda") for u in us]
    sx.project(mesh, [x.data_ptr() for x in du], dp.data_ptr(), [x.data_ptr() for x in du], nz, stride, dt, nu,
               ndim=ndim, ncom=ncom, prandtl=pr)  # in place
    for x, w in zip(du, want):
        _close(x.cpu().numpy()[:, :n], w)


def test_smooth_bitwise(sx, torch):
    m = _mesh(8, nx=6, ny=5, periodic_x=True, bc={"bottom": "D", "top": "N"})
    geo = dns.Geometry(m)
    mesh = sx.Mesh(m)
    a = _planes(np.random.default_rng(7), 3, m, m.nplane + 1)
    d = torch.tensor(a, device="cuda")
    sx.field_smooth(mesh, d.data_ptr(), 3, m.nplane + 1)
    got = d.cpu().numpy()
    assert np.array_equal(got[:, :m.nplane], dns.smooth(geo, a[:, :m.nplane]))
    assert np.all(got[:, m.nplane:] == 7.25)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_wave_prop_bitwise(sx, torch, order):
    rng = np.random.default_rng(8 + order)
    nadv, npts = 3, 10007
    us = [[rng.standard_normal(npts) for _ in range(nadv)] for _ in range(order)]
    uf = [[rng.standard_normal(npts) for _ in range(nadv)] for _ in range(order)]
    dus = [[torch.tensor(x, device="cuda") for x in lev] for lev in us]
    duf = [[torch.tensor(x, device="cuda") for x in lev] for lev in uf]
    h = [dus[0][i] for i in range(nadv)]  # in place over the newest level
    sx.wave_prop([[x.data_ptr() for x in lev] for lev in dus], [[x.data_ptr() for x in lev] for lev in duf],
                 [x.data_ptr() for x in h], npts, 0.02)
    want = dns.wave_prop(us, uf, 0.02)
    for x, w in zip(h, want):
        assert np.array_equal(x.cpu().numpy(), w)


def test_elliptic_phase_chain(sx, torch):
    """waveProp -> setPForce -> pressure solve -> project -> viscous solves,
    every step on the device, against the same chain on the CPU."""
    from oracle.oracle import DIRECT, OracleMesh, solve_planes
    kw = dict(nx=8, ny=4, jitter=0.15, seed=11, periodic_x=True)
    mv = _mesh(9, bc={"bottom": "D", "top": "D"}, **kw)
    mp = _mesh(9, bc={"bottom": "N", "top": "N"}, **kw)
    gv = dns.Geometry(mv)
    nz, n = 8, mv.nplane
    dt, nu, beta, order = 0.01, 0.02, 1.0, 2
    rng = np.random.default_rng(12)
    us = [[rng.standard_normal((nz, n)) for _ in range(3)] for _ in range(order)]
    uf = [[rng.standard_normal((nz, n)) for _ in range(3)] for _ in range(order)]
    lam_v = dns.STIFFLY_STABLE[order][0] / (dt * nu)

    # CPU chain
    h = dns.wave_prop(us, uf, dt)
    fp = dns.pressure_forcing(gv, h, dt, beta)
    p, _ = solve_planes(OracleMesh(mp), 0.0, beta, fp, None, DIRECT)
    fv = dns.project(gv, h, p, dt, nu, ndim=3, beta=beta)
    omv = OracleMesh(mv)
    want = [solve_planes(omv, lam_v, beta, f, None, DIRECT)[0] for f in fv]

    # GPU chain
    mesh_v, mesh_p = sx.Mesh(mv), sx.Mesh(mp)
    Sp = sx.ModalMatrixSys(mesh_p, 0.0, beta, 0, nz // 2, sx.DIRECT)
    Sv = sx.ModalMatrixSys(mesh_v, lam_v, beta, 0, nz // 2, sx.DIRECT)
    dus = [[torch.tensor(x, device="cuda") for x in lev] for lev in us]
    duf = [[torch.tensor(x, device="cuda") for x in lev] for lev in uf]
    dh = [torch.empty_like(dus[0][0]) for _ in range(3)]
    ptr = lambda ts: [t.data_ptr() for t in ts]  # noqa: E731
    sx.wave_prop([ptr(lev) for lev in dus], [ptr(lev) for lev in duf], ptr(dh), nz * n, dt)
    dfp = torch.empty_like(dh[0])
    sx.pressure_forcing(mesh_v, ptr(dh), dfp.data_ptr(), nz, n, dt, beta)
    dp = torch.zeros_like(dfp)
    Sp.solve_device(dp.data_ptr(), dfp.data_ptr(), 0, nz, n)
    sx.project(mesh_v, ptr(dh), dp.data_ptr(), ptr(dh), nz, n, dt, nu, ndim=3, beta=beta)
    got = []
    for f in dh:
        u = torch.zeros_like(f)
        Sv.solve_device(u.data_ptr(), f.data_ptr(), 0, nz, n)
        got.append(u)
    torch.cuda.synchronize()
    for g, w in zip(got, want):
        g = g.cpu().numpy()
        rel = np.linalg.norm(g - w) / np.linalg.norm(w)
        assert rel <= 1e-10, rel


def test_refused_arguments(sx, torch):
    m = _mesh(5)
    mesh = sx.Mesh(m)
    n = m.nplane
    d = [torch.zeros((4, n), dtype=torch.float64, device="cuda") for _ in range(4)]
    L = sx.lib
    ptrs = sx._ptrs([x.data_ptr() for x in d[:3]])
    assert L.sx_dns_pressure_forcing(mesh.h, ptrs, 3, d[3].data_ptr(), 4, n, 0.0, 1.0, 0, 0) == SX_ERR_ARG
    assert L.sx_dns_pressure_forcing(mesh.h, ptrs, 3, d[2].data_ptr(), 4, n, 0.1, 1.0, 0, 0) == SX_ERR_ARG
    assert L.sx_dns_pressure_forcing(mesh.h, ptrs, 3, d[3].data_ptr(), 3, n, 0.1, 1.0, 0, 0) == SX_ERR_ARG
    assert L.sx_field_gradient(mesh.h, d[0].data_ptr(), 3, n, 2, 1.0, 0, 0) == SX_ERR_ARG
    assert L.sx_field_gradient(mesh.h, d[0].data_ptr(), 4, n - 1, 0, 1.0, 0, 0) == SX_ERR_ARG
    assert L.sx_dns_project(mesh.h, ptrs, d[0].data_ptr(), ptrs, 3, 3, 3, 4, n, 0.1, 0.01, 1.0, 1.0, 0,
                            0) == SX_ERR_ARG  # p is uf[0]
    assert L.sx_dns_project(mesh.h, ptrs, d[3].data_ptr(), ptrs, 3, 2, 3, 4, n, 0.1, 0.01, 1.0, 1.0, 0,
                            0) == SX_ERR_ARG  # ncom < ndim
    torch.cuda.synchronize()

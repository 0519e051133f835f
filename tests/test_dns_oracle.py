"""CPU tests that pin the DNS elliptic-phase oracle (oracle/dns.py) to
mathematics, the reference having no test that fixes these routines'
outputs:

* the spectral x / y derivative of a polynomial of degree <= N is exact on
  affine elements -- rectangles (where the null mapping drops dr/dy and
  ds/dx, src/element.cpp:1431-1434) and sheared parallelograms (where it
  drops none) -- and converges spectrally on jittered quads;
* d/dz of Fourier planes: Re' = -beta k Im, Im' = beta k Re, mode 0 and
  Nyquist zeroed for base mode 0, kept for a rank's block;
* setPForce of a known field is its divergence over dt; project combines
  the u^ and grad P parts with the reference's constants;
* smooth leaves a continuous field unchanged and averages a broken one by
  the Q4 weights;
* the wave step's stiffly-stable and extrapolation weights are exact for
  polynomials in time of their order.
"""
import numpy as np
import pytest

from oracle import dns
from semtex_b200.mesh import rect_mesh


def _sheared(nx, ny, np_):
    """Parallelograms: the unit-square grid under x' = x + 0.3 y, y' = y + 0.2 x."""
    xs, ys = np.linspace(0.0, 1.0, nx + 1), np.linspace(0.0, 1.0, ny + 1)
    VX, VY = np.meshgrid(xs, ys, indexing="xy")
    return rect_mesh(nx, ny, np_, vertex_xy=(VX + 0.3 * VY, VY + 0.2 * VX))


@pytest.mark.parametrize("kind", ["rect", "sheared"])
def test_gradient_exact_for_polynomials_on_affine_elements(kind):
    np_ = 7  # N = 6
    m = rect_mesh(3, 2, np_, 0.0, 2.0, 0.0, 1.0) if kind == "rect" else _sheared(3, 2, np_)
    geo = dns.Geometry(m)
    nul = [np.all(p == 0.0, axis=1) for p in (geo.drdx, geo.drdy, geo.dsdx, geo.dsdy)]
    if kind == "rect":
        assert nul[1].all() and nul[2].all() and not nul[0].any() and not nul[3].any()
    else:
        assert not any(n.any() for n in nul)
    f = m.eval_nodes(lambda x, y: x ** 4 * y ** 2 - 3 * x * y ** 5 + 2 * y ** 6)
    fx = m.eval_nodes(lambda x, y: 4 * x ** 3 * y ** 2 - 3 * y ** 5)
    fy = m.eval_nodes(lambda x, y: 2 * x ** 4 * y - 15 * x * y ** 4 + 12 * y ** 5)
    gx = dns.gradient(geo, f[None], 0)[0]
    gy = dns.gradient(geo, f[None], 1)[0]
    scale = np.abs(fx).max() + np.abs(fy).max()
    assert np.abs(gx - fx).max() < 1e-12 * scale
    assert np.abs(gy - fy).max() < 1e-12 * scale


def test_gradient_converges_on_jittered_quads():
    errs = []
    for np_ in (6, 9, 12):
        m = rect_mesh(4, 4, np_, 0.0, 2.0, 0.0, 1.0, jitter=0.15, seed=5)
        geo = dns.Geometry(m)
        f = m.eval_nodes(lambda x, y: np.sin(2 * x) * np.cos(3 * y))
        fx = m.eval_nodes(lambda x, y: 2 * np.cos(2 * x) * np.cos(3 * y))
        errs.append(np.abs(dns.gradient(geo, f[None], 0)[0] - fx).max())
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-8, errs


@pytest.mark.parametrize("base", [0, 3])
def test_gradient_z(base):
    rng = np.random.default_rng(1)
    w = rng.standard_normal((8, 5))
    g = dns.gradient_z(w, beta=0.5, base_mode=base)
    for z in range(8):
        k = z // 2 + base
        if base == 0 and z < 2:
            assert np.all(g[z] == 0.0)
        elif z % 2 == 0:
            assert np.array_equal(g[z], -(0.5 * k) * w[z + 1])
        else:
            assert np.array_equal(g[z], (0.5 * k) * w[z - 1])


def test_pressure_forcing_is_divergence_over_dt():
    m = rect_mesh(3, 3, 8, 0.0, 1.0, 0.0, 1.0)
    geo = dns.Geometry(m)
    u = m.eval_nodes(lambda x, y: x ** 3 * y)[None]
    v = m.eval_nodes(lambda x, y: y ** 2 - x * y ** 3)[None]
    div = m.eval_nodes(lambda x, y: 3 * x ** 2 * y + 2 * y - 3 * x * y ** 2)
    got = dns.pressure_forcing(geo, [u, v], dt=0.01)[0]
    assert np.abs(got - div / 0.01).max() < 1e-10 * np.abs(div / 0.01).max()
    # three components: the z part of w is added before the 1/dt
    rng = np.random.default_rng(2)
    u3, v3, w3 = (rng.standard_normal((4, m.nplane)) for _ in range(3))
    want = (dns.gradient(geo, u3, 0) + dns.gradient(geo, v3, 1) + dns.gradient_z(w3, 2.0)) * (1.0 / 0.5)
    assert np.array_equal(dns.pressure_forcing(geo, [u3, v3, w3], 0.5, beta=2.0), want)


def test_project_constants():
    m = rect_mesh(2, 2, 5)
    geo = dns.Geometry(m)
    rng = np.random.default_rng(3)
    us = [rng.standard_normal((4, m.nplane)) for _ in range(4)]
    p = rng.standard_normal((4, m.nplane))
    dt, nu, pr = 0.02, 0.05, 0.7
    out = dns.project(geo, us, p, dt, nu, ndim=3, ncom=3, prandtl=pr, beta=1.5)
    alpha, bv = -1.0 / (dt * nu), 1.0 / nu
    assert np.array_equal(out[0], alpha * us[0] + bv * dns.gradient(geo, p, 0))
    assert np.array_equal(out[2], alpha * us[2] + bv * dns.gradient_z(p, 1.5))
    assert np.array_equal(out[3], (alpha * us[3]) * pr)  # the scalar: no pressure term


def test_smooth_continuous_field_unchanged_and_broken_field_averaged():
    m = rect_mesh(3, 2, 6, 0.0, 1.0, 0.0, 1.0, jitter=0.2, seed=4)
    geo = dns.Geometry(m)
    f = m.eval_nodes(lambda x, y: 1.0 + np.sin(3 * x) * y)
    s = dns.smooth(geo, f[None])[0]
    assert np.abs(s - f).max() <= 4 * np.finfo(float).eps * np.abs(f).max()
    # element-wise constants: a shared node gets sum(Q4 c) / sum(Q4)
    c = np.arange(1.0, m.nel + 1.0)
    g = np.repeat(c, m.npnp)
    sg = dns.smooth(geo, g[None])[0].reshape(m.nel, m.npnp)
    em = dns.edge_map(m.np)
    # slot 1 lies inside element 0's bottom side, on the domain boundary: no other holder
    assert sg[0, em[1]] == pytest.approx(1.0, rel=1e-15)
    # the node at element 0's top-right corner is shared by elements 0, 1, 3, 4
    corner = m.btog[0][2 * (m.np - 1)]
    holders = [(e, i) for e in range(m.nel) for i in range(m.next) if m.btog[e][i] == corner]
    assert sorted(e for e, _ in holders) == [0, 1, 3, 4]
    w = {e: geo.Q4[e, em[i]] for e, i in holders}
    want = sum(w[e] * c[e] for e in w) / sum(w.values())
    for e, i in holders:
        assert sg[e, em[i]] == pytest.approx(want, rel=1e-14)
    # interiors untouched
    inner = em[m.next:]
    assert np.array_equal(sg[:, inner], g.reshape(m.nel, m.npnp)[:, inner])


@pytest.mark.parametrize("order", [1, 2, 3])
def test_wave_prop_weights_exact_for_polynomials(order):
    dt, t1 = 0.1, 1.0  # new level t1; stored levels t1 - dt, t1 - 2 dt, ...
    u = lambda t: 0.3 + 1.7 * t - 0.9 * t ** 2 + 0.4 * t ** 3 if order == 3 else (  # noqa: E731
        0.3 + 1.7 * t - 0.9 * t ** 2 if order == 2 else 0.3 + 1.7 * t)
    du = lambda t: 1.7 - 1.8 * t + 1.2 * t ** 2 if order == 3 else (  # noqa: E731
        1.7 - 1.8 * t if order == 2 else 1.7)
    N = lambda t: 2.0 - 0.5 * t + 0.25 * t ** 2 if order == 3 else (  # noqa: E731
        2.0 - 0.5 * t if order == 2 else 2.0)
    levels = [t1 - (q + 1) * dt for q in range(order)]
    us = [[np.array([u(t)])] for t in levels]
    uf = [[np.array([N(t)])] for t in levels]
    h = dns.wave_prop(us, uf, dt)[0][0]
    a0 = dns.STIFFLY_STABLE[order][0]
    # sum_q alpha_q u(t1 - q dt) = dt u'(t1) and sum_q beta_q N(t1-(q+1)dt) = N(t1)
    assert h == pytest.approx(a0 * u(t1) - dt * du(t1) + dt * N(t1), rel=1e-12, abs=1e-13)

"""CPU restatement of the DNS elliptic-phase field operations: the checker
for semtex_b200's sx_field_gradient, sx_dns_pressure_forcing,
sx_dns_project, sx_field_smooth and sx_dns_wave_prop.

TEST INFRASTRUCTURE ONLY: imported by tests/ and the cpu_baseline leg of
bench.py, as the checker.  The product never imports this module.

Fields are arrays (nz, nel*np*np): planes of element-major, np x np
row-major element data, the layout the solve entry points take.  Sums run
over k in ascending order and every elementwise step is rounded where the
reference's veclib call rounds, so a difference from the GPU comes from the
GPU's fused multiply-adds inside the derivative sums only (and from none in
smooth and the wave step).

Parity: no test of the reference pins these routines' outputs, and the
reference cannot be built here (it needs BLAS/LAPACK and a parser).  The
restatement is pinned instead by mathematics, in tests/test_dns_oracle.py:
spectral derivatives of polynomials of degree <= N are exact on affine
elements, the stiffly-stable and extrapolation weights are exact for
polynomials in time of their order, and smoothing leaves a continuous field
unchanged and averages a broken one by the mass weights.
"""
from __future__ import annotations

import numpy as np

from .oracle import gll

EPSDP = 6.0e-14   # femlib/cfemdef.h
EPS = 4 * EPSDP   # the null-mapping threshold, src/element.cpp:1334


def _seq_rows(a, D):
    """a D^T per element with the k-sum in ascending order: out[e,i,j] =
    sum_k a[e,i,k] D[j,k] (Blas::mxm (a, np, DT, np, out, np))."""
    out = np.zeros_like(a)
    for k in range(a.shape[-1]):
        out = out + a[:, :, k, None] * D[None, None, :, k]
    return out


def _seq_cols(a, D):
    """D a per element: out[e,i,j] = sum_k D[i,k] a[e,k,j]."""
    out = np.zeros_like(a)
    for k in range(a.shape[-2]):
        out = out + D[None, :, k, None] * a[:, None, k, :]
    return out


def edge_map(np_):
    """emap: element-boundary slots in counter-clockwise, side-major order
    from the (0,0) corner, then the interior row by row
    (femlib/mapping.c:46-132)."""
    nm = np_ - 1
    e = [i for i in range(nm)]                             # side 0: bottom row
    e += [i * np_ + nm for i in range(nm)]                 # side 1: right column
    e += [nm * np_ + (nm - i) for i in range(nm)]          # side 2: top row, reversed
    e += [(nm - i) * np_ for i in range(nm)]               # side 3: left column, down
    e += [i * np_ + j for i in range(1, nm) for j in range(1, nm)]
    return np.array(e, dtype=np.int64)


class Geometry:
    """Per-element mapping of a QuadMesh: Q4 (mass with weights) and the
    inverse partials with the null-mapping rule (Element::mapping,
    src/element.cpp:1346-1436)."""

    def __init__(self, m):
        self.m = m
        n = m.np
        _, w, D = gll(n)
        self.D = D
        x = np.asarray(m.x, dtype=np.float64).reshape(m.nel, n, n)
        y = np.asarray(m.y, dtype=np.float64).reshape(m.nel, n, n)
        dxdr, dxds = _seq_rows(x, D), _seq_cols(x, D)
        dydr, dyds = _seq_rows(y, D), _seq_cols(y, D)
        jac = dxdr * dyds - dxds * dydr
        ww = w[:, None] * w[None, :]
        self.Q4 = (jac * ww[None]).reshape(m.nel, n * n)
        parts = [dyds / jac, -dxds / jac, -dydr / jac, dxdr / jac]   # drdx, drdy, dsdx, dsdy
        out = []
        for p in parts:
            p = p.reshape(m.nel, n * n)
            nul = np.sqrt(np.sum(p * p, axis=1)) < EPS
            p = p.copy()
            p[nul] = 0.0
            out.append(p)
        self.drdx, self.drdy, self.dsdx, self.dsdy = out
        # inverse assembled boundary mass (src/bcmgr.cpp:805-821)
        em = edge_map(n)[:m.next]
        mass = np.zeros(m.nglobal)
        q4b = self.Q4[:, em]
        for e in range(m.nel):
            np.add.at(mass, m.btog[e], q4b[e])
        self.imass = 1.0 / mass
        self.emap = em


def gradient_xy(geo, planes, dir):
    """AuxField::gradient, dir 0 or 1 (src/auxfield.cpp:583-596, Element::grad
    src/element.cpp:552-596): tgt = (D u) * ds/dx_i + ((u D^T) * dr/dx_i)."""
    m = geo.m
    n = m.np
    u = np.asarray(planes, dtype=np.float64).reshape(-1, m.nel, n, n)
    pr = (geo.drdx if dir == 0 else geo.drdy).reshape(m.nel, n, n)
    ps = (geo.dsdx if dir == 0 else geo.dsdy).reshape(m.nel, n, n)
    out = np.empty_like(u)
    for z in range(u.shape[0]):
        a = _seq_rows(u[z], geo.D) * pr
        b = _seq_cols(u[z], geo.D) * ps
        out[z] = b + a
    return out.reshape(u.shape[0], -1)


def gradient_z(planes, beta, base_mode=0):
    """AuxField::gradient, dir 2 (src/auxfield.cpp:597-610)."""
    w = np.asarray(planes, dtype=np.float64)
    out = w.copy()
    nmodes = w.shape[0] // 2
    klo = 0
    if base_mode == 0:
        out[0:2] = 0.0
        klo = 1
    for k in range(klo, nmodes):
        bk = beta * (k + base_mode)
        out[2 * k] = -bk * w[2 * k + 1]
        out[2 * k + 1] = bk * w[2 * k]
    return out


def gradient(geo, planes, dir, beta=1.0, base_mode=0):
    return gradient_z(planes, beta, base_mode) if dir == 2 else gradient_xy(geo, planes, dir)


def pressure_forcing(geo, us, dt, beta=1.0, base_mode=0):
    """setPForce (dns/integrate.cpp:262-277)."""
    s = gradient(geo, us[0], 0) + gradient(geo, us[1], 1)
    if len(us) == 3:
        s = s + gradient(geo, us[2], 2, beta, base_mode)
    return s * (1.0 / dt)


def project(geo, us, p, dt, kinvis, ndim, ncom=None, prandtl=1.0, beta=1.0, base_mode=0):
    """project (dns/integrate.cpp:280-310)."""
    ncom = len(us) if ncom is None else ncom
    alpha = -1.0 / (dt * kinvis)
    bvisc = 1.0 / kinvis
    out = []
    for i, u in enumerate(us):
        v = alpha * np.asarray(u, dtype=np.float64)
        if i == ncom:
            v = v * prandtl
        if i < ndim:
            v = v + bvisc * gradient(geo, p, i, beta, base_mode)
        out.append(v)
    return out


def smooth(geo, planes):
    """Field::smooth (src/field.cpp:190-231): dssum[btog] += Q4 u over the
    element boundaries, element after element; times imass; written back."""
    m = geo.m
    u = np.array(planes, dtype=np.float64).reshape(-1, m.nel, m.npnp)
    q4b = geo.Q4[:, geo.emap]
    for z in range(u.shape[0]):
        ds = np.zeros(m.nglobal)
        ub = u[z][:, geo.emap]
        for e in range(m.nel):
            np.add.at(ds, m.btog[e], q4b[e] * ub[e])
        ds = ds * geo.imass
        for e in range(m.nel):
            u[z, e, geo.emap] = ds[m.btog[e]]
    return u.reshape(u.shape[0], -1)


# Stiffly-stable (backward differentiation) weights of order 1-3, the new
# level first, and the extrapolation weights (Gear 1971, Table 11.1;
# src/integration.cpp:98-163).
STIFFLY_STABLE = {1: (1.0, -1.0), 2: (1.5, -2.0, 0.5), 3: (11.0 / 6.0, -3.0, 1.5, -1.0 / 3.0)}
EXTRAPOLATION = {1: (1.0,), 2: (2.0, -1.0), 3: (3.0, -3.0, 1.0)}


def wave_prop(us, uf, dt):
    """waveProp (dns/integrate.cpp:227-259): us[q][i], uf[q][i] = level q of
    field i; returns h[i]."""
    order = len(us)
    a = STIFFLY_STABLE[order]
    b = [c * dt for c in EXTRAPOLATION[order]]
    out = []
    for i in range(len(us[0])):
        h = np.zeros_like(np.asarray(us[0][i], dtype=np.float64))
        for q in range(order):
            h = h + (-a[q + 1]) * us[q][i]
            h = h + b[q] * uf[q][i]
        out.append(h)
    return out

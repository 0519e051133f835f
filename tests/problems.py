"""The reference's elliptic regression problems, restated as test inputs.

Each entry restates one session file of the reference (mesh/<name>: 2 x 2
quads on the unit square or [-1,1]^2, its TOKENS, USER forcing/exact
strings and BCS) and the golden line ``compare -n`` prints for it
(regress/<name>.ok): the infinity-norm error of the DIRECT solve against the
analytic solution, "noise-level" meaning < 1e-12 (utility/compare.cpp:85,
229-235), otherwise 3 significant digits.
"""
import numpy as np

from semtex_b200.mesh import rect_mesh

PI = np.pi
NOISE = 1e-12

# name: (np, lambda2, forcing(x,y), exact(x,y), bc spec, bc values, periodic, golden)
PROBLEMS_2D = {
    # mesh/helmholtz1, regress/helmholtz1.ok
    "helmholtz1": dict(
        np=11, lambda2=16.0,
        forcing=lambda x, y: np.sin(PI * x) * np.sin(PI * y),
        exact=lambda x, y: -np.sin(PI * x) * np.sin(PI * y) / (2 * PI * PI + 16.0),
        bc=None, bcval={}, periodic=False, golden=None),
    # mesh/poisson1, regress/poisson1.ok
    "poisson1": dict(
        np=11, lambda2=0.0,
        forcing=lambda x, y: np.sin(PI * x) * np.sin(PI * y),
        exact=lambda x, y: -1.0 / (2 * PI * PI) * np.sin(PI * x) * np.sin(PI * y),
        bc=None, bcval={}, periodic=False, golden=None),
    # mesh/laplace1, regress/laplace1.ok
    "laplace1": dict(
        np=11, lambda2=0.0,
        forcing=lambda x, y: 0.0 * x,
        exact=lambda x, y: np.sin(2 * PI * x) * np.sinh(2 * PI * y) / np.sinh(2 * PI),
        bc=None, bcval={"top": lambda x, y: np.sin(2 * PI * x)}, periodic=False,
        golden=1.052e-10),
    # mesh/laplace4, regress/laplace4.ok (natural BC du/dn = sin(pi x) on top)
    "laplace4": dict(
        np=12, lambda2=0.0,
        forcing=lambda x, y: 0.0 * x,
        exact=lambda x, y: np.sin(PI * x) * np.sinh(PI * y) / (PI * np.cosh(PI)),
        bc={"top": "N"}, bcval={"top": lambda x, y: np.sin(PI * x)}, periodic=False,
        golden=None),
    # mesh/mixed1, regress/mixed1.ok (Robin K=3, C=7 on top, periodic sides)
    "mixed1": dict(
        np=11, lambda2=0.0,
        forcing=lambda x, y: -20.0 + 0.0 * x,
        exact=lambda x, y: 4 + 14.75 * y - 10 * y * y,
        bc={"top": ("M", 3.0, 7.0), "bottom": "D"},
        bcval={"bottom": lambda x, y: 4.0 + 0.0 * x}, periodic=True, golden=None),
}


def _sin_exp(x, y):
    return np.sin(x) * np.exp(-y)


# Two more of the reference's 2 x 2, N_P = 11 Laplace problems on the unit
# square, exact solution sin(x) exp(-y), goldens "noise-level"; pinned on the
# oracle (CPU tests) in addition to the five above.
PROBLEMS_2D_MORE = {
    # mesh/laplace5, regress/laplace5.ok: the exact solution as essential BC
    # on every side
    "laplace5": dict(
        np=11, lambda2=0.0,
        forcing=lambda x, y: 0.0 * x,
        exact=_sin_exp,
        bc=None, bcval={s: _sin_exp for s in ("bottom", "right", "top", "left")}, periodic=False,
        golden=None),
    # mesh/laplace7, regress/laplace7.ok: essential on top, natural (the
    # outward normal derivative) on the other three sides
    "laplace7": dict(
        np=11, lambda2=0.0,
        forcing=lambda x, y: 0.0 * x,
        exact=_sin_exp,
        bc={"bottom": "N", "right": "N", "left": "N"},
        bcval={"top": _sin_exp, "bottom": _sin_exp,
               "right": lambda x, y: np.cos(x) * np.exp(-y),
               "left": lambda x, y: -np.cos(x) * np.exp(-y)},
        periodic=False, golden=None),
}


def build_2d(name):
    p = PROBLEMS_2D[name] if name in PROBLEMS_2D else PROBLEMS_2D_MORE[name]
    m = rect_mesh(2, 2, p["np"], bc=p["bc"], periodic_x=p["periodic"])
    f = m.eval_nodes(p["forcing"])[None]
    bc = m.bc_line(p["bcval"])[None]
    exact = m.eval_nodes(p["exact"])
    return m, p, f, bc, exact


def golden_ok(err, golden):
    """True when err prints as the golden line would (3 significant digits)."""
    if golden is None:
        return err < NOISE
    return float(f"{err:.3e}") == golden


# mesh/laplace3, regress/laplace3.ok: 3-D, N_Z = 8, BETA = 1, [-1,1]^2,
# c = exp(sqrt(2) x) sin(y) sin(z) as essential BC and exact solution.
LAPLACE3 = dict(np=10, nz=8, beta=1.0)


def laplace3_fn(x, y, z):
    return np.exp(np.sqrt(2.0) * x) * np.sin(y) * np.sin(z)


def to_fourier(phys):
    """Physical planes (nz, ...) -> semtex Fourier plane order with 1/nz
    scaling: plane 0 mode 0, plane 1 Nyquist, 2k/2k+1 Re/Im of mode k
    (femlib/fourier.c:47-70)."""
    nz = phys.shape[0]
    F = np.fft.rfft(phys, axis=0) / nz
    out = np.zeros_like(phys)
    out[0] = F[0].real
    out[1] = F[nz // 2].real
    for k in range(1, nz // 2):
        out[2 * k] = F[k].real
        out[2 * k + 1] = F[k].imag
    return out


def to_physical(four):
    nz = four.shape[0]
    F = np.zeros((nz // 2 + 1,) + four.shape[1:], dtype=complex)
    F[0] = four[0]
    F[nz // 2] = four[1]
    for k in range(1, nz // 2):
        F[k] = four[2 * k] + 1j * four[2 * k + 1]
    return np.fft.irfft(F * nz, n=nz, axis=0)


def build_laplace3():
    p = LAPLACE3
    m = rect_mesh(2, 2, p["np"], -1.0, 1.0, -1.0, 1.0)
    nz = p["nz"]
    zs = np.arange(nz) * 2 * np.pi / p["beta"] / nz
    bcp = np.stack([m.bc_line({0: (lambda x, y, z=z: laplace3_fn(x, y, z))}) for z in zs])
    exact = np.stack([m.eval_nodes(lambda x, y, z=z: laplace3_fn(x, y, z)) for z in zs])
    return m, to_fourier(bcp), exact

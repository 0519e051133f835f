"""Seeded synthetic Helmholtz workloads.

The reference publishes no benchmark data set.  These builders are
seeded stand-ins with the shapes of the five benchmark configurations (mesh,
order, planes, per-mode Helmholtz constants, forcing law); each returns a
``Workload`` with the mesh, the per-mode (lambda2, betak2) and the forcing
planes in semtex's Fourier plane order (plane 0 mode 0, plane 1 Nyquist,
planes 2k / 2k+1 Re / Im of mode k).

Equation convention: semtex solves  div grad u - lambda^2 u = f
(src/field.h:15-21), so manufactured forcings carry that sign.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import QuadMesh, edge_maps, rect_mesh


@dataclass
class Workload:
    name: str
    mesh: QuadMesh
    nz: int
    beta: float
    lambda2: np.ndarray          # per local mode
    betak2: np.ndarray           # per local mode
    forcing: np.ndarray          # (nz, nplane)
    exact: np.ndarray | None = None
    seed: int = 0
    info: dict = field(default_factory=dict)
    base_mode: int = 0           # first local mode (a rank's block of modes)

    @property
    def num_modes(self):
        return len(self.lambda2)

    @property
    def planes_solved(self):
        """Planes the solve touches: plane 1 (Nyquist) is skipped when the
        block starts at mode 0."""
        if self.nz == 1:
            return 1
        return self.nz - 1 if self.base_mode == 0 else self.nz

    @property
    def solved_planes(self):
        """Indices of the solved planes."""
        if self.nz == 1:
            return [0]
        return ([0] + list(range(2, self.nz))) if self.base_mode == 0 else list(range(self.nz))

    @property
    def dof_per_plane(self):
        return self.mesh.n_unique

    @property
    def dof_solves(self):
        return self.dof_per_plane * self.planes_solved


def scatter_global(m: QuadMesh, gvals: np.ndarray) -> np.ndarray:
    """Continuous field from values per unique node: gvals has
    nglobal + nel*nint entries (element-boundary globals first, then each
    element's interior nodes in edge-map order); returns the element plane.
    A leading axis of gvals (planes) is kept: (..., n) -> (..., nplane)."""
    emap, _ = edge_maps(m.np)
    # source of every element-plane value: a boundary slot's global node, or
    # the element's own interior node
    src = np.empty((m.nel, m.npnp), dtype=np.int64)
    src[:, emap[: m.next]] = m.btog
    src[:, emap[m.next:]] = m.nglobal + np.arange(m.nel * m.nint, dtype=np.int64).reshape(m.nel, m.nint)
    g = np.asarray(gvals)
    return np.take(g, src.reshape(-1), axis=-1)


def _jittered_channel(nx, ny, np_, jitter, seed, lx=2 * np.pi):
    return rect_mesh(nx, ny, np_, 0.0, lx, 0.0, 1.0, jitter=jitter, seed=seed, periodic_x=True,
                     bc={"bottom": "D", "top": "D"})


def config1():
    """Unit square, 4x4 straight quads, N=8, lambda2=1, u = sin(pi x) sin(pi y)."""
    m = rect_mesh(4, 4, 9)
    f = -(2 * np.pi ** 2 + 1.0) * m.eval_nodes(lambda x, y: np.sin(np.pi * x) * np.sin(np.pi * y))
    exact = m.eval_nodes(lambda x, y: np.sin(np.pi * x) * np.sin(np.pi * y))
    return Workload("cfg1_unit_square_4x4_N8", m, 1, 0.0, np.array([1.0]), np.array([0.0]),
                    f[None], exact[None], seed=1)


def fourier_forcing(m: QuadMesh, nz: int, rng, decay=8.0):
    """Gaussian random Fourier coefficients N(0,1) e^{-k/decay} per unique
    node, Re and Im planes independent, scattered continuously."""
    n = m.n_unique
    f = np.zeros((nz, m.nplane))
    planes = [p for p in range(nz) if not (p == 1 and nz > 1)]   # the Nyquist plane stays zero
    # one draw for every plane is the same stream as one draw per plane in turn
    g = rng.standard_normal((len(planes), n))
    g *= np.exp(-(np.array(planes) >> 1) / decay)[:, None]
    f[planes] = scatter_global(m, g)
    return f


def config2(nx=32, ny=32, np_=9, nz=64, seed=2):
    """[0,2pi]x[0,1], 32x32 quads jittered +-15%, N=8, nz=64 (modes 0..31),
    beta=1, lambda2 = 1/(nu dt) = 1e6 with nu = dt = 1e-3, betak2 = k^2."""
    m = _jittered_channel(nx, ny, np_, 0.15, seed)
    rng = np.random.default_rng(seed)
    nm = max(nz // 2, 1)
    lam = np.full(nm, 1.0 / (1e-3 * 1e-3))
    bk2 = np.arange(nm, dtype=np.float64) ** 2
    f = fourier_forcing(m, nz, rng)
    return Workload(f"cfg2_channel_{nx}x{ny}_N{np_ - 1}_nz{nz}", m, nz, 1.0, lam, bk2, f, seed=seed,
                    info={"jitter": 0.15, "nu": 1e-3, "dt": 1e-3})


def config3(nx=64, ny=64, np_=11, nz=128, seed=3):
    """64x64 quads jittered +-20%, N=10, nz=128 (65 modes incl. Nyquist),
    lambda2_k log-uniform in [1e-2, 1e4] (total Helmholtz constant per mode),
    manufactured u = sum_k a_k sin(pi y) cos(k z) cos(3x), a_k ~ N(0,1) k^-2
    (a_0 uses k=1 scaling).  Only cos(kz): Im planes zero."""
    m = _jittered_channel(nx, ny, np_, 0.20, seed)
    rng = np.random.default_rng(seed)
    nm = nz // 2
    lam = np.exp(rng.uniform(np.log(1e-2), np.log(1e4), size=nm))
    bk2 = np.zeros(nm)
    a = rng.standard_normal(nm) * np.maximum(np.arange(nm), 1.0) ** -2.0
    shape = m.eval_nodes(lambda x, y: np.sin(np.pi * y) * np.cos(3 * x))
    f = np.zeros((nz, m.nplane))
    exact = np.zeros((nz, m.nplane))
    for k in range(nm):
        # semtex sign: div grad u - lam u = f, with -(pi^2 + 9) from the x,y parts
        plane = 2 * k
        exact[plane] = a[k] * shape
        f[plane] = -(np.pi ** 2 + 9.0 + lam[k]) * a[k] * shape
    return Workload(f"cfg3_channel_{nx}x{ny}_N{np_ - 1}_nz{nz}", m, nz, 1.0, lam, bk2, f, exact,
                    seed=seed, info={"jitter": 0.20})


def config3_block(world=1, rank=0, nx=64, ny=64, np_=11, modes_per_rank=64, seed=3):
    """Rank `rank`'s block of a config-3 problem with modes_per_rank * world
    Fourier modes (nz = 2 modes_per_rank world planes), split as the
    reference splits modes across processes (contiguous blocks,
    src/geometry.cpp:72-101; partition.mode_block): the per-GPU work stays
    that of config 3 as ranks are added (weak scaling).  The per-mode lambda2
    and a_k of all modes come from one seeded stream, so world = 1 is
    config3() exactly.  Only the block's planes are built: planes 2l, 2l+1 of
    local mode l, with the Nyquist datum at plane 1 when the block starts at
    mode 0."""
    from .partition import mode_block
    nm = modes_per_rank * world
    base, count = mode_block(nm, world, rank)
    m = _jittered_channel(nx, ny, np_, 0.20, seed)
    rng = np.random.default_rng(seed)
    lam = np.exp(rng.uniform(np.log(1e-2), np.log(1e4), size=nm))
    a = rng.standard_normal(nm) * np.maximum(np.arange(nm), 1.0) ** -2.0
    shape = m.eval_nodes(lambda x, y: np.sin(np.pi * y) * np.cos(3 * x))
    nzl = 2 * count
    f = np.zeros((nzl, m.nplane))
    exact = np.zeros((nzl, m.nplane))
    for l in range(count):
        k = base + l
        exact[2 * l] = a[k] * shape
        f[2 * l] = -(np.pi ** 2 + 9.0 + lam[k]) * a[k] * shape
    return Workload(f"cfg3_channel_{nx}x{ny}_N{np_ - 1}_nz{2 * nm}", m, nzl, 1.0, lam[base:base + count].copy(),
                    np.zeros(count), f, exact, seed=seed,
                    info={"jitter": 0.20, "modes_total": nm, "rank": rank, "world": world}, base_mode=base)


def config5(nx=128, ny=64, np_=11, nz=256, seed=5, nu=5e-4, dt=5e-4):
    """The elliptic phase of one DNS timestep on a jittered periodic channel
    (+-15 %, [0,2pi] x [0,1]): three viscous Helmholtz solves (velocity,
    Dirichlet walls) with lambda2 = 1/(nu dt), betak2 = k^2, and the pressure
    Poisson solve (natural walls) with lambda2 = 0, betak2 = k^2, whose k = 0
    mode is singular and pinned like the reference's.  Forcing: seeded random
    smooth velocity-like fields with spectral energy ~ k^-5/3 up to k = 32 (the
    viscous forcing -u/(nu dt), the pressure forcing of the same law scaled by
    1/dt).  Returns [u, v, w, p] workloads; u, v, w share one mesh."""
    mv = _jittered_channel(nx, ny, np_, 0.15, seed)
    mp = rect_mesh(nx, ny, np_, 0.0, 2 * np.pi, 0.0, 1.0, jitter=0.15, seed=seed, periodic_x=True,
                   bc={"bottom": "N", "top": "N"})
    rng = np.random.default_rng(seed)
    nm = max(nz // 2, 1)
    k = np.arange(nm, dtype=np.float64)
    amp = np.where(k < 32, np.maximum(k, 1.0) ** (-5.0 / 6.0), 0.0)  # energy ~ k^-5/3

    def field(m):
        f = np.zeros((nz, m.nplane))
        for plane in range(nz):
            if plane == 1 and nz > 1:
                continue
            f[plane] = scatter_global(m, rng.standard_normal(m.n_unique) * amp[plane >> 1])
        return f

    out = []
    for name in ("u", "v", "w"):
        lam = np.full(nm, 1.0 / (nu * dt))
        out.append(Workload(f"cfg5_{name}_{nx}x{ny}_N{np_ - 1}_nz{nz}", mv, nz, 1.0, lam, k ** 2,
                            -field(mv) / (nu * dt), seed=seed, info={"solve": "viscous"}))
    out.append(Workload(f"cfg5_p_{nx}x{ny}_N{np_ - 1}_nz{nz}", mp, nz, 1.0, np.zeros(nm), k ** 2,
                        field(mp) / dt, seed=seed, info={"solve": "pressure"}))
    return out


@dataclass
class DnsBlock:
    """One rank's share of a DNS elliptic step: its block of Fourier modes
    of the velocity (Dirichlet walls) and pressure (natural walls) meshes of
    one geometry, with the viscous and pressure Helmholtz constants of the
    block's modes."""
    name: str
    mesh_v: QuadMesh
    mesh_p: QuadMesh
    base_mode: int
    num_modes: int
    beta: float
    nu: float
    dt: float
    lambda2_v: np.ndarray        # per local mode: 1/(nu dt)
    lambda2_p: np.ndarray        # per local mode: 0
    betak2: np.ndarray           # per local mode: (beta k)^2
    info: dict = field(default_factory=dict)

    @property
    def nz(self):
        return 2 * self.num_modes

    @property
    def planes_solved(self):
        return self.nz - 1 if self.base_mode == 0 else self.nz


def config5_block(world=8, rank=0, nx=128, ny=64, np_=11, modes_per_rank=16, seed=5, nu=5e-4, dt=5e-4):
    """Rank `rank`'s block of config 5 (128 x 64 quads jittered +-15 %,
    N = 10, [0, 2pi] x [0, 1], periodic in x) split over `world` ranks as
    the reference splits modes (partition.mode_block): with the default
    8 x 16 modes, nz = 256 planes in all.  All 128 pressure factors (about
    5.9 GB each) exceed one GPU; a block of 16 holds about 94 GB."""
    from .partition import mode_block
    nm = modes_per_rank * world
    base, count = mode_block(nm, world, rank)
    mv = _jittered_channel(nx, ny, np_, 0.15, seed)
    mp = rect_mesh(nx, ny, np_, 0.0, 2 * np.pi, 0.0, 1.0, jitter=0.15, seed=seed, periodic_x=True,
                   bc={"bottom": "N", "top": "N"})
    k = np.arange(base, base + count, dtype=np.float64)
    return DnsBlock(f"cfg5_channel_{nx}x{ny}_N{np_ - 1}_nz{2 * nm}", mv, mp, base, count, 1.0, nu, dt,
                    np.full(count, 1.0 / (nu * dt)), np.zeros(count), k ** 2,
                    info={"modes_total": nm, "rank": rank, "world": world, "jitter": 0.15})


@dataclass
class ServeRequest:
    t_arrival: float             # seconds after the first arrival
    mesh: QuadMesh
    lambda2: np.ndarray          # per mode
    betak2: np.ndarray           # per mode, k^2
    forcing: np.ndarray          # (nz, nplane)

    @property
    def nz(self):
        return self.forcing.shape[0]

    @property
    def dof_solves(self):
        """Unique nodes per plane x planes solved (Nyquist excluded)."""
        return self.mesh.n_unique * (1 if self.nz == 1 else self.nz - 1)


@dataclass
class ServeSpec:
    """One request of the serving stream before its mesh and forcing are built."""
    index: int
    t_arrival: float
    ex: int
    ey: int
    order: int
    modes: int
    lam: float


def serving_plan(n_requests, seed=4, rate=2000.0):
    """The mixed-size request stream (config 4): Poisson arrivals at
    `rate`/s; each request a straight-sided E_x x E_y quad mesh of [0,1]^2
    with E_x, E_y uniform in [2, 64], order N uniform in {4..10}, a mode count
    uniform in [1, 64], lambda2 log-uniform in [1e-2, 1e4] (plus k^2 per
    mode, beta = 1), Dirichlet on every side.  The sizes, constants and
    arrival times of the first `n_requests` come from one seeded stream."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        ex, ey = (int(v) for v in rng.integers(2, 65, size=2))
        order = int(rng.integers(4, 11))
        modes = int(rng.integers(1, 65))
        lam = float(np.exp(rng.uniform(np.log(1e-2), np.log(1e4))))
        out.append(ServeSpec(i, t, ex, ey, order, modes, lam))
        t += float(rng.exponential(1.0 / rate))
    return out


def serving_request(spec: ServeSpec, seed=4) -> ServeRequest:
    """Build one planned request: its mesh and seeded Gaussian Fourier
    forcing (fourier_forcing, from the request's own stream (seed, index), so
    that requests can be built in any order or in parallel)."""
    m = rect_mesh(spec.ex, spec.ey, spec.order + 1, 0.0, 1.0, 0.0, 1.0)
    nz = 1 if spec.modes == 1 else 2 * spec.modes
    f = fourier_forcing(m, nz, np.random.default_rng([seed, spec.index]))
    return ServeRequest(spec.t_arrival, m, np.full(spec.modes, spec.lam),
                        np.arange(spec.modes, dtype=np.float64) ** 2, f)


def serving_trace(n_requests, seed=4, rate=2000.0):
    """The first `n_requests` of the serving stream, built (serving_plan,
    serving_request)."""
    return [serving_request(s, seed) for s in serving_plan(n_requests, seed, rate)]


def small_mesh_mix(n_meshes=24, seed=9):
    """Many small meshes of uneven size and order, the case a multi-mesh
    batch is for: straight-sided E_x x E_y quads of [0,1]^2 with E_x, E_y
    uniform in [2, 12], order N uniform in {4..10}, a mode count uniform in
    [1, 12], lambda2 log-uniform in [1e3, 1e5] (plus k^2 per mode), seeded
    Gaussian Fourier forcing, Dirichlet on every side."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_meshes):
        ex, ey = (int(v) for v in rng.integers(2, 13, size=2))
        order = int(rng.integers(4, 11))
        modes = int(rng.integers(1, 13))
        lam = float(np.exp(rng.uniform(np.log(1e3), np.log(1e5))))
        m = rect_mesh(ex, ey, order + 1, 0.0, 1.0, 0.0, 1.0)
        nz = 1 if modes == 1 else 2 * modes
        out.append(ServeRequest(0.0, m, np.full(modes, lam), np.arange(modes, dtype=np.float64) ** 2,
                                fourier_forcing(m, nz, rng)))
    return out


def small_channel(nx=8, ny=6, np_=9, nz=16, lam=1e6, seed=7, jitter=0.15):
    """Small config-2-shaped case for parity tests."""
    m = _jittered_channel(nx, ny, np_, jitter, seed)
    rng = np.random.default_rng(seed)
    nm = max(nz // 2, 1)
    lamv = np.full(nm, float(lam))
    bk2 = np.arange(nm, dtype=np.float64) ** 2
    return Workload(f"channel_{nx}x{ny}_N{np_ - 1}_nz{nz}", m, nz, 1.0, lamv, bk2,
                    fourier_forcing(m, nz, rng), seed=seed)

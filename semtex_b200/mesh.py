"""Quad meshes and semtex-style global numbering for the Helmholtz solve.

This module builds, on the host, the inputs that semtex's setup layers hand to
the elliptic solve:

* element node coordinates, straight sides at GLL spacing and a Coons patch
  inside (``Mesh::meshElmt``, src/mesh.cpp:772-886);
* the element-boundary-to-global map ``btog`` in edge-major CCW order
  (``Mesh::buildMap``/``Side::connect``, src/mesh.cpp:889-1017;
  femlib/mapping.c:46-132), with essential-BC nodes numbered last
  (``Nsys::sortGid``, utility/enumerate.cpp:621-677) and the solve nodes
  renumbered by reverse Cuthill-McKee to cut the band
  (``Nsys::renumber``, utility/enumerate.cpp:680-809);
* ``bmask``/``emask`` (src/bcmgr.cpp:786-803), ``nglobal``, ``nsolve`` and
  the band width including the diagonal (``Nsys::globalBandwidth``,
  utility/enumerate.cpp:903-943);
* the ordered list of boundary edges with their condition kind (essential,
  natural, mixed), as ``BoundarySys`` holds them.

It is pure numpy/scipy: numbering is set-up work done once per mesh.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

ESSENTIAL, NATURAL, MIXED = 0, 1, 2
_KIND = {"D": ESSENTIAL, "N": NATURAL, "M": MIXED,
         "essential": ESSENTIAL, "natural": NATURAL, "mixed": MIXED}


def gll_points(np_: int) -> np.ndarray:
    """GLL points on [-1, 1] (roots of (1-z^2) P'_N), Newton in long double.

    Same points as femlib/polylib.c:312-352 (``zwglj`` with alpha=beta=0).
    """
    n = np_ - 1
    z = np.zeros(np_, dtype=np.longdouble)
    z[0], z[n] = -1, 1
    for i in range(1, n):
        x = -np.cos(np.longdouble(np.pi) * i / n)
        for _ in range(100):
            p0, p1, d0, d1 = np.longdouble(1), x, np.longdouble(0), np.longdouble(1)
            for k in range(2, n + 1):
                p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
                d2 = d0 + (2 * k - 1) * p1
                p0, p1, d0, d1 = p1, p2, d1, d2
            dd = (2 * x * d1 - n * (n + 1) * p1) / (1 - x * x)
            dx = d1 / dd
            x = x - dx
            if abs(dx) < 1e-30:
                break
        z[i] = x
    for i in range(np_ // 2):
        a = (z[n - i] - z[i]) / 2
        z[i], z[n - i] = -a, a
    if np_ % 2:
        z[n // 2] = 0
    return z.astype(np.float64)


def edge_maps(np_: int):
    """emap / pmap of femlib/mapping.c:46-132 (CCW exterior, then interior)."""
    em = [0]
    n = 0
    for step in (1, np_, -1, -np_):
        for _ in range(1, np_):
            n += step
            em.append(n)
    em = em[:-1]
    for i in range(1, np_ - 1):
        for j in range(1, np_ - 1):
            em.append(i * np_ + j)
    emap = np.array(em, dtype=np.int32)
    pmap = np.empty_like(emap)
    pmap[emap] = np.arange(np_ * np_, dtype=np.int32)
    return emap, pmap


def element_nodes(np_: int, z: np.ndarray, vx, vy):
    """Node coordinates (np x np, row-major) of a straight-sided quad.

    Side points at GLL spacing, interior by the Coons patch exactly as in
    src/mesh.cpp:772-886 (sides 2 and 3 use the reversed, negated spacing).
    """
    nm = np_ - 1
    x = np.zeros((np_, np_))
    y = np.zeros((np_, np_))
    for s in range(4):
        x1, y1 = vx[s], vy[s]
        x2, y2 = vx[(s + 1) % 4], vy[(s + 1) % 4]
        sp = z if s < 2 else -z[::-1]
        px = x1 + (x2 - x1) * 0.5 * (sp + 1.0)
        py = y1 + (y2 - y1) * 0.5 * (sp + 1.0)
        # side s's first nm points, CCW from its start vertex
        if s == 0:
            idx = (0, slice(0, nm))
        elif s == 1:
            idx = (slice(0, nm), nm)
        elif s == 2:
            idx = (nm, slice(nm, 0, -1))
        else:
            idx = (slice(nm, 0, -1), 0)
        x[idx], y[idx] = px[:nm], py[:nm]
    # Coons interior, node by node the same arithmetic as a scalar loop
    zr = z[None, 1:nm]  # along j
    zs = z[1:nm, None]  # along i
    for a in (x, y):
        a[1:nm, 1:nm] = (0.50 * ((1.0 - zr) * a[1:nm, 0:1] + (1.0 + zr) * a[1:nm, nm:nm + 1]
                                 + (1.0 - zs) * a[0:1, 1:nm] + (1.0 + zs) * a[nm:nm + 1, 1:nm])
                         - 0.25 * ((1.0 - zr) * (1.0 - zs) * a[0, 0]
                                   + (1.0 - zr) * (1.0 + zs) * a[nm, 0]
                                   + (1.0 - zs) * (1.0 + zr) * a[0, nm]
                                   + (1.0 + zs) * (1.0 + zr) * a[nm, nm]))
    return x, y


def side_node_index(np_: int, side: int):
    """Row-major node indices along an element side, CCW from its start vertex."""
    nm = np_ - 1
    if side == 0:
        return [0 * np_ + i for i in range(np_)]
    if side == 1:
        return [i * np_ + nm for i in range(np_)]
    if side == 2:
        return [nm * np_ + (nm - i) for i in range(np_)]
    return [(nm - i) * np_ for i in range(np_)]


@dataclass
class Boundary:
    """One element side on the domain boundary (a semtex ``Boundary``)."""
    elmt: int
    side: int
    kind: int
    K: float = 0.0     # mixed: dc/dn + K (c - C) = 0
    C: float = 0.0
    group: str = ""


@dataclass
class QuadMesh:
    """Element geometry + numbering system + boundary list for one mesh."""
    np: int
    nel: int
    x: np.ndarray            # (nel, np, np)
    y: np.ndarray
    btog: np.ndarray         # (nel, next) int32
    bmask: np.ndarray        # (nel, next) int32
    nglobal: int
    nsolve: int
    nband: int
    boundaries: list = field(default_factory=list)
    vx: np.ndarray | None = None   # (nel, 4)
    vy: np.ndarray | None = None

    @property
    def next(self):
        return 4 * (self.np - 1)

    @property
    def nint(self):
        return (self.np - 2) ** 2

    @property
    def npnp(self):
        return self.np * self.np

    @property
    def nplane(self):
        """Element data points per plane (Geometry::nPlane)."""
        return self.nel * self.npnp

    @property
    def n_unique(self):
        """Unique nodes per plane: element-boundary globals + interiors."""
        return self.nglobal + self.nel * self.nint

    def bc_arrays(self):
        nb = len(self.boundaries)
        be = np.array([b.elmt for b in self.boundaries] or [0], dtype=np.int32)[:max(nb, 1)]
        bs = np.array([b.side for b in self.boundaries] or [0], dtype=np.int32)[:max(nb, 1)]
        bk = np.array([b.kind for b in self.boundaries] or [0], dtype=np.int32)[:max(nb, 1)]
        bK = np.array([b.K for b in self.boundaries] or [0.0], dtype=np.float64)[:max(nb, 1)]
        bC = np.array([b.C for b in self.boundaries] or [0.0], dtype=np.float64)[:max(nb, 1)]
        return nb, be, bs, bk, bK, bC

    def side_xy(self, b: Boundary):
        idx = side_node_index(self.np, b.side)
        return self.x[b.elmt].ravel()[idx], self.y[b.elmt].ravel()[idx]

    def bc_line(self, funcs):
        """Boundary-line values (nbound, np) for one plane.

        ``funcs`` maps a condition kind (or a group name) to ``f(x, y)``;
        missing entries give zero.  Values are at the side nodes in CCW order
        (``Element::sideEval``).
        """
        out = np.zeros((max(len(self.boundaries), 1), self.np))
        for k, b in enumerate(self.boundaries):
            f = funcs.get(b.group, funcs.get(b.kind))
            if f is not None:
                xs, ys = self.side_xy(b)
                out[k] = np.broadcast_to(f(xs, ys), (self.np,))
        return out

    def eval_nodes(self, f):
        """Evaluate f(x, y) at every element node: plane layout (nel*np*np)."""
        return np.asarray(f(self.x, self.y), dtype=np.float64).reshape(-1).copy()

    def global_to_element(self):
        """CSR inverse of btog: for each global node, the (element, local)
        contributions in element-major order (the summation order of
        ``Veclib::scatr_sum`` over elements)."""
        flat = self.btog.reshape(-1)
        order = np.argsort(flat, kind="stable")
        counts = np.bincount(flat, minlength=self.nglobal)
        ptr = np.zeros(self.nglobal + 1, dtype=np.int32)
        np.cumsum(counts, out=ptr[1:])
        return ptr, order.astype(np.int32)


def _rcm_order(adj_rows, adj_cols, n):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    if n == 0:
        return np.zeros(0, dtype=np.int64)
    A = sp.csr_matrix((np.ones(len(adj_rows)), (adj_rows, adj_cols)), shape=(n, n))
    return np.asarray(reverse_cuthill_mckee(A, symmetric_mode=True))


def number_mesh(np_, elem_vids, canon, essential_sides, renumber="rcm"):
    """Global numbering for a conforming quad mesh.

    elem_vids        (nel, 4) vertex ids, CCW
    canon            vertex id -> canonical id (periodic identification)
    essential_sides  set of (elmt, side) carrying an essential BC
    renumber         "rcm" (reverse Cuthill-McKee over solve nodes),
                     "none" (naive element-traverse order)

    Returns btog, bmask (nel, next), nglobal, nsolve, nband.

    Each element boundary slot gets a code: a vertex its canonical id, the
    t-th interior node of an edge (t counted from the edge's lower vertex)
    nv + edge id (nm - 1) + t - 1.  Global ids are given in order of first
    appearance over elements and their slots (Side::connect's traverse
    order), essential nodes are moved last (sortGid), then the solve nodes
    are renumbered by RCM over the element coupling graph.
    """
    nel = elem_vids.shape[0]
    nm = np_ - 1
    next_ = 4 * nm
    canon = np.asarray(canon, dtype=np.int64)
    nv = int(canon.max()) + 1 if canon.size else 0
    P = canon[np.asarray(elem_vids, dtype=np.int64)]   # side start vertex, (nel, 4)
    Q = np.roll(P, -1, axis=1)                          # side end vertex
    lo, hi = np.minimum(P, Q), np.maximum(P, Q)
    _, eid = np.unique(lo * max(nv, 1) + hi, return_inverse=True)
    eid = eid.reshape(nel, 4)
    codes = np.empty((nel, 4, nm), dtype=np.int64)
    codes[:, :, 0] = P
    if nm > 1:
        t = np.arange(1, nm, dtype=np.int64)[None, None, :]
        tt = np.where((P < Q)[:, :, None], t, nm - t)
        codes[:, :, 1:] = nv + eid[:, :, None] * (nm - 1) + (tt - 1)
    # naive numbering in element/side traverse order (Side::connect)
    uc, first, inv = np.unique(codes.reshape(-1), return_index=True, return_inverse=True)
    rank = np.empty(len(uc), dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uc))
    btog = rank[inv].reshape(nel, next_)
    nglobal = len(uc)
    ess = np.zeros(nglobal, dtype=bool)
    if essential_sides:
        es = np.array(sorted(essential_sides), dtype=np.int64).reshape(-1, 2)
        ks = (es[:, 1:2] * nm + np.arange(np_)[None, :]) % next_
        ess[btog[es[:, 0:1], ks]] = True
    # sortGid: unknowns first, each partition in ascending naive order
    unknown = np.flatnonzero(~ess)
    known = np.flatnonzero(ess)
    nsolve = len(unknown)
    new = np.empty(nglobal, dtype=np.int64)
    new[unknown] = np.arange(nsolve)
    new[known] = nsolve + np.arange(len(known))
    btog = new[btog]
    if renumber == "rcm" and nsolve > 0:
        solve = btog < nsolve
        pair = solve[:, :, None] & solve[:, None, :]
        rows = np.broadcast_to(btog[:, :, None], pair.shape)[pair]
        cols = np.broadcast_to(btog[:, None, :], pair.shape)[pair]
        perm = _rcm_order(rows, cols, nsolve)
        inv2 = np.empty(nglobal, dtype=np.int64)
        inv2[perm] = np.arange(nsolve)
        inv2[nsolve:] = np.arange(nsolve, nglobal)
        btog = inv2[btog]
    bmask = (btog >= nsolve).astype(np.int32)
    solve = bmask == 0
    nband = 0
    if solve.any():
        gmax = np.where(solve, btog, -1).max(axis=1)
        gmin = np.where(solve, btog, np.iinfo(np.int64).max).min(axis=1)
        has = solve.any(axis=1)
        nband = int((gmax[has] - gmin[has]).max())
    nband += 1
    return btog.astype(np.int32), bmask, nglobal, nsolve, nband


def elements_nodes(np_: int, z: np.ndarray, vx: np.ndarray, vy: np.ndarray):
    """element_nodes for every element at once: vx, vy (nel, 4) -> X, Y
    (nel, np, np), the same arithmetic element by element."""
    nel = vx.shape[0]
    nm = np_ - 1
    X = np.zeros((nel, np_, np_))
    Y = np.zeros((nel, np_, np_))
    for s in range(4):
        sp = z if s < 2 else -z[::-1]
        for A, V in ((X, vx), (Y, vy)):
            v1 = V[:, s][:, None]
            v2 = V[:, (s + 1) % 4][:, None]
            pv = v1 + (v2 - v1) * 0.5 * (sp + 1.0)[None, :]
            if s == 0:
                A[:, 0, 0:nm] = pv[:, :nm]
            elif s == 1:
                A[:, 0:nm, nm] = pv[:, :nm]
            elif s == 2:
                A[:, nm, nm:0:-1] = pv[:, :nm]
            else:
                A[:, nm:0:-1, 0] = pv[:, :nm]
    zr = z[None, None, 1:nm]
    zs = z[None, 1:nm, None]
    for a in (X, Y):
        a[:, 1:nm, 1:nm] = (0.50 * ((1.0 - zr) * a[:, 1:nm, 0:1] + (1.0 + zr) * a[:, 1:nm, nm:nm + 1]
                                    + (1.0 - zs) * a[:, 0:1, 1:nm] + (1.0 + zs) * a[:, nm:nm + 1, 1:nm])
                            - 0.25 * ((1.0 - zr) * (1.0 - zs) * a[:, 0:1, 0:1]
                                      + (1.0 - zr) * (1.0 + zs) * a[:, nm:nm + 1, 0:1]
                                      + (1.0 - zs) * (1.0 + zr) * a[:, 0:1, nm:nm + 1]
                                      + (1.0 + zs) * (1.0 + zr) * a[:, nm:nm + 1, nm:nm + 1]))
    return X, Y


def rect_mesh(nx, ny, np_, x0=0.0, x1=1.0, y0=0.0, y1=1.0, jitter=0.0, seed=None,
              periodic_x=False, bc=None, renumber="rcm", vertex_xy=None):
    """Structured nx x ny quad mesh of [x0,x1] x [y0,y1].

    Elements are ordered row by row from the bottom-left (as semtex sessions
    list them); vertices CCW.  ``jitter`` moves interior vertices by a seeded
    uniform fraction of the local spacing (boundary vertices stay put, so a
    periodic pair stays matched).  ``bc`` maps "bottom"/"right"/"top"/"left"
    to (kind, K, C) or a kind letter "D"/"N"/"M"; default all essential.
    Boundaries are listed bottom (left->right), right (bottom->top), top
    (right->left), left (top->bottom): a CCW walk of the domain boundary.
    """
    bc = dict(bc or {})
    for side in ("bottom", "right", "top", "left"):
        bc.setdefault(side, "D")
    if periodic_x:
        bc["left"] = bc["right"] = None
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    VX, VY = np.meshgrid(xs, ys, indexing="xy")  # (ny+1, nx+1)
    VX = VX.copy()
    VY = VY.copy()
    if vertex_xy is not None:
        VX, VY = vertex_xy
    elif jitter > 0.0:
        rng = np.random.default_rng(seed)
        dx = (x1 - x0) / nx
        dy = (y1 - y0) / ny
        jx = rng.uniform(-jitter, jitter, size=VX.shape) * dx
        jy = rng.uniform(-jitter, jitter, size=VY.shape) * dy
        inner = np.zeros(VX.shape, dtype=bool)
        inner[1:-1, 1:-1] = True
        VX[inner] += jx[inner]
        VY[inner] += jy[inner]
    vid = lambda i, j: j * (nx + 1) + i  # noqa: E731
    canon = np.arange((nx + 1) * (ny + 1))
    if periodic_x:
        for j in range(ny + 1):
            canon[vid(nx, j)] = vid(0, j)
    nel = nx * ny
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()                      # element e = j nx + i
    ci = np.stack([ii, ii + 1, ii + 1, ii], axis=1)      # CCW corners
    cj = np.stack([jj, jj, jj + 1, jj + 1], axis=1)
    evids = (cj * (nx + 1) + ci).astype(np.int64)
    vx = np.asarray(VX)[cj, ci].astype(np.float64)
    vy = np.asarray(VY)[cj, ci].astype(np.float64)
    bnds = []

    def add(side_name, e, s):
        spec = bc[side_name]
        if spec is None:
            return
        if isinstance(spec, str):
            spec = (spec,)
        kind = _KIND[spec[0]]
        K = spec[1] if len(spec) > 1 else 0.0
        C = spec[2] if len(spec) > 2 else 0.0
        bnds.append(Boundary(e, s, kind, K, C, group=side_name))

    for i in range(nx):
        add("bottom", i, 0)
    for j in range(ny):
        add("right", j * nx + nx - 1, 1)
    for i in reversed(range(nx)):
        add("top", (ny - 1) * nx + i, 2)
    for j in reversed(range(ny)):
        add("left", j * nx, 3)
    ess = {(b.elmt, b.side) for b in bnds if b.kind == ESSENTIAL}
    btog, bmask, nglobal, nsolve, nband = number_mesh(np_, evids, canon, ess, renumber)
    z = gll_points(np_)
    X, Y = elements_nodes(np_, z, vx, vy)
    return QuadMesh(np_, nel, X, Y, btog, bmask, nglobal, nsolve, nband, bnds, vx, vy)

"""Numberings of one jittered channel whose band-factor envelopes differ, and
the envelope tables read off a LAPACK band factor (shared by the CPU and GPU
envelope tests).

Numberings: reverse Cuthill-McKee (the front-end's default, a smooth
staircase), Cuthill-McKee (the same order reversed), the naive element order
(a ragged envelope), a seeded random permutation of the solve nodes (a
nearly full band), and RCM with runs of nodes exchanged (a staircase that
falls and rises, so that the envelope's monotone hull is what bounds it).
"""
import dataclasses

import numpy as np


def numbered_mesh(order, nx=10, ny=8, np_=7, seed=4):
    """A jittered periodic channel whose solve nodes are numbered by `order`."""
    from semtex_b200.mesh import rect_mesh
    kw = dict(x0=0.0, x1=2 * np.pi, y0=0.0, y1=1.0, jitter=0.15, seed=seed, periodic_x=True,
              bc={"bottom": "D", "top": "D"})
    if order == "none":
        return rect_mesh(nx, ny, np_, renumber="none", **kw)
    m = rect_mesh(nx, ny, np_, **kw)
    ns = m.nsolve
    if order == "rcm":
        return m
    if order == "cm":
        perm = np.arange(ns)[::-1]
    elif order == "random":
        perm = np.random.default_rng(seed).permutation(ns)
    elif order == "swapped":
        # RCM with two pairs of 64-node runs exchanged: the lowest row block
        # that a block column reaches then falls and rises along the band
        perm = np.arange(ns)
        for a, b in ((3, 5), (8, 9)):
            ra, rb = perm[64 * a:64 * (a + 1)].copy(), perm[64 * b:64 * (b + 1)].copy()
            perm[64 * a:64 * (a + 1)], perm[64 * b:64 * (b + 1)] = rb, ra
    else:
        raise ValueError(order)
    new = np.concatenate([perm, np.arange(ns, m.nglobal)])
    btog = new[m.btog].astype(np.int32)
    solve = btog < ns
    gmax = np.where(solve, btog, -1).max(axis=1)
    gmin = np.where(solve, btog, np.iinfo(np.int32).max).min(axis=1)
    has = solve.any(axis=1)
    nband = int((gmax[has] - gmin[has]).max()) + 1
    return dataclasses.replace(m, btog=btog, nband=nband)


ORDERS = ["rcm", "cm", "none", "random", "swapped"]


def lapack_tile_hull(ab, nsolve, nband, nb=64):
    """The tables the envelope must equal, from the oracle's factor alone:
    for each block column the lowest row block holding a non-zero of the
    factor, its suffix minimum over the later columns (the monotone hull),
    and from it the tiles above each diagonal and right of it."""
    kd = nband - 1
    nblk = (nsolve + nb - 1) // nb
    low = np.arange(nblk)
    cols, offs = np.nonzero(ab)
    rows = cols + offs - kd
    np.minimum.at(low, cols // nb, rows // nb)
    fm = np.minimum.accumulate(low[::-1])[::-1]
    J = (kd + nb - 1) // nb
    above = np.minimum(np.arange(nblk) - fm, J)
    right = np.zeros(nblk, dtype=np.int64)
    for k in range(nblk):
        c = k
        while c + 1 < nblk and fm[c + 1] <= k:
            c += 1
        right[k] = min(J, c - k)
    return above, right

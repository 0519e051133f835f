"""Fourier-mode partition across ranks (one process per GPU).

semtex splits the Fourier modes of a field across MPI ranks in contiguous
blocks before the solve (src/geometry.cpp:72-101; Geometry::baseMode /
nModeProc, src/geometry.h:53-58) and the solve itself never communicates
(src/field.cpp:564-723 touches only local planes).  The same split is used
here: rank r owns modes [base, base + count); its local planes are 2l and
2l+1 for local mode l, except that plane 1 of rank 0 is the Nyquist datum,
which is not solved (src/field.cpp:566).
"""
from __future__ import annotations


def mode_block(num_modes: int, world: int, rank: int):
    """Contiguous block of modes owned by `rank`: (base_mode, count)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    per, extra = divmod(num_modes, world)
    count = per + (1 if rank < extra else 0)
    base = rank * per + min(rank, extra)
    return base, count


def local_planes(base_mode: int, count: int):
    """Global plane indices a rank solves, in local order."""
    planes = []
    for mode in range(base_mode, base_mode + count):
        if mode == 0:
            planes.append(0)
        else:
            planes += [2 * mode, 2 * mode + 1]
    return planes


def betak2(base_mode: int, count: int, beta: float):
    """(beta k)^2 for the rank's modes (Field::modeConstant, Cartesian)."""
    return [(beta * k) ** 2 for k in range(base_mode, base_mode + count)]

"""Generate tests/golden/gll_ref.npz from the reference's own femlib/polylib.c.

The reference source is compiled (by `make -C oracle ref`) into
oracle/_ref/libref_polylib.so; this script calls its zwglj/Dglj for
np = 3..16 and stores the tables, so the GLL pin also holds where the
reference tree is absent.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    so = os.path.join(ROOT, "oracle", "_ref", "libref_polylib.so")
    L = C.CDLL(so)
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    L.zwglj.argtypes = [dp, dp, C.c_int, C.c_double, C.c_double]
    L.Dglj.argtypes = [dp, dp, dp, C.c_int, C.c_double, C.c_double]
    out = {}
    for n in range(3, 17):
        z, w = np.zeros(n), np.zeros(n)
        D, Dt = np.zeros(n * n), np.zeros(n * n)
        L.zwglj(z, w, n, 0.0, 0.0)
        L.Dglj(D, Dt, z, n, 0.0, 0.0)
        out[f"z{n}"], out[f"w{n}"], out[f"D{n}"] = z, w, D.reshape(n, n)
    np.savez(os.path.join(HERE, "gll_ref.npz"), **out)


if __name__ == "__main__":
    main()

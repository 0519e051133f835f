"""Generate tests/golden/edgemap_ref.npz from the reference's own
femlib/mapping.c.

The reference source is compiled (by `make -C oracle ref`) into
oracle/_ref/libref_mapping.so; this script calls its edgemaps for np = 2..16
in two dimensions (and in one, the side maps) and stores emap and pmap, so
the edge-map pin also holds where the reference tree is absent.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_mapping.so"))
    IP = C.POINTER(C.c_int)
    L.edgemaps.argtypes = [C.c_int, C.c_int, C.POINTER(IP), C.POINTER(IP)]
    L.edgemaps.restype = None
    out = {}
    for dim in (1, 2):
        for n in range(2, 17):
            em, pm = IP(), IP()
            L.edgemaps(n, dim, C.byref(em), C.byref(pm))
            length = n * n if dim == 2 else n
            out[f"emap{dim}_{n}"] = np.array(em[:length], dtype=np.int32)
            out[f"pmap{dim}_{n}"] = np.array(pm[:length], dtype=np.int32)
    np.savez(os.path.join(HERE, "edgemap_ref.npz"), **out)


if __name__ == "__main__":
    main()

"""Mode-partitioned solves across ranks (CPU, gloo, world_size 2).

Each rank solves its own block of Fourier modes with the oracle (no
collective in the solve); the blocks are then gathered and must equal the
single-process solve of all modes exactly, since every mode is independent.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import DIRECT, OracleMesh, OracleSystem
        from semtex_b200.partition import betak2, local_planes, mode_block
        from semtex_b200.workloads import small_channel
        w = small_channel(nx=4, ny=3, np_=5, nz=8, lam=10.0, seed=4)
        base, count = mode_block(w.num_modes, world, rank)
        om = OracleMesh(w.mesh)
        planes = local_planes(base, count)
        sol = np.zeros((w.nz, w.mesh.nplane))
        for mode, bk2 in zip(range(base, base + count), betak2(base, count, w.beta)):
            S = OracleSystem(om, float(w.lambda2[mode]), bk2, DIRECT)
            for p in ([0] if mode == 0 else [2 * mode, 2 * mode + 1]):
                sol[p], _ = S.solve_plane(w.forcing[p], None)
        t = torch.tensor(sol)
        gathered = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(gathered, t)  # result collection only, after the solve
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), sum(g.numpy() for g in gathered))
            np.save(os.path.join(out_dir, "planes.npy"), np.array(planes))
    finally:
        dist.destroy_process_group()


def test_partition_blocks_cover_modes():
    from semtex_b200.partition import local_planes, mode_block
    for nm in (1, 5, 32, 33):
        for world in (1, 2, 3, 8):
            blocks = [mode_block(nm, world, r) for r in range(world)]
            assert sum(c for _, c in blocks) == nm
            assert blocks[0][0] == 0
            for (b0, c0), (b1, _) in zip(blocks, blocks[1:]):
                assert b0 + c0 == b1
    assert local_planes(0, 3) == [0, 2, 3, 4, 5]
    assert local_planes(3, 2) == [6, 7, 8, 9]


def test_two_rank_mode_partition_matches_single(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    got = np.load(tmp_path / "gathered.npy")
    from oracle.oracle import OracleMesh, solve_planes
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=4, ny=3, np_=5, nz=8, lam=10.0, seed=4)
    ref, _ = solve_planes(OracleMesh(w.mesh), 0.0, w.beta, w.forcing, None,
                          lambda2_per_mode=w.lambda2)
    assert np.array_equal(got, ref)

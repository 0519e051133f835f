"""CPU tests of the parts of bench.py's output contract that need no GPU:
the per-launch DRAM traffic it reports for each dominant kernel comes from
the committed ncu summaries, and the profiler-run flag exists."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_traffic_of_each_roofline_kernel_is_committed():
    # the kernels a bench line reports a roofline for, on their workloads
    for kernel, tag in (("k_cg", "config2"), ("k_band_sweep", "config2")):
        t = bench._ncu_traffic(kernel, tag)
        assert isinstance(t, int) and t > 0, kernel


def test_traffic_lookup_of_an_unprofiled_kernel_is_none():
    assert bench._ncu_traffic("k_not_a_kernel", "config3") is None


def test_sample_modes_spread_over_lambda2():
    lam = [5.0, 0.1, 300.0, 2.0, 40.0]
    # sorted by lambda2: modes 1, 3, 0, 4, 2
    assert bench.sample_modes(lam, 3) == [0, 1, 2]      # lowest (1), median (0), highest (2)
    assert bench.sample_modes(lam, 1) == [0]
    assert bench.sample_modes(lam, 10) == [0, 1, 2, 3, 4]


def test_compulsory_bytes_of_a_direct_solve():
    from semtex_b200.workloads import config3_block
    m = config3_block().mesh
    # one mode of two planes: factor + element matrices + Q8 + forcing in/out
    b = bench.direct_bytes(m, [2])
    nn, nint, nxt = 121, 81, 40
    assert b == 8 * (m.nsolve * m.nband + m.nel * (nxt * nint + nint * nint) + m.nel * nn + 4 * m.nel * nn)
    assert bench.sweep_bytes(m, [2], 2) - bench.sweep_bytes(m, [2], 1) == m.nsolve * m.nband * 8


def test_profile_summaries_give_their_command():
    d = os.path.join(ROOT, "profiles")
    for name in sorted(os.listdir(d)):
        assert name.endswith((".md", ".txt")), name
        with open(os.path.join(d, name)) as fh:
            text = fh.read()
        # every summary carries the ncu command that made it, with the
        # clock-control flag, and runs committed files only
        assert "ncu " in text and "--clock-control none" in text, name
        assert "_work" not in text, name


def test_bench_flags():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True,
                         text=True, check=True).stdout
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--no-extras", "--serve-requests"):
        assert flag in out, flag

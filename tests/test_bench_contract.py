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
    # the two kernels a bench line names in "roofline" / "roofline_other_form"
    for kernel in ("k_cg", "k_band_sweep"):
        t = bench._ncu_traffic(kernel)
        assert isinstance(t, int) and t > 0, kernel


def test_traffic_lookup_of_an_unprofiled_kernel_is_none():
    assert bench._ncu_traffic("k_not_a_kernel") is None


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
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--no-config3", "--serve-requests"):
        assert flag in out, flag

#!/usr/bin/env python
"""Benchmark: per-Fourier-mode Helmholtz solve (semtex Field::solve) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (N=1): the largest configuration that fits one GPU -- the
mixed-precision channel: [0,2pi] x [0,1], 64 x 64 quads jittered +-20 %
(seed 3), N = 10, nz = 128 planes (modes 0..63, 127 planes solved, Nyquist
skipped), lambda2 log-uniform in [1e-2, 1e4] per mode, Dirichlet walls,
periodic in x, manufactured solution u = sum_k a_k sin(pi y) cos(kz) cos(3x).
Every mode is factored (121 GB of band factors, set-up).  A step is one solve
of every plane of every mode.

Metric: Helmholtz DoF-solves/s (unique nodes per plane x planes solved /
seconds) at <= 1e-10 relative error.  ``value`` is the batched
mixed-precision form on device-resident inputs; ``e2e`` the same through the
host-pointer C-ABI call with the host<->device copies inside the timed region;
the plain FP64 mode-by-mode form and the batched FP64 form are reported
beside it, and the lowest-, median- and highest-lambda2 modes are checked
against the oracle.  Config 2 (32 x 32, N = 8, nz = 64, lambda2 = 1e6 + k^2),
the multi-mesh batch, the z-transform, the DNS elliptic-phase field
operations (config 5's field shape), one DNS elliptic step of config 5 at
full size (one rank's 16-mode block of an 8-GPU split) and the serving loop
are extra keys.

Multi-GPU (torchrun): Fourier modes are independent, so the modes of a
64 N-mode problem are split in contiguous blocks of 64 (the reference's mode
split; weak scaling, no collective in the data path); the timing is the max
over ranks.

``--impl reference`` times the reference algorithm on the host cores (the
C oracle port, one process per core over config-3 modes) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Helmholtz DoF-solves/s at <=1e-10 rel err, mixed vs plain FP64; serve p50/p99 ms"
UNIT = "DoF-solves/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# clocks sampling during the timed region
# --------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        busy = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": float(np.median(busy)) if busy else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# reference arm / cpu baseline: the C oracle on the host cores
# --------------------------------------------------------------------------

def _oracle_mode_worker(mode, reps, barrier, queue, want_solution):
    """One config-3 mode on one core (a spawned process): mesh, element
    condensation and band assembly with the oracle, the band factored by
    LAPACK dpbtrf (set-up, untimed), then both planes of the mode solved
    `reps` times after every worker is ready (timed; median)."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    try:
        from oracle.oracle import DIRECT, OracleMesh, OracleSystem
        from semtex_b200.workloads import config3_block
        w = config3_block(world=64, rank=mode, modes_per_rank=1)  # mode k of config 3 alone
        om = OracleMesh(w.mesh)
        sysm = OracleSystem(om, float(w.lambda2[0]), 0.0, DIRECT, factor="lapack")
        planes = w.solved_planes
        err = None
    except Exception as exc:  # reported, never hangs the barrier
        planes, err = [], repr(exc)
    barrier.wait()
    if err:
        queue.put((mode, None, 0, None, err))
        return
    times, sols = [], None
    for _ in range(max(1, reps)):
        t0 = time.perf_counter()
        sols = [sysm.solve_plane(w.forcing[p], None)[0] for p in planes]
        times.append(time.perf_counter() - t0)
    queue.put((mode, float(np.median(times)), len(planes), sols if want_solution else None, None))


def oracle_modes(modes, reps, want_solution=False):
    """Solve config-3 modes with the oracle, one process per mode, all at
    once.  Returns {mode: (seconds per solve of its planes, planes,
    solutions)} and the wall time of the whole run."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(len(modes))
    q = ctx.Queue()
    t0 = time.perf_counter()
    procs = [ctx.Process(target=_oracle_mode_worker, args=(m, reps, barrier, q, want_solution))
             for m in modes]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        mode, t, planes, sols, err = q.get()
        if err:
            raise RuntimeError(f"oracle worker for mode {mode}: {err}")
        out[mode] = (t, planes, sols)
    for p in procs:
        p.join()
    return out, time.perf_counter() - t0


def sample_modes(lambda2, n):
    """n modes spread evenly over the modes sorted by lambda2 (lowest,
    ..., highest)."""
    order = np.argsort(lambda2)
    n = max(1, min(n, len(order)))
    if n == 1:
        return [int(order[len(order) // 2])]
    idx = np.round(np.linspace(0, len(order) - 1, n)).astype(int)
    return sorted({int(order[i]) for i in idx})


def _host_workers():
    """Processes the host can run at once for the reference arm: one per core,
    at most one per mode, and no more than available memory allows (about
    2.5 GB for a config-3 mode: band factor 1.45 GB, element matrices 0.32 GB)."""
    cores = os.cpu_count() or 1
    try:
        import psutil
        mem = int(psutil.virtual_memory().available * 0.7 / 2.5e9)
    except Exception:
        mem = cores
    return max(1, min(cores, 64, mem)), cores


def run_reference(args, rank, world):
    """The reference's algorithm on the host cores (the oracle port: element
    condensation, band assembly, LAPACK dpbtrf factor as set-up; the solve's
    condensed right-hand side, dpbtrs-style band sweeps and interior
    back-substitution timed), on the config-3 workload: as many modes as the
    host can hold, one process per core, all solving at once (the
    reference's mode split without MPI).  A step is one solve of every
    sampled mode; DoF-solves/s = unique nodes per plane x planes / step."""
    if rank != 0:
        return
    from semtex_b200.workloads import config3_block
    w = config3_block()
    nwork, cores = _host_workers()
    modes = sample_modes(w.lambda2, nwork)
    res, wall = oracle_modes(modes, max(1, args.steps))
    step_s = max(r[0] for r in res.values())
    planes = sum(r[1] for r in res.values())
    value = w.dof_per_plane * planes / step_s
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded manufactured solution)",
        "config": {"workload": w.name, "planes_solved": w.planes_solved, "dof_per_plane": w.dof_per_plane,
                   "sample_modes": modes, "host_cores": cores},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(modes), "kind": "port",
                         "sample": f"{len(modes)} of the {w.num_modes} modes of {w.name} ({planes} planes), spread "
                                   "over the lambda2 range, one process per core solving at once; oracle C port "
                                   "with LAPACK dpbtrf for the factor (untimed set-up), median of "
                                   f"{max(1, args.steps)} solves per process; run wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------

def rel_err(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return (float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)),
            float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)))


def _ncu_traffic(kernel, tag):
    """DRAM bytes (read + write) per launch of `kernel` on workload `tag`,
    from the committed ncu summary profiles/<kernel>_<tag>.md (its line
    `dram_bytes_per_launch: N`); None when there is none."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{tag}.md")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        for line in fh:
            if line.strip().startswith("dram_bytes_per_launch:"):
                return int(line.split(":", 1)[1].strip().split()[0])
    return None


def direct_bytes(m, modes_planes):
    """Compulsory bytes of a direct FP64 solve (each operand read once, each
    output written once), per mode with P planes: the band factor, the
    element matrices hbi hii^-1 and hii^-1, the mass Q8, forcing in and
    solution out."""
    nn, nint, nxt = m.np * m.np, (m.np - 2) ** 2, 4 * (m.np - 1)
    tot = 0
    for P in modes_planes:
        tot += 8 * (m.nsolve * m.nband + m.nel * (nxt * nint + nint * nint) + m.nel * nn + P * 2 * m.nel * nn)
    return tot


def sweep_bytes(m, modes_planes, reads_of_factor):
    """Bytes of the band sweeps of one solve: the factor `reads_of_factor`
    times per system, and each right-hand side read and written by each
    sweep."""
    return sum(reads_of_factor * m.nsolve * m.nband * 8 + 2 * 2 * P * m.nsolve * 8 for P in modes_planes)


TILE_BYTES = 64 * 65 * 8   # one 64 x 64 band tile as stored (rows padded to 65)


def envelope_sweep_bytes(mesh, m, modes_planes):
    """Bytes the two sweeps move: per system and sweep, the factor tiles
    inside the envelope (the tiles above each diagonal tile, and the diagonal
    inverse) once, and each right-hand side read and written."""
    above, _ = mesh.envelope()
    tiles = int(above.sum()) + len(above)
    return sum(2 * tiles * TILE_BYTES + 2 * 2 * P * m.nsolve * 8 for P in modes_planes)


def run_ours(args, rank, world):
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import config3_block

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sx.lib.sx_set_device(dev.index)
    dist = None
    if world > 1:
        import torch.distributed as dist
    # this rank's block of modes (the reference's contiguous mode split)
    w = config3_block(world, rank)
    m = w.mesh
    nz, base, nmodes = w.nz, w.base_mode, w.num_modes
    stride = m.nplane
    sp = w.solved_planes
    planes_solved = len(sp)
    dofs = w.dof_per_plane * planes_solved
    mode_planes = [1 if (base + l) == 0 else 2 for l in range(nmodes)]
    mesh = sx.Mesh(m)
    t0 = time.perf_counter()
    S = sx.ModalMatrixSys(mesh, base_mode=base, num_modes=nmodes, method=sx.DIRECT,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    f_src = torch.tensor(w.forcing, device=dev)
    f_work = torch.empty_like(f_src)
    u_dev = torch.zeros_like(f_src)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def restore():
        f_work.copy_(f_src)  # the solve overwrites its forcing (src/field.cpp:525-526)

    # 256 MB written between timed steps: evicts the 126 MB L2 (the step's
    # working set, 121 GB of factors, is far above L2 anyway)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)

    def timed(fn, k, wu):
        for _ in range(wu):
            restore()
            fn()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        for e0, e1 in ev:
            restore()
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / k
        if dist is not None:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # plain FP64, mode by mode (the reference-compatible form)
    def step_plain():
        S.solve_device(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, stream=sptr)

    restore()
    step_plain()
    torch.cuda.synchronize()
    u_plain = u_dev.cpu().numpy()[sp]
    ms_plain = timed(step_plain, max(1, min(args.steps, 3)), 1)

    # batched FP64, schedule picked by the autotuner on this data (set-up)
    fp64_stats = {}

    def step_batched():
        fp64_stats.update(S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, sx.FP64,
                                          stream=sptr))

    tune64 = S.autotune(u_dev.data_ptr(), f_src.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)
    restore()
    step_batched()
    torch.cuda.synchronize()
    u_batched = u_dev.cpu().numpy()[sp]
    clk = ClockSampler(dev.index)
    clk.start()
    ms_batched = timed(step_batched, args.steps, args.warmup)

    # batched mixed precision (the headline form): per mode, FP32 CG inside
    # FP64 refinement or the FP64 band Cholesky, whichever streams fewer bytes
    mixed_stats = {}

    def step_mixed():
        mixed_stats.update(S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride,
                                           sx.MIXED_FP32, tol_rel=args.tol, max_refine=20, stream=sptr))

    tunemx = S.autotune(u_dev.data_ptr(), f_src.data_ptr(), 0, nz, stride, sx.MIXED_FP32,
                        tol_rel=args.tol, max_refine=20, stream=sptr)
    restore()
    step_mixed()
    torch.cuda.synchronize()
    u_mixed = u_dev.cpu().numpy()[sp]
    ms_mixed = timed(step_mixed, args.steps, args.warmup)
    clocks = clk.stop()
    mixed_err = rel_err(u_mixed, u_batched)
    mixed_ok = max(mixed_err) <= 1e-10
    if dist is not None:
        t = torch.tensor([0.0 if mixed_ok else 1.0], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mixed_ok = t.item() == 0.0
    if not mixed_ok:
        raise SystemExit(f"mixed form misses the 1e-10 bar against the FP64 form: {mixed_err}")
    ex = w.exact[sp]
    launches_per_step = int(mixed_stats.get("kernel_launches", 0))

    def kernel_ms(replay, reps):
        """Average duration of one replayed launch, CUDA events on its stream."""
        replay(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        replay(reps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    hbm, peak_kind = _peaks()
    # the dominant kernel: the banded sweeps (both sweeps of every system in
    # one launch).  Algorithmic bytes per launch: each system's band factor
    # as LAPACK stores it (nsolve x nband) once and each right-hand side in
    # and out.  The kernel's own bytes (design): each sweep reads the factor
    # tiles inside the envelope once (the other tiles are exact zeros and
    # are skipped) and each right-hand side in and out.
    restore()
    S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)
    sweep_ms = kernel_ms(lambda r: S.profile_band_sweeps(r, sptr), max(3, min(args.steps, 5)))
    alg = sweep_bytes(m, mode_planes, 1)
    design = envelope_sweep_bytes(mesh, m, mode_planes)
    band_gbs = alg / (sweep_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_band_sweep", "achieved": band_gbs, "peak": hbm, "unit": "GB/s",
                "frac": band_gbs / hbm, "peak_kind": peak_kind, "traffic": _ncu_traffic("k_band_sweep", "config3"),
                "algorithmic_bytes_per_launch": alg, "launch_ms": sweep_ms,
                "design_bytes_per_launch": design,
                "design_achieved": design / (sweep_ms * 1e-3) / 1e9,
                "design_frac": design / (sweep_ms * 1e-3) / 1e9 / hbm,
                "note": "algorithmic = band factor (nsolve x nband, LAPACK's storage) once + RHS in/out per "
                        "sweep; design = the factor tiles inside the envelope (exact zeros outside it are "
                        "skipped) read by each of the two sweeps + RHS in/out"}
    solve_alg = direct_bytes(m, mode_planes)
    solve_gbs = solve_alg / (ms_mixed * 1e-3) / 1e9

    # end to end through the host-pointer C-ABI call, pinned buffers
    f_host = torch.tensor(w.forcing).pin_memory()
    u_host = torch.zeros_like(f_host).pin_memory()
    fh, uh = f_host.numpy(), u_host.numpy()
    for _ in range(max(1, args.warmup)):
        S.solve_batched_host(fh, out=uh, precision=sx.MIXED_FP32, tol_rel=args.tol, max_refine=20)
    if dist is not None:
        dist.barrier()
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        S.solve_batched_host(fh, out=uh, precision=sx.MIXED_FP32, tol_rel=args.tol, max_refine=20)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_t))
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_err = rel_err(uh[sp], u_mixed)
    d2h = int(len(sp) * stride * 8)

    total_dofs = dofs * world
    value = total_dofs / (ms_mixed * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded manufactured solution on the 64 x 64, N = 10, nz = 128 jittered channel)",
        "config": {"workload": w.name, "elements": m.nel, "order": m.np - 1, "nz_per_gpu": nz,
                   "modes_per_gpu": nmodes, "planes_solved_per_gpu": planes_solved,
                   "dof_per_plane": w.dof_per_plane, "nglobal": m.nglobal, "nsolve": m.nsolve,
                   "nband": m.nband, "lambda2": "log-uniform [1e-2, 1e4] per mode (seed 3)",
                   "form": "batched mixed precision (per mode: FP32 CG in FP64 refinement, or the FP64 "
                           "band Cholesky when it streams fewer bytes)",
                   "parallelism": f"modes split over {world} GPU(s) in contiguous blocks, no collective",
                   "l2": "factors %.1f GB per GPU >> L2; 256 MB written between timed steps"
                         % (S.device_bytes / 1e9)},
        "plain_fp64": {"value": total_dofs / (ms_plain * 1e-3), "ms_per_step": ms_plain,
                       "form": "mode by mode, as Field::solve's plane loop"},
        "batched_fp64": {"value": total_dofs / (ms_batched * 1e-3), "ms_per_step": ms_batched,
                         "rel_err_vs_plain": rel_err(u_batched, u_plain),
                         "kernel_launches": int(fp64_stats.get("kernel_launches", 0))},
        "batched_mixed": {"value": value, "ms_per_step": ms_mixed, "rel_err_vs_fp64": mixed_err,
                          "meets_1e-10": mixed_ok, "refinements": mixed_stats.get("refinements"),
                          "inner_iterations": mixed_stats.get("iterations_max"),
                          "planes_to_band": mixed_stats.get("planes_direct"),
                          "final_rel_residual": mixed_stats.get("final_rel_residual"),
                          "max_rel_err_vs_manufactured": float(np.abs(u_mixed - ex).max() / np.abs(ex).max())},
        "speedup_mixed_vs_plain": ms_plain / ms_mixed,
        "speedup_mixed_vs_batched_fp64": ms_batched / ms_mixed,
        "autotuned": {"batched_fp64": tune64, "batched_mixed": tunemx},
        "setup_s": setup_s,
        "roofline": roofline,
        "solve_roofline": {"bound": "hbm", "algorithmic_bytes_per_step": solve_alg, "achieved": solve_gbs,
                           "peak": hbm, "unit": "GB/s", "frac": solve_gbs / hbm, "peak_kind": peak_kind,
                           "note": "whole direct solve, each operand once: factor, hbi hii^-1, hii^-1, Q8, "
                                   "forcing in, solution out"},
        "e2e": {"value": total_dofs / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": int(fh.nbytes), "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_s * 1e3, "rel_err_vs_device_call": e2e_err,
                "call": "sx_field_solve_batched_host (pinned host buffers; copies and solve in the timed "
                        "region; the modes in chunks whose copies and solves overlap, 8 modes a chunk "
                        "when every mode goes to the band solve)"},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        # CPU baseline + full-size parity: the oracle on the lowest-, median-
        # and highest-lambda2 modes, one process per mode
        pm = sample_modes(w.lambda2, 3)
        res, wall = oracle_modes(pm, 2, want_solution=True)
        step_s = max(r[0] for r in res.values())
        planes = sum(r[1] for r in res.values())
        line["cpu_baseline"] = {"value": w.dof_per_plane * planes / step_s, "unit": UNIT, "cores": len(pm),
                                "kind": "port",
                                "sample": f"modes {pm} of {w.name} (lowest, median, highest lambda2; {planes} "
                                          "planes), one process per core at once; oracle C port, LAPACK "
                                          f"dpbtrf factor untimed, median of 2 solves; wall {wall:.1f} s"}
        par = {}
        for k in pm:
            sols = res[k][2]
            rows = [sp.index(2 * k), sp.index(2 * k + 1)] if k > 0 else [0]
            got_m = [u_mixed[r] for r in rows]
            got_b = [u_batched[r] for r in rows]
            got_p = [u_plain[r] for r in rows]
            par[str(k)] = {"lambda2": float(w.lambda2[k]),
                           "mixed": rel_err(np.array(got_m), np.array(sols)),
                           "batched_fp64": rel_err(np.array(got_b), np.array(sols)),
                           "plain_fp64": rel_err(np.array(got_p), np.array(sols))}
        worst = max(max(v["mixed"] + v["batched_fp64"] + v["plain_fp64"]) for v in par.values())
        line["rel_err_vs_oracle"] = {"modes": par, "worst": worst, "meets_1e-10": worst <= 1e-10,
                                     "meets_1e-12": worst <= 1e-12}
        if worst > 1e-10:
            print(json.dumps(line), flush=True)
            raise SystemExit(f"GPU solution differs from the oracle by {worst:.3e} (> 1e-10)")
    del S
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_extras:
        line["config2"] = run_config2(args)
        line["multi_mesh"] = run_multi()
        line["transform_z"] = run_transform()
        line["dns_elliptic_phase"] = run_dns()
        line["config5_full"] = run_config5(ranks=(0,))
    if rank == 0 and world == 1 and args.serve_requests > 0:
        line["serving"] = run_serving(args.serve_requests, check_oracle=not args.no_cpu,
                                      precision=args.serve_precision, slots=args.serve_slots)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_config2(args, reps=None):
    """Config 2 (32 x 32 jittered quads, N = 8, nz = 64, lambda2 = 1e6 +
    k^2): plain FP64 mode by mode, batched FP64 and batched mixed, autotuned,
    device-resident inputs, CUDA events, L2 flushed between steps; mode 1
    checked against the oracle (its parity bar: 1e-12 for the FP64 forms)."""
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import config2
    reps = reps or max(3, args.steps)
    w = config2(seed=2)
    m = w.mesh
    nz, stride = w.nz, m.nplane
    S = sx.ModalMatrixSys(sx.Mesh(m), num_modes=w.num_modes, method=sx.DIRECT, lambda2_modes=w.lambda2,
                          betak2_modes=w.betak2)
    f0 = torch.tensor(w.forcing, device="cuda")
    f, u = torch.empty_like(f0), torch.zeros_like(f0)
    sptr = torch.cuda.current_stream().cuda_stream
    l2 = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    sp = w.solved_planes

    def timed(fn, k):
        for _ in range(2):
            f.copy_(f0)
            fn()
        ts = []
        for _ in range(k):
            f.copy_(f0)
            l2.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        f.copy_(f0)
        fn()
        torch.cuda.synchronize()
        return float(np.mean(ts)), u.cpu().numpy()[sp]

    t_plain, u_plain = timed(lambda: S.solve_device(u.data_ptr(), f.data_ptr(), 0, nz, stride, stream=sptr), 3)
    S.autotune(u.data_ptr(), f0.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)
    t_b, u_b = timed(lambda: S.solve_batched(u.data_ptr(), f.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr),
                     reps)
    S.autotune(u.data_ptr(), f0.data_ptr(), 0, nz, stride, sx.MIXED_FP32, tol_rel=args.tol, max_refine=20,
               stream=sptr)
    t_m, u_m = timed(lambda: S.solve_batched(u.data_ptr(), f.data_ptr(), 0, nz, stride, sx.MIXED_FP32,
                                             tol_rel=args.tol, max_refine=20, stream=sptr), reps)
    # the mixed form's kernel: one fused FP32 CG iteration over every plane
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    S.profile_mixed_iterations(1, sptr)
    e0.record()
    S.profile_mixed_iterations(reps, sptr)
    e1.record()
    e1.synchronize()
    cg_ms = e0.elapsed_time(e1) / reps
    nn, npts = m.np * m.np, m.nglobal + m.nel * (m.np - 2) ** 2
    # section 8(d): per iteration per plane 4 B x (5 node vectors + the
    # element operator's q), geometry once per launch
    cg_alg = 4 * len(sp) * (5 * npts + m.nel * nn) + 4 * 4 * m.nel * nn
    hbm, kind = _peaks()
    dofs = w.dof_per_plane * len(sp)
    out = {"workload": w.name, "dof_per_plane": w.dof_per_plane, "planes_solved": len(sp),
           "plain_fp64_ms": t_plain, "batched_fp64_ms": t_b, "batched_mixed_ms": t_m,
           "plain_fp64_dof_solves_per_s": dofs / (t_plain * 1e-3),
           "batched_fp64_dof_solves_per_s": dofs / (t_b * 1e-3),
           "batched_mixed_dof_solves_per_s": dofs / (t_m * 1e-3),
           "speedup_mixed_vs_plain": t_plain / t_m,
           "mixed_vs_batched_fp64_rel_err": rel_err(u_m, u_b),
           "batched_vs_plain_rel_err": rel_err(u_b, u_plain),
           "k_cg": {"launch_ms": cg_ms, "algorithmic_bytes_per_launch": cg_alg,
                    "achieved_gbs": cg_alg / (cg_ms * 1e-3) / 1e9,
                    "frac": cg_alg / (cg_ms * 1e-3) / 1e9 / hbm, "peak_kind": kind,
                    "traffic": _ncu_traffic("k_cg", "config2")}}
    if not args.no_cpu:
        from oracle.oracle import DIRECT, OracleMesh, OracleSystem
        om = OracleMesh(m)
        osys = OracleSystem(om, float(w.lambda2[1]), float(w.betak2[1]), DIRECT, factor="lapack")
        sols = np.array([osys.solve_plane(w.forcing[p], None)[0] for p in (2, 3)])
        rows = [sp.index(2), sp.index(3)]
        e_p = rel_err(u_plain[rows], sols)
        e_b = rel_err(u_b[rows], sols)
        e_m = rel_err(u_m[rows], sols)
        out["rel_err_vs_oracle_mode1"] = {"plain_fp64": e_p, "batched_fp64": e_b, "mixed": e_m}
        if max(e_p + e_b) > 1e-12 or max(e_m) > 1e-10:
            raise SystemExit(f"config 2 mode 1 vs oracle: plain {e_p}, batched {e_b}, mixed {e_m}")
    del S
    torch.cuda.empty_cache()
    return out


def run_multi(n_meshes=24, reps=5):
    """Form (a) on many small meshes (workloads.small_mesh_mix: orders 4-10,
    4 to 144 elements, 1-12 modes): the same solves (i) one mesh after
    another with the single-mesh batched form and (ii) as one multi-mesh
    batch, mixed precision to 1e-12, device-resident inputs, CUDA events on
    one stream, median of `reps` after a warm-up (graph capture)."""
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import small_mesh_mix
    torch.cuda.set_device(0)
    reqs = small_mesh_mix(n_meshes)
    st = torch.cuda.Stream()
    sptr = st.cuda_stream
    mem = []
    for r in reqs:
        S = sx.ModalMatrixSys(sx.Mesh(r.mesh), num_modes=len(r.lambda2), method=sx.AUTO,
                              lambda2_modes=r.lambda2, betak2_modes=r.betak2)
        f0 = torch.tensor(r.forcing, device="cuda")
        mem.append((S, f0, torch.empty_like(f0), torch.zeros_like(f0), r))
    dofs = sum(r.dof_solves for r in reqs)
    B = sx.Batch()

    def one_by_one():
        for S, _, f, u, r in mem:
            S.solve_batched(u.data_ptr(), f.data_ptr(), 0, r.nz, r.mesh.nplane, sx.MIXED_FP32, 1e-12,
                            max_refine=30, stream=sptr)

    def batched():
        B.solve([(S, u.data_ptr(), f.data_ptr(), None, r.nz, r.mesh.nplane) for S, _, f, u, r in mem],
                sx.MIXED_FP32, 1e-12, max_refine=30, stream=sptr)

    l2 = torch.empty(64 << 20, dtype=torch.float32, device="cuda")

    def timed(fn):
        out = []
        for k in range(reps + 1):
            with torch.cuda.stream(st):
                for _, f0, f, _, _ in mem:
                    f.copy_(f0)  # the band-routed modes overwrite their forcing
                l2.zero_()       # 256 MB: nothing of the last solve stays in L2
            st.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            if k > 0:
                out.append(e0.elapsed_time(e1))
        return float(np.median(out))

    t_one = timed(one_by_one)
    u_one = [u.cpu().numpy() for _, _, _, u, _ in mem]
    t_bat = timed(batched)
    worst = 0.0
    for (_, _, _, u, r), a in zip(mem, u_one):
        sp = [0] + list(range(2, r.nz)) if r.nz > 1 else [0]
        worst = max(worst, rel_err(u.cpu().numpy()[sp], a[sp])[0])
    return {"meshes": n_meshes, "orders": sorted({r.mesh.np - 1 for r in reqs}),
            "elements": [min(r.mesh.nel for r in reqs), max(r.mesh.nel for r in reqs)],
            "dof_solves": dofs, "one_by_one_ms": t_one, "batch_ms": t_bat,
            "one_by_one_dof_solves_per_s": dofs / (t_one * 1e-3),
            "batch_dof_solves_per_s": dofs / (t_bat * 1e-3), "speedup": t_one / t_bat,
            "batch_vs_one_by_one_rel_l2": worst,
            "note": "mixed precision to 1e-12; routing per mode (SX_AUTO); CUDA events on one stream; "
                    "L2 flushed before each timed call"}


def run_transform(reps=20):
    """The z-direction transform (dDFTr) on the bench workload's field
    shape: nz = 64 planes of 82,944 points (1024 elements x 81 nodes),
    forward and inverse in place, CUDA events, median of `reps`; the
    roofline is one read and one write of the field per direction."""
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import config2
    torch.cuda.set_device(0)
    w = config2()
    nz, stride = w.nz, w.mesh.nplane
    d = torch.tensor(w.forcing, device="cuda")
    sptr = torch.cuda.current_stream().cuda_stream
    sx.transform_z(d.data_ptr(), nz, stride, stride, +1, sptr)   # warm-up
    sx.transform_z(d.data_ptr(), nz, stride, stride, -1, sptr)
    # the field (42 MB) fits in L2: 256 MB written between timed calls
    l2 = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    out = {}
    for name, sign in (("forward", +1), ("inverse", -1)):
        ts = []
        for _ in range(reps):
            l2.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sx.transform_z(d.data_ptr(), nz, stride, stride, sign, sptr)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        gbs = 2.0 * nz * stride * 8 / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "achieved_gbs": gbs}
    peak, kind = _peaks()
    back = d.cpu().numpy()
    out.update({"nz": nz, "points": stride, "bytes_per_direction": 2 * nz * stride * 8,
                "peak_gbs": peak, "peak_kind": kind,
                "frac_forward": out["forward"]["achieved_gbs"] / peak,
                "round_trip_max_rel_err": float(np.abs(back - w.forcing).max() / np.abs(w.forcing).max()),
                "l2": "flushed between timed calls (256 MB written)",
                "kernel": "k_z_fwd<64> / k_z_inv<64>: one pass, each point's z-line in registers"})
    # config 3 and 5 field shapes: one pass through shared memory
    for name, nz2, pts in (("nz128_config3", 128, 64 * 64 * 121), ("nz256_config5", 256, 128 * 64 * 121)):
        x = torch.randn((nz2, pts), dtype=torch.float64, device="cuda")
        sx.transform_z(x.data_ptr(), nz2, pts, pts, +1, sptr)
        ts = []
        for _ in range(max(3, reps // 4)):
            l2.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sx.transform_z(x.data_ptr(), nz2, pts, pts, +1, sptr)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        gbs = 2.0 * nz2 * pts * 8 / (ms * 1e-3) / 1e9
        out[name] = {"forward_ms": ms, "achieved_gbs": gbs, "frac": gbs / peak,
                     "kernel": f"k_z_fwd_s<{nz2}>"}
        del x
    return out


def _dns_fields(nz, n, count, seed):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return [torch.randn((nz, n), dtype=torch.float64, device="cuda", generator=g) for _ in range(count)]


def run_dns(reps=5, nz=256, check=True):
    """The DNS elliptic-phase field operations (waveProp, setPForce, project,
    Field::smooth, AuxField::gradient) on config 5's field shape: 128 x 64
    quads jittered +-15 %, N = 10 (8192 elements, 991,232 points a plane),
    nz = 256 planes -- 2.03 GB a field, every operand larger than L2.
    Seeded random device fields (synthetic: these operations are linear and
    their cost does not depend on the values).  CUDA events on the launching
    stream, median of `reps`; the roofline is each operand read once and each
    result written once (the partials and numbering, 40 MB, are counted
    once).  Planes of modes 0, 1 and 127 are checked against the oracle, which
    is also timed on them (one core)."""
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import _jittered_channel
    torch.cuda.set_device(0)
    m = _jittered_channel(128, 64, 11, 0.15, 5)
    mesh = sx.Mesh(m)
    n, nel, npnp = m.nplane, m.nel, m.npnp
    f8 = nz * n * 8
    peak, kind = _peaks()
    sptr = torch.cuda.current_stream().cuda_stream
    order, dt, nu, beta = 2, 5e-4, 5e-4, 1.0
    us = [_dns_fields(nz, n, 3, 50 + q) for q in range(order)]
    uf = [_dns_fields(nz, n, 3, 60 + q) for q in range(order)]
    h = _dns_fields(nz, n, 3, 70)
    p, fp, gx = _dns_fields(nz, n, 3, 80)
    out3 = [torch.empty_like(p) for _ in range(3)]
    ptr = lambda ts: [t.data_ptr() for t in ts]  # noqa: E731
    geo_bytes = 4 * nel * npnp * 8
    num_bytes = m.nglobal * 8 + m.nglobal * 4 + nel * m.next * 4 + nel * npnp * 8
    ops = {
        "wave_prop": (lambda: sx.wave_prop([ptr(x) for x in us], [ptr(x) for x in uf], ptr(h), nz * n, dt,
                                           stream=sptr),
                      (2 * order + 1) * 3 * f8, "k_wave_prop"),
        "pressure_forcing": (lambda: sx.pressure_forcing(mesh, ptr(h), fp.data_ptr(), nz, n, dt, beta, stream=sptr),
                             4 * f8 + geo_bytes, "k_elem<11, PFORCE>"),
        "project": (lambda: sx.project(mesh, ptr(h), p.data_ptr(), ptr(out3), nz, n, dt, nu, ndim=3, beta=beta,
                                       stream=sptr),
                    7 * f8 + geo_bytes, "k_elem<11, PROJECT>"),
        "gradient_x": (lambda: sx.field_gradient(mesh, gx.data_ptr(), nz, n, 0, stream=sptr),
                       2 * f8 + geo_bytes // 2, "k_elem<11, GRAD>"),
        # the element-boundary values of every plane read and written once
        "smooth": (lambda: sx.field_smooth(mesh, out3[0].data_ptr(), nz, n, stream=sptr),
                   2 * nz * nel * m.next * 8 + num_bytes, "k_smooth"),
    }
    res = {}
    for name, (fn, nbytes, kern) in ops.items():
        fn()  # warm-up
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        gbs = nbytes / (ms * 1e-3) / 1e9
        res[name] = {"ms": ms, "algorithmic_bytes": int(nbytes), "achieved_gbs": gbs, "frac": gbs / peak,
                     "kernel": kern}
    out = {"workload": f"cfg5 field shape: {m.nel} elements N=10, {n} points a plane, nz={nz}",
           "field_bytes": f8, "peak_gbs": peak, "peak_kind": kind, "ops": res,
           "l2": "every operand 2.03 GB, larger than L2; no flush"}
    if check:
        from oracle import dns
        geo = dns.Geometry(m)
        # fresh inputs: run each operation once more and compare the sample
        sx.pressure_forcing(mesh, ptr(h), fp.data_ptr(), nz, n, dt, beta, stream=sptr)
        sx.project(mesh, ptr(h), p.data_ptr(), ptr(out3), nz, n, dt, nu, ndim=3, beta=beta, stream=sptr)
        torch.cuda.synchronize()
        errs, cpu = {}, {}
        for k in (0, 1, nz // 2 - 1):
            sl = slice(2 * k, 2 * k + 2)
            hh = [x[sl].cpu().numpy() for x in h]
            pp = p[sl].cpu().numpy()
            t0 = time.perf_counter()
            want_f = dns.pressure_forcing(geo, hh, dt, beta, base_mode=k)
            t1 = time.perf_counter()
            want_u = dns.project(geo, hh, pp, dt, nu, ndim=3, beta=beta, base_mode=k)
            t2 = time.perf_counter()
            cpu.setdefault("pressure_forcing", []).append((t1 - t0) / 2 * 1e3)
            cpu.setdefault("project", []).append((t2 - t1) / 2 * 1e3)
            got_f = fp[sl].cpu().numpy()
            e = np.abs(got_f - want_f).max() / np.abs(want_f).max()
            for c in range(3):
                got = out3[c][sl].cpu().numpy()
                e = max(e, np.abs(got - want_u[c]).max() / np.abs(want_u[c]).max())
            errs[str(k)] = float(e)
        out["max_rel_err_vs_oracle"] = {"modes": errs, "worst": max(errs.values()),
                                        "scale": "max |GPU - oracle| over max |oracle|, per mode"}
        out["cpu_oracle_ms_per_plane"] = {k: float(np.median(v)) for k, v in cpu.items()}
        out["gpu_ms_per_plane"] = {k: res[k]["ms"] / nz for k in ("pressure_forcing", "project")}
        out["cpu_oracle"] = "numpy restatement (oracle/dns.py), one core, modes 0, 1 and 127"
    del us, uf, h, p, fp, gx, out3
    torch.cuda.empty_cache()
    return out


def run_config5(ranks=(0,), pressure_checks=None, viscous_checks=None, reps=3):
    """One DNS elliptic step of config 5 at full size (128 x 64 quads, N = 10,
    nz = 256: 128 modes) as the ranks of an 8-GPU node take it, one rank's
    block of 16 modes at a time on this GPU (modes are independent: the step
    time of the node is the slowest rank's).  Per rank the step is, all on
    the device: the wave step (order 2) of the velocity levels, the pressure
    forcing, the pressure solve (natural walls, every mode's band factor
    resident: 16 x 6.1 GB; k = 0 singular, pinned), project, and the three
    viscous solves (lambda2 = 1/(nu dt) = 4e6 + k^2) in the mixed form.
    Inputs: seeded random velocity levels and nonlinear terms, made
    continuous by Field::smooth.  Checked against the oracle: the pressure
    solve of `pressure_checks` modes (LAPACK dpbtrf factor), the viscous
    solve of `viscous_checks` modes (oracle Jacobi PCG to 1e-14), and the
    forcing operations on those modes' planes."""
    import torch
    import semtex_b200 as sx
    from oracle import dns
    from oracle.oracle import DIRECT as O_DIRECT
    from oracle.oracle import JACPCG as O_JACPCG
    from oracle.oracle import OracleMesh, OracleSystem
    from semtex_b200.workloads import config5_block
    torch.cuda.set_device(0)
    sptr = torch.cuda.current_stream().cuda_stream
    pressure_checks = [1] if pressure_checks is None else list(pressure_checks)
    viscous_checks = [1] if viscous_checks is None else list(viscous_checks)
    out = {"workload": None, "ranks": {}}
    ptr = lambda ts: [t.data_ptr() for t in ts]  # noqa: E731
    for rank in ranks:
        b = config5_block(rank=rank)
        out["workload"] = b.name
        mv, mp = b.mesh_v, b.mesh_p
        nz, n = b.nz, mv.nplane
        t0 = time.perf_counter()
        mesh_v, mesh_p = sx.Mesh(mv), sx.Mesh(mp)
        Sp = sx.ModalMatrixSys(mesh_p, base_mode=b.base_mode, num_modes=b.num_modes, method=sx.DIRECT,
                               lambda2_modes=b.lambda2_p, betak2_modes=b.betak2)
        Sv = sx.ModalMatrixSys(mesh_v, base_mode=b.base_mode, num_modes=b.num_modes, method=sx.JACPCG,
                               lambda2_modes=b.lambda2_v, betak2_modes=b.betak2)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        order = 2
        us = [_dns_fields(nz, n, 3, 500 + 10 * rank + q) for q in range(order)]
        uf = [_dns_fields(nz, n, 3, 600 + 10 * rank + q) for q in range(order)]
        for lev in us + uf:
            for x in lev:
                sx.field_smooth(mesh_v, x.data_ptr(), nz, n, stream=sptr)
        h = [torch.empty_like(us[0][0]) for _ in range(3)]
        fp, p = torch.empty_like(h[0]), torch.zeros_like(h[0])
        uo = [torch.zeros_like(h[0]) for _ in range(3)]
        stats = {}

        def step(keep=None):
            sx.wave_prop([ptr(x) for x in us], [ptr(x) for x in uf], ptr(h), nz * n, b.dt, stream=sptr)
            sx.pressure_forcing(mesh_v, ptr(h), fp.data_ptr(), nz, n, b.dt, b.beta, b.base_mode, stream=sptr)
            if keep is not None:
                keep["h"] = [x.clone() for x in h]
                keep["fp"] = fp.clone()
            stats["p"] = Sp.solve_batched(p.data_ptr(), fp.data_ptr(), 0, nz, n, sx.FP64, stream=sptr)
            sx.project(mesh_v, ptr(h), p.data_ptr(), ptr(h), nz, n, b.dt, b.nu, ndim=3, beta=b.beta,
                       base_mode=b.base_mode, stream=sptr)
            if keep is not None:
                keep["fv"] = [x.clone() for x in h]
            for c in range(3):
                stats[f"v{c}"] = Sv.solve_batched(uo[c].data_ptr(), h[c].data_ptr(), 0, nz, n, sx.MIXED_FP32,
                                                  tol_rel=1e-12, max_refine=20, stream=sptr)

        step()  # warm-up: graphs captured, iteration counts settled
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        dof = (3 * mv.n_unique + mp.n_unique) * b.planes_solved
        res = {"modes": [b.base_mode, b.base_mode + b.num_modes - 1], "setup_s": setup_s, "ms_per_step": ms,
               "dof_solves_per_s": dof / (ms * 1e-3), "dof_solves_per_step": dof,
               "pressure_band_gb": Sp.device_bytes / 1e9,
               "viscous_iterations": [stats[f"v{c}"]["iterations_total"] for c in range(3)],
               "viscous_refinements": [stats[f"v{c}"]["refinements"] for c in range(3)],
               "viscous_final_rel_residual": max(stats[f"v{c}"]["final_rel_residual"] for c in range(3)),
               "nband_p": mp.nband, "nband_v": mv.nband}
        keep = {}
        step(keep)
        torch.cuda.synchronize()
        errs = {}
        mine_p = [k for k in pressure_checks if b.base_mode <= k < b.base_mode + b.num_modes]
        mine_v = [k for k in viscous_checks if b.base_mode <= k < b.base_mode + b.num_modes]
        if mine_p or mine_v:
            geo = dns.Geometry(mv)
        for k in sorted(set(mine_p + mine_v)):
            lo = 2 * (k - b.base_mode)
            sl = slice(lo, lo + 2)
            hh = [x[sl].cpu().numpy() for x in keep["h"]]
            pp = p[sl].cpu().numpy()
            e = {}
            want_f = dns.pressure_forcing(geo, hh, b.dt, b.beta, base_mode=k)
            got_f = keep["fp"][sl].cpu().numpy()
            e["pressure_forcing"] = float(np.abs(got_f - want_f).max() / np.abs(want_f).max())
            want_v = dns.project(geo, hh, pp, b.dt, b.nu, ndim=3, beta=b.beta, base_mode=k)
            got_v = [x[sl].cpu().numpy() for x in keep["fv"]]
            e["project"] = float(max(np.abs(g - w).max() / np.abs(w).max() for g, w in zip(got_v, want_v)))
            planes = [0] if k == 0 else [0, 1]
            if k in mine_p:
                t1 = time.perf_counter()
                osys = OracleSystem(OracleMesh(mp), 0.0, float(k * k), O_DIRECT, factor="lapack")
                uo_p = np.array([osys.solve_plane(got_f[q], None)[0] for q in planes])
                del osys
                e["pressure_solve"] = rel_err(pp[planes], uo_p)
                e["oracle_pressure_s"] = time.perf_counter() - t1
            if k in mine_v:
                osys = OracleSystem(OracleMesh(mv), float(b.lambda2_v[0]), float(k * k), O_JACPCG)
                uo_v = np.array([osys.solve_plane(got_v[0][q], None, tol_rel=1e-14, step_max=20000)[0]
                                 for q in planes])
                del osys
                e["viscous_solve"] = rel_err(uo[0][sl].cpu().numpy()[planes], uo_v)
            errs[str(k)] = e
        res["rel_err_vs_oracle"] = errs
        out["ranks"][str(rank)] = res
        del Sp, Sv, mesh_v, mesh_p, us, uf, h, fp, p, uo, keep
        torch.cuda.empty_cache()
    worst = [v for r in out["ranks"].values() for e in r["rel_err_vs_oracle"].values()
             for key, v in e.items() if key.endswith("solve")]
    out["worst_solve_err"] = max(max(x) for x in worst) if worst else None
    out["node_ms_per_step"] = max(r["ms_per_step"] for r in out["ranks"].values())
    out["note"] = ("ranks of an 8-GPU node (16 modes each), run one after another on this GPU; the node's step "
                   "time is its slowest rank's (no collective in the elliptic phase)")
    return out


def _build_request(args):
    """Build one planned serving request (a spawned worker process)."""
    spec, seed = args
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from semtex_b200.workloads import ServeSpec, serving_request
    return serving_request(ServeSpec(*spec), seed)


def run_serving(n_requests, check_oracle=True, precision="mixed", slots=4, window=48, builders=None):
    """The serving loop on the first `n_requests` of the mixed-size request
    stream (config 4: Poisson arrivals at 2000/s).  Requests are built by
    worker processes a little ahead of need (mesh and seeded forcing) and
    submitted in arrival order once their arrival time has passed and fewer
    than `window` are in the server; a request's latency is counted from its
    scheduled arrival, so the time it spends waiting outside the window is
    queueing like any other (the server admits in arrival order, and with
    `window` above slots x max_batch it always has the next requests at
    hand).  This keeps the host memory of the stream bounded: a request holds
    its forcing, the server's copy and its result only while in the window.
    The three smallest requests are checked against the oracle's FP64 direct
    solve."""
    import dataclasses
    import multiprocessing as mp
    import queue as _queue
    import semtex_b200 as sx
    from semtex_b200.workloads import serving_plan
    plan = serving_plan(n_requests)
    size = [(s.ex * s.order + 1) * (s.ey * s.order + 1) * (1 if s.modes == 1 else 2 * s.modes - 1) for s in plan]
    check = set(sorted(range(n_requests), key=lambda k: size[k])[:3]) if check_oracle else set()
    nb = builders or max(1, min(8, (os.cpu_count() or 2) - 2))
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(nb)
    prefetch = 2 * nb
    builds = []
    nbuilt = 0

    def top_up(upto):
        nonlocal nbuilt
        while nbuilt < min(n_requests, upto):
            builds.append(pool.apply_async(_build_request, ((dataclasses.astuple(plan[nbuilt]), 4),)))
            nbuilt += 1

    top_up(prefetch)
    builds[0].get(timeout=600)  # the workers are up before the clock starts
    prec = sx.MIXED_FP32 if precision == "mixed" else sx.FP64
    srv = sx.Server(slots=slots, precision=prec, tol_rel=1e-12, max_refine=30, inner_iters=12, max_batch=8)
    results = [None] * n_requests
    kept = {}
    ids = _queue.Queue()
    completed = [0]

    def waiter():
        while True:
            item = ids.get()
            if item is None:
                return
            k, rid, t_sub = item
            st, lat, u = srv.wait(rid, timeout_s=3600.0)
            results[k] = (st, t_sub + lat * 1e-3)
            if k in check:
                kept[k] = kept[k] + (u,)
            completed[0] += 1

    th = threading.Thread(target=waiter, daemon=True)
    th.start()
    dofs = 0
    try:
        start = time.perf_counter()
        for k in range(n_requests):
            top_up(k + 1 + prefetch)
            r = builds[k].get(timeout=600)
            builds[k] = None
            dofs += r.dof_solves
            while k - completed[0] >= window:
                time.sleep(0.0005)
            while time.perf_counter() - start < r.t_arrival:
                pass
            rid = srv.submit(r.mesh, r.lambda2, r.betak2, r.forcing)
            if k in check:
                kept[k] = (r,)
            ids.put((k, rid, time.perf_counter() - start))
        ids.put(None)
        th.join()
        makespan = max(t for _, t in results)
        st = srv.stats()
    finally:
        srv.close()
        pool.terminate()
    lat = np.array([(results[k][1] - plan[k].t_arrival) * 1e3 for k in range(n_requests)])
    ok = sum(1 for s, _ in results if s == sx.OK)
    statuses = {}
    for s_, _ in results:
        statuses[sx.status_string(s_)] = statuses.get(sx.status_string(s_), 0) + 1
    out = {"requests": n_requests,
           "trace": "cfg4: E_x,E_y~U[2,64], N~U{4..10}, modes~U[1,64], lambda2~logU[1e-2,1e4], Poisson 2000/s "
                    "(plan seed 4; request k's forcing from seed (4, k))",
           "slots": slots,
           "precision": ("mixed (FP32 CG / FP64 band per mode, FP64 refinement)" if precision == "mixed"
                         else "FP64 band Cholesky for every mode"),
           "latency": "scheduled arrival to result on the host",
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "makespan_s": makespan,
           "throughput_dof_solves_per_s": dofs / makespan, "requests_per_s": n_requests / makespan,
           "arrival_window_s": plan[-1].t_arrival, "in_server_window": window,
           "converged_to_1e-12": ok, "statuses": statuses, "failed": st["failed"],
           "mesh_hits": st["mesh_hits"], "system_misses": st["system_misses"],
           "evictions": st["evictions"], "max_batch": 8, "batches": st["batches"],
           "mean_batch": st["completed"] / max(st["batches"], 1),
           # per request, averaged, as the server sees them: waiting for
           # admission, mesh/system builds and factorisation, the batch solve
           "queue_ms_mean": st["queue_ms"] / n_requests, "build_ms_mean": st["build_ms"] / n_requests,
           "solve_ms_mean": st["solve_ms"] / n_requests}
    if check_oracle:
        from oracle.oracle import OracleMesh, solve_planes
        worst = 0.0
        for k in sorted(kept):
            r, u = kept[k]
            uo, _ = solve_planes(OracleMesh(r.mesh), 0.0, 1.0, r.forcing, None, lambda2_per_mode=r.lambda2)
            sp = [0] + list(range(2, r.nz)) if r.nz > 1 else [0]
            worst = max(worst, rel_err(u[sp], uo[sp])[0])
        out["rel_err_vs_oracle_3_smallest"] = worst
    return out


def run_profile(args):
    """Bounded runs of one kernel family for ncu captures (not a bench line).

    band : band sweeps of a config-2-shaped channel with 32 x 16 quads and
           nz = 16 (8 systems, ~0.5 GB of factors, larger than L2)
    band3: band sweeps of two config-3 systems (the full 64 x 64, N = 10
           mesh, modes 0 and 1: 2.9 GB of factors, the config-3 band)
    solve3: `steps` batched FP64 solves of config 3 at full size (every
           mode factored, 121 GB), for a launch list (one-pass metrics only)
    mixed: the mixed-precision batched form on the full config-2 workload
           with Jacobi systems only (no band factors, ~0.3 GB resident)
    transform: the z-direction transform of the config-2 field (nz = 64,
           82,944 points, 42 MB), forward and inverse, `steps` times each,
           a 256 MB write between calls
    transform256: the transform at config 5's length (nz = 256) on 99,840
           points (205 MB), forward and inverse, `steps` times each
    dns:   the DNS elliptic-phase operations on config 5's plane shape with
           nz = 32 (254 MB a field), `steps` + 1 launches of each
    """
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import config2
    torch.cuda.set_device(0)
    if args.profile == "transform":
        w = config2()
        d = torch.tensor(w.forcing, device="cuda")
        l2 = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
        sptr = torch.cuda.current_stream().cuda_stream
        for _ in range(max(1, args.steps)):
            for sign in (+1, -1):
                l2.zero_()
                sx.transform_z(d.data_ptr(), w.nz, w.mesh.nplane, w.mesh.nplane, sign, sptr)
        torch.cuda.synchronize()
        print(json.dumps({"profile": "transform", "nz": w.nz, "points": w.mesh.nplane}), flush=True)
        return
    if args.profile == "transform256":
        # config 5's transform length on 99,840 points (205 MB, above L2)
        x = torch.randn((256, 99840), dtype=torch.float64, device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(5))
        l2 = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
        sptr = torch.cuda.current_stream().cuda_stream
        for _ in range(max(1, args.steps)):
            for sign in (+1, -1):
                l2.zero_()
                sx.transform_z(x.data_ptr(), 256, 99840, 99840, sign, sptr)
        torch.cuda.synchronize()
        print(json.dumps({"profile": "transform256", "nz": 256, "points": 99840}), flush=True)
        return
    if args.profile == "dns":
        print(json.dumps({"profile": "dns", "run": run_dns(reps=max(1, args.steps), nz=32, check=False)}),
              flush=True)
        return
    if args.profile == "band3":
        from semtex_b200.workloads import config3_block
        w = config3_block(world=32, rank=0, modes_per_rank=2)
        method = sx.DIRECT
    elif args.profile == "solve3":
        from semtex_b200.workloads import config3_block
        w = config3_block()
        method = sx.DIRECT
    elif args.profile == "band":
        w = config2(ny=16, nz=16)
        method = sx.DIRECT
    else:
        w = config2()
        method = sx.JACPCG
    m = w.mesh
    S = sx.ModalMatrixSys(sx.Mesh(m), num_modes=w.num_modes, method=method,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    if args.band_cluster or args.band_stages or args.band_lead:
        S.tune(band_cluster=args.band_cluster, band_stages=args.band_stages, band_lead=args.band_lead)
    f_src = torch.tensor(w.forcing, device="cuda")
    f = torch.empty_like(f_src)
    u = torch.zeros_like(f_src)
    sptr = torch.cuda.current_stream().cuda_stream
    for _ in range(max(1, args.steps)):
        f.copy_(f_src)
        if args.profile in ("band", "band3", "solve3"):
            S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, sx.FP64, stream=sptr)
        else:
            S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, sx.MIXED_FP32,
                            tol_rel=args.tol, max_refine=20, stream=sptr)
    ms = None
    if args.profile in ("band", "band3"):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        S.profile_band_sweeps(max(1, args.steps), sptr)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / max(1, args.steps)
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile, "workload": w.name, "nband": m.nband,
                      "nsolve": m.nsolve, "modes": w.num_modes, "sweep_launch_ms": ms}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the extra keys (config 2, multi-mesh batch, z-transform, DNS operations)")
    ap.add_argument("--serve-only", type=int, default=0, metavar="N",
                    help="run only the serving loop on the first N requests of the config-4 stream "
                         "and print its JSON (not a bench line)")
    ap.add_argument("--serve-precision", choices=["mixed", "fp64"], default="mixed",
                    help="serving loop: mixed (per mode FP32 CG or FP64 band) or fp64 (band for every mode)")
    ap.add_argument("--serve-slots", type=int, default=8, help="serving loop: requests on the device at once")
    ap.add_argument("--serve-requests", type=int, default=1000,
                    help="requests of the mixed-size serving trace to run (0 skips it)")
    ap.add_argument("--config5-ranks", default=None, metavar="R,R,...",
                    help="run only the config-5 elliptic step for these ranks of the 8-GPU split, checking "
                         "pressure modes 0, 1, 2, 31, 127 and viscous modes 1, 127 where they fall, and print "
                         "its JSON (not a bench line)")
    ap.add_argument("--tol", type=float, default=1e-12,
                    help="FP64 relative residual at which the mixed form stops")
    ap.add_argument("--profile", choices=["band", "band3", "solve3", "mixed", "transform", "transform256", "dns"],
                    default=None,
                    help="bounded run of one kernel family for ncu (no bench line)")
    ap.add_argument("--band-cluster", type=int, default=0, help="--profile band*: CTAs per cluster (0: default)")
    ap.add_argument("--band-stages", type=int, default=0, help="--profile band*: ring depth (0: default)")
    ap.add_argument("--band-lead", type=int, default=0, help="--profile band*: leader share K (1: none; 0: default)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.serve_only > 0:
        print(json.dumps({"serving_only": run_serving(args.serve_only, check_oracle=False,
                                                      precision=args.serve_precision, slots=args.serve_slots)}),
              flush=True)
        return
    if args.config5_ranks:
        ranks = tuple(int(r) for r in args.config5_ranks.split(","))
        print(json.dumps({"config5_full": run_config5(ranks, pressure_checks=(0, 1, 2, 31, 127),
                                                      viscous_checks=(1, 127))}), flush=True)
        return
    if args.profile:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

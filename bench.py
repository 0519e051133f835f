#!/usr/bin/env python
"""Benchmark: per-Fourier-mode Helmholtz solve (semtex Field::solve) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (N=1): the batched 2-D x Fourier channel -- [0,2pi] x [0,1],
32 x 32 quads jittered +-15 % (seed 2), N = 8, nz = 64 planes (modes 0..31,
63 planes solved, Nyquist skipped), beta = 1, lambda2 = 1/(nu dt) = 1e6,
Dirichlet walls, periodic in x, seeded Gaussian Fourier forcing decaying as
e^{-k/8}.  A step is one solve of every plane of every mode.

Metric: Helmholtz DoF-solves/s (unique nodes per plane x planes solved /
seconds) at <= 1e-10 relative error against the FP64 solve.  ``value`` is the
best batched form on device-resident inputs; ``e2e`` the same through the
host-pointer C-ABI call with the host<->device copies inside the timed region.
The plain FP64 mode-by-mode form is reported beside it.

Multi-GPU (torchrun): Fourier modes are independent, so each rank solves its
own block of 32 modes (weak scaling, no collective in the data path); the
timing is the max over ranks.

``--impl reference`` times the reference algorithm on the host cores (the
C oracle port, one process per core over modes) on the same workload.
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

def _oracle_worker(args):
    """Factor + solve one mode's planes with the oracle (runs in a spawned
    process).  Returns (solve seconds per repetition, planes, solution)."""
    mode, reps, seed = args
    sys.path.insert(0, ROOT)
    from oracle.oracle import DIRECT, OracleMesh, OracleSystem
    from semtex_b200.workloads import config2
    w = config2(seed=seed)
    om = OracleMesh(w.mesh)
    sysm = OracleSystem(om, float(w.lambda2[mode]), float(w.betak2[mode]), DIRECT)
    planes = [0] if mode == 0 else [2 * mode, 2 * mode + 1]
    times, sols = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        sols = [sysm.solve_plane(w.forcing[p], None)[0] for p in planes]
        times.append(time.perf_counter() - t0)
    return float(np.median(times)), len(planes), sols


def cpu_baseline_sample(reps=2):
    """One mode (k = 1, two planes) of the workload solved by the oracle on
    one core; factorisation untimed (set-up), solve timed."""
    t, planes, sols = _oracle_worker((1, reps, 2))
    from semtex_b200.workloads import config2
    w = config2()
    return w.dof_per_plane * planes / t, sols, w


def run_reference(args, rank, world):
    if rank != 0:
        return
    import multiprocessing as mp
    from semtex_b200.workloads import config2
    w = config2()
    cores = os.cpu_count() or 1
    nm = w.num_modes
    nproc = max(1, min(cores, nm))
    modes = list(range(nproc))
    ctx = mp.get_context("spawn")
    with ctx.Pool(nproc) as pool:
        res = pool.map(_oracle_worker, [(m, max(1, args.steps), 2) for m in modes])
    # every worker solved its mode concurrently; a step is the slowest one
    step_s = max(r[0] for r in res)
    planes = sum(r[1] for r in res)
    value = w.dof_per_plane * planes / step_s
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": w.name, "planes_solved": w.planes_solved,
                   "dof_per_plane": w.dof_per_plane, "sample_modes": modes},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port",
                         "sample": f"modes {modes[0]}..{modes[-1]} ({planes} planes) of {w.name}, "
                                   f"one process per core, solve timed, factor untimed"},
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


def _ncu_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` on this workload, from
    the committed ncu summary profiles/<kernel>_*.md (its line
    `dram_bytes_per_launch: N`); None when there is none."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for name in sorted(os.listdir(d)):
        if not (name.startswith(kernel + "_") and name.endswith(".md")):
            continue
        with open(os.path.join(d, name)) as fh:
            for line in fh:
                if line.strip().startswith("dram_bytes_per_launch:"):
                    return int(line.split(":", 1)[1].strip().split()[0])
    return None


def run_ours(args, rank, world):
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import config2

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sx.lib.sx_set_device(dev.index)
    dist = None
    if world > 1:
        import torch.distributed as dist
    w = config2(seed=2)
    m = w.mesh
    nz = w.nz
    nmodes = w.num_modes
    base = rank * nmodes
    # each rank owns modes [base, base + nmodes); betak2 = (beta k)^2
    bk2 = (np.arange(base, base + nmodes, dtype=np.float64) * w.beta) ** 2
    mesh = sx.Mesh(m)
    t0 = time.perf_counter()
    S = sx.ModalMatrixSys(mesh, base_mode=base, num_modes=nmodes, method=sx.DIRECT,
                          lambda2_modes=w.lambda2, betak2_modes=bk2)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    planes_solved = nz - 1 if base == 0 else nz
    dofs = w.dof_per_plane * planes_solved
    stride = m.nplane
    f_src = torch.tensor(w.forcing, device=dev)
    f_work = torch.empty_like(f_src)
    u_dev = torch.zeros_like(f_src)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def restore():
        f_work.copy_(f_src)  # the solve overwrites its forcing (src/field.cpp:525-526)

    def step_batched():
        S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)

    def step_plain():
        S.solve_device(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, stream=sptr)

    # 256 MB written between timed steps: evicts the 126 MB L2
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

    # plain FP64, mode by mode (reference-compatible form)
    restore()
    step_plain()
    torch.cuda.synchronize()
    u_plain = u_dev.cpu().numpy().copy()
    ms_plain = timed(step_plain, max(1, min(args.steps, 3)), 1)

    # batched FP64, its band-sweep cluster size picked by the autotuner on
    # this data (untimed set-up)
    tune64 = S.autotune(u_dev.data_ptr(), f_src.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)
    clk = ClockSampler(dev.index)
    restore()
    step_batched()
    torch.cuda.synchronize()
    u_batched = u_dev.cpu().numpy().copy()
    clk.start()
    ms_batched = timed(step_batched, args.steps, args.warmup)

    restore()
    st_b = S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)
    launches_fp64 = int(st_b["kernel_launches"])

    # batched mixed precision: FP32 CG inner iterations, FP64 refinement
    mixed_stats = {}

    def step_mixed():
        mixed_stats.update(S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride,
                                           sx.MIXED_FP32, tol_rel=args.tol, max_refine=20,
                                           stream=sptr))

    tunemx = S.autotune(u_dev.data_ptr(), f_src.data_ptr(), 0, nz, stride, sx.MIXED_FP32,
                        tol_rel=args.tol, max_refine=20, stream=sptr)
    restore()
    step_mixed()
    torch.cuda.synchronize()
    u_mixed = u_dev.cpu().numpy().copy()
    sp = [0] + list(range(2, nz)) if base == 0 else list(range(nz))
    mixed_err = rel_err(u_mixed[sp], u_batched[sp])
    ms_mixed = timed(step_mixed, args.steps, args.warmup)
    clocks = clk.stop()
    mixed_ok = max(mixed_err) <= 1e-10
    if dist is not None:
        t = torch.tensor([0.0 if mixed_ok else 1.0], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mixed_ok = t.item() == 0.0
    # headline: the fastest batched form that meets the 1e-10 bar
    use_mixed = mixed_ok and ms_mixed < ms_batched
    head_prec = sx.MIXED_FP32 if use_mixed else sx.FP64
    ms_head = ms_mixed if use_mixed else ms_batched
    launches_per_step = int(mixed_stats.get("kernel_launches", 0)) if use_mixed else launches_fp64

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
    reps = max(3, args.steps)
    # batched FP64's dominant kernel: the banded sweeps.  Algorithmic bytes
    # per launch: the band factor read by each sweep (forward and backward)
    # + each sweep's RHS read and write.
    restore()
    S.solve_batched(u_dev.data_ptr(), f_work.data_ptr(), 0, nz, stride, sx.FP64, stream=sptr)
    sweep_ms = kernel_ms(lambda r: S.profile_band_sweeps(r, sptr), reps)
    band_bytes = 0
    for mode in range(nmodes):
        P = 1 if (base + mode) == 0 else 2
        band_bytes += 2 * m.nsolve * m.nband * 8 + 2 * 2 * P * m.nsolve * 8
    band_gbs = band_bytes / (sweep_ms * 1e-3) / 1e9
    roof_band = {"bound": "hbm", "kernel": "k_band_sweep", "achieved": band_gbs, "peak": hbm,
                 "unit": "GB/s", "frac": band_gbs / hbm, "peak_kind": peak_kind,
                 "traffic": _ncu_traffic("k_band_sweep"), "algorithmic_bytes_per_launch": band_bytes,
                 "launch_ms": sweep_ms}
    # the mixed form's dominant kernel: one fused FP32 CG iteration (k_cg)
    # over every plane.  Algorithmic bytes per launch: r, s, p, d read and
    # written at every node, A u (element boundary slots + interior nodes)
    # read and written, per plane solved; + the preconditioner columns and the
    # FP32 geometry read once.
    restore()
    step_mixed()
    cg_ms = kernel_ms(lambda r: S.profile_mixed_iterations(r, sptr), reps)
    nn = m.np * m.np
    npts = m.nglobal + m.nel * (m.np - 2) ** 2
    cg_bytes = 4 * planes_solved * (8 * npts + 2 * m.nel * nn) + 4 * npts * nmodes + 16 * m.nel * nn
    cg_gbs = cg_bytes / (cg_ms * 1e-3) / 1e9
    roof_cg = {"bound": "hbm", "kernel": "k_cg", "achieved": cg_gbs, "peak": hbm, "unit": "GB/s",
               "frac": cg_gbs / hbm, "peak_kind": peak_kind, "traffic": _ncu_traffic("k_cg"),
               "algorithmic_bytes_per_launch": cg_bytes, "launch_ms": cg_ms}
    roofline = roof_cg if use_mixed else roof_band

    # end to end through the host-pointer C-ABI call, pinned buffers
    f_host = torch.tensor(w.forcing).pin_memory()
    u_host = torch.empty_like(f_host).pin_memory()
    fh, uh = f_host.numpy(), u_host.numpy()
    for _ in range(args.warmup):
        S.solve_batched_host(fh, out=uh, precision=head_prec, tol_rel=args.tol, max_refine=20)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        S.solve_batched_host(fh, out=uh, precision=head_prec, tol_rel=args.tol, max_refine=20)
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    total_dofs = dofs * world
    value = total_dofs / (ms_head * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_head, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if use_mixed else "f64",
        "data": "synthetic (seeded Gaussian Fourier forcing)",
        "config": {"workload": w.name, "elements": m.nel, "order": m.np - 1, "nz": nz,
                   "modes_per_gpu": nmodes, "planes_solved_per_gpu": planes_solved,
                   "dof_per_plane": w.dof_per_plane, "nglobal": m.nglobal, "nsolve": m.nsolve,
                   "nband": m.nband, "lambda2": float(w.lambda2[0]),
                   "form": "batched mixed (FP32 PCG + FP64 refinement)" if use_mixed else "batched FP64",
                   "parallelism": f"modes split over {world} GPU(s), no collective",
                   "l2": "working set (factors %.1f GB) >> L2" % (S.device_bytes / 1e9)},
        "plain_fp64": {"value": total_dofs / (ms_plain * 1e-3), "ms_per_step": ms_plain},
        "batched_fp64": {"value": total_dofs / (ms_batched * 1e-3), "ms_per_step": ms_batched,
                         "rel_err_vs_plain": rel_err(u_batched[[0] + list(range(2, nz))],
                                                     u_plain[[0] + list(range(2, nz))])},
        "batched_mixed": {"value": total_dofs / (ms_mixed * 1e-3), "ms_per_step": ms_mixed,
                          "rel_err_vs_fp64": mixed_err, "meets_1e-10": mixed_ok,
                          "refinements": mixed_stats.get("refinements"),
                          "inner_iterations": mixed_stats.get("iterations_max"),
                          "final_rel_residual": mixed_stats.get("final_rel_residual")},
        "speedup_mixed_vs_plain": ms_plain / ms_mixed,
        "autotuned": {"batched_fp64": tune64, "batched_mixed": tunemx},
        "setup_s": setup_s,
        "roofline": roofline,
        "roofline_other_form": roof_band if use_mixed else roof_cg,
        "e2e": {"value": total_dofs / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": int(fh.nbytes), "d2h_bytes_per_step": int(uh.nbytes),
                "ms_per_step": e2e_s * 1e3, "call": "sx_field_solve_batched_host (pinned)"},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        # CPU baseline + full-size parity: the oracle on mode 1 (one core)
        cpu_val, sols, _ = cpu_baseline_sample()
        line["cpu_baseline"] = {"value": cpu_val, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"mode 1 (planes 2,3) of {w.name}; oracle C port, "
                                          "factor untimed, median of 2 solves"}
        l2a, mxa = rel_err(u_batched[2], sols[0])
        l2b, mxb = rel_err(u_batched[3], sols[1])
        line["batched_fp64"]["rel_err_vs_oracle_mode1"] = [max(l2a, l2b), max(mxa, mxb)]
    if rank == 0 and world == 1:
        line["multi_mesh"] = run_multi()
        line["transform_z"] = run_transform()
        if not args.no_config3:
            line["config3_full"] = run_config3_full()
    if rank == 0 and world == 1 and args.serve_requests > 0:
        line["serving"] = run_serving(args.serve_requests, check_oracle=not args.no_cpu)
    if rank == 0:
        print(json.dumps(line), flush=True)


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


def run_config3_full(reps=3):
    """Config 3 at full size -- 64 x 64 jittered quads, N = 10, nz = 128
    (127 planes, 410,240 DoF each), lambda2 log-uniform in [1e-2, 1e4] over
    the modes, manufactured solution: every mode factored (FP64 band
    Cholesky, ~120 GB resident), then the batched FP64 form and the mixed
    form on the same systems (the mixed form routes the ill-conditioned
    modes to the band solve and the rest to the FP32 iterations).  CUDA
    events, median of `reps` after a warm-up; the working set is far above
    L2."""
    import torch
    import semtex_b200 as sx
    from semtex_b200.workloads import config3
    torch.cuda.set_device(0)
    w = config3()
    m = w.mesh
    t0 = time.perf_counter()
    S = sx.ModalMatrixSys(sx.Mesh(m), num_modes=w.num_modes, method=sx.DIRECT, lambda2_modes=w.lambda2,
                          betak2_modes=w.betak2)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    f0 = torch.tensor(w.forcing, device="cuda")
    f = torch.empty_like(f0)
    u = torch.zeros_like(f0)
    st = torch.cuda.current_stream().cuda_stream

    def timed(prec):
        ts, stats = [], None
        for k in range(reps + 1):
            f.copy_(f0)  # the band solve overwrites its forcing
            u.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            stats = S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, prec, 1e-12, max_refine=30,
                                    stream=st)
            e1.record()
            e1.synchronize()
            if k:
                ts.append(e0.elapsed_time(e1))
        return float(np.median(ts)), stats, u.cpu().numpy()

    f.copy_(f0)
    tune = S.autotune(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, sx.FP64, stream=st)
    t64, s64, u64 = timed(sx.FP64)
    tmx, smx, umx = timed(sx.MIXED_FP32)
    sp = [0] + list(range(2, w.nz))
    dofs = w.dof_per_plane * len(sp)
    ex = w.exact[sp]
    out = {"workload": w.name, "dof_per_plane": w.dof_per_plane, "planes_solved": len(sp),
           "nsolve": m.nsolve, "nband": m.nband, "setup_s_factor_all_modes": setup_s,
           "factor_bytes": int(S.device_bytes),
           "fp64_ms": t64, "fp64_dof_solves_per_s": dofs / (t64 * 1e-3),
           "mixed_ms": tmx, "mixed_dof_solves_per_s": dofs / (tmx * 1e-3),
           "mixed_planes_to_band": smx["planes_direct"], "mixed_refinements": smx["refinements"],
           "mixed_vs_fp64_rel_err": rel_err(umx[sp], u64[sp]),
           "fp64_vs_manufactured_max_rel_err": float(np.abs(u64[sp] - ex).max() / np.abs(ex).max()),
           "speedup_mixed_vs_fp64": t64 / tmx, "autotuned_fp64": tune}
    del S, f0, f, u
    torch.cuda.empty_cache()
    return out


def run_serving(n_requests, check_oracle=True):
    """The serving loop on a bounded sample of the mixed-size request stream
    (config 4): requests are submitted at their Poisson arrival times
    (2000/s) to a mixed-precision server with 4 slots, each solving up to 8
    requests per multi-mesh batch; latency is submit to result on the host,
    as the server measures it.  The smallest requests
    are checked against the oracle's FP64 direct solve."""
    import semtex_b200 as sx
    from semtex_b200.workloads import serving_trace
    t0 = time.perf_counter()
    trace = serving_trace(n_requests)
    prep_s = time.perf_counter() - t0
    srv = sx.Server(slots=4, precision=sx.MIXED_FP32, tol_rel=1e-12, max_refine=30, inner_iters=12,
                    max_batch=8)
    try:
        ids = []
        start = time.perf_counter()
        for r in trace:
            while time.perf_counter() - start < r.t_arrival:
                pass
            ids.append(srv.submit(r.mesh, r.lambda2, r.betak2, r.forcing))
        res = [srv.wait(i, timeout_s=600.0) for i in ids]
        makespan = time.perf_counter() - start
        st = srv.stats()
    finally:
        srv.close()
    lat = np.array([lt for _, lt, _ in res])
    ok = sum(1 for s, _, _ in res if s == sx.OK)
    dofs = sum(r.dof_solves for r in trace)
    out = {"requests": n_requests, "trace": "cfg4: E_x,E_y~U[2,64], N~U{4..10}, modes~U[1,64], "
                                            "lambda2~logU[1e-2,1e4], Poisson 2000/s, seed 4",
           "slots": 4, "precision": "mixed (FP32 CG / FP64 band per mode, FP64 refinement)",
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "makespan_s": makespan,
           "throughput_dof_solves_per_s": dofs / makespan, "requests_per_s": n_requests / makespan,
           "converged_to_1e-12": ok, "mesh_hits": st["mesh_hits"], "system_misses": st["system_misses"],
           "evictions": st["evictions"], "host_prep_s_untimed": prep_s,
           "max_batch": 8, "batches": st["batches"],
           "mean_batch": st["completed"] / max(st["batches"], 1),
           # per request, averaged: waiting for admission, mesh/system builds
           # and factorisation, the batch solve with its copies
           "queue_ms_mean": st["queue_ms"] / n_requests, "build_ms_mean": st["build_ms"] / n_requests,
           "solve_ms_mean": st["solve_ms"] / n_requests}
    if check_oracle:
        from oracle.oracle import OracleMesh, solve_planes
        worst = 0.0
        for k in sorted(range(n_requests), key=lambda k: trace[k].dof_solves)[:3]:
            r, u = trace[k], res[k][2]
            uo, _ = solve_planes(OracleMesh(r.mesh), 0.0, 1.0, r.forcing, None, lambda2_per_mode=r.lambda2)
            sp = [0] + list(range(2, r.nz)) if r.nz > 1 else [0]
            worst = max(worst, rel_err(u[sp], uo[sp])[0])
        out["rel_err_vs_oracle_3_smallest"] = worst
    return out


def run_profile(args):
    """Bounded runs of one kernel family for ncu captures (not a bench line).

    band : band sweeps of a config-2-shaped channel with 32 x 16 quads and
           nz = 16 (8 systems, ~0.5 GB of factors, larger than L2)
    mixed: the mixed-precision batched form on the full config-2 workload
           with Jacobi systems only (no band factors, ~0.3 GB resident)
    transform: the z-direction transform of the config-2 field (nz = 64,
           82,944 points, 42 MB), forward and inverse, `steps` times each,
           a 256 MB write between calls
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
    if args.profile == "band":
        w = config2(ny=16, nz=16)
        method = sx.DIRECT
    else:
        w = config2()
        method = sx.JACPCG
    m = w.mesh
    S = sx.ModalMatrixSys(sx.Mesh(m), num_modes=w.num_modes, method=method,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    f_src = torch.tensor(w.forcing, device="cuda")
    f = torch.empty_like(f_src)
    u = torch.zeros_like(f_src)
    sptr = torch.cuda.current_stream().cuda_stream
    for _ in range(max(1, args.steps)):
        f.copy_(f_src)
        if args.profile == "band":
            S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, sx.FP64, stream=sptr)
        else:
            S.solve_batched(u.data_ptr(), f.data_ptr(), 0, w.nz, m.nplane, sx.MIXED_FP32,
                            tol_rel=args.tol, max_refine=20, stream=sptr)
    if args.profile == "band":
        S.profile_band_sweeps(max(1, args.steps), sptr)
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile, "workload": w.name, "nband": m.nband,
                      "nsolve": m.nsolve, "modes": w.num_modes}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-config3", action="store_true",
                    help="skip config 3 at full size (121 GB of band factors; keep it out of profiler runs)")
    ap.add_argument("--serve-only", type=int, default=0, metavar="N",
                    help="run only the serving loop on the first N requests of the config-4 stream "
                         "and print its JSON (not a bench line)")
    ap.add_argument("--serve-requests", type=int, default=32,
                    help="requests of the mixed-size serving trace to run (0 skips it)")
    ap.add_argument("--tol", type=float, default=1e-12,
                    help="FP64 relative residual at which the mixed form stops")
    ap.add_argument("--profile", choices=["band", "mixed", "transform"], default=None,
                    help="bounded run of one kernel family for ncu (no bench line)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.serve_only > 0:
        print(json.dumps({"serving_only": run_serving(args.serve_only, check_oracle=False)}), flush=True)
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

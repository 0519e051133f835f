"""GPU tests of the batched forms.

* batched FP64 (all modes per launch, captured graph) equals the plain
  mode-by-mode form to rounding (rel <= 1e-13), for every band-sweep
  cluster size;
* the mixed-precision form (FP32 Jacobi-PCG inner iterations, FP64
  refinement) matches the oracle's FP64 direct solve within 1e-10 relative
  L2 and max norm, on the config-2 shape and on the reference goldens;
* results are deterministic (bitwise equal on repeat).
"""
import numpy as np
import pytest

from oracle.oracle import OracleMesh, solve_planes
from tests.problems import PROBLEMS_2D, build_2d, golden_ok

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-10


def rel_errs(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return (np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300),
            np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def solved_planes(nz):
    return [0] + list(range(2, nz)) if nz > 1 else [0]


def _setup(sx, w, method=0):
    mesh = sx.Mesh(w.mesh)
    S = sx.ModalMatrixSys(mesh, num_modes=w.num_modes, method=method,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    return mesh, S


def _run_device(torch, S, w, batched=True, precision=0, tol=1e-12, bc=None):
    f = torch.tensor(w.forcing, device="cuda")
    u = torch.zeros_like(f)
    b = None if bc is None else torch.tensor(bc, device="cuda")
    bptr = 0 if b is None else b.data_ptr()
    if batched:
        st = S.solve_batched(u.data_ptr(), f.data_ptr(), bptr, w.nz, w.mesh.nplane, precision, tol,
                             max_refine=40)
    else:
        st = S.solve_device(u.data_ptr(), f.data_ptr(), bptr, w.nz, w.mesh.nplane)
    torch.cuda.synchronize()
    S.status()
    return u.cpu().numpy(), st


@pytest.mark.parametrize("cluster,stages", [(0, 0), (1, 0), (2, 0), (3, 0), (5, 0), (2, 2), (5, 2), (3, 3), (1, 1),
                                            (4, 1)])
def test_batched_fp64_equals_plain(sx, torch, cluster, stages):
    """Every band-sweep cluster size and ring depth (tiles in flight per
    CTA) gives the plain form's answer to rounding."""
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=8, np_=9, nz=12, lam=1e6, seed=11)
    _, S = _setup(sx, w)
    S.tune(band_cluster=cluster, band_stages=stages)
    up, _ = _run_device(torch, S, w, batched=False)
    ub, st = _run_device(torch, S, w, batched=True)
    sp = solved_planes(w.nz)
    l2, mx = rel_errs(ub[sp], up[sp])
    assert l2 <= 1e-13 and mx <= 1e-13, (cluster, l2, mx)
    assert st["planes_solved"] == w.nz - 1


@pytest.mark.parametrize("cluster,stages,lead", [(2, 2, 2), (3, 2, 3), (3, 4, 4), (4, 2, 5), (4, 1, 8),
                                                  (5, 2, 6), (2, 1, 3), (4, 2, 1)])
def test_batched_fp64_leader_share_equals_plain(sx, torch, cluster, stages, lead):
    """The cluster leader working a step ahead on its share of the band tiles
    (the last of every `lead` tiles j >= 2; 1 = none) gives the plain form's
    answer to rounding, for every cluster size and ring depth: a band of
    9 tiles per block column, 54 block columns, so every CTA owns tiles."""
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=24, ny=10, np_=9, nz=8, lam=1e4, seed=11)
    _, S = _setup(sx, w)
    S.tune(band_cluster=cluster, band_stages=stages, band_lead=lead)
    up, _ = _run_device(torch, S, w, batched=False)
    ub, st = _run_device(torch, S, w, batched=True)
    sp = solved_planes(w.nz)
    l2, mx = rel_errs(ub[sp], up[sp])
    assert l2 <= 1e-13 and mx <= 1e-13, (cluster, lead, l2, mx)
    uo, _ = solve_planes(OracleMesh(w.mesh), 0.0, 1.0, w.forcing, None, lambda2_per_mode=w.lambda2)
    l2, mx = rel_errs(ub[sp], uo[sp])
    assert l2 <= 1e-12 and mx <= 1e-12, (cluster, lead, l2, mx)


@pytest.mark.parametrize("lam,inner", [(1e6, 12), (1e3, 30)])
def test_mixed_matches_oracle(sx, torch, lam, inner):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=6, ny=5, np_=9, nz=6, lam=lam, seed=5)
    _, S = _setup(sx, w)
    S.tune(inner_iters=inner, mixed_route=sx.ROUTE_CG)
    um, st = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32, tol=1e-12)
    assert st["planes_direct"] == 0
    assert st["final_rel_residual"] <= 1e-12
    uo, _ = solve_planes(OracleMesh(w.mesh), 0.0, 1.0, w.forcing, None,
                         lambda2_per_mode=w.lambda2)
    sp = solved_planes(w.nz)
    l2, mx = rel_errs(um[sp], uo[sp])
    assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (lam, l2, mx, st)


@pytest.mark.parametrize("name", ["helmholtz1", "laplace1", "laplace4"])
def test_mixed_regress_goldens(sx, torch, name):
    m, p, f, bc, exact = build_2d(name)
    from semtex_b200.workloads import Workload
    w = Workload(name, m, 1, 0.0, np.array([p["lambda2"]]), np.array([0.0]), f)
    _, S = _setup(sx, w)
    S.tune(inner_iters=200, mixed_route=sx.ROUTE_CG)
    um, st = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32, tol=1e-13, bc=bc)
    uo, _ = solve_planes(OracleMesh(m), p["lambda2"], 0.0, f, bc)
    l2, mx = rel_errs(um, uo)
    assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (name, l2, mx, st)
    err = np.abs(um[0] - exact).max()
    if p["golden"] is not None:
        assert golden_ok(err, p["golden"]), err


def test_mixed_deterministic(sx, torch):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=6, ny=6, np_=7, nz=8, lam=1e5, seed=9)
    _, S = _setup(sx, w)
    S.tune(mixed_route=sx.ROUTE_CG)
    a, _ = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32)
    b, _ = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32)
    assert np.array_equal(a, b)


def test_mixed_route_band_equals_fp64(sx, torch):
    """Modes routed to the band Cholesky run the batched FP64 form's kernels:
    their planes equal the FP64 form's bit for bit."""
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=8, np_=9, nz=12, lam=1e6, seed=11)
    _, S = _setup(sx, w)
    ub, _ = _run_device(torch, S, w, batched=True)
    S.tune(mixed_route=sx.ROUTE_BAND)
    um, st = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32)
    sp = solved_planes(w.nz)
    assert st["planes_direct"] == len(sp) == st["planes_solved"]
    assert np.array_equal(um[sp], ub[sp])


@pytest.mark.parametrize("method", ["direct", "auto"])
def test_mixed_hybrid_route_vs_oracle(sx, torch, method):
    """lambda2 from 1e-2 to 1e6 across the modes: the ill-conditioned modes
    go to the FP64 band Cholesky, the others to the FP32 iterations, both in
    one call; every plane meets the 1e-10 bar against the oracle."""
    from semtex_b200.workloads import small_channel
    # 20 x 12 elements at N = 8: modes 0-5 (lambda2 <= 5.2e3) to the band,
    # predicted CG / band time 2.7 on mode 5; modes 6-7 to CG, ratio 0.76
    w = small_channel(nx=20, ny=12, np_=9, nz=16, lam=1e6, seed=13)
    w.lambda2 = np.logspace(-2, 6, w.num_modes)
    mesh = sx.Mesh(w.mesh)
    S = sx.ModalMatrixSys(mesh, num_modes=w.num_modes, method=sx.DIRECT if method == "direct" else sx.AUTO,
                          lambda2_modes=w.lambda2, betak2_modes=w.betak2)
    um, st = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32, tol=1e-12)
    sp = solved_planes(w.nz)
    assert 0 < st["planes_direct"] < len(sp), st
    assert st["planes_solved"] == len(sp)
    uo, _ = solve_planes(OracleMesh(w.mesh), 0.0, 1.0, w.forcing, None, lambda2_per_mode=w.lambda2)
    for p in sp:
        l2, mx = rel_errs(um[p], uo[p])
        assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (p, l2, mx, st)


def test_autotune_first_call_finds_clusters(sx, torch):
    """The autotuner as the first band-sweep call of the process-fresh
    system: it still finds (and times) several cluster schedules."""
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=8, np_=10, nz=12, lam=1e6, seed=29)
    _, S = _setup(sx, w)
    f = torch.tensor(w.forcing, device="cuda")
    u = torch.zeros_like(f)
    r = S.autotune(u.data_ptr(), f.data_ptr(), 0, w.nz, w.mesh.nplane, sx.FP64)
    assert r["trials"] > 1 and r["band_cluster"] >= 1, r


def test_autotune_keeps_results(sx, torch):
    """The autotuner picks a schedule among the candidates, leaves the
    forcing untouched, and the batched forms give the same answers after it:
    bit for bit for FP64 (the cluster size does not change the arithmetic),
    within the mixed form's bar for the mixed form."""
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=8, ny=8, np_=9, nz=12, lam=1e6, seed=11)
    _, S = _setup(sx, w)
    ub, _ = _run_device(torch, S, w, batched=True)
    f = torch.tensor(w.forcing, device="cuda")
    u = torch.zeros_like(f)
    r64 = S.autotune(u.data_ptr(), f.data_ptr(), 0, w.nz, w.mesh.nplane, sx.FP64)
    assert r64["trials"] >= 1 and r64["band_cluster"] >= 1 and r64["ms"] > 0.0
    assert r64["band_stages"] in (1, 2, 3, 4)
    assert np.array_equal(f.cpu().numpy(), w.forcing)
    ub2, _ = _run_device(torch, S, w, batched=True)
    sp = solved_planes(w.nz)
    assert np.array_equal(ub2[sp], ub[sp])
    rm = S.autotune(u.data_ptr(), f.data_ptr(), 0, w.nz, w.mesh.nplane, sx.MIXED_FP32)
    assert rm["inner_iters"] in (8, 12, 16, 24)
    um, st = _run_device(torch, S, w, batched=True, precision=sx.MIXED_FP32)
    l2, mx = rel_errs(um[sp], ub[sp])
    assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (l2, mx, st, rm)


def test_batched_host_entry(sx, torch):
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=5, ny=4, np_=6, nz=6, lam=10.0, seed=3)
    _, S = _setup(sx, w)
    ud, _ = _run_device(torch, S, w, batched=True)
    uh = S.solve_batched_host(w.forcing)
    sp = solved_planes(w.nz)
    assert np.array_equal(uh[sp], ud[sp])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_host_entry_pipelined(sx, torch, precision):
    """More than 16 modes: the host entry solves chunks of 16 modes with
    their copies overlapped; every plane matches the single device-side
    batched solve (FP64: to rounding; mixed: within the 1e-10 bar), and the
    Nyquist plane is left as the caller passed it."""
    from semtex_b200.workloads import small_channel
    w = small_channel(nx=4, ny=3, np_=6, nz=40, lam=1e5, seed=23)
    _, S = _setup(sx, w)
    prec = sx.FP64 if precision == "fp64" else sx.MIXED_FP32
    ud, _ = _run_device(torch, S, w, batched=True, precision=prec, tol=1e-12)
    out = np.full_like(w.forcing, 7.0)
    uh = S.solve_batched_host(w.forcing, out=out, precision=prec, tol_rel=1e-12, max_refine=40)
    sp = solved_planes(w.nz)
    l2, mx = rel_errs(uh[sp], ud[sp])
    tol = 1e-13 if precision == "fp64" else MIXED_TOL
    assert l2 <= tol and mx <= tol, (precision, l2, mx)
    assert np.all(uh[1] == 7.0)
    assert S.last_stats["planes_solved"] == len(sp)

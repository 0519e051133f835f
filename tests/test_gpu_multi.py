"""GPU tests of the multi-mesh batch (sx_batch_solve).

Members differ in mesh, element count, order, mode count and lambda2.

* mixed precision: every member's planes meet the 1e-10 bar against the
  oracle's FP64 direct solve, and agree within it with the same member
  solved alone by the single-mesh batched form;
* FP64: every member equals its single-mesh batched FP64 solve bit for bit
  (the band sweeps of all members share one launch; each system's
  arithmetic is unchanged);
* modes routed to the band Cholesky and to the FP32 iterations in one call;
* replaying the captured graphs on new forcing values gives the new answer.
"""
import numpy as np
import pytest

from oracle.oracle import OracleMesh, solve_planes

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-10


def rel_errs(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return (np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300),
            np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def solved_planes(nz):
    return [0] + list(range(2, nz)) if nz > 1 else [0]


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _workloads():
    from semtex_b200.workloads import small_channel
    # orders 8, 5, 8, 10; 30, 12, 28, 9 elements; 3, 5, 2, 1 modes
    return [small_channel(nx=6, ny=5, np_=9, nz=6, lam=1e6, seed=5),
            small_channel(nx=4, ny=3, np_=6, nz=10, lam=1e4, seed=6),
            small_channel(nx=7, ny=4, np_=9, nz=4, lam=1e5, seed=8),
            small_channel(nx=3, ny=3, np_=11, nz=2, lam=1e3, seed=12)]


class Member:
    def __init__(self, sx, torch, w, method=0):
        self.w = w
        self.mesh = sx.Mesh(w.mesh)
        self.S = sx.ModalMatrixSys(self.mesh, num_modes=w.num_modes, method=method,
                                   lambda2_modes=w.lambda2, betak2_modes=w.betak2)
        self.f = torch.tensor(w.forcing, device="cuda")
        self.u = torch.zeros_like(self.f)

    def args(self):
        return (self.S, self.u.data_ptr(), self.f.data_ptr(), None, self.w.nz, self.w.mesh.nplane)

    def alone(self, torch, precision, tol=1e-12):
        # a fresh copy: the direct form overwrites its forcing, as
        # Field::solve does (src/field.cpp:525-526)
        f = torch.tensor(self.w.forcing, device="cuda")
        u = torch.zeros_like(f)
        self.S.solve_batched(u.data_ptr(), f.data_ptr(), 0, self.w.nz, self.w.mesh.nplane, precision,
                             tol, max_refine=40)
        torch.cuda.synchronize()
        return u.cpu().numpy()

    def oracle(self):
        uo, _ = solve_planes(OracleMesh(self.w.mesh), 0.0, 1.0, self.w.forcing, None,
                             lambda2_per_mode=self.w.lambda2)
        return uo


def test_multi_mixed_vs_oracle_and_alone(sx, torch):
    ms = [Member(sx, torch, w) for w in _workloads()]
    for m in ms:
        m.S.tune(mixed_route=sx.ROUTE_CG)
    B = sx.Batch()
    stats = B.solve([m.args() for m in ms], sx.MIXED_FP32, 1e-12, max_refine=40)
    torch.cuda.synchronize()
    for m, st in zip(ms, stats):
        sp = solved_planes(m.w.nz)
        assert st["planes_solved"] == len(sp) and st["planes_direct"] == 0, st
        assert st["final_rel_residual"] <= 1e-12, st
        um = m.u.cpu().numpy()
        l2, mx = rel_errs(um[sp], m.oracle()[sp])
        assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (m.w.name, l2, mx, st)
        ua = m.alone(torch, sx.MIXED_FP32)
        l2, mx = rel_errs(um[sp], ua[sp])
        assert l2 <= MIXED_TOL and mx <= MIXED_TOL, ("alone vs mix", m.w.name, l2, mx)


@pytest.mark.parametrize("cluster", [0, 2])
def test_multi_fp64_equals_alone(sx, torch, cluster):
    """With the band-sweep cluster size left to the batch (0) the sweeps may
    split the tiles differently from the member's own solve: equal to
    rounding.  With the same cluster size forced on both: bit for bit."""
    ms = [Member(sx, torch, w) for w in _workloads()]
    for m in ms:
        m.S.tune(band_cluster=cluster)
    B = sx.Batch()
    stats = B.solve([m.args() for m in ms], sx.FP64)
    torch.cuda.synchronize()
    for m, st in zip(ms, stats):
        sp = solved_planes(m.w.nz)
        assert st["planes_solved"] == len(sp) == st["planes_direct"], st
        um = m.u.cpu().numpy()
        ua = m.alone(torch, sx.FP64)
        if cluster:
            assert np.array_equal(um[sp], ua[sp]), m.w.name
        else:
            l2, mx = rel_errs(um[sp], ua[sp])
            assert l2 <= 1e-13 and mx <= 1e-13, (m.w.name, l2, mx)
        l2, mx = rel_errs(um[sp], m.oracle()[sp])
        assert l2 <= 1e-12 and mx <= 1e-12, (m.w.name, l2, mx)


def test_multi_hybrid_routes(sx, torch):
    """One member's low-lambda2 modes go to the band Cholesky (their sweeps
    in the batch's one sweep launch), the rest of the batch to the FP32
    iterations."""
    from semtex_b200.workloads import small_channel
    wh = small_channel(nx=20, ny=12, np_=9, nz=16, lam=1e6, seed=13)
    wh.lambda2 = np.logspace(-2, 6, wh.num_modes)
    ws = [wh] + _workloads()[:2]
    ms = [Member(sx, torch, w, method=sx.AUTO) for w in ws]
    B = sx.Batch()
    stats = B.solve([m.args() for m in ms], sx.MIXED_FP32, 1e-12, max_refine=40)
    torch.cuda.synchronize()
    assert 0 < stats[0]["planes_direct"] < stats[0]["planes_solved"], stats[0]
    for m, st in zip(ms, stats):
        sp = solved_planes(m.w.nz)
        assert st["planes_solved"] == len(sp), st
        um = m.u.cpu().numpy()
        uo = m.oracle()
        for p in sp:
            l2, mx = rel_errs(um[p], uo[p])
            assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (m.w.name, p, l2, mx, st)


def test_multi_replay_new_forcing(sx, torch):
    """Second call on the same members and buffers replays the captured
    graphs; new forcing values give the new answer, and a repeat is bitwise
    the same."""
    ms = [Member(sx, torch, w) for w in _workloads()[:3]]
    for m in ms:
        m.S.tune(mixed_route=sx.ROUTE_CG)
    B = sx.Batch()
    B.solve([m.args() for m in ms], sx.MIXED_FP32, 1e-12, max_refine=40)
    rng = np.random.default_rng(21)
    for m in ms:
        m.w.forcing = m.w.forcing * rng.uniform(0.5, 2.0) + 0.1 * np.roll(m.w.forcing, 1, axis=1)
        m.f.copy_(torch.tensor(m.w.forcing, device="cuda"))
    B.solve([m.args() for m in ms], sx.MIXED_FP32, 1e-12, max_refine=40)
    torch.cuda.synchronize()
    first = [m.u.cpu().numpy() for m in ms]
    B.solve([m.args() for m in ms], sx.MIXED_FP32, 1e-12, max_refine=40)
    torch.cuda.synchronize()
    for m, a in zip(ms, first):
        sp = solved_planes(m.w.nz)
        um = m.u.cpu().numpy()
        assert np.array_equal(um, a)
        l2, mx = rel_errs(um[sp], m.oracle()[sp])
        assert l2 <= MIXED_TOL and mx <= MIXED_TOL, (m.w.name, l2, mx)


def test_multi_rejects_duplicate_member(sx, torch):
    m = Member(sx, torch, _workloads()[1])
    B = sx.Batch()
    with pytest.raises(sx.SolverError):
        B.solve([m.args(), m.args()], sx.MIXED_FP32)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_multi_with_boundary_values(sx, torch, precision):
    """Members with essential and natural boundary data (the reference
    goldens laplace1: sin(2 pi x) on the top wall; laplace4: du/dn on the
    top) beside a channel member without any: each member's essential
    values and <h, w> terms come from its own BC lines inside the batch,
    within the form's bar of the oracle."""
    from tests.problems import build_2d
    from semtex_b200.workloads import Workload, small_channel
    prec = sx.MIXED_FP32 if precision == "mixed" else sx.FP64
    tol = MIXED_TOL if precision == "mixed" else 1e-12
    members, oracles = [], []
    for name in ("laplace1", "laplace4"):
        m, p, f, bc, _ = build_2d(name)
        w = Workload(name, m, 1, 0.0, np.array([p["lambda2"]]), np.array([0.0]), f)
        mem = Member(sx, torch, w)
        mem.bc = torch.tensor(bc, device="cuda")
        members.append(mem)
        uo, _ = solve_planes(OracleMesh(m), p["lambda2"], 0.0, f, bc)
        oracles.append(uo)
    wc = small_channel(nx=4, ny=3, np_=7, nz=4, lam=1e4, seed=17)
    mc = Member(sx, torch, wc)
    mc.bc = None
    members.append(mc)
    oracles.append(mc.oracle())
    for m in members:
        if precision == "mixed":
            m.S.tune(mixed_route=sx.ROUTE_CG, inner_iters=200)
    B = sx.Batch()
    args = [(m.S, m.u.data_ptr(), m.f.data_ptr(), m.bc.data_ptr() if m.bc is not None else None,
             m.w.nz, m.w.mesh.nplane) for m in members]
    B.solve(args, prec, 1e-13, max_refine=40)
    torch.cuda.synchronize()
    for m, uo in zip(members, oracles):
        sp = solved_planes(m.w.nz)
        l2, mx = rel_errs(m.u.cpu().numpy()[sp], uo[sp])
        assert l2 <= tol and mx <= tol, (m.w.name, precision, l2, mx)

"""CPU tests of the synthetic workload builders."""
import numpy as np

from semtex_b200.workloads import serving_trace


def test_serving_trace_shapes_and_ranges():
    tr = serving_trace(6, seed=4)
    assert len(tr) == 6
    assert tr[0].t_arrival == 0.0
    assert all(b.t_arrival > a.t_arrival for a, b in zip(tr, tr[1:]))
    for r in tr:
        m = r.mesh
        assert 4 <= m.np - 1 <= 10
        assert 4 <= m.nel <= 64 * 64
        modes = len(r.lambda2)
        assert 1 <= modes <= 64
        assert r.nz == (1 if modes == 1 else 2 * modes)
        assert r.forcing.shape == (r.nz, m.nplane)
        assert np.all(r.lambda2 == r.lambda2[0]) and 1e-2 <= r.lambda2[0] <= 1e4
        assert np.array_equal(r.betak2, np.arange(modes) ** 2.0)
        if r.nz > 1:
            assert not r.forcing[1].any()  # Nyquist plane
    # seeded: the same stream twice
    again = serving_trace(6, seed=4)
    assert all(np.array_equal(a.forcing, b.forcing) for a, b in zip(tr, again))


def test_serving_requests_build_in_any_order():
    from semtex_b200.workloads import serving_plan, serving_request
    plan = serving_plan(5, seed=4)
    fwd = [serving_request(s) for s in plan]
    rev = [serving_request(s) for s in reversed(plan)][::-1]
    assert all(np.array_equal(a.forcing, b.forcing) and a.t_arrival == b.t_arrival for a, b in zip(fwd, rev))
    # a plan is a prefix of a longer plan
    assert [(s.ex, s.ey, s.order, s.modes, s.lam) for s in serving_plan(3)] == \
        [(s.ex, s.ey, s.order, s.modes, s.lam) for s in plan[:3]]

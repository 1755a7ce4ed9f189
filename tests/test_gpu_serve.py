"""GPU tests of the serving loop (continuous batching by device-memory budget):
requests that arrive while others run are admitted and run alongside them,
the budget bounds how many are resident, and every result is the same alone
and in the mix (relative L2 position difference <= 1e-6; FP32 grid sums are
accumulated in a different order in a different mix) and within the FP32
target of the FP64 oracle."""
import numpy as np
import pytest

from icempm_multi_b200.batch import device_bytes
from icempm_multi_b200.serve import Request, Server
from scenarios import standard, stress
from test_gpu_parity import field_errors
from test_gpu_split import POS_TOL

pytestmark = pytest.mark.gpu

MIX_TOL = 1e-6


def scenes():
    return [standard(seed=51), standard(n_cells_x=20, n_cells_y=6, grid=(64, 32), seed=52), stress(seed=53),
            standard(n_cells_x=36, n_cells_y=9, grid=(128, 48), seed=54, IndVelocity=2.5)]


def requests(sc, arrivals, steps):
    return [Request(rid=k, arrival=a, params=sc[k % len(sc)][0].copy(), soa=sc[k % len(sc)][1], steps=s)
            for k, (a, s) in enumerate(zip(arrivals, steps))]


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


def test_serving_mix_matches_alone(oracle):
    sc = scenes()
    arrivals = [0.0, 0.0, 0.05, 0.1, 0.15, 0.2]
    steps = [120, 60, 80, 100, 40, 60]
    srv = Server(budget_bytes=8e9, round_steps=20)
    stats = srv.run(requests(sc, arrivals, steps))
    srv.close()
    assert stats["requests"] == 6
    assert stats["peak_live"] > 1                     # work overlapped on the device
    done = {r.rid: r for r in srv.completed}
    # a request that arrived while others were running joined them
    assert any(r.admitted < max(o.done for o in done.values() if o.rid != r.rid) and r.arrival > 0
               for r in done.values())
    for rid in (0, 2, 3):
        alone = Server(budget_bytes=8e9, round_steps=20)
        alone.run(requests(sc, [0.0], [steps[rid]]) if rid == 0 else
                  [Request(rid=0, arrival=0.0, params=sc[rid % len(sc)][0].copy(), soa=sc[rid % len(sc)][1],
                           steps=steps[rid])])
        a = alone.completed[0]
        alone.close()
        m = done[rid]
        assert m.steps_done == a.steps_done == steps[rid]
        assert m.sim_time == a.sim_time
        e = field_errors(m.result, a.result)
        assert e["pos"] <= MIX_TOL, (rid, e)
        ref = sc[rid % len(sc)][1].clone()
        assert oracle.run(sc[rid % len(sc)][0], ref, 0, steps[rid])[0] == 0
        assert field_errors(m.result, ref)["pos"] <= POS_TOL


def test_serving_budget_bounds_residency():
    sc = [scenes()[0]]                       # five requests of the same size
    one = device_bytes(sc[0][0], sc[0][1].capacity)
    srv = Server(budget_bytes=2.2 * one, round_steps=20)
    stats = srv.run(requests(sc, [0.0] * 5, [40] * 5))
    srv.close()
    assert stats["requests"] == 5
    assert stats["peak_live"] <= 2
    assert stats["peak_device_bytes"] <= 2.2 * one


def test_serving_evict_resume_and_cancel():
    """Host-side interventions in a running serve: request 0 is evicted after
    the second round (state, time, step and force bins to the host, device
    memory freed) and resumes; request 2 is cancelled.  The evicted request
    ends where it would have ended alone."""
    sc = scenes()[:3]
    events = {}

    def on_round(srv, k):
        if k == 2:
            events["evicted"] = srv.evict(0)
        if k == 3:
            events["cancelled"] = srv.cancel(2)

    srv = Server(budget_bytes=8e9, round_steps=20)
    stats = srv.run(requests(sc, [0.0, 0.0, 0.0], [100, 60, 200]), on_round=on_round)
    srv.close()
    assert events == {"evicted": True, "cancelled": True}
    assert stats["requests"] == 2 and stats["cancelled"] == 1 and stats["evictions"] == 1
    done = {r.rid: r for r in srv.completed}
    assert set(done) == {0, 1} and srv.cancelled[0].rid == 2
    r0 = done[0]
    assert r0.evictions == 1 and r0.steps_done == 100
    alone = Server(budget_bytes=8e9, round_steps=20)
    alone.run(requests(sc, [0.0], [100]))
    a = alone.completed[0]
    alone.close()
    assert r0.sim_time == a.sim_time
    assert field_errors(r0.result, a.result)["pos"] <= MIX_TOL
    assert np.allclose(r0.bins, a.bins, rtol=1e-5, atol=1e-6 * (np.abs(a.bins).max() + 1))


def test_request_larger_than_the_budget_is_refused():
    sc = scenes()[:1]
    one = device_bytes(sc[0][0], sc[0][1].capacity)
    srv = Server(budget_bytes=0.5 * one, round_steps=20)
    with pytest.raises(RuntimeError, match="budget"):
        srv.run(requests(sc, [0.0], [40]))
    srv.close()

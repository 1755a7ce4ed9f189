"""Host-side tests of the serving loop (icempm_multi_b200/serve.py) on the CPU:
the Server drives a stand-in for the batch that keeps each member's step
count and clock the way icy_batch_* does (a round advances every live
member; a retired member leaves after the rounds queued before it; its slot
is reserved until collected), so the scheduling -- admission by budget and
slots, pipelining of rounds, retirement, cancel and evict -- is checked
without a device."""
import numpy as np
import pytest

from icempm_multi_b200 import serve as S
from icempm_multi_b200.batch import device_bytes
from icempm_multi_b200.hssoa import HostSideSOA
from scenarios import standard


class FakeBatch:
    def __init__(self, max_instances, device=0):
        self.nslots = max_instances
        self.members = {}        # slot -> dict(params, soa, step, t)
        self.retiring = {}       # slot -> (state, soa buffer)
        self.steps_queued = 0
        self.log = []

    def _free_slot(self):
        for s in range(self.nslots):
            if s not in self.members and s not in self.retiring:
                return s
        raise RuntimeError("no slot")

    def add_async(self, params, soa):
        s = self._free_slot()
        self.members[s] = {"params": params, "soa": soa, "step": 0, "t": 0.0}
        self.log.append(("add", s))
        return s

    add = add_async

    def step(self, n):
        for m in self.members.values():
            m["step"] += n
            m["t"] += n * m["params"].InitialTimeStep
        self.steps_queued += 1
        self.log.append(("step", n, sorted(self.members)))

    def set_clock(self, slot, t, step):
        self.members[slot]["t"], self.members[slot]["step"] = t, step

    def retire(self, slot, soa=None, bins=True):
        m = self.members.pop(slot)
        if soa is not None:
            soa.size = m["soa"].size
            soa.buf[:, :soa.size] = m["soa"].buf[:, :soa.size]
        self.retiring[slot] = (m, soa)
        self.log.append(("retire", slot))

    def collect(self, slot, wait=True):
        m, _ = self.retiring.pop(slot)
        self.log.append(("collect", slot))
        return m["t"], m["step"], np.zeros(2 * m["params"].n_indenter_subdivisions)

    def download(self, slot, soa):
        m = self.members[slot]
        soa.size = m["soa"].size
        return m["t"], m["step"], np.ones(2 * m["params"].n_indenter_subdivisions)

    def remove(self, slot):
        self.members.pop(slot)

    def wait_steps(self, in_flight):
        pass

    def reserve(self, nbytes):
        pass

    def close(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    made = []

    def factory(*a, **k):
        b = FakeBatch(*a, **k)
        made.append(b)
        return b

    monkeypatch.setattr(S, "Batch", factory)
    return made


def _requests(n, steps, arrivals=None):
    p, soa = standard(seed=3)
    arrivals = arrivals or [0.0] * n
    return [S.Request(rid=k, arrival=arrivals[k], params=p.copy(), soa=soa, steps=steps[k]) for k in range(n)]


def test_every_request_runs_its_steps_and_retires_after_its_last_round(fake):
    reqs = _requests(4, [40, 100, 60, 20])
    srv = S.Server(budget_bytes=1e12, round_steps=20)
    stats = srv.run(reqs)
    b = fake[0]
    assert stats["requests"] == 4 and stats["rounds"] == 5
    for r in srv.completed:
        assert r.steps_done == r.steps and r.sim_time == pytest.approx(r.steps * r.params.InitialTimeStep)
    # a member is retired right after the round that completes it, before the next round
    retired_after = {e[1]: i for i, e in enumerate(b.log) if e[0] == "retire"}
    for r in srv.completed:
        k = r.steps // 20
        rounds = [i for i, e in enumerate(b.log) if e[0] == "step"]
        assert rounds[k - 1] < retired_after[r.slot] < (rounds[k] if k < len(rounds) else len(b.log))
    # collected one pipelined round later, and every slot is free at the end
    assert not b.members and not b.retiring


def test_budget_bounds_residency_including_retiring_members(fake):
    p, soa = standard(seed=3)
    one = device_bytes(p, soa.capacity)
    reqs = _requests(5, [40] * 5)
    srv = S.Server(budget_bytes=2.2 * one, round_steps=20)
    stats = srv.run(reqs)
    assert stats["requests"] == 5
    assert stats["peak_live"] <= 2 and stats["peak_device_bytes"] <= 2.2 * one
    b = fake[0]
    # never more than two members resident, counting those whose results are being copied
    live = set()
    for e in b.log:
        if e[0] == "add":
            live.add(e[1])
        elif e[0] == "collect":
            live.discard(e[1])
        assert len(live) <= 2


def test_slots_bound_residency_including_retiring_members(fake):
    """With slots, not memory, the limit: a retired member holds its slot
    until its results are collected, so admission counts it (the batch has
    no free slot for a new member before that)."""
    reqs = _requests(9, [20, 40, 20, 60, 20, 40, 20, 20, 40])
    srv = S.Server(budget_bytes=1e12, max_instances=3, round_steps=20)
    stats = srv.run(reqs)
    assert stats["requests"] == 9 and stats["peak_live"] <= 3
    held = set()
    for e in fake[0].log:
        if e[0] == "add":
            held.add(e[1])
        elif e[0] == "collect":
            held.discard(e[1])
        assert len(held) <= 3


def test_request_larger_than_the_budget_is_refused(fake):
    p, soa = standard(seed=3)
    srv = S.Server(budget_bytes=0.5 * device_bytes(p, soa.capacity), round_steps=20)
    with pytest.raises(RuntimeError, match="budget"):
        srv.run(_requests(1, [40]))


def test_evict_resumes_and_cancel_drops(fake):
    def on_round(srv, k):
        if k == 1:
            assert srv.evict(0)
        if k == 2:
            assert srv.cancel(1)

    srv = S.Server(budget_bytes=1e12, round_steps=20)
    stats = srv.run(_requests(3, [60, 200, 40]), on_round=on_round)
    assert stats["requests"] == 2 and stats["cancelled"] == 1 and stats["evictions"] == 1
    done = {r.rid: r for r in srv.completed}
    assert set(done) == {0, 2} and srv.cancelled[0].rid == 1
    r0 = done[0]
    assert r0.evictions == 1 and r0.steps_done == 60
    # resumed where it stopped: its clock continued from the evicted state
    assert r0.sim_time == pytest.approx(60 * r0.params.InitialTimeStep)
    # the force bins of the part before the eviction are kept
    assert np.all(r0.bins == 1.0)


def test_late_arrival_joins_a_running_batch(fake):
    reqs = _requests(2, [200, 40], arrivals=[0.0, 0.02])
    srv = S.Server(budget_bytes=1e12, round_steps=20)

    def on_round(srv, k):   # make the rounds take a little host time
        import time
        time.sleep(0.005)

    srv.run(reqs, on_round=on_round)
    b = fake[0]
    both = [e for e in b.log if e[0] == "step" and len(e[2]) == 2]
    assert both, "the second request never ran beside the first"
    done = {r.rid: r for r in srv.completed}
    assert done[1].admitted < done[0].done


def test_saturated_rate_is_reported_when_requests_wait(fake):
    """With more requests than slots, rounds run while requests wait: the
    stats carry the rate over those rounds (and None when nothing waited)."""
    reqs = _requests(9, [40] * 9)
    srv = S.Server(budget_bytes=1e12, max_instances=3, round_steps=20)
    stats = srv.run(reqs)
    assert stats["saturated_s"] >= 0.0
    assert stats["saturated_particle_steps_per_s"] is None or stats["saturated_particle_steps_per_s"] > 0
    srv2 = S.Server(budget_bytes=1e12, max_instances=16, round_steps=20)
    stats2 = srv2.run(_requests(3, [40] * 3))
    assert stats2["saturated_particle_steps_per_s"] is None and stats2["saturated_s"] == 0.0

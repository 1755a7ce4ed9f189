"""GPU tests of batches of independent scenarios (icy_batch_*): every member
matches its own single-instance FP32 run and the FP64 oracle, members added
at different times keep their own clocks, slots are reused after removal."""
import numpy as np
import pytest

from icempm_multi_b200 import GPUImplementation
from icempm_multi_b200._lib import PRECISION_FP32_SPLIT
from icempm_multi_b200.batch import Batch
from icempm_multi_b200.hssoa import HostSideSOA
from scenarios import standard, stress
from test_gpu_parity import field_errors
from test_gpu_split import POS_TOL

pytestmark = pytest.mark.gpu


def single_f32(p, soa, steps, chunk):
    out = soa.clone()
    g = GPUImplementation(p, out, precision=PRECISION_FP32_SPLIT)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    t, done = 0.0, 0
    while done < steps:
        k = min(chunk, steps - done)
        t = g.run_steps(done, k, t)
        done += k
    g.transfer_from_device()
    g.close()
    return out, t


def scenarios():
    return [standard(seed=31), standard(n_cells_x=20, n_cells_y=6, grid=(64, 32), seed=32, IndVelocity=2.0),
            stress(seed=33), standard(n_cells_x=40, n_cells_y=10, grid=(128, 48), seed=34, DP_phi=45),
            standard(n_cells_x=12, n_cells_y=12, grid=(64, 64), seed=35, YoungsModulus=5e8)]


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


def test_batch_members_match_single_and_oracle(oracle):
    sc = scenarios()
    b = Batch(8)
    slots = [b.add(p, soa) for p, soa in sc]
    b.step(40)
    b.step(40)
    for (p, soa), s in zip(sc, slots):
        out = soa.clone()
        t, step, bins = b.download(s, out)
        assert step == 80
        tt = 0.0
        for _ in range(80):
            tt += p.InitialTimeStep
        assert t == tt                       # the host recurrence of Model::Step, exactly
        one, t1 = single_f32(p, soa, 80, 40)
        assert t1 == t
        e1 = field_errors(out, one)
        assert e1["pos"] <= 1e-6, e1
        ref = soa.clone()
        assert oracle.run(p, ref, 0, 80)[0] == 0
        assert field_errors(out, ref)["pos"] <= POS_TOL
    info = b.info()
    assert info["live"] == 5 and info["kernel_launches"] > 0
    b.close()


def test_batch_members_keep_their_own_clock(oracle):
    (pa, sa), (pb, sb) = standard(seed=41), standard(n_cells_x=16, n_cells_y=6, grid=(64, 32), seed=42)
    b = Batch(4)
    a = b.add(pa, sa)
    b.step(30)
    c = b.add(pb, sb)
    b.step(30)
    oa, ob = sa.clone(), sb.clone()
    _, step_a, _ = b.download(a, oa)
    _, step_c, _ = b.download(c, ob)
    assert (step_a, step_c) == (60, 30)
    ra, rb = sa.clone(), sb.clone()
    oracle.run(pa, ra, 0, 60)
    oracle.run(pb, rb, 0, 30)
    assert field_errors(oa, ra)["pos"] <= POS_TOL
    assert field_errors(ob, rb)["pos"] <= POS_TOL
    # free a slot and reuse it
    b.remove(a)
    d = b.add(pa, sa)
    assert d == a
    b.step(10)
    od = sa.clone()
    _, step_d, _ = b.download(d, od)
    assert step_d == 10
    b.close()


def test_async_admission_and_retirement(oracle):
    """icy_batch_add_async while a round is queued, icy_batch_retire /
    icy_batch_collect behind the next one: the same clocks and states as the
    synchronous calls, and the slot is reused only after its collection."""
    (pa, sa), (pb, sb) = standard(seed=41), standard(n_cells_x=16, n_cells_y=6, grid=(64, 32), seed=42)
    b = Batch(4)
    a = b.add(pa, sa)
    b.step(30)
    c = b.add_async(pb, sb)          # joins behind the queued round
    b.step(30)
    oa = HostSideSOA(sa.capacity, pinned=True)
    oc = HostSideSOA(sb.capacity, pinned=True)
    b.retire(a, oa)
    b.retire(c, oc)
    d = b.add_async(pa, sa)          # a and c are still reserved
    assert d not in (a, c)
    b.step(10)
    ta, step_a, bins_a = b.collect(a)
    tc, step_c, _ = b.collect(c)
    assert (step_a, step_c) == (60, 30)
    assert ta == pytest.approx(60 * pa.InitialTimeStep) and tc == pytest.approx(30 * pb.InitialTimeStep)
    assert oa.size == sa.size and np.all(np.isfinite(bins_a))
    ra, rb = sa.clone(), sb.clone()
    oracle.run(pa, ra, 0, 60)
    oracle.run(pb, rb, 0, 30)
    assert field_errors(oa, ra)["pos"] <= POS_TOL
    assert field_errors(oc, rb)["pos"] <= POS_TOL
    e = b.add(pb, sb)                # a freed slot is taken again
    assert e in (a, c)
    b.wait_steps(0)
    assert b.info()["live"] == 2
    b.close()


def test_two_small_batches_at_once(oracle):
    """Two batches alive together, stepped in turns: the first owns the device's
    constant-bank copy of its member arguments, the second reads its own global
    table; each member matches the oracle, and after both are closed a new
    batch takes the table over."""
    (pa, sa), (pb, sb) = standard(seed=43), standard(n_cells_x=16, n_cells_y=6, grid=(64, 32), seed=44)
    b1, b2 = Batch(4), Batch(4)
    s1, s2 = b1.add(pa, sa), b2.add(pb, sb)
    for _ in range(3):
        b1.step(20)
        b2.step(20)
    o1, o2 = sa.clone(), sb.clone()
    assert b1.download(s1, o1)[1] == 60 and b2.download(s2, o2)[1] == 60
    ra, rb = sa.clone(), sb.clone()
    assert oracle.run(pa, ra, 0, 60)[0] == 0 and oracle.run(pb, rb, 0, 60)[0] == 0
    assert field_errors(o1, ra)["pos"] <= POS_TOL
    assert field_errors(o2, rb)["pos"] <= POS_TOL
    b1.close()
    b2.close()
    b3 = Batch(4)
    s3 = b3.add(pb, sb)
    b3.step(60)
    o3 = sb.clone()
    b3.download(s3, o3)
    assert field_errors(o3, rb)["pos"] <= POS_TOL
    b3.close()


def test_batch_beyond_the_constant_bank(oracle):
    """A batch of more slots than the constant-bank table holds (300) reads
    its members' arguments from the global table: members still match their
    single-instance runs (the constant-bank path is the one of the tests
    above)."""
    sc = scenarios()[:3]
    b = Batch(400)
    slots = [b.add(p, soa) for p, soa in sc]
    b.step(30)
    b.step(30)
    for (p, soa), s in zip(sc, slots):
        out = soa.clone()
        assert b.download(s, out)[1] == 60
        one, _ = single_f32(p, soa, 60, 30)
        assert field_errors(out, one)["pos"] <= 1e-6
    b.close()


@pytest.mark.parametrize("shape", [0, 1])
def test_batch_rebinning_matches_single(oracle, shape):
    """All members re-binned together on the device every 20 steps (one
    launch per phase for the whole batch): each member still matches its
    single-instance run and the oracle, after six re-binnings."""
    sc = scenarios()
    b = Batch(8)
    b.set_option("tile_shape", shape)
    b.set_option("resort_every", 20)
    slots = [b.add(p, soa) for p, soa in sc]
    for _ in range(6):
        b.step(20)
    for (p, soa), s in zip(sc, slots):
        out = soa.clone()
        assert b.download(s, out)[1] == 120
        one, _ = single_f32(p, soa, 120, 40)
        assert field_errors(out, one)["pos"] <= 1e-6
        ref = soa.clone()
        assert oracle.run(p, ref, 0, 120)[0] == 0
        assert field_errors(out, ref)["pos"] <= POS_TOL
    b.close()


def test_reserved_pool_serves_members(oracle):
    """icy_mpm_reserve maps device memory into the instance pool up front
    (a negative size is refused); members admitted afterwards still match
    their single-instance runs."""
    import ctypes as C
    from icempm_multi_b200._lib import ICY_ERR_INVALID_ARGUMENT, lib
    assert lib().icy_mpm_reserve(0, C.c_int64(-1)) == ICY_ERR_INVALID_ARGUMENT
    b = Batch(4)
    b.reserve(256 << 20)
    p, soa = standard(seed=47)
    s = b.add_async(p, soa)
    b.step(40)
    out = soa.clone()
    assert b.download(s, out)[1] == 40
    one, _ = single_f32(p, soa, 40, 40)
    assert field_errors(out, one)["pos"] <= 1e-6
    b.close()

"""GPU tests of one instance in slabs of grid columns (icy_part_*): the
reference's multi-partition GPU_Implementation5
(simulation/gpu_implementation5.cpp:31-204,221-326; kernels
simulation/kernels.cuh:416-513), here with 1 to 4 partitions on one GPU (as
the reference places partition i on device i % deviceCount) and, where two
GPUs are present, on two devices over peer access.

Against the FP64 oracle, within the FP64 tolerances of the parity tests (the
sums add in another order: each slab sums its own points, then the
neighbour's boundary columns): every field after 120 steps with points
handed between slabs, the indenter force bins with the indenter pressing on
a slab boundary, and a block translating across three slabs."""
import numpy as np
import pytest

from icempm_multi_b200._lib import ICY_ERR_CAPACITY, IcyError
from icempm_multi_b200.partition import Partitioned, plan
from scenarios import standard, stress
from test_gpu_parity import assert_close, field_errors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


def run_parts(p, soa, n, steps, chunk=37, devices=None):
    out = soa.clone()
    part = Partitioned(p, n, devices=devices, size_hint=soa.size)
    part.upload(soa)
    t, done = 0.0, 0
    while done < steps:
        k = min(chunk, steps - done)
        t = part.run_steps(done, k, t)
        done += k
    bins = part.download(out)
    slots = [part.info(i)["slots"] for i in range(n)]
    part.close()
    return out, bins, t, slots


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_partitions_match_oracle(oracle, n):
    p, soa = stress(seed=11, n_cells_x=80, grid=(200, 48))
    p.UpdateEveryNthStep, p.PointTransferFrequency = 20, 2   # points change slabs every 10 steps
    ref = soa.clone()
    err, t_ref, bins_ref = oracle.run(p, ref, 0, 120)
    assert err == 0
    out, bins, t, slots = run_parts(p, soa, n, 120)
    assert t == t_ref
    e = field_errors(out, ref)
    print("partitions", n, e, slots)
    assert_close(e)
    assert np.allclose(bins, bins_ref, rtol=1e-9, atol=1e-9 * max(np.abs(bins_ref).max(), 1e-300))


def test_indenter_on_a_slab_boundary(oracle):
    """The indenter presses into the block where two slabs meet: each node's
    force is counted once, the bins match the one-domain oracle."""
    p, soa = standard(n_cells_x=48, n_cells_y=12, grid=(128, 48), seed=31, IndVelocity=3.0, IndDepth=0.6)
    p.UpdateEveryNthStep, p.PointTransferFrequency = 20, 2
    x0, w, _, _ = plan(p, soa, 2)[1]
    # start the indenter over the boundary column
    p.indenter_x_initial = p.indenter_x = x0 * p.cellsize - 0.3
    ref = soa.clone()
    err, _, bins_ref = oracle.run(p, ref, 0, 200)
    assert err == 0 and np.abs(bins_ref).max() > 0
    out, bins, _, _ = run_parts(p, soa, 2, 200)
    assert_close(field_errors(out, ref))
    assert np.allclose(bins, bins_ref, rtol=1e-9, atol=1e-9 * np.abs(bins_ref).max())


def test_block_translating_across_slabs(oracle):
    """Points moving at 100 m/s (16 cells in 400 steps) cross slab
    boundaries: they are handed over as they go, nothing is lost, the state
    matches the oracle."""
    p, soa = standard(n_cells_x=54, n_cells_y=6, grid=(200, 48), seed=4, Gravity=0.0, IndDepth=0.05)
    soa.vel[0, :] = 100.0
    p.indenter_x_initial = p.indenter_x = 0.5   # keep the indenter away from the block
    p.indenter_y = 0.5
    p.UpdateEveryNthStep, p.PointTransferFrequency = 20, 4   # an exchange every 5 steps
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 400)[0] == 0
    moved = (ref.pos[0] - soa.pos[0]).mean() / p.cellsize
    assert moved > 10
    out, _, _, slots = run_parts(p, soa, 3, 400)
    assert_close(field_errors(out, ref))
    first = plan(p, soa, 3)
    assert slots[2] > first[2][3], (slots, first)   # the rightmost slab received points


def test_partition_capacity_is_checked(built):
    p, soa = standard(n_cells_x=48, grid=(128, 48), seed=2)
    part = Partitioned(p, 2, capacity_per_partition=soa.size // 4)
    with pytest.raises(IcyError) as e:
        part.upload(soa)
    assert e.value.code == ICY_ERR_CAPACITY
    part.close()


def test_partitions_on_two_devices(oracle):
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU: the two-device placement needs two")
    p, soa = stress(seed=11, n_cells_x=80, grid=(200, 48))
    p.UpdateEveryNthStep, p.PointTransferFrequency = 20, 2
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 120)[0] == 0
    out, _, _, _ = run_parts(p, soa, 2, 120, devices=[0, 1])
    assert_close(field_errors(out, ref))

"""Seeded randomized scenes (grid, cell size, block, points per cell, material,
cohesion, strengths, grain variability, indenter, CFL time step; see
scenarios.randomized) for 200 steps through the C-ABI against the FP64
oracle: the tiled FP64 path and the one-thread-per-item FP64 kernels within
the parity tolerances, the FP32 split path within its position target."""
import pytest

from scenarios import randomized
from test_gpu_parity import TOL, assert_close, field_errors, run_gpu
from test_gpu_split import POS_TOL, run_split

pytestmark = pytest.mark.gpu

STEPS = 200
# FP32 field bounds of these scenes (up to 74 % of the points crushed, the
# return mapping taken at every step by most of them): about ten times the
# largest errors measured over the twelve scenes (4.1e-4, 3.6e-4, 8.8e-4, 3.5e-4)
TOL32_SCENES = {"vel": 4e-3, "Fe": 4e-3, "Bp": 1e-2, "Jp": 4e-3}


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


@pytest.mark.parametrize("seed", range(12))
def test_randomized_scene_matches_oracle(oracle, seed):
    p, soa = randomized(seed)
    ref = soa.clone()
    assert oracle.run(p, ref, 0, STEPS)[0] == 0
    out, _, _, _ = run_gpu(p, soa, STEPS)
    e64 = field_errors(out, ref)
    simple = soa.clone()
    from icempm_multi_b200 import GPUImplementation
    g = GPUImplementation(p, simple)
    g.set_option("tiled", 0)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    g.run_steps(0, STEPS, 0.0)
    g.transfer_from_device()
    g.close()
    es = field_errors(simple, ref)
    out32, _, _ = run_split(p, soa, STEPS)
    e32 = field_errors(out32, ref)
    print("randomized", seed, soa.size, "fp64", e64, "simple", es, "fp32", e32)
    assert_close(e64)
    assert_close(es)
    assert e32["pos"] <= POS_TOL
    for k, v in TOL32_SCENES.items():
        assert e32[k] <= v, (k, e32)


def test_randomized_scenes_as_one_batch(oracle):
    """The twelve scenes as members of one batch (each with its own time step,
    material and grid), half of them admitted while the first round is
    queued, all retired together: every member against the oracle for its own
    step count."""
    from icempm_multi_b200.batch import Batch
    from icempm_multi_b200.hssoa import HostSideSOA
    scenes = [randomized(s) for s in range(12)]
    b = Batch(16)
    slots = [b.add(p, soa) for p, soa in scenes[:6]]
    b.step(100)
    slots += [b.add_async(p, soa) for p, soa in scenes[6:]]
    b.step(100)
    outs = []
    for (p, soa), slot in zip(scenes, slots):
        out = HostSideSOA(soa.capacity, pinned=True)
        b.retire(slot, out)
        outs.append(out)
    for k, ((p, soa), slot, out) in enumerate(zip(scenes, slots, outs)):
        _, step, _ = b.collect(slot)
        n = 200 if k < 6 else 100
        assert step == n
        ref = soa.clone()
        assert oracle.run(p, ref, 0, n)[0] == 0
        e = field_errors(out, ref)
        assert e["pos"] <= POS_TOL, (k, e)
    b.close()

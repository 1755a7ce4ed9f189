"""GPU tests of the FP32 tile shapes (option "tile_shape": 32 x 8, 16 x 16,
16 x 8 cells per tile) and of the autotuner that picks them.

Every shape against the FP64 oracle within the FP32 bounds (crushed, liquid
and disabled points, call boundaries, re-binning every 16 steps); a batch
whose members take the 16 x 8 shape; the options refused where they cannot
apply; the tuner timing each shape on an instance and on batches of a sample
of scenarios, applying and caching the fastest."""
import json

import pytest

from icempm_multi_b200 import GPUImplementation
from icempm_multi_b200._lib import ICY_ERR_NOT_SUPPORTED, PRECISION_FP32_SPLIT, IcyError
from icempm_multi_b200.batch import Batch
from scenarios import randomized, standard, stress
from test_gpu_parity import field_errors
from test_gpu_split import POS_TOL, run_split

pytestmark = pytest.mark.gpu

BOUND = {"vel": 1e-3, "Fe": 1e-3, "Bp": 2e-3, "Jp": 4e-3}   # the stress scene's FP32 bounds (measured <= 1e-3 Jp)


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_tile_shapes_match_oracle(oracle, shape):
    p, soa = stress(seed=5)
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 200)[0] == 0
    out, _, _ = run_split(p, soa, 200, chunk=37, resort_every=16, tile_shape=shape)
    e = field_errors(out, ref)
    print("shape", shape, e)
    assert e["pos"] <= POS_TOL
    for k, v in BOUND.items():
        assert e[k] <= v, (k, e)


def test_batch_members_with_16x8_tiles(oracle):
    scenes = [randomized(s) for s in range(4)]
    b = Batch(8)
    b.set_option("tile_shape", 2)
    slots = [b.add(p, soa) for p, soa in scenes]
    with pytest.raises(IcyError) as e:   # the shape is the batch's: set while it is empty
        b.set_option("tile_shape", 0)
    assert e.value.code == ICY_ERR_NOT_SUPPORTED
    b.step(120)
    b.synchronize()
    for (p, soa), slot in zip(scenes, slots):
        out = soa.clone()
        b.download(slot, out)
        ref = soa.clone()
        assert oracle.run(p, ref, 0, 120)[0] == 0
        assert field_errors(out, ref)["pos"] <= POS_TOL
    b.close()


def test_shape_option_on_fp64_is_refused(built):
    p, soa = standard(seed=3)
    g = GPUImplementation(p, soa.clone())
    g.set_option("tile_shape", 0)
    with pytest.raises(IcyError) as e:
        g.set_option("tile_shape", 2)
    assert e.value.code == ICY_ERR_NOT_SUPPORTED
    g.close()


def test_autotune_instance_shapes_and_cache(tmp_path, oracle):
    from icempm_multi_b200.autotune import tune_instance
    p, soa = standard(n_cells_x=96, n_cells_y=24, grid=(160, 64), seed=8)
    out = soa.clone()
    g = GPUImplementation(p, out, precision=PRECISION_FP32_SPLIT)
    g.update_constants()
    g.transfer_ponts_to_device()
    cache = str(tmp_path / "tune.json")
    res = tune_instance(g, p, soa.size, steps=8, resorts=(64, 128), cache=cache)
    st = res["settings"]
    shapes = [t for t in res["trials"] if "tile_shape" in t]
    assert sorted(t["tile_shape"] for t in shapes) == [0, 1, 2] and not res["cached"]
    assert st["tile_shape"] == min(shapes, key=lambda t: t["ms_per_step"])["tile_shape"]
    assert st["resort_every"] in (64, 128)
    assert json.load(open(cache))[res["signature"]]["settings"] == st
    again = tune_instance(g, p, soa.size, steps=8, resorts=(64, 128), cache=cache)
    assert again["cached"] and again["settings"] == st
    g.close()
    # the tuned shape runs the scene as the oracle does
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 150)[0] == 0
    tuned, _, _ = run_split(p, soa, 150, chunk=50, **st)
    assert field_errors(tuned, ref)["pos"] <= POS_TOL


def test_autotune_batch_shape(built):
    from icempm_multi_b200.autotune import tune_batch_shape
    scenes = [standard(seed=70 + k) for k in range(6)]
    res = tune_batch_shape(scenes, sample=3, steps=6)
    assert sorted(t["tile_shape"] for t in res["trials"]) == [0, 1, 2] and res["sample"] == 3
    assert res["tile_shape"] == min(res["trials"], key=lambda t: t["ms_per_step"])["tile_shape"]

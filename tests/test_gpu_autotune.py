"""GPU test of the batch autotuner: it tries every candidate of each knob,
keeps the fastest, applies it, caches it per workload signature, and the
tuned batch still matches the single-instance FP32 path."""
import json

import numpy as np
import pytest

from icempm_multi_b200 import GPUImplementation
from icempm_multi_b200._lib import PRECISION_FP32_SPLIT
from icempm_multi_b200.autotune import tune_batch
from icempm_multi_b200.batch import Batch
from scenarios import standard
from test_gpu_parity import field_errors

pytestmark = pytest.mark.gpu


def test_autotune_picks_and_caches(tmp_path):
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    scenes = [standard(seed=60 + k) for k in range(3)]
    b = Batch(8)
    slots = [b.add(p, s) for p, s in scenes]
    cache = str(tmp_path / "tune.json")
    res = tune_batch(b, steps=4, cache=cache)
    st = res["settings"]
    assert st["tile_ctas"] in [sms * k for k in (2, 3, 4)]
    assert st["update_ctas"] in [sms * k for k in (4, 8, 16)]
    assert st["resort_every"] in (128, 256, 512)
    assert len(res["trials"]) == 9 and not res["cached"]
    for knob in ("tile_ctas", "update_ctas"):
        tr = [t for t in res["trials"] if knob in t]
        assert st[knob] == min(tr, key=lambda t: t["ms_per_step"])[knob]
    assert json.load(open(cache))[res["signature"]]["settings"] == st
    again = tune_batch(b, steps=4, cache=cache)
    assert again["cached"] and again["settings"] == st
    # the tuned batch steps on; each member against the same scene run alone
    b.step(50)
    b.synchronize()
    for (p, soa), slot in zip(scenes, slots):
        out = soa.clone()
        t, step, _ = b.download(slot, out)
        alone = soa.clone()
        g = GPUImplementation(p, alone, precision=PRECISION_FP32_SPLIT)
        g.update_constants()
        g.transfer_ponts_to_device()
        assert g.run_steps(0, step, 0.0) == t
        g.transfer_from_device()
        g.close()
        assert field_errors(out, alone)["pos"] <= 1e-5   # float atomic order differs over ~3,700 steps
    b.close()

"""The CUDA paths on the reference's own geometry: the 70,534-point cloud
build/geometries_2d/2d_70k.h5 under the reference's build/p1.json, placed as
SnapshotManager::LoadRawPoints places it, one frame of 500 sub-steps
(tests/golden/ref_2d_70k.npz, written by tests/golden/make_geometry_golden.py
from the reference's kernels compiled for the host).

Checks: the tiled FP64 path and the one-thread-per-item FP64 path against the
reference's frame (positions, Jp_inv, status words) and against the oracle
(every field, which the CPU tests pin to the same frame bit for bit) within
the FP64 tolerances of the parity tests; the FP32 split path within the FP32
bounds of the split tests, on absolute position and on displacement."""
import numpy as np
import pytest

from icempm_multi_b200 import GPUImplementation
from icempm_multi_b200._lib import PRECISION_FP32_SPLIT, PRECISION_FP64
from test_gpu_parity import STATUS_MISMATCH_MAX, TOL, assert_close, field_errors
from test_gpu_split import POS_TOL, TOL32, displacement_errors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(built):
    from golden.make_geometry_golden import load_geometry
    from oracle.oracle import Oracle
    p, soa, steps, ref = load_geometry()
    full = soa.clone()
    err, t, bins = Oracle().run(p, full, 0, steps)
    assert err == 0 and t == ref["t_end"]
    assert np.array_equal(full.pos, ref["pos_out"])   # the oracle is the reference's frame
    return p, soa, steps, ref, full, bins


def run(p, soa, steps, precision, **opts):
    out = soa.clone()
    g = GPUImplementation(p, out, precision=precision)
    for k, v in opts.items():
        g.set_option(k, v)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    t = g.run_steps(0, steps, 0.0)
    g.transfer_from_device()
    bins = g.indenter_bins.copy()
    g.close()
    return out, t, bins


def rel(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


@pytest.mark.parametrize("tiled", [1, 0])
def test_fp64_paths_on_reference_geometry(case, tiled):
    p, soa, steps, ref, full, bins = case
    out, t, b = run(p, soa, steps, PRECISION_FP64, tiled=tiled)
    assert t == ref["t_end"]
    assert rel(out.pos, ref["pos_out"]) <= TOL["pos"]
    assert rel(out.Jp_inv - 1.0, ref["jp_out"] - 1.0) <= TOL["Jp"] or np.array_equal(out.Jp_inv, ref["jp_out"])
    assert np.mean(out.utility != ref["util_out"]) <= STATUS_MISMATCH_MAX
    errs = field_errors(out, full)
    print("2d_70k FP64 tiled=%d" % tiled, errs)
    assert_close(errs)
    assert np.allclose(b, bins, rtol=1e-9, atol=1e-9 * max(np.abs(bins).max(), 1e-300))


def test_fp32_split_on_reference_geometry(case):
    p, soa, steps, ref, full, bins = case
    out, t, _ = run(p, soa, steps, PRECISION_FP32_SPLIT)
    assert t == ref["t_end"]
    errs = field_errors(out, full)
    disp = displacement_errors(p, soa, out, full)
    print("2d_70k FP32 split", errs, disp)
    assert rel(out.pos, ref["pos_out"]) <= POS_TOL
    for k, v in TOL32.items():
        assert errs[k] <= v, (k, errs)
    assert np.array_equal(out.utility, ref["util_out"])
    # one frame moves the points 0.002 h at most: the displacement-relative
    # error (measured 2.1e-3) is near the FP32 offset resolution
    assert disp["disp_rel"] <= 2e-2 and disp["max_dx_h"] <= 1e-4, disp

"""GPU parity: the CUDA library against the CPU oracle (and the reference's own
CUDA kernels), called through the C-ABI.

FP64 results differ from the oracle only by FMA contraction and the order of
floating-point atomic sums, so the comparison uses per-field relative errors
with the tolerances written below.  All cases keep every particle well inside
the grid (checked on the oracle's trajectory before the reference's CUDA
kernels, which do not stop at out-of-grid particles, are run).
"""
import ctypes as C

import numpy as np
import pytest

from icempm_multi_b200 import GPUImplementation, Model
from icempm_multi_b200._lib import ICY_ERR_OUT_OF_GRID, PRECISION_FP64, IcyError, lib
from scenarios import standard, stress

pytestmark = pytest.mark.gpu

# FP64 tolerances (relative L2 over all non-disabled points)
TOL = {"pos": 1e-12, "vel": 1e-7, "Fe": 1e-9, "Bp": 1e-6, "Jp": 1e-9}
STATUS_MISMATCH_MAX = 0.01   # fraction of points whose crushed bit may differ


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


def field_errors(a, b):
    """Relative L2 errors of the GPU result a against the oracle result b."""
    m = ~b.disabled()
    def rel(x, y, shift=0.0):
        den = np.linalg.norm(y - shift)
        return float(np.linalg.norm(x - y) / (den if den > 0 else 1.0))
    I = np.array([1.0, 0.0, 0.0, 1.0])[:, None]
    return {
        "pos": rel(a.pos[:, m], b.pos[:, m]),
        "vel": rel(a.vel[:, m], b.vel[:, m]),
        "Fe": rel(a.Fe[:, m] - I, b.Fe[:, m] - I),
        "Bp": rel(a.Bp[:, m], b.Bp[:, m]),
        "Jp": rel(a.Jp_inv[m] - 1.0, b.Jp_inv[m] - 1.0),
        "status": float(np.mean(a.utility[m] != b.utility[m])),
    }


def run_gpu(p, soa, steps, phases=False):
    out = soa.clone()
    g = GPUImplementation(p, out)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    t = 0.0
    if phases:
        for k in range(steps):   # the per-phase calls of icy::Model::Step (model.cpp:40-49)
            t += p.InitialTimeStep
            ix = p.indenter_x_initial + t * p.IndVelocity
            g.reset_grid()
            g.p2g()
            g.receive_halos()
            g.update_nodes(t, ix, p.indenter_y)
            g.g2p(k % p.UpdateEveryNthStep == 0)
            g.receive_points()
    else:
        t = g.run_steps(0, steps, 0.0)
    g.transfer_from_device()
    bins = g.indenter_bins.copy()
    launches = g.kernel_launches()
    g.close()
    return out, t, bins, launches


def assert_close(errs, tol=TOL):
    for k, v in tol.items():
        assert errs[k] <= v, (k, errs)
    assert errs["status"] <= STATUS_MISMATCH_MAX, errs


@pytest.mark.parametrize("make,steps", [(standard, 100), (stress, 40)])
def test_step_matches_oracle(oracle, make, steps):
    p, soa = make()
    ref = soa.clone()
    err, t_ref, bins_ref = oracle.run(p, ref, 0, steps)
    assert err == 0
    out, t, bins, launches = run_gpu(p, soa, steps)
    assert t == t_ref
    assert launches > 0
    errs = field_errors(out, ref)
    print(make.__name__, errs)
    assert_close(errs)
    # indenter force: total over bins
    fr, fo = bins_ref.reshape(-1, 2).sum(0), bins.reshape(-1, 2).sum(0)
    assert np.allclose(fo, fr, rtol=1e-6, atol=1e-6 * (np.abs(fr).max() + 1))


def test_phase_api_matches_step_api(oracle):
    p, soa = standard(seed=3)
    a, _, ba, _ = run_gpu(p, soa, 50, phases=True)
    b, _, bb, _ = run_gpu(p, soa, 50, phases=False)
    errs = field_errors(a, b)
    assert_close(errs)


def test_larger_block_matches_oracle(oracle):
    p, soa = standard(n_cells_x=96, n_cells_y=24, grid=(192, 64), seed=5)
    ref = soa.clone()
    err, _, _ = oracle.run(p, ref, 0, 150)
    assert err == 0
    out, _, _, _ = run_gpu(p, soa, 150)
    errs = field_errors(out, ref)
    print("larger", soa.size, errs)
    assert_close(errs)


def test_reference_cuda_kernels_match_oracle(oracle):
    """The reference's own kernels built for sm_100a agree with the oracle to
    the same tolerance (parity check against the reference GPU build)."""
    from oracle.oracle import RefCuda
    p, soa = standard(seed=6)
    ref = soa.clone()
    err, _, _ = oracle.run(p, ref, 0, 80)
    assert err == 0
    # every point stays > 4 cells inside the grid along the oracle trajectory
    h = p.cellsize
    assert ref.pos[0].min() > 4 * h and ref.pos[0].max() < (p.GridXTotal - 4) * h
    assert ref.pos[1].min() > 2 * h and ref.pos[1].max() < (p.GridY - 4) * h
    out = soa.clone()
    rc, _, _, ms = RefCuda().run(p, out, 0, 80)
    assert rc == 0
    assert_close(field_errors(out, ref))


def test_model_frame_loop(oracle):
    """icy::Model::Step: one frame = UpdateEveryNthStep sub-steps + download,
    force averaged over the frame (model.cpp:27-114)."""
    p, soa = standard(seed=8)
    log = []
    m = Model(p, soa.clone(), force_log=log)
    m.gpu.transfer_ponts_to_device()
    m.Prepare()
    m.Step()
    m.Step()
    n = 2 * p.UpdateEveryNthStep
    assert p.SimulationStep == n and len(log) == 2
    ref = soa.clone()
    oracle.run(p, ref, 0, n)
    assert_close(field_errors(m.gpu.hssoa, ref))
    m.gpu.close()


def run_gpu_opts(p, soa, steps, **opts):
    out = soa.clone()
    g = GPUImplementation(p, out)
    for k, v in opts.items():
        g.set_option(k, v)
    g.update_constants()
    g.transfer_ponts_to_device()
    t = 0.0
    done = 0
    while done < steps:                 # several calls: exercises the first-P2G / last-G2P seams
        k = min(37, steps - done)
        t = g.run_steps(done, k, t)
        done += k
    g.transfer_from_device()
    g.close()
    return out


@pytest.mark.parametrize("opts", [{"tiled": 0}, {"tiled": 1, "resort_every": 0}, {"tiled": 1, "resort_every": 3},
                                  {"tiled": 1, "pipe": 1}, {"tiled": 1, "pipe": 1, "resort_every": 5}])
def test_kernel_paths_match_oracle(oracle, opts):
    p, soa = stress(seed=11)
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 80)[0] == 0
    out = run_gpu_opts(p, soa, 80, **opts)
    assert_close(field_errors(out, ref))


def test_drift_beyond_staged_region(oracle):
    """Points translating at 60 m/s cross several cells without re-binning, so
    their stencils leave the tile's staged region and take the global-memory
    path; the result must still match the oracle."""
    p, soa = standard(n_cells_x=20, n_cells_y=6, grid=(128, 48), seed=4, Gravity=0.0, IndDepth=0.05)
    soa.vel[0, :] = 60.0
    p.indenter_x_initial = p.indenter_x = 0.5   # keep the indenter away from the block
    p.indenter_y = 0.5
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 120)[0] == 0
    moved_cells = (ref.pos[0] - soa.pos[0]).mean() / p.cellsize
    assert moved_cells > 2.0
    out = run_gpu_opts(p, soa, 120, resort_every=0)
    assert_close(field_errors(out, ref))
    out2 = run_gpu_opts(p, soa, 120, resort_every=10)
    assert_close(field_errors(out2, ref))


def test_out_of_grid_reports_reference_code(oracle):
    """A point whose stencil leaves the grid yields the reference's error code
    (70..73) at download instead of a memory fault: the kernels skip it."""
    p, soa = standard(seed=2)
    soa.pos[1, 0] = -0.6 * p.cellsize    # (int)(y/h - 0.5) = -1 < 0  -> code 71
    g = GPUImplementation(p, soa.clone())
    g.update_constants()
    g.transfer_ponts_to_device()
    g.run_steps(0, 2, 0.0)
    with pytest.raises(IcyError) as e:
        g.transfer_from_device()
    assert e.value.code in ICY_ERR_OUT_OF_GRID
    g.close()


def test_pipe_wait_timeout_is_reported_and_recoverable(oracle):
    """The bounded waits of the bulk-copy pipeline: with the first ring stage
    left unfilled on purpose, every wait on it gives up after 1 s, the kernel
    returns and the download reports ICY_ERR_TIMEOUT; the context stays usable
    and the same instance then steps normally."""
    import time
    from icempm_multi_b200._lib import ICY_ERR_TIMEOUT
    p, soa = standard(seed=41)
    g = GPUImplementation(p, soa.clone())
    g.set_option("pipe", 1)
    g.set_option("pipe_fault_test", 1)
    g.update_constants()
    g.transfer_ponts_to_device()
    t0 = time.time()
    g.run_steps(0, 2, 0.0)
    with pytest.raises(IcyError) as e:
        g.transfer_from_device()
    assert e.value.code == ICY_ERR_TIMEOUT
    assert time.time() - t0 < 30
    # recover: clear the status, upload the state again, step without the fault
    g.set_option("pipe_fault_test", 0)
    g.update_constants()
    g.hssoa.copy_from(soa)
    g.transfer_ponts_to_device()
    g.run_steps(0, 40, 0.0)
    g.transfer_from_device()
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 40)[0] == 0
    assert_close(field_errors(g.hssoa, ref))
    g.close()


@pytest.mark.parametrize("precision", [PRECISION_FP64, 1])
def test_matches_reference_cuda_build_directly(oracle, precision):
    """Parity check (a): this library against the reference's own kernels
    built for sm_100a (oracle/_ref/libref_cuda.so, one partition) on the same
    seeded input, 300 steps of a 9,216-point block under the indenter.  Both
    sum node contributions with float atomics in different orders, so the
    FP64 comparison uses the FP64 tolerances (TOL); FP32 split uses POS_TOL."""
    from oracle.oracle import RefCuda
    from test_gpu_split import POS_TOL, run_split
    p, soa = standard(n_cells_x=96, n_cells_y=24, grid=(192, 64), seed=44)
    ref = soa.clone()
    err, _, _ = oracle.run(p, ref, 0, 300)
    assert err == 0
    h = p.cellsize     # the reference kernels do not stop at out-of-grid points: stay well inside
    assert ref.pos[0].min() > 4 * h and ref.pos[0].max() < (p.GridXTotal - 4) * h
    assert ref.pos[1].min() > 2 * h and ref.pos[1].max() < (p.GridY - 4) * h
    rc_out = soa.clone()
    rc, _, _, _ = RefCuda().run(p, rc_out, 0, 300)
    assert rc == 0
    if precision == PRECISION_FP64:
        out, _, _, _ = run_gpu(p, soa, 300)
        assert_close(field_errors(out, rc_out))
    else:
        out, _, _ = run_split(p, soa, 300)
        assert field_errors(out, rc_out)["pos"] <= POS_TOL

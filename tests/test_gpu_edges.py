"""GPU edge cases of the hot path, through the C-ABI, against the FP64 oracle:
an empty instance, stencil bases exactly on the truncation boundary of
(int)(x/h - 0.5) (simulation/kernels.cuh:90), the indenter centre exactly on
a node with mass (normalize of a zero vector, kernels.cuh:270), points next
to every wall, tiles holding more points than one staged chunk, and the full
9.6 M-point instance through size-independent checks (FP32 against FP64,
tiled FP64 against the one-thread-per-item kernels), the largest grid
dimensions the packed cell indices take, and an allocation the device
refuses."""
import numpy as np
import pytest

from icempm_multi_b200 import GPUImplementation
from icempm_multi_b200._lib import PRECISION_FP32_SPLIT, PRECISION_FP64
from icempm_multi_b200.hssoa import HostSideSOA, make_block
from scenarios import params_for, standard
from test_gpu_parity import TOL, assert_close, field_errors, run_gpu
from test_gpu_split import POS_TOL, run_split

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_FP32_SPLIT])
def test_empty_instance(precision):
    p, _ = standard()
    p.nPtsTotal = 0
    empty = HostSideSOA(16)
    g = GPUImplementation(p, empty, precision=precision)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    t = g.run_steps(0, 25, 0.0)
    assert t == pytest.approx(25 * p.InitialTimeStep)
    g.transfer_from_device()
    assert empty.size == 0 and np.all(g.indenter_bins == 0)
    g.close()


def _exact_positions(p, soa):
    """Move some points onto exact truncation boundaries: x/h - 0.5 integer
    (base = that integer, weight w2 = 0), x/h integer, and one ulp either side."""
    h = p.cellsize
    n = soa.size
    idx = np.arange(0, n, max(n // 24, 1))[:24]
    cx = np.floor(soa.pos[0, idx] / h)
    cy = np.floor(soa.pos[1, idx] / h)
    kinds = np.arange(len(idx)) % 4
    fx = np.where(kinds == 0, cx + 0.5, np.where(kinds == 1, cx + 1.0, cx + 0.5))
    x = fx * h
    x = np.where(kinds == 2, np.nextafter(x, -np.inf), np.where(kinds == 3, np.nextafter(x, np.inf), x))
    y = (cy + np.where(kinds % 2 == 0, 0.5, 1.0)) * h
    soa.pos[0, idx] = x
    soa.pos[1, idx] = y
    return idx


def test_truncation_boundaries_match_oracle(oracle):
    p, soa = standard(seed=31)
    _exact_positions(p, soa)
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 60)[0] == 0
    out, _, _, _ = run_gpu(p, soa, 60)
    assert_close(field_errors(out, ref))
    out32, _, _ = run_split(p, soa, 60)
    assert field_errors(out32, ref)["pos"] <= POS_TOL


def test_indenter_centre_on_a_node(oracle):
    p, soa = standard(seed=32, IndVelocity=0.0)
    h = p.cellsize
    k = soa.size // 2
    bx = int(soa.pos[0, k] / h - 0.5)
    by = int(soa.pos[1, k] / h - 0.5)
    # the centre exactly on node (bx + 1, by + 1), which holds mass from point k
    p.indenter_x = p.indenter_x_initial = (bx + 1) * h
    p.indenter_y = p.indenter_y_initial = (by + 1) * h
    ref = soa.clone()
    err, _, bins_ref = oracle.run(p, ref, 0, 40)
    assert err == 0
    out, _, bins, _ = run_gpu(p, soa, 40)
    assert np.all(np.isfinite(out.pos)) and np.all(np.isfinite(out.vel)) and np.all(np.isfinite(bins))
    assert_close(field_errors(out, ref))
    fr, fo = bins_ref.reshape(-1, 2).sum(0), bins.reshape(-1, 2).sum(0)
    assert np.allclose(fo, fr, rtol=1e-6, atol=1e-6 * (np.abs(fr).max() + 1))
    out32, _, bins32 = run_split(p, soa, 40)
    assert np.all(np.isfinite(out32.pos)) and np.all(np.isfinite(bins32))
    assert field_errors(out32, ref)["pos"] <= POS_TOL


def test_points_at_every_wall(oracle):
    """A block lifted off the floor and moved against the left wall, with a
    downward and leftward velocity: the wall conditions of kernels.cuh:290-294
    act on the nodes next to the floor and to the left and right walls."""
    p = params_for(64, 48, 0.25, 1e-4, IndVelocity=0.0, IndDepth=0.0)
    soa = make_block(p, 10 * 0.25, 6 * 0.25, ppc=4, seed=33, n_grains=4)
    h = p.cellsize
    half = soa.size // 2
    # left half of the points against the left wall (base x = 1), the rest at the right wall
    soa.pos[0, :half] += (1.6 * h) - soa.pos[0, :half].min()
    soa.pos[0, half:] += (p.GridXTotal - 4.4) * h - soa.pos[0, half:].max()
    soa.pos[1] += (1.6 * h) - soa.pos[1].min()
    soa.vel[0, :half] = -2.0
    soa.vel[0, half:] = 2.0
    soa.vel[1] = -1.0
    p.indenter_x = p.indenter_x_initial = -100.0   # far away
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 30)[0] == 0
    out, _, _, _ = run_gpu(p, soa, 30)
    assert_close(field_errors(out, ref))
    out32, _, _ = run_split(p, soa, 30)
    assert field_errors(out32, ref)["pos"] <= POS_TOL


def test_tiles_with_more_points_than_a_chunk(oracle):
    """16 points per cell: a 32 x 8-cell tile holds up to 4,096 points, more
    than one staged chunk (1,056 FP64 / 1,280 FP32), so the chunk loop runs."""
    p = params_for(96, 48, 0.25, 5e-5)
    soa = make_block(p, 40 * 0.25, 10 * 0.25, ppc=16, seed=34, n_grains=8)
    assert soa.size == 40 * 10 * 16
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 40)[0] == 0
    out, _, _, _ = run_gpu(p, soa, 40)
    assert_close(field_errors(out, ref))
    out32, _, _ = run_split(p, soa, 40)
    assert field_errors(out32, ref)["pos"] <= POS_TOL


def test_full_size_instance_consistency():
    """The 9.6 M-point bench instance, 20 steps: tiled FP64 against the
    one-thread-per-item FP64 kernels (same arithmetic, other summation order)
    and FP32 split against FP64."""
    from icempm_multi_b200.workloads import LARGE, make_workload
    p, soa = make_workload(LARGE)      # pageable buffers: 4 x 1.2 GB pinned would stay cached in this process
    res = {}
    for name, prec, opts in (("tiled", PRECISION_FP64, {}), ("simple", PRECISION_FP64, {"tiled": 0}),
                             ("fp32", PRECISION_FP32_SPLIT, {})):
        out = soa.clone()
        g = GPUImplementation(p, out, precision=prec)
        for k, v in opts.items():
            g.set_option(k, v)
        g.update_constants()
        g.transfer_ponts_to_device()
        g.run_steps(0, 20, 0.0)
        g.transfer_from_device()
        g.close()
        res[name] = out
    e = field_errors(res["tiled"], res["simple"])
    assert e["pos"] <= TOL["pos"] and e["vel"] <= TOL["vel"] and e["status"] == 0.0, e
    e32 = field_errors(res["fp32"], res["tiled"])
    assert e32["pos"] <= 1e-6, e32


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_FP32_SPLIT])
def test_allocation_refused_is_reported(precision):
    """An instance larger than the device (4e9 points) is refused with
    ICY_ERR_OUT_OF_MEMORY, the device memory the pool took for it goes back to
    the driver (a refused FP32 request left the pool holding all but 23 MB of
    the device, so a second process could not create its context), and the
    next instance is created normally."""
    import torch
    from icempm_multi_b200._lib import ICY_ERR_OUT_OF_MEMORY, IcyError
    p, soa = standard()
    huge = HostSideSOA(1)
    free0 = torch.cuda.mem_get_info()[0]
    with pytest.raises(IcyError) as e:
        GPUImplementation(p, huge, precision=precision, capacity=4_000_000_000)
    assert e.value.code == ICY_ERR_OUT_OF_MEMORY
    assert torch.cuda.mem_get_info()[0] >= free0 - (1 << 30)
    g = GPUImplementation(p, soa.clone(), precision=precision)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.run_steps(0, 5, 0.0)
    g.transfer_from_device()
    g.close()


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_FP32_SPLIT])
def test_grid_beyond_the_packed_indices_is_refused(precision):
    """Node columns (GridX + 2 halo) and rows are packed into 16 bits: 32,768
    columns are refused with ICY_ERR_INVALID_ARGUMENT."""
    from icempm_multi_b200._lib import ICY_ERR_INVALID_ARGUMENT, IcyError
    p = params_for(32768 - 16, 16, 0.25, 1e-4)
    with pytest.raises(IcyError) as e:
        GPUImplementation(p, HostSideSOA(16), precision=precision)
    assert e.value.code == ICY_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("shape", ["widest", "tallest"])
def test_largest_grid_dimensions(oracle, shape):
    """32,767 node columns (or rows), the largest the packed indices take, with
    a block of points at the far end: cell indices near the 16-bit limit, the
    far wall conditions, 20 steps against the oracle."""
    h = 0.25
    if shape == "widest":
        p = params_for(32767 - 16, 16, h, 1e-4, IndVelocity=0.0, IndDepth=0.0)
    else:
        p = params_for(16, 32767, h, 1e-4, IndVelocity=0.0, IndDepth=0.0)
    soa = make_block(p, 8 * h, 4 * h, ppc=4, seed=36, n_grains=4)
    if shape == "widest":
        soa.pos[0] += (p.GridXTotal - 4.5) * h - soa.pos[0].max()   # against the right wall
        soa.vel[0] = 1.0
    else:
        soa.pos[1] += (p.GridY - 6.5) * h - soa.pos[1].max()        # at the top, falling
        soa.vel[0] = 2.0 * (soa.pos[1] - soa.pos[1].mean())          # and sheared (Fe - I, Bp not zero)
    p.indenter_x = p.indenter_x_initial = -100.0
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 20)[0] == 0
    out, _, _, _ = run_gpu(p, soa, 20)
    assert_close(field_errors(out, ref))
    out32, _, _ = run_split(p, soa, 20)
    assert field_errors(out32, ref)["pos"] <= POS_TOL


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_FP32_SPLIT])
def test_kernel_timing_samples_every_nth_launch(precision):
    """With the option profile_every = 4, 16 sub-steps time launches 0, 4, 8
    and 12 of the grid update (16 launches) and of the fused step kernel (15),
    with positive durations; profile_every = 1 times every launch."""
    p, soa = standard(seed=8)
    g = GPUImplementation(p, soa.clone(), precision=precision)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.set_option("resort_every", 0)
    for every, expect in ((4, 4), (1, None)):
        g.set_option("profile_every", every)
        g.profile(True)
        g.run_steps(0, 16, 0.0)
        prof = g.profile_read()
        g.profile(False)
        ms_u, n_u = prof["k_update_nodes"]
        ms_t, n_t = prof["k_tile_g2p2g"]
        assert ms_u > 0 and ms_t > 0
        assert (n_u, n_t) == ((4, 4) if expect else (16, 15))
    from icempm_multi_b200._lib import ICY_ERR_INVALID_ARGUMENT, IcyError
    with pytest.raises(IcyError) as e:
        g.set_option("profile_every", 0)
    assert e.value.code == ICY_ERR_INVALID_ARGUMENT
    g.close()

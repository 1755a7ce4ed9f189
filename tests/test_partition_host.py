"""CPU tests of the slab (multi-partition) decomposition's bookkeeping.

* icy_part_plan against a restatement of the reference's split
  (GPU_Implementation5::split_hssoa_into_partitions,
  simulation/gpu_implementation5.cpp:284-326, with ProxyPoint::getXIndex,
  simulation/hssoa/proxypoint2d.cpp:171-176), on a synthetic block and on the
  reference's own 70k-point geometry;
* the exchange itself, run as two gloo ranks on the CPU (one slab each):
  each rank scatters its points' mass and momentum into its slab's columns
  plus `halo` on each side (quadratic B-spline weights, as P2G), sends its
  2*halo boundary columns to the neighbour and adds what it receives -- the
  column ranges partition.cu copies -- and the result must equal the
  one-domain scatter on those columns; then points moved more than 3 columns
  past the slab are handed over (sizes first, then the packed points) and
  every point ends in the slab that owns its stencil base, none lost."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from icempm_multi_b200._lib import ICY_ERR_INVALID_ARGUMENT, IcyError
from icempm_multi_b200.partition import plan
from scenarios import standard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def plan_like_reference(p, soa, n):
    """split_hssoa_into_partitions restated: equal shares of the sorted
    points, each boundary at the x index (int)(x h^-1 + 0.5) of the first
    point of the next share, the last slab to the end of the grid."""
    out, done, off = [], 0, 0
    for i in range(n):
        share = (soa.size - done) // (n - i)
        if i < n - 1:
            cell = int(soa.pos[0][done + share] * p.cellsize_inv + 0.5)
            out.append((off, cell - off, done, share))
            off = cell
        else:
            out.append((off, p.GridXTotal - off, done, share))
        done += share
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_plan_matches_reference_split(built, n):
    p, soa = standard(n_cells_x=64, n_cells_y=8, grid=(160, 48), seed=3)
    want = plan_like_reference(p, soa, n)
    if min(w for _, w, _, _ in want) < 2 * p.GridHaloSize:
        # a slab narrower than its two boundary regions is refused
        with pytest.raises(IcyError) as e:
            plan(p, soa, n)
        assert e.value.code == ICY_ERR_INVALID_ARGUMENT
        return
    got = plan(p, soa, n)
    assert got == want
    assert sum(c for _, _, _, c in got) == soa.size
    assert got[-1][0] + got[-1][1] == p.GridXTotal and all(w > 0 for _, w, _, _ in got)


def test_plan_on_reference_geometry(built):
    from golden.make_geometry_golden import load_geometry
    p, soa, _, _ = load_geometry()
    for n in (2, 4):
        assert plan(p, soa, n) == plan_like_reference(p, soa, n)


# ---------------------------------------------------------------- gloo ranks
def _weights(f):
    return np.stack([0.5 * (1.5 - f) ** 2, 0.75 - (f - 1.0) ** 2, 0.5 * (f - 0.5) ** 2])


def scatter(x, y, mv, h, ny, col0, ncols):
    """Mass-and-momentum scatter of points (x, y, m v) into columns
    [col0, col0 + ncols) of a grid of ny rows (one array per quantity)."""
    g = np.zeros((3, ncols, ny))
    bx = (x / h - 0.5).astype(np.int64)
    by = (y / h - 0.5).astype(np.int64)
    wx, wy = _weights(x / h - bx), _weights(y / h - by)
    for a in range(3):
        for b in range(3):
            w = wx[a] * wy[b]
            c = bx + a - col0
            ok = (c >= 0) & (c < ncols)
            np.add.at(g[0], (c[ok], (by + b)[ok]), w[ok])
            np.add.at(g[1], (c[ok], (by + b)[ok]), (w * mv[0])[ok])
            np.add.at(g[2], (c[ok], (by + b)[ok]), (w * mv[1])[ok])
    return g


def _slab_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from icempm_multi_b200.partition import plan as plan_
    from scenarios import standard as standard_
    p, soa = standard_(n_cells_x=64, n_cells_y=8, grid=(160, 48), seed=3)
    halo, ny, h = p.GridHaloSize, p.GridY, p.cellsize
    rng = np.random.default_rng(5)
    mv = rng.normal(size=(2, soa.size))
    x0, width, first, count = plan_(p, soa, world)[rank]
    sl = slice(first, first + count)
    # the slab's grid: columns x0 - halo .. x0 + width + halo
    g = scatter(soa.pos[0][sl], soa.pos[1][sl], mv[:, sl], h, ny, x0 - halo, width + 2 * halo)
    # boundary columns: local [0, 2 halo) with the left neighbour, [width, width + 2 halo) with the right
    sides = [(rank - 1, 0), (rank + 1, width)]
    reqs, recv = [], {}
    for nb, c0 in sides:
        if 0 <= nb < world:
            send = torch.from_numpy(np.ascontiguousarray(g[:, c0:c0 + 2 * halo, :]))
            recv[nb] = torch.empty_like(send)
            reqs.append(dist.isend(send, nb))
            reqs.append(dist.irecv(recv[nb], nb))
    for r in reqs:
        r.wait()
    for nb, c0 in sides:
        if nb in recv:
            g[:, c0:c0 + 2 * halo, :] += recv[nb].numpy()
    whole = scatter(soa.pos[0], soa.pos[1], mv, h, ny, x0 - halo, width + 2 * halo)
    grid_ok = bool(np.allclose(g, whole, rtol=1e-12, atol=1e-12))
    # migration: shift every point by 5 columns, hand over those past the slab by more than 3 columns
    x = soa.pos[0][sl] + 5.0 * h
    bx = (x / h - 0.5).astype(np.int64)
    go_left, go_right = bx - x0 < -3, bx - (x0 + width - 3) > 3
    keep = ~(go_left | go_right)
    mine = [x[keep]]
    for nb, mask in ((rank - 1, go_left), (rank + 1, go_right)):
        if 0 <= nb < world:
            n_out = torch.tensor([int(mask.sum())], dtype=torch.int64)
            n_in = torch.empty(1, dtype=torch.int64)
            a, b = dist.isend(n_out, nb), dist.irecv(n_in, nb)
            a.wait()
            b.wait()
            pts_in = torch.empty(int(n_in.item()), dtype=torch.float64)
            a = dist.isend(torch.from_numpy(np.ascontiguousarray(x[mask])), nb)
            b = dist.irecv(pts_in, nb)
            a.wait()
            b.wait()
            mine.append(pts_in.numpy())
        else:
            assert not mask.any()   # the outer slabs keep the grid's ends
    mine = np.concatenate(mine)
    bmine = (mine / h - 0.5).astype(np.int64)
    in_slab = bool(np.all((bmine - x0 >= -3) & (bmine - (x0 + width - 3) <= 3)))
    total = torch.tensor([mine.size], dtype=torch.int64)
    dist.all_reduce(total)
    dist.destroy_process_group()
    out.put((rank, grid_ok, in_slab, int(total.item()), soa.size))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.timeout(120)
def test_two_slabs_over_gloo_exchange_halos_and_points(built):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=100) for _ in range(world))
    for pr in procs:
        pr.join(timeout=30)
        assert pr.exitcode == 0
    for rank, grid_ok, in_slab, total, size in res:
        assert grid_ok, rank
        assert in_slab, rank
        assert total == size

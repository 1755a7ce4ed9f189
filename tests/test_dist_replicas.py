"""CPU test of the multi-process logic of bench.py: N independent replicas
(one process per GPU under torchrun), no collective on the data path, the
timed region bracketed by barriers, the slowest rank's time reported.  Run
here as two gloo ranks on the CPU (127.0.0.1 rendezvous)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, pg = bench.dist_setup(world, backend="gloo")
    assert (r, w, local) == (rank, world, rank)
    bench.barrier(pg, local)
    ms = 10.0 + 5.0 * rank                      # this rank's device time
    ms_max = bench.max_over_ranks(pg, ms, local)
    value = bench.replica_rate(1000, 200, w, ms_max)
    # the reference arm: rank 0 alone measures; the others return at once
    class A:
        pass
    a = A()
    a.gpus, a.steps, a.warmup = w, 1, 1
    ref_rc = bench.run_reference_arm(a) if rank != 0 else 0
    bench.barrier(pg, local)
    pg.destroy_process_group()
    out.put((rank, ms_max, value, ref_rc))


@pytest.mark.timeout(120)
def test_two_replicas_report_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    res.sort()
    ms_max = 10.0 + 5.0 * (world - 1)
    for rank, m, value, ref_rc in res:
        assert m == ms_max
        assert value == 1000 * 200 * world / (ms_max / 1e3)
        assert ref_rc == 0

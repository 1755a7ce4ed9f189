#!/usr/bin/env python
"""Benchmark of the MLS-MPM hot path (particle-steps/s) on one or more B200s.

Headline workload: the single large instance -- grid 4096 x 2048 cells at
h = 0.05 m, an ice block of 150 m x 40 m at 4 points per cell (9.6 M points),
dt = 2e-5 s, E = 1 GPa, nu = 0.3, rho = 980, friction angle 62 deg, cohesion 0,
gravity 9.81, indenter radius 1 m at 1 m/s; seeded synthetic points (no
point-cloud files are available).  One bench step = one MPM sub-step (P2G,
grid update, G2P + return mapping) over the whole instance.  `value` is the
FP32 split-precision path (its accuracy, <= 1e-4 relative position error
against the FP64 oracle after 1000 steps, is a GPU test); the plain FP64
drop-in path is measured on the same instance and reported under "fp64".
The particle state (0.65 GB FP32, 1.23 GB FP64) is larger than L2, so no extra
flush is done between steps.  Also reported: a batch of independent
scenarios ("batched") and a served Poisson request stream ("served").

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs its own replica (the instances are
independent: weak scaling, no collective on the data path); the reported time
is the maximum over ranks of the device-timed region.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from icempm_multi_b200.workloads import LARGE, MEDIUM, SMALL  # noqa: E402
from icempm_multi_b200.workloads import make_workload as _make, workload_params  # noqa: E402

METRIC = "particle-steps/s"
# Algorithmic bytes per particle-step, per kernel: the fields of the particle
# layout each phase of the reference step must touch (P2G reads utility, pos,
# vel, Fe, Bp; G2P reads utility, pos, Fe, Jp and writes pos, vel, Fe, Bp, Jp,
# utility), at the stored width of the layout:
#   FP64 HSSOA: P2G 13 x 8 = 104 B, G2P 8 x 8 + 14 x 8 = 176 B, step 280 B
#   FP32 split: P2G 56 B (utility 4, pos 12, vel 8, Fe 16, Bp 16), G2P 36 + 60 B, step 152 B
# A fused G2P(n)+P2G(n+1) launch does one whole step's work: 280 / 152 B.
ALG_BYTES = {"k_p2g_simple": 104, "k_g2p_simple": 176, "k_tile_g2p2g": 280, "k_tile_p2g": 104,
             "k_tile_g2p": 176}
ALG_BYTES_F32 = {"k_tile_g2p2g": 152, "k_tile_p2g": 56, "k_tile_g2p": 96}
# Bytes per particle-step the fused launch itself has to move: the persistent
# state read once and written once (velocity and Bp stay in registers from
# G2P(n) to P2G(n+1)): FP64 8 + 8 doubles, FP32 split 9 + 9 words.
MOVED_BYTES = {"fp64": 128, "fp32": 72}


WORKLOAD = LARGE


def workload_desc():
    w = WORKLOAD
    return (f"single instance: grid {w['grid_x']}x{w['grid_y']} h={w['h']} m, {w['block_w']:g}x{w['block_h']:g} m "
            f"block, {w['ppc']} ppc, dt={w['dt']:g}, E={w['E']:g}, phi={w['phi']:g}, "
            f"indenter r={w['ind_radius']:g} m at {w['ind_velocity']:g} m/s")


def make_workload(pinned):
    return _make(WORKLOAD, pinned=pinned)


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = ""

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_setup(n_gpus, backend=None):
    """One process per GPU under torchrun (RANK / WORLD_SIZE / LOCAL_RANK from
    the environment, rendezvous at MASTER_ADDR): NCCL on GPUs, gloo on a host
    without CUDA (the CPU tests of this logic).  Each rank runs an independent
    replica; the only collectives are the barrier and the max of the timings."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        pg = dist
    return rank, world, local, pg


def _on_gpu(pg):
    return pg is not None and pg.get_backend() == "nccl"


def max_over_ranks(pg, value, local):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}" if _on_gpu(pg) else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        if _on_gpu(pg):
            pg.barrier(device_ids=[local])
        else:
            pg.barrier()


def replica_rate(points_per_rank, steps, world, ms_max):
    """Whole-job particle-steps/s of `world` independent replicas, timed by the
    slowest rank."""
    return points_per_rank * steps * world / (ms_max / 1e3)


def cpu_reference_rate(p, soa, target_s=15.0, max_steps=50, min_steps=2):
    """The reference's own kernels compiled for the host (oracle/_ref, OpenMP on all
    host cores) on the same workload; returns (particle-steps/s, steps, threads, seconds)."""
    from oracle.oracle import RefHost
    ref = RefHost()
    threads = ref.max_threads()
    work = soa.clone()
    t0 = time.perf_counter()
    ref.run(p, work, 0, 1, 0.0, threads=threads)
    t1 = time.perf_counter() - t0
    steps = int(max(min_steps, min(max_steps, target_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    err, _, _ = ref.run(p, work, 1, steps, p.InitialTimeStep, threads=threads)
    dt = time.perf_counter() - t0
    return soa.size * steps / dt, steps, threads, dt, err


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    p, soa = make_workload(pinned=False)
    p_full = p   # the placed parameters of the full instance (p is rebound to the sample below)
    from oracle.oracle import RefHost
    ref = RefHost()
    threads = ref.max_threads()
    work = soa.clone()
    # one sub-step of the full instance, to size the sample
    t0 = time.perf_counter()
    ref.run(p, work, 0, 1, 0.0, threads=threads)
    t_step = time.perf_counter() - t0
    budget = 150.0
    frac = min(1.0, budget / max((args.steps + args.warmup) * t_step, 1e-9))
    sample = soa
    desc = f"full instance ({soa.size} points) per step"
    if frac < 1.0:
        # a narrower block of the same grid, density and material (bounded sample)
        from icempm_multi_b200 import make_block
        w = dict(WORKLOAD)
        w["block_w"] = max(2.0, WORKLOAD["block_w"] * frac)
        pp = workload_params(w)
        sample = make_block(pp, w["block_w"], w["block_h"], ppc=w["ppc"], seed=w["seed"], n_grains=w["n_grains"])
        p = pp
        desc = f"{w['block_w']:.2f} m x {w['block_h']} m block ({sample.size} points) per step"
    work = sample.clone()
    t = 0.0
    _, t, _ = ref.run(p, work, 0, args.warmup, t, threads=threads)
    t0 = time.perf_counter()
    err, t, _ = ref.run(p, work, args.warmup, args.steps, t, threads=threads)
    el = time.perf_counter() - t0
    v = sample.size * args.steps / el
    ref_gpu = reference_gpu_rate(p_full, soa, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "error_code": err,
        "config": {"workload": workload_desc() + ", FP64",
                   "points": soa.size, "dt": WORKLOAD["dt"]},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
                         "sample": desc + ", reference kernels (simulation/kernels.cuh) built for the host, OpenMP"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": ref_gpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu_rate(p, soa, steps, warmup):
    """The reference's own CUDA kernels (simulation/kernels.cuh, built for
    sm_100a by oracle/Makefile into oracle/_ref/libref_cuda.so) run as one
    partition on the full instance on this GPU: device time of the step loop
    (CUDA events around its launches), after `warmup` untimed steps.  The
    reference's GPU implementation of the path, beside its CPU one."""
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        from oracle.oracle import RefCuda
        ref = RefCuda()
        work = soa.clone()
        err, t, _, _ = ref.run(p, work, 0, warmup, 0.0)
        err2, _, _, ms = ref.run(p, work, warmup, steps, t)
        return {"value": soa.size * steps / (ms / 1e3), "unit": METRIC, "steps": steps, "ms_per_step": ms / steps,
                "error_code": err or err2, "sample": f"the full {soa.size}-point instance, FP64, one partition"}
    except Exception as e:
        return {"unavailable": str(e)[:200]}




PROFILE_EVERY = 8


def measure_instance(p, soa, precision, steps, warmup, local, pg, opts=(), profile=True, clocks=True, tune=False):
    """Device-timed steps of one instance (inputs resident in HBM); with
    `tune`, the FP32 tile shape is picked first by timing each shape on this
    instance (before the warm-up: the tuning steps are not timed)."""
    import torch
    from icempm_multi_b200 import GPUImplementation
    from icempm_multi_b200._lib import PRECISION_FP32_SPLIT, PRECISION_FP64
    prec = PRECISION_FP32_SPLIT if precision == "fp32" else PRECISION_FP64
    stream = torch.cuda.Stream(device=local)
    g = GPUImplementation(p, soa, device=local, precision=prec)
    g.set_stream(stream.cuda_stream)
    for o in opts:
        k, v = o.split("=", 1)
        g.set_option(k, float(v))
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    tuned = None
    if tune and precision == "fp32" and not any(o.startswith("tile_shape=") for o in opts):
        from icempm_multi_b200.autotune import SHAPES, tune_instance
        tuned = tune_instance(g, p, soa.size, steps=10, resorts=(), stream=stream)
        tuned = {"tile_shape": SHAPES[tuned["settings"]["tile_shape"]],
                 "trials": [{"tile_shape": SHAPES[t["tile_shape"]], "ms_per_step": round(t["ms_per_step"], 5)}
                            for t in tuned["trials"]]}
    # the clock sampler runs from before the warm-up to the end of the timed region
    sampler = ClockSampler(local) if clocks else None
    if sampler:
        sampler.__enter__()
        time.sleep(0.5)
    t_sim = g.run_steps(0, warmup, 0.0)
    torch.cuda.synchronize()
    barrier(pg, local)
    torch.cuda.synchronize()
    l0 = g.kernel_launches()
    if profile:
        # every PROFILE_EVERY-th launch of each kernel gets an event pair: each pair
        # costs the stream a few microseconds between kernels
        g.set_option("profile_every", PROFILE_EVERY)
        g.profile(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    t_sim = g.run_steps(warmup, steps, t_sim)
    ev1.record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    barrier(pg, local)
    ms = ev0.elapsed_time(ev1)
    launches = g.kernel_launches() - l0
    prof = g.profile_read() if profile else {}
    g.profile(False)
    timing = amortise_binning(g, ms, steps, prof, opts)
    return g, stream, {"ms": ms, "ms_amortised": timing["ms_amortised"], "timing": timing, "launches": launches,
                       "prof": prof, "clocks": sampler.summary() if sampler else None, "tuned": tuned}


RESORT_EVERY = 64   # the library's default re-binning interval (icy_mpm "resort_every")


def amortise_binning(g, ms, steps, prof, opts):
    """The timed region's time with its re-binnings replaced by their
    amortised share: the points are re-binned every R steps, so K steps carry
    K/R re-binnings whatever the window.  Every re-binning is timed with CUDA
    events (it is rare); if none fell inside the region, R more steps are run
    afterwards to time one.  Returns the raw and amortised milliseconds."""
    R = RESORT_EVERY
    for o in opts:
        k, v = o.split("=", 1)
        if k == "resort_every":
            R = int(float(v))
    b_ms, b_n = prof.get("bin_sort", (0.0, 0))
    per_bin = b_ms / b_n if b_n else None
    if R > 0 and per_bin is None:
        g.set_option("profile_every", 1 << 20)
        g.profile(True)
        g.run_steps(0, R + 1, 0.0)
        extra = g.profile_read().get("bin_sort", (0.0, 0))
        g.profile(False)
        per_bin = extra[0] / extra[1] if extra[1] else 0.0
    amort = ms - b_ms + (steps / R * per_bin if R > 0 else 0.0)
    return {"ms_timed": ms, "bins_in_region": b_n, "bin_ms": per_bin, "resort_every": R, "ms_amortised": amort}


def measure_e2e(g, stream, soa, steps, frame, local, pg):
    """End to end through the C-ABI with host buffers: upload the HSSOA from
    pinned host memory, run the steps with the reference's frame structure (a
    full HSSOA download every UpdateEveryNthStep sub-steps and at the end)."""
    import torch
    barrier(pg, local)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    downloads = 0
    w0 = time.perf_counter()
    e0.record(stream)
    g.transfer_ponts_to_device()
    done, t2 = 0, 0.0
    while done < steps:
        k = min(frame, steps - done)
        t2 = g.run_steps(done, k, t2)
        done += k
        g.transfer_from_device()   # synchronous download, as Model::Step does
        downloads += 1
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    return max(e0.elapsed_time(e1), wall * 1e3), downloads


def measure_batch(n_instances=256, steps=500, seed=7):
    """The batched workload: n_instances floe scenarios (points log-uniform
    10k-500k, grids 128 x 128 to 1024 x 512, E 5e8-2e9 Pa, friction angle
    45-70 deg, indenter 0.5-3 m/s, CFL time steps) advanced together for 500
    steps each in one timed call (one graph replay), which holds the members'
    re-binnings of those steps (every 256 steps)."""
    import torch
    from icempm_multi_b200.batch import Batch
    from icempm_multi_b200.workloads import batch_scenarios, make_workload as mk
    ws = batch_scenarios(n_instances, seed=seed)
    scenes = [mk(w) for w in ws]
    from icempm_multi_b200.autotune import SHAPES, tune_batch_shape
    shape = tune_batch_shape(scenes, sample=32, steps=10)
    b = Batch(n_instances)
    b.set_option("tile_shape", shape["tile_shape"])
    npts = 0
    for p, soa in scenes:
        b.add(p, soa)
        npts += soa.size
    from icempm_multi_b200.autotune import tune_batch
    # launch shape by timing this batch (6 candidates x 30 steps; the re-binning interval stays 256)
    tuned = tune_batch(b, steps=10, resort=False)
    b.step(steps)            # captures the graph for this step count, warms up
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.info()["stream"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.info()["kernel_launches"]
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    b.synchronize()
    ms = e0.elapsed_time(e1)
    launches = b.info()["kernel_launches"] - l0
    b.close()
    return {"value": npts * steps / (ms / 1e3), "unit": METRIC, "instances": n_instances, "points": npts,
            "steps": steps, "ms_per_step": ms / steps, "gpu_launches": int(launches),
            "autotuned": dict(tuned["settings"], tile_shape=SHAPES[shape["tile_shape"]]),
            "shape_trials": [{"tile_shape": SHAPES[t["tile_shape"]], "ps_per_point_step": round(t["ps_per_point_step"], 2)}
                             for t in shape["trials"]],
            "timing": f"one call of {steps} steps, the members' re-binnings (every 256 steps) included",
            "workload": "floe scenarios: points log-uniform 10k-500k, grids 128x128..1024x512 (h=0.1 m), "
                        "E U(5e8,2e9), phi U(45,70), indenter U(0.5,3) m/s, CFL dt, FP32 split, CUDA graph"}


def measure_serve(rate=10.0, duration=12.0, seed=11, budget=150e9, max_instances=128):
    """Served Poisson request stream (the serving workload): every request its
    own seeded floe-indentation scenario -- points log-uniform 5k-2M, E, friction
    angle and indenter speed drawn per request, steps uniform 200-5000 --
    arriving at `rate` per second for `duration` seconds (the same trace every
    run), admitted by a device-memory budget, continuous batching in rounds of
    50 steps; p50/p99 completion latency; the offered load (requested
    particle-steps per second of arrivals) beside the served throughput.  The
    requests' scenarios are built before the run (a request arrives with its
    input) and each host copy is released once uploaded."""
    from concurrent.futures import ThreadPoolExecutor

    from icempm_multi_b200.serve import Server, seeded_requests
    n_req = max(8, int(rate * duration))
    reqs = seeded_requests(rate, n_req, round_steps=50, seed=seed)
    # a request arrives with its scenario: the inputs are built before the run
    # (the generator releases the interpreter lock), not by the serving loop
    with ThreadPoolExecutor(8) as ex:
        list(ex.map(lambda r: r.ensure(), reqs))
    srv = Server(budget_bytes=budget, max_instances=max_instances, round_steps=50, keep_results=False,
                 keep_inputs=False)
    st = srv.run(reqs)
    srv.close()
    offered = sum(r.npts * r.steps for r in reqs) / max(reqs[-1].arrival, 1e-9)
    st.update({"arrival_rate_per_s": rate, "offered_particle_steps_per_s": offered, "round_steps": 50,
               "slots": max_instances, "unit": METRIC,
               "workload": "Poisson arrivals, a seeded scenario per request: points log-uniform 5k-2M, "
                           "steps U(200,5000), FP32 split, continuous batching"})
    return st


def measure_slabs(p, soa, parts=(1, 2, 4), steps=50, warmup=5):
    """One instance in slabs of grid columns on this GPU (icy_part_*, the
    reference's multi-partition layout): the same instance split 1, 2 and 4
    ways, FP64 one-thread-per-item kernels, boundary columns added between
    neighbours at every step and points handed over every
    UpdateEveryNthStep / PointTransferFrequency steps.  Wall time of `steps`
    steps between device synchronisations."""
    import time
    import torch
    from icempm_multi_b200.partition import Partitioned
    out = {}
    for n in parts:
        part = Partitioned(p, n, size_hint=soa.size)
        part.upload(soa)
        t = part.run_steps(0, warmup, 0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        part.run_steps(warmup, steps, t)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        part.close()
        out[f"{n}"] = {"value": soa.size * steps / secs, "ms_per_step": secs * 1e3 / steps}
    return {"unit": METRIC, "steps": steps, "partitions": out,
            "workload": "the single-instance workload in 1, 2 and 4 slabs on one GPU, FP64, one thread per "
                        "point / node (the reference's kernel structure)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default tile shape (no autotuning)")
    ap.add_argument("--no-extra", action="store_true",
                    help="time only the headline path (no other precision, batched or served legs)")
    ap.add_argument("--workload", default="large", choices=["large", "medium", "small"],
                    help="large: the 9.6 M-point headline instance; medium: the 4.8 M-point profiling case; "
                         "small: the 65,536-point CPU-runnable case (L2-resident, launch bound)")
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"],
                    help="path of the headline value: fp32 split precision (default) or fp64")
    ap.add_argument("--opt", action="append", default=[],
                    help="instance option name=value (icy_mpm_set_option), repeatable")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global WORKLOAD
    WORKLOAD = {"large": LARGE, "medium": MEDIUM, "small": SMALL}[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    p, soa = make_workload(pinned=True)
    n = soa.size
    # the other-precision leg starts from the same state (the end-to-end leg downloads into soa)
    soa0 = soa.clone() if not args.no_extra else None

    # ---- headline path, device-resident timed region ----------------------------------
    g, stream, r = measure_instance(p, soa, args.precision, args.steps, args.warmup, local, pg, args.opt,
                                    tune=not args.no_tune)
    ms = max_over_ranks(pg, r["ms_amortised"], local)
    value = replica_rate(n, args.steps, world, ms)

    # ---- end to end through the C-ABI with host buffers ----------------------------------
    frame = p.UpdateEveryNthStep
    ms_e2e, downloads = measure_e2e(g, stream, soa, args.steps, frame, local, pg)
    ms_e2e = max_over_ranks(pg, ms_e2e, local)
    e2e_value = replica_rate(n, args.steps, world, ms_e2e)
    g.close()

    # ---- roofline of the dominant kernel ------------------------------------------------
    peak, peak_kind = peaks()
    prof = r["prof"]
    name, (tot_ms, cnt) = max(prof.items(), key=lambda kv: kv[1][0]) if prof else (None, (0, 0))
    per_launch_ms = tot_ms / max(cnt, 1)
    alg = (ALG_BYTES_F32 if args.precision == "fp32" else ALG_BYTES).get(name, 0) * n
    achieved = alg / (per_launch_ms / 1e3) / 1e9 if per_launch_ms > 0 else 0.0
    moved = MOVED_BYTES[args.precision] * n if name == "k_tile_g2p2g" else alg
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            per_point = json.load(open(tf))["bytes_per_point"].get(f"{name}:{args.precision}")
            traffic = per_point * n if per_point is not None else None
        except Exception:
            traffic = None

    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "timing": dict(r["timing"], note="value = points x steps / ms_amortised: the timed region's re-binnings "
                                         "replaced by steps / resort_every of them (each timed with CUDA events)"),
        "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": workload_desc(),
                   "points": n, "precision": args.precision + (" split" if args.precision == "fp32" else ""),
                   "l2": f"inputs larger than L2 (particle state {n * (36 if args.precision == 'fp32' else 128) / 1e9:.2f} GB "
                         "read and written per step; no extra flush)", "replicas": world,
                   "options": args.opt,
                   "tile_shape": (r["tuned"] or {}).get("tile_shape", "32x8"),
                   "autotune": r["tuned"]},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 16 * 8 * n / args.steps,
                "d2h_bytes_per_step": 16 * 8 * n * downloads / args.steps, "frame_steps": frame,
                "downloads": downloads},
        "gpu_launches": int(r["launches"]),
        "kernels": {k: {"ms_total": v[0], "launches": v[1], "ms_per_launch": v[0] / max(v[1], 1)}
                    for k, v in prof.items()},
        "kernels_timed": f"CUDA events around every {PROFILE_EVERY}th launch of each kernel in the timed "
                         "region (ms_total and launches are those of the timed launches)",
        "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg,
                     # the same launch against the bytes the fused design moves (no vel/Bp round trip)
                     "moved_bytes_per_launch": moved,
                     "moved_frac": (moved / (per_launch_ms / 1e3) / 1e9) / peak if peak and per_launch_ms > 0
                     else None},
        "clocks": r["clocks"],
    }

    # ---- the other precision on the same instance -----------------------------------------
    if not args.no_extra:
        other = "fp64" if args.precision == "fp32" else "fp32"
        k2 = min(args.steps, 100)
        soa2 = soa0.clone(pinned=True)
        g2, st2, r2 = measure_instance(p, soa2, other, k2, args.warmup, local, pg, profile=True, clocks=False)
        ms2 = max_over_ranks(pg, r2["ms_amortised"], local)
        ms2_e2e, dl2 = measure_e2e(g2, st2, soa2, k2, frame, local, pg)
        ms2_e2e = max_over_ranks(pg, ms2_e2e, local)
        g2.close()
        out[other] = {"value": n * k2 * world / (ms2 / 1e3), "unit": METRIC, "ms_per_step": ms2 / k2, "steps": k2,
                      "timing": r2["timing"],
                      "kernels": {k: v[0] / max(v[1], 1) for k, v in r2["prof"].items()},
                      "e2e": {"value": replica_rate(n, k2, world, ms2_e2e), "unit": METRIC,
                              "h2d_bytes_per_step": 16 * 8 * n / k2, "d2h_bytes_per_step": 16 * 8 * n * dl2 / k2,
                              "frame_steps": frame, "downloads": dl2}}

    if rank == 0 and world == 1:
        if not args.no_extra:
            try:
                out["batched"] = measure_batch()
                out["served"] = measure_serve()
                # the same kind of trace at six times the arrival rate: more than the GPU
                # can take, so throughput shows the serving capacity and latency the queueing
                out["served_overload"] = measure_serve(rate=60.0, duration=4.0)
                # over capacity with a budget the admitted scenarios fill: admission is
                # held back by device memory, not by slots (at these request sizes the
                # 150 GB budget would need about 1,300 resident requests to bind)
                out["served_budget"] = measure_serve(rate=20.0, duration=6.0, budget=2.5e9, max_instances=300)
            except Exception as e:
                out["batched_or_served_error"] = str(e)[:300]
            try:
                out["slabs"] = measure_slabs(p, soa)
            except Exception as e:
                out["slabs"] = {"unavailable": str(e)[:200]}
        # ---- CPU baseline ------------------------------------------------------------------
        if not args.no_cpu_baseline:
            try:
                v, steps, threads, secs, err = cpu_reference_rate(p, soa)
                out["cpu_baseline"] = {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
                                       "sample": f"{steps} sub-steps of the full {n}-point instance "
                                                 f"({secs:.1f} s), reference kernels built for the host, OpenMP"}
            except Exception as e:
                out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

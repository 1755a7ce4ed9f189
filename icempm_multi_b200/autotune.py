"""Autotuner: picks the tile shape, launch shape and re-binning interval of
a batch or of a single FP32 instance by timing real steps on its own stream.

Knobs (icy_batch_set_option / icy_mpm_set_option):
  tile_shape   cells per tile of the binned kernels: 32 x 8, 16 x 16, 16 x 8
               (the points a CTA stages and processes at a time, the span of
               the sort bins; a batch takes it while empty, so
               tune_batch_shape tries it on batches of a sample of the
               scenarios)
  tile_ctas    persistent CTAs of the fused tile kernel (multiples of the SM count)
  update_ctas  CTAs of the list-driven grid update
  resort_every steps between re-binnings of the points by tile (the binning
               costs a few hundred microseconds per member set; between
               re-binnings points drift off their cells and take the slower
               scatter path)

The search is coordinate descent in that order: every candidate is applied,
one step call captures its graph, then two calls of `steps` sub-steps are
timed with CUDA events and the faster counts (a re-binning falls in one of
them at most); the best value of a knob is kept before the next knob is
tried.  The
re-binning interval is timed over two intervals so a re-binning is included.
The tuning steps advance the simulation like any other steps.  Results can be
cached per workload signature in a JSON file.
"""
import json
import os

import torch


def _sm_count(device):
    return torch.cuda.get_device_properties(device).multi_processor_count


def _time_steps(batch, steps, reps=1):
    """ms per step of `steps`-step calls: the fastest of `reps` timed calls
    (a re-binning of the members lands in one call at most when steps is
    small against the re-binning interval)."""
    info = batch.info()
    stream = torch.cuda.ExternalStream(info["stream"])
    batch.step(steps)                          # graph capture for this step count + warm-up
    batch.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.step(steps)
        e1.record(stream)
        batch.synchronize()
        ms = e0.elapsed_time(e1) / steps
        best = ms if best is None else min(best, ms)
    return best


def signature(batch):
    info = batch.info()
    name = torch.cuda.get_device_name()
    return f"{name}|members={info['live']}|points={round(info['points'], -4)}"


def tune_batch(batch, steps=20, device=0, cache=None, log=None, resort=True):
    """Tune `batch` in place; returns {"settings": {...}, "trials": [...]}.
    resort=False keeps the re-binning interval (and the tuning short: the
    interval trials run 2 x 1,792 steps)."""
    key = signature(batch)
    if cache and os.path.exists(cache):
        try:
            known = json.load(open(cache))
            if key in known:
                for k, v in known[key]["settings"].items():
                    batch.set_option(k, v)
                return dict(known[key], cached=True)
        except (OSError, ValueError):
            pass
    sms = _sm_count(device)
    space = [
        ("tile_ctas", [sms * k for k in (4, 3, 2)]),
        ("update_ctas", [sms * k for k in (8, 4, 16)]),
    ]
    settings = {}
    trials = []
    for knob, values in space:
        best = None
        for v in values:
            batch.set_option(knob, v)
            ms = _time_steps(batch, steps, reps=2)
            trials.append({knob: v, "ms_per_step": ms})
            if log:
                log(f"autotune {knob}={v}: {ms:.4f} ms/step")
            if best is None or ms < best[1]:
                best = (v, ms)
        batch.set_option(knob, best[0])
        settings[knob] = best[0]
    # re-binning interval: time two intervals of each candidate so each includes re-binnings
    best = None
    for every in ((128, 256, 512) if resort else ()):
        batch.set_option("resort_every", every)
        ms = _time_steps(batch, 2 * every)
        trials.append({"resort_every": every, "ms_per_step": ms})
        if log:
            log(f"autotune resort_every={every}: {ms:.4f} ms/step")
        if best is None or ms < best[1]:
            best = (every, ms)
    if best is not None:
        batch.set_option("resort_every", best[0])
        settings["resort_every"] = best[0]
    out = {"settings": settings, "trials": trials, "signature": key, "cached": False}
    if cache:
        try:
            known = json.load(open(cache)) if os.path.exists(cache) else {}
        except (OSError, ValueError):
            known = {}
        known[key] = {"settings": settings, "trials": trials, "signature": key}
        with open(cache, "w") as f:
            json.dump(known, f, indent=1)
    return out


SHAPES = {0: "32x8", 1: "16x16", 2: "16x8"}


def _time_instance(g, stream, steps, reps=2, step0=0):
    """ms per step of an instance: the fastest of `reps` timed calls of
    `steps` sub-steps after an untimed one (re-binning, warm-up)."""
    t = g.run_steps(step0, steps, 0.0)
    torch.cuda.synchronize()
    best = None
    for r in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t = g.run_steps(step0 + (r + 1) * steps, steps, t)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        best = ms if best is None else min(best, ms)
    return best


def instance_signature(g, params, points):
    name = torch.cuda.get_device_name()
    return f"{name}|grid={params.GridXTotal}x{params.GridY}|points={round(points, -4)}"


def tune_instance(g, params, points, steps=20, shapes=(0, 1, 2), resorts=(64, 128, 256), cache=None, log=None,
                  stream=None):
    """Tune a single FP32 split-precision instance (GPUImplementation, points
    uploaded) in place: tile shape, then re-binning interval, each candidate
    timed on real steps of the instance (which advance its simulation).
    Returns {"settings": {...}, "trials": [...], "signature": ..., "cached": bool}."""
    key = instance_signature(g, params, points)
    if cache and os.path.exists(cache):
        try:
            known = json.load(open(cache))
            if key in known:
                for k, v in known[key]["settings"].items():
                    g.set_option(k, v)
                return dict(known[key], cached=True)
        except (OSError, ValueError):
            pass
    if stream is None:
        stream = torch.cuda.Stream()
        g.set_stream(stream.cuda_stream)
    settings, trials = {}, []
    best = None
    for sh in shapes:
        g.set_option("tile_shape", sh)   # the points are binned again at the next step
        ms = _time_instance(g, stream, steps)
        trials.append({"tile_shape": sh, "ms_per_step": ms})
        if log:
            log(f"autotune tile_shape={SHAPES[sh]}: {ms:.4f} ms/step")
        if best is None or ms < best[1]:
            best = (sh, ms)
    g.set_option("tile_shape", best[0])
    settings["tile_shape"] = best[0]
    best = None
    for every in resorts:
        g.set_option("resort_every", every)
        ms = _time_instance(g, stream, every, reps=1)   # one interval: one re-binning
        trials.append({"resort_every": every, "ms_per_step": ms})
        if log:
            log(f"autotune resort_every={every}: {ms:.4f} ms/step")
        if best is None or ms < best[1]:
            best = (every, ms)
    if best is not None:
        g.set_option("resort_every", best[0])
        settings["resort_every"] = best[0]
    out = {"settings": settings, "trials": trials, "signature": key, "cached": False}
    if cache:
        try:
            known = json.load(open(cache)) if os.path.exists(cache) else {}
        except (OSError, ValueError):
            known = {}
        known[key] = {"settings": settings, "trials": trials, "signature": key}
        with open(cache, "w") as f:
            json.dump(known, f, indent=1)
    return out


def tune_batch_shape(scenes, shapes=(0, 1, 2), sample=32, steps=20, device=0, log=None):
    """The tile shape for a batch of `scenes` [(params, soa)]: each shape timed
    on a temporary batch of (up to) `sample` of them, evenly spread over the
    list (a batch takes its shape while empty).  Returns
    {"tile_shape": best, "trials": [...]}; the caller sets the shape on its
    own batch before adding members."""
    from .batch import Batch
    pick = scenes[::max(1, len(scenes) // sample)][:sample]
    trials, best = [], None
    for sh in shapes:
        b = Batch(len(pick), device=device)
        b.set_option("tile_shape", sh)
        for p, soa in pick:
            b.add(p, soa)
        ms = _time_steps(b, steps, reps=2)
        npts = b.info()["points"]
        b.close()
        ps = ms * 1e-3 / max(npts, 1) * 1e12   # picoseconds per point-step
        trials.append({"tile_shape": sh, "ms_per_step": ms, "ps_per_point_step": ps})
        if log:
            log(f"autotune batch tile_shape={SHAPES[sh]}: {ps:.1f} ps per point-step")
        if best is None or ms < best[1]:
            best = (sh, ms)
    return {"tile_shape": best[0], "trials": trials, "sample": len(pick)}

"""Autotuner for batches: picks the launch shape and the re-binning interval
of a Batch by timing real steps of that batch on its own stream.

Knobs (icy_batch_set_option):
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

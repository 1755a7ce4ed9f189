"""Batches of independent floe scenarios advanced together (FP32 split precision).

Python face of the icy_batch_* C-ABI (include/icempm.h): members are added
with their own SimParams and HSSOA, every batch step advances all of them by
the same number of sub-steps with a handful of kernel launches replayed as a
CUDA graph, and each member keeps its own simulation time and step index.
"""
import ctypes as C

import numpy as np

from ._lib import PRECISION_FP32_SPLIT, check, lib


class Batch:
    def __init__(self, max_instances, device=0):
        self.device = device
        self._b = C.c_void_p()
        check(lib().icy_batch_create(device, int(max_instances), C.byref(self._b)), "icy_batch_create")
        self.params = {}
        self._keep = {}         # host buffers of asynchronous admissions
        self._retiring = {}     # slot -> (state buffer, bins) of retirements in flight

    def close(self):
        if self._b:
            lib().icy_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, params, soa):
        """Admit a scenario; returns its slot."""
        slot = C.c_int(-1)
        check(lib().icy_batch_add(self._b, C.byref(params), soa.ptr, soa.capacity, soa.size, C.byref(slot)),
              "icy_batch_add")
        self.params[slot.value] = params
        return slot.value

    def add_async(self, params, soa):
        """Admit a scenario without waiting for its upload (icy_batch_add_async):
        soa must stay unchanged until a round queued after this call has run;
        returns its slot."""
        slot = C.c_int(-1)
        check(lib().icy_batch_add_async(self._b, C.byref(params), soa.ptr, soa.capacity, soa.size, C.byref(slot)),
              "icy_batch_add_async")
        self.params[slot.value] = params
        self._keep[slot.value] = soa
        return slot.value

    def retire(self, slot, soa=None, bins=True):
        """Take a member out after the queued work; its state goes into soa (if
        given) and its force bins into a new array while later rounds run.
        Finish with collect(slot)."""
        p = self.params[slot]
        b = np.zeros(2 * p.n_indenter_subdivisions) if bins else None
        check(lib().icy_batch_retire(self._b, int(slot), soa.ptr if soa is not None else None,
                                     soa.capacity if soa is not None else 0,
                                     b.ctypes.data_as(C.c_void_p) if b is not None else None), "icy_batch_retire")
        self._keep.pop(slot, None)
        self._retiring[slot] = (soa, b)

    def collect(self, slot, wait=True):
        """None while a retirement's copy runs (wait=False); else frees the slot
        and returns (sim_time, next_step, bins)."""
        done, n, t, st = C.c_int(0), C.c_uint(0), C.c_double(0), C.c_int64(0)
        rc = lib().icy_batch_collect(self._b, int(slot), 1 if wait else 0, C.byref(done), C.byref(n), C.byref(t),
                                     C.byref(st))
        if not done.value:
            check(rc, "icy_batch_collect")
            return None
        soa, b = self._retiring.pop(slot)
        self.params.pop(slot, None)
        if soa is not None:
            soa.size = n.value
        check(rc, "icy_batch_collect")
        return t.value, st.value, b

    def wait_steps(self, in_flight):
        """Block until at most in_flight of the step() calls so far are unfinished."""
        check(lib().icy_batch_wait_steps(self._b, int(in_flight)), "icy_batch_wait_steps")

    def remove(self, slot):
        check(lib().icy_batch_remove(self._b, int(slot)), "icy_batch_remove")
        self.params.pop(slot, None)
        self._keep.pop(slot, None)

    def step(self, nsteps):
        check(lib().icy_batch_step(self._b, int(nsteps)), "icy_batch_step")

    def synchronize(self):
        check(lib().icy_batch_synchronize(self._b), "icy_batch_synchronize")

    def download(self, slot, soa):
        """Member state into soa (upload order); returns (sim_time, next_step, bins)."""
        p = self.params[slot]
        bins = np.zeros(2 * p.n_indenter_subdivisions)
        n = C.c_uint(0)
        t = C.c_double(0)
        st = C.c_int64(0)
        rc = lib().icy_batch_download(self._b, int(slot), soa.ptr, soa.capacity, C.byref(n),
                                      bins.ctypes.data_as(C.c_void_p), C.byref(t), C.byref(st))
        soa.size = n.value
        check(rc, "icy_batch_download")
        return t.value, st.value, bins

    def set_clock(self, slot, sim_time, step):
        """Resume a member at (sim_time, step): its clock and indenter position."""
        check(lib().icy_batch_set_clock(self._b, int(slot), float(sim_time), int(step)), "icy_batch_set_clock")

    def set_option(self, name, value):
        check(lib().icy_batch_set_option(self._b, name.encode(), float(value)), "icy_batch_set_option")

    def reserve(self, nbytes):
        """Grow the device's instance memory pool to at least nbytes (icy_mpm_reserve):
        members admitted later take their buffers from memory already mapped."""
        check(lib().icy_mpm_reserve(self.device, int(nbytes)), "icy_mpm_reserve")

    def info(self):
        live, pts, launches, stream = C.c_int(0), C.c_int64(0), C.c_int64(0), C.c_void_p()
        check(lib().icy_batch_info(self._b, C.byref(live), C.byref(pts), C.byref(launches), C.byref(stream)),
              "icy_batch_info")
        return {"live": live.value, "points": pts.value, "kernel_launches": launches.value,
                "stream": stream.value}

    def device_bytes(self, slot):
        return lib().icy_batch_device_bytes(self._b, int(slot))


def device_bytes(params, capacity, precision=PRECISION_FP32_SPLIT):
    """Device memory an instance of this size allocates."""
    return lib().icy_mpm_device_bytes(C.byref(params), int(capacity), int(precision))


def main():
    """python -m icempm_multi_b200.batch [--instances 256] [--steps 10] [--seed 7] [--repeat 2]
                                        [--workload large|medium|small]

    Builds the batched workload (icempm_multi_b200.workloads.batch_scenarios,
    or copies of one single-instance workload) and advances it `repeat` times by `steps` sub-steps (the first call
    captures the CUDA graph), printing the device time of each call."""
    import argparse
    import time

    from .workloads import batch_scenarios, make_workload
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--workload", choices=["large", "medium", "small"],
                    help="every member a copy of this single-instance workload instead of the floe scenarios")
    a = ap.parse_args()
    b = Batch(a.instances)
    n = 0
    if a.workload:
        from . import workloads
        members = [getattr(workloads, a.workload.upper())] * a.instances
    else:
        members = batch_scenarios(a.instances, seed=a.seed)
    for w in members:
        p, soa = make_workload(w)
        b.add(p, soa)
        n += soa.size
    for r in range(a.repeat):
        t0 = time.perf_counter()
        b.step(a.steps)
        b.synchronize()
        print(f"call {r}: {a.steps} steps of {a.instances} members ({n} points) in "
              f"{1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)
    b.close()


if __name__ == "__main__":
    main()

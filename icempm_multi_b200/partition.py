"""One instance in slabs of grid columns (partitions) over the C-ABI
(include/icempm.h, icy_part_*): the multi-partition GPU_Implementation5 of
the reference (simulation/gpu_implementation5.cpp:31-204,221-326), with
several partitions on one GPU or one GPU each."""
import ctypes as C

import numpy as np

from ._lib import check, lib


def plan(params, soa, n_partitions):
    """The split of GPU_Implementation5::split_hssoa_into_partitions as the
    library computes it: per partition (first column, columns, first point,
    points)."""
    x0 = np.zeros(n_partitions, dtype=np.int32)
    width = np.zeros(n_partitions, dtype=np.int32)
    first = np.zeros(n_partitions, dtype=np.uint32)
    count = np.zeros(n_partitions, dtype=np.uint32)
    vp = C.c_void_p
    check(lib().icy_part_plan(C.byref(params), soa.ptr, soa.capacity, soa.size, n_partitions,
                              x0.ctypes.data_as(vp), width.ctypes.data_as(vp), first.ctypes.data_as(vp),
                              count.ctypes.data_as(vp)), "icy_part_plan")
    return [(int(a), int(b), int(c), int(d)) for a, b, c, d in zip(x0, width, first, count)]


class Partitioned:
    """An instance split into `n_partitions` slabs, partition i on
    devices[i] (default: all on device 0), each with room for
    `capacity_per_partition` points (default: the HSSOA's capacity share
    with the reference's ExtraSpaceForIncomingPoints)."""

    def __init__(self, params, n_partitions, devices=None, capacity_per_partition=None, size_hint=None):
        self.params = params
        self.n = n_partitions
        if capacity_per_partition is None:
            total = size_hint if size_hint is not None else params.nPtsTotal
            capacity_per_partition = int(total / n_partitions * (1 + max(params.ExtraSpaceForIncomingPoints, 0.5))) + 64
        self.capacity_per_partition = capacity_per_partition
        dev = None
        if devices is not None:
            dev = (C.c_int * n_partitions)(*devices)
        h = C.c_void_p()
        check(lib().icy_part_create(C.byref(params), n_partitions, dev, capacity_per_partition, C.byref(h)),
              "icy_part_create")
        self._h = h

    def upload(self, soa):
        check(lib().icy_part_upload(self._h, soa.ptr, soa.capacity, soa.size), "icy_part_upload")

    def run_steps(self, step0, nsteps, sim_time):
        t = C.c_double(sim_time)
        check(lib().icy_part_step(self._h, step0, nsteps, C.byref(t)), "icy_part_step")
        return t.value

    def download(self, soa):
        """Points back into `soa` in upload order; returns the indenter force bins."""
        bins = np.zeros(2 * self.params.n_indenter_subdivisions)
        size = C.c_uint(0)
        check(lib().icy_part_download(self._h, soa.ptr, soa.capacity, C.byref(size),
                                      bins.ctypes.data_as(C.c_void_p)), "icy_part_download")
        soa.size = size.value
        return bins

    def info(self, part):
        x0, w, dev = C.c_int(0), C.c_int(0), C.c_int(0)
        cnt = C.c_uint(0)
        check(lib().icy_part_info(self._h, part, C.byref(x0), C.byref(w), C.byref(cnt), C.byref(dev)),
              "icy_part_info")
        return {"x0": x0.value, "width": w.value, "slots": cnt.value, "device": dev.value}

    def close(self):
        if self._h:
            lib().icy_part_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

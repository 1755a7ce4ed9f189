"""Python mirror of the reference's step interface over the C-ABI.

``GPUImplementation`` follows GPU_Implementation5 (simulation/gpu_implementation5.h:25-59)
for one partition on one GPU; ``Model`` follows icy::Model
(simulation/model.h:32-57, model.cpp:27-139): Reset / Prepare / Step, where
Step runs UpdateEveryNthStep sub-steps, downloads the particles, averages the
indenter force over the frame and logs it.  Every call raises IcyError on a
non-zero status, as the reference throws std::runtime_error.
"""
import ctypes as C
import threading

import numpy as np

from ._lib import PRECISION_FP64, check, lib
from .hssoa import HostSideSOA


class GPUImplementation:
    def __init__(self, params, hssoa=None, device=0, precision=PRECISION_FP64, capacity=None):
        self.prms = params
        self.hssoa = hssoa
        self.device = device
        self.precision = precision
        self.indenter_force = np.zeros(2)
        self.transfer_completion_callback = None
        self._h = C.c_void_p()
        cap = capacity or (hssoa.capacity if hssoa is not None else max(params.nPtsTotal, 1))
        check(lib().icy_mpm_create(C.byref(params), device, int(cap), precision, C.byref(self._h)),
              "icy_mpm_create")

    # --- life cycle -----------------------------------------------------------
    def close(self):
        if self._h:
            lib().icy_mpm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr):
        check(lib().icy_mpm_set_stream(self._h, C.c_void_p(stream_ptr)), "icy_mpm_set_stream")

    def get_stream(self):
        return lib().icy_mpm_get_stream(self._h)

    # --- GPU_Implementation5 interface ------------------------------------------
    def update_constants(self):
        check(lib().icy_mpm_update_constants(self._h, C.byref(self.prms)), "update_constants")

    def transfer_ponts_to_device(self):
        s = self.hssoa
        check(lib().icy_mpm_transfer_points_to_device(self._h, s.ptr, s.capacity, s.size),
              "transfer_ponts_to_device")

    def transfer_from_device(self):
        s = self.hssoa
        bins = np.zeros(2 * self.prms.n_indenter_subdivisions)
        n = C.c_uint(0)
        rc = lib().icy_mpm_transfer_from_device(self._h, s.ptr, s.capacity, C.byref(n),
                                                bins.ctypes.data_as(C.c_void_p))
        s.size = n.value
        check(rc, "transfer_from_device")
        self.indenter_force = np.array([bins[0::2].sum(), bins[1::2].sum()])
        self.indenter_bins = bins
        if self.transfer_completion_callback:
            self.transfer_completion_callback()

    def reset_indenter_force_accumulator(self):
        check(lib().icy_mpm_reset_indenter_force_accumulator(self._h), "reset_indenter_force_accumulator")

    def reset_grid(self):
        check(lib().icy_mpm_reset_grid(self._h), "reset_grid")

    def p2g(self):
        check(lib().icy_mpm_p2g(self._h), "p2g")

    def receive_halos(self):
        check(lib().icy_mpm_receive_halos(self._h), "receive_halos")

    def update_nodes(self, simulation_time, indenter_x=None, indenter_y=None):
        ix = self.prms.indenter_x if indenter_x is None else indenter_x
        iy = self.prms.indenter_y if indenter_y is None else indenter_y
        check(lib().icy_mpm_update_nodes(self._h, ix, iy, simulation_time), "update_nodes")

    def g2p(self, recordPQ, enablePointTransfer=False):
        check(lib().icy_mpm_g2p(self._h, int(recordPQ), int(enablePointTransfer)), "g2p")

    def receive_points(self):
        check(lib().icy_mpm_receive_points(self._h), "receive_points")

    def synchronize(self):
        check(lib().icy_mpm_synchronize(self._h), "synchronize")

    def status(self):
        return lib().icy_mpm_status(self._h)

    def kernel_launches(self):
        return lib().icy_mpm_kernel_launches(self._h)

    def counters(self):
        """Device counters: points off their binned cell (per P2G), FP32 launches
        that fused the grid update, launches that fell back to the update kernel."""
        c = [C.c_int64(0) for _ in range(3)]
        check(lib().icy_mpm_counters(self._h, *[C.byref(x) for x in c]), "icy_mpm_counters")
        return {"moved_points": c[0].value, "fused_launches": c[1].value, "fallback_launches": c[2].value}

    def set_option(self, name, value):
        """Instance tuning option (include/icempm.h: icy_mpm_set_option)."""
        check(lib().icy_mpm_set_option(self._h, name.encode(), float(value)), "icy_mpm_set_option")

    def profile(self, enable):
        """Start (clearing) or stop per-kernel CUDA-event timing on the instance stream."""
        check(lib().icy_mpm_profile(self._h, int(bool(enable))), "icy_mpm_profile")

    def profile_read(self):
        """{kernel name: (total ms, timed launches)} recorded since profiling was
        enabled (every launch, or every n-th with the option "profile_every")."""
        mx = 32
        names = C.create_string_buffer(48 * mx)
        ms = np.zeros(mx)
        n = np.zeros(mx, dtype=np.int64)
        cnt = C.c_int(0)
        check(lib().icy_mpm_profile_read(self._h, mx, names, ms.ctypes.data_as(C.c_void_p),
                                         n.ctypes.data_as(C.c_void_p), C.byref(cnt)), "icy_mpm_profile_read")
        out = {}
        for k in range(min(cnt.value, mx)):
            name = names.raw[48 * k:48 * (k + 1)].split(b"\0", 1)[0].decode()
            out[name] = (float(ms[k]), int(n[k]))
        return out

    # --- fused multi-step path ------------------------------------------------
    def run_steps(self, step0, nsteps, sim_time):
        """Queue nsteps sub-steps of Model::Step on the device; returns the new time."""
        t = C.c_double(sim_time)
        check(lib().icy_mpm_step(self._h, int(step0), int(nsteps), C.byref(t)), "icy_mpm_step")
        return t.value


class Model:
    """icy::Model for one GPU (simulation/model.cpp:27-139)."""

    def __init__(self, params, hssoa, device=0, precision=PRECISION_FP64, force_log=None):
        self.prms = params
        self.gpu = GPUImplementation(params, hssoa, device=device, precision=precision)
        self.processing_current_cycle_data = threading.Lock()
        self.accessing_point_data = threading.Lock()
        self.force_log = force_log  # list or file-like receiving "t,|F|,Fx,Fy" lines
        self.abort_requested = False
        self.Reset()

    def Reset(self):
        self.prms.SimulationStep = 0
        self.prms.SimulationTime = 0.0

    def Prepare(self):
        self.abort_requested = False
        self.gpu.update_constants()

    def UnlockCycleMutex(self):
        self.processing_current_cycle_data.release()

    def Step(self):
        """One frame: UpdateEveryNthStep sub-steps, then download (model.cpp:27-114)."""
        p = self.prms
        t = p.SimulationTime
        self.gpu.reset_indenter_force_accumulator()
        n = p.UpdateEveryNthStep - (p.SimulationStep % p.UpdateEveryNthStep)
        t = self.gpu.run_steps(p.SimulationStep, n, t)
        self.processing_current_cycle_data.acquire()
        with self.accessing_point_data:
            self.gpu.transfer_from_device()
            p.SimulationTime = t
            p.SimulationStep += n
            self.gpu.indenter_force = self.gpu.indenter_force / float(n)
            f = self.gpu.indenter_force
            line = f"{p.SimulationTime},{np.hypot(f[0], f[1])},{f[0]},{f[1]}"
            if self.force_log is not None:
                if hasattr(self.force_log, "append"):
                    self.force_log.append(line)
                else:
                    self.force_log.write(line + "\n")
        if self.gpu.transfer_completion_callback is None:
            self.UnlockCycleMutex()
        return p.SimulationTime < p.SimulationEndTime

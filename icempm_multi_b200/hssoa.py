"""Host-side particle SoA in the reference layout.

Mirror of ``HostSideSOA`` (simulation/hssoa/host_side_soa.h:52-74): one buffer
of 16 lines x ``capacity`` doubles, ``size`` points in use, line 0 holding the
64-bit utility word bit-cast into a double.  The buffer can be page-locked
(icy_host_alloc, released by icy_host_free when the object is collected) so
that uploads and downloads run at full PCIe/C2C speed.
"""
import ctypes as C
import weakref

import numpy as np

from ._lib import (BP00, FE00, IDX_JP_INV, IDX_P, IDX_Q, N_PTS_ARRAYS, POSX, STATUS_CRUSHED, STATUS_DISABLED,
                   STATUS_LIQUID, VELX, check, lib)


class HostSideSOA:
    def __init__(self, capacity, pinned=False):
        self.capacity = int(capacity)
        self.size = 0
        self._keep = None
        if pinned:
            n = N_PTS_ARRAYS * self.capacity
            ptr = C.c_void_p()
            check(lib().icy_host_alloc(n * 8, C.byref(ptr)), "icy_host_alloc")
            mem = (C.c_double * n).from_address(ptr.value)
            # freed when the last numpy view of the buffer is gone
            self._keep = weakref.finalize(mem, lib().icy_host_free, ptr)
            self.buf = np.ctypeslib.as_array(mem).reshape(N_PTS_ARRAYS, self.capacity)
        else:
            self.buf = np.zeros((N_PTS_ARRAYS, self.capacity), dtype=np.float64)

    # --- access -----------------------------------------------------------
    @property
    def ptr(self):
        return self.buf.ctypes.data_as(C.c_void_p)

    def line(self, k):
        return self.buf[k, :self.size]

    @property
    def utility(self):
        return self.buf[0, :self.size].view(np.int64)

    @property
    def pos(self):
        return self.buf[POSX:POSX + 2, :self.size]

    @property
    def vel(self):
        return self.buf[VELX:VELX + 2, :self.size]

    @property
    def Fe(self):
        return self.buf[FE00:FE00 + 4, :self.size]

    @property
    def Bp(self):
        return self.buf[BP00:BP00 + 4, :self.size]

    @property
    def Jp_inv(self):
        return self.buf[IDX_JP_INV, :self.size]

    @property
    def PQ(self):
        return self.buf[IDX_P:IDX_Q + 1, :self.size]

    def crushed(self):
        return (self.utility & STATUS_CRUSHED) != 0

    def disabled(self):
        return (self.utility & STATUS_DISABLED) != 0

    def liquid(self):
        return (self.utility & STATUS_LIQUID) != 0

    def grains(self):
        return (self.utility & 0xFFFF).astype(np.int64)

    def copy_from(self, other):
        n = other.size
        assert n <= self.capacity
        self.buf[:, :n] = other.buf[:, :n]
        self.size = n
        return self

    def clone(self, pinned=False):
        c = HostSideSOA(max(self.size, 1), pinned=pinned)
        return c.copy_from(self)

    def active_count(self):
        """Non-disabled points (simulation/gpu_implementation5.cpp:399-405)."""
        return int((~self.disabled()).sum())


def make_block(params, block_w, block_h, ppc=4, seed=1, n_grains=0, extra_space=0.0, pinned=False):
    """Seeded synthetic ice block placed as LoadRawPoints places a cloud
    (simulation/snapshotmanager.cpp:29-121).  Updates ``params`` in place
    (nPtsTotal, Volume, ParticleVolume, indenter start, derived constants)."""
    n = lib().icy_scene_block_count(C.byref(params), block_w, block_h, ppc)
    cap = int(n * (1 + extra_space)) if extra_space else int(n)
    soa = HostSideSOA(max(cap, 1), pinned=pinned)
    out_n = C.c_uint(0)
    rc = lib().icy_scene_block(C.byref(params), block_w, block_h, ppc, seed, n_grains, soa.ptr, soa.capacity,
                               C.byref(out_n))
    check(rc, "icy_scene_block")
    soa.size = out_n.value
    return soa


def load_h5(params, path, extra_space=None, pinned=False):
    """A point cloud of the reference's HDF5 format ("x", "y", "llGrainIDs" with
    its "volume" attribute), read and placed as SnapshotManager::LoadRawPoints
    does (simulation/snapshotmanager.cpp:29-109).  Capacity = points x (1 +
    ExtraSpaceForIncomingPoints) unless extra_space is given.  Updates
    ``params`` in place."""
    from ._lib import host_lib
    H = host_lib()
    n = C.c_uint(0)
    rc = H.icy_h5_count(str(path).encode(), C.byref(n))
    if rc != 0:
        raise RuntimeError(f"icy_h5_count({path}) failed with status {rc}: {H.icy_host_last_error().decode()}")
    es = params.ExtraSpaceForIncomingPoints if extra_space is None else extra_space
    soa = HostSideSOA(max(int(n.value * (1 + es)), 1), pinned=pinned)
    got = C.c_uint(0)
    rc = H.icy_h5_load(C.byref(params), str(path).encode(), soa.ptr, soa.capacity, C.byref(got))
    if rc != 0:
        raise RuntimeError(f"icy_h5_load({path}) failed with status {rc}: {H.icy_host_last_error().decode()}")
    soa.size = got.value
    return soa

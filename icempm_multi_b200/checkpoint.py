"""Checkpoints of a model's state, in the file format written and read by
icy::SnapshotManager::SaveSnapshot / ReadSnapshot of the C++ host layer
(icempm_multi_b200/host/icy_host.cpp):

    8 bytes   "ICYCKPT1"
    6 x u32   format version (1), sizeof(icy_sim_params), HSSOA capacity,
              points stored, precision (0 FP64, 1 FP32 split), 0
    icy_sim_params (SimulationStep and SimulationTime included)
    16 lines of `points` doubles (the HSSOA lines, utility word bit-cast)

The reference's own snapshot code is disabled (cli/main.cpp:57); these files
are the resume path of long runs and of evicted served scenarios.
"""
import ctypes as C
import struct

import numpy as np

from ._lib import N_PTS_ARRAYS, SimParams
from .hssoa import HostSideSOA

MAGIC = b"ICYCKPT1"


def write_checkpoint(path, params, soa, precision=0):
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<6I", 1, C.sizeof(SimParams), soa.capacity, soa.size, int(precision), 0))
        f.write(bytes(params))
        for line in range(N_PTS_ARRAYS):
            f.write(np.ascontiguousarray(soa.buf[line, :soa.size]).tobytes())


def read_checkpoint(path):
    """-> (SimParams, HostSideSOA, precision)"""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError(f"{path} is not a checkpoint")
    ver, psize, cap, size, precision, _ = struct.unpack_from("<6I", data, 8)
    if ver != 1 or psize != C.sizeof(SimParams) or size > cap:
        raise ValueError(f"{path}: unsupported checkpoint header")
    off = 8 + 24
    params = SimParams.from_buffer_copy(data[off:off + psize])
    off += psize
    soa = HostSideSOA(max(cap, 1))
    soa.size = size
    need = off + 8 * size * N_PTS_ARRAYS
    if len(data) < need:
        raise ValueError(f"{path}: truncated checkpoint")
    lines = np.frombuffer(data, dtype=np.float64, count=size * N_PTS_ARRAYS, offset=off)
    soa.buf[:, :size] = lines.reshape(N_PTS_ARRAYS, size)
    return params, soa, precision

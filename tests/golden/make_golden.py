"""Writes the golden vectors in this directory.

Each case is a seeded scenario run for a few steps by the REFERENCE's own
kernel sources compiled for the host (oracle/_ref/libref_host.so, one thread,
built by oracle/Makefile from the reference tree).  The .npz holds the input
HSSOA, the parameters, the output HSSOA, the indenter force bins and the end
time, so the oracle can be checked against the reference where the reference
tree is absent.

    python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from icempm_multi_b200._lib import SimParams  # noqa: E402
from icempm_multi_b200.hssoa import HostSideSOA  # noqa: E402


def save_case(path, p, soa_in, steps, soa_out, bins, t_end):
    raw = np.frombuffer(bytes(p), dtype=np.uint8)
    np.savez_compressed(path, params=raw, soa_in=soa_in.buf[:, :soa_in.size], steps=steps,
                        soa_out=soa_out.buf[:, :soa_out.size], bins=bins, t_end=t_end)


def load_case(path):
    z = np.load(path)
    p = SimParams()
    C.memmove(C.byref(p), z["params"].tobytes(), C.sizeof(SimParams))
    a = z["soa_in"]
    soa = HostSideSOA(a.shape[1])
    soa.buf[:, :] = a
    soa.size = a.shape[1]
    return p, soa, int(z["steps"]), z["soa_out"], z["bins"], float(z["t_end"])


def main():
    from oracle.oracle import RefHost, build
    from scenarios import standard, stress
    build()
    ref = RefHost()
    cases = [("standard_s1", standard(seed=1), 60), ("stress_s7", stress(seed=7), 40),
             ("standard_s2_small", standard(n_cells_x=12, n_cells_y=6, seed=2, grid=(48, 32)), 100)]
    for name, (p, soa), steps in cases:
        out = soa.clone()
        err, t, bins = ref.run(p, out, 0, steps, threads=1)
        assert err == 0
        save_case(os.path.join(HERE, name + ".npz"), p, soa, steps, out, bins, t)
        print(name, soa.size, steps, "crushed", int(out.crushed().sum()))


if __name__ == "__main__":
    main()

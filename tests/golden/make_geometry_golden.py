"""Writes tests/golden/ref_2d_70k.npz: the reference's own 70,534-point
geometry (build/geometries_2d/2d_70k.h5 under build/p1.json) as placed by
SnapshotManager::LoadRawPoints (simulation/snapshotmanager.cpp:29-121; read
and placed here by the project's HDF5 reader, icy_h5_load, which the CPU
tests pin to an independent decoder), and the state after one frame of the
reference's p1.json (UpdateEveryNthStep = 500 sub-steps) computed by the
REFERENCE's own kernel sources compiled for the host
(oracle/_ref/libref_host.so, one thread).

Stored: the parameters (icy::SimParams bytes), the placed points (x, y,
utility word; Fe = I, Jp_inv = 1, the rest zero), and of the reference's
output the positions, Jp_inv and utility words, the indenter force bins and
the end time.  The GPU tests run the CUDA paths on it where the reference
tree is absent, and compare every other field with the reference host build
run live when oracle/_ref/libref_host.so is present.

    python tests/golden/make_geometry_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

STEPS = 500


def load_geometry(path=None):
    """(params, placed HSSOA, steps, reference output dict) of the fixture."""
    import ctypes as C
    from icempm_multi_b200._lib import SimParams
    from icempm_multi_b200.hssoa import HostSideSOA
    z = np.load(path or os.path.join(HERE, "ref_2d_70k.npz"))
    p = SimParams()
    C.memmove(C.byref(p), z["params"].tobytes(), C.sizeof(SimParams))
    n = z["pos_in"].shape[1]
    soa = HostSideSOA(int(z["capacity"]))
    soa.size = n
    soa.pos[:, :n] = z["pos_in"]
    soa.utility[:n] = z["util_in"]
    soa.Fe[0][:n] = 1.0
    soa.Fe[3][:n] = 1.0
    soa.Jp_inv[:n] = 1.0
    ref = {k: z[k] for k in ("pos_out", "jp_out", "util_out", "bins")}
    ref["t_end"] = float(z["t_end"])
    return p, soa, int(z["steps"]), ref


def main():
    from icempm_multi_b200 import load_h5, parse_file
    from oracle.oracle import RefHost, build
    from refpaths import GEOM, REF
    build()
    p, _ = parse_file(os.path.join(REF, "build", "p1.json"))
    soa = load_h5(p, os.path.join(GEOM, "2d_70k.h5"))
    assert p.UpdateEveryNthStep == STEPS
    n = soa.size
    out = soa.clone()
    err, t, bins = RefHost().run(p, out, 0, STEPS, threads=1)
    assert err == 0
    raw = np.frombuffer(bytes(p), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "ref_2d_70k.npz"), params=raw, capacity=soa.capacity,
                        pos_in=soa.pos[:, :n], util_in=soa.utility[:n], steps=STEPS,
                        pos_out=out.pos[:, :n], jp_out=out.Jp_inv[:n], util_out=out.utility[:n],
                        bins=bins, t_end=t)
    print("2d_70k", n, "points,", STEPS, "steps, crushed", int(out.crushed().sum()),
          "largest displacement / h", float(np.abs(out.pos[:, :n] - soa.pos[:, :n]).max() / p.cellsize))


if __name__ == "__main__":
    main()

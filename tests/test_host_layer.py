"""CPU tests of the C++ host layer (libicempm_host.so, icy_cli): exported
symbols, the frame-log number format, the HDF5 point-cloud reader and the
LoadRawPoints placement, and -- where the reference tree is present -- the
oracle against the reference's own kernels on the reference's 70k-point
geometry.  No compute call is made on a device here."""
import ctypes as C
import os
import re
import subprocess
import zlib

import numpy as np
import pytest

from icempm_multi_b200 import format_double, load_h5, parse_file
from icempm_multi_b200._lib import (CLI_PATH, HOST_EXPORTED, HOST_LIB_PATH, STATUS_DISABLED, host_lib, lib)
from icempm_multi_b200.hssoa import HostSideSOA
from scenarios import comparable_bits

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "icempm_host.h")
from refpaths import GEOM, REF
have_geom = pytest.mark.skipif(not os.path.exists(os.path.join(GEOM, "2d_70k.h5")),
                               reason="reference point clouds absent")


def test_host_library_exports_every_declared_symbol(built):
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    syms = sorted(set(re.findall(r"\b(icy_[a-z0-9_]+)\s*\(", txt)))
    assert set(syms) == set(HOST_EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", HOST_LIB_PATH], capture_output=True, text=True).stdout
    defined = set(l.split()[-1] for l in out.splitlines() if l.strip())
    assert not [s for s in syms if s not in defined]
    H = host_lib()
    for s in syms:
        assert getattr(H, s) is not None


@pytest.mark.parametrize("v,text", [
    (0.0, "0"), (1.0, "1"), (-3.0, "-3"), (100.0, "100"), (0.1, "0.1"), (0.0001, "0.0001"),
    (1e-05, "1e-05"), (2.5e-05, "2.5e-05"), (0.00012, "0.00012"), (123.456, "123.456"),
    (1e16, "1e+16"), (1234567890123456.0, "1234567890123456"), (1.2345678901234568e+17, "1.2345678901234568e+17"),
    (0.30000000000000004, "0.30000000000000004"), (6.02e23, "6.02e+23"), (-7.5e-300, "-7.5e-300"),
])
def test_force_log_number_format(built, v, text):
    # the fmt library's "{}" for a double: shortest round trip, fixed for 1e-4 <= |v| < 1e16
    assert format_double(v) == text
    assert float(format_double(v)) == v


def test_cli_usage(built):
    r = subprocess.run([CLI_PATH, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage: icy_cli" in r.stderr
    r = subprocess.run([CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([CLI_PATH, "/nonexistent.json"], capture_output=True, text=True, cwd="/tmp")
    assert r.returncode == 1 and "configuration file is not found" in r.stderr


# ---------------------------------------------------------------- HDF5 point clouds

def _py_read_h5(path):
    """Independent decoder of the subset of HDF5 the reference's clouds use
    (superblock 0, v1 object headers, v1 B-trees, chunked + deflate), written
    from the file-format specification: {name: (values, attrs)}."""
    f = open(path, "rb").read()
    u = lambda o, n: int.from_bytes(f[o:o + n], "little")
    assert f[:8] == b"\x89HDF\r\n\x1a\n" and f[8] == 0
    root = 24 + 32
    btree, heap = u(root + 24, 8), u(root + 32, 8)
    heap_data = u(heap + 24, 8)

    def msgs(a):
        n, size = u(a + 2, 2), u(a + 8, 4)
        out, blocks = [], [(a + 16, size)]
        while blocks and len(out) < n:
            q, sz = blocks.pop(0)
            end = q + sz
            while q + 8 <= end and len(out) < n:
                t, s = u(q, 2), u(q + 2, 2)
                out.append((t, q + 8, s))
                if t == 0x10:
                    blocks.append((u(q + 8, 8), u(q + 16, 8)))
                q += 8 + s
        return out

    objs = {}
    node = btree
    used = u(node + 6, 2)
    q = node + 24 + 8
    for _ in range(used):
        sn = u(q, 8)
        q += 16
        for k in range(u(sn + 6, 2)):
            e = sn + 8 + 40 * k
            no = heap_data + u(e, 8)
            name = f[no:f.index(b"\0", no)].decode()
            objs[name] = u(e + 8, 8)
    out = {}
    for name, oh in objs.items():
        dims = None; dt = None; chunk = None; attrs = {}
        for t, d, s in msgs(oh):
            if t == 1:
                dims = [u(d + 8 + 8 * i, 8) for i in range(f[d + 1])]
            elif t == 3:
                dt = (f[d] & 15, u(d + 4, 4), bool(f[d + 1] & 8))
            elif t == 8:
                assert f[d] == 3 and f[d + 1] == 2
                chunk = (u(d + 3, 8), [u(d + 11 + 4 * i, 4) for i in range(f[d + 2])])
            elif t == 0xC:
                nn, nt, ns = u(d + 2, 2), u(d + 4, 2), u(d + 6, 2)
                an = f[d + 8:d + 8 + nn].split(b"\0")[0].decode()
                r8 = lambda x: (x + 7) // 8 * 8
                tpos = d + 8 + r8(nn)
                dpos = tpos + r8(nt) + r8(ns)
                cls, size = f[tpos] & 15, u(tpos + 4, 4)
                attrs[an] = np.frombuffer(f[dpos:dpos + size], dtype={(1, 4): "<f4", (1, 8): "<f8"}[(cls, size)])[0]
        es = dt[1]
        raw = bytearray(dims[0] * es)
        stack = [chunk[0]]
        while stack:
            nd = stack.pop()
            lvl, used = f[nd + 5], u(nd + 6, 2)
            q = nd + 24
            for _ in range(used):
                csize, off = u(q, 4), u(q + 8, 8)
                child = u(q + 24, 8)
                q += 32
                if lvl:
                    stack.append(child)
                    continue
                data = zlib.decompress(f[child:child + csize])
                m = min(chunk[1][0], dims[0] - off)
                raw[off * es:(off + m) * es] = data[:m * es]
        kind = "<f8" if dt[0] == 1 else ("<i8" if dt[2] else "<u8")
        out[name] = (np.frombuffer(bytes(raw), dtype=kind), attrs)
    return out


def _place_like_reference(p, x, y, grains):
    """LoadRawPoints' placement in numpy (simulation/snapshotmanager.cpp:62-109)."""
    h = p.cellsize
    x = x + ((p.GridXTotal * h) - (x.max() - x.min())) / 2
    y = y + 2 * h
    key = (x * p.cellsize_inv + 0.5).astype(np.int32).astype(np.int64) * p.GridY + \
        (y * p.cellsize_inv + 0.5).astype(np.int32)
    order = np.argsort(key, kind="stable")
    return x[order], y[order], grains[order]


@have_geom
@pytest.mark.parametrize("name", ["2d_70k", "2d_250k"])
def test_h5_reader_and_placement(built, name):
    path = os.path.join(GEOM, name + ".h5")
    ref = _py_read_h5(path)
    x0, y0 = ref["x"][0], ref["y"][0]
    g0, attrs = ref["llGrainIDs"]
    p, _ = parse_file(os.path.join(REF, "build", "p1.json"))
    soa = load_h5(p, path)
    n = len(x0)
    assert soa.size == n == p.nPtsTotal
    assert soa.capacity == int(n * (1 + p.ExtraSpaceForIncomingPoints))
    vol = float(np.float32(attrs["volume"]))
    assert p.Volume == vol and p.ParticleVolume == vol / n
    x, y, g = _place_like_reference(p, x0, y0, g0.view(np.int64))
    assert np.array_equal(soa.pos[0], x) and np.array_equal(soa.pos[1], y)
    assert np.array_equal(soa.utility, g)
    assert np.all(soa.Fe[0] == 1) and np.all(soa.Fe[3] == 1) and np.all(soa.Fe[1:3] == 0)
    assert np.all(soa.Jp_inv == 1) and np.all(soa.vel == 0) and np.all(soa.Bp == 0)
    # indenter start (snapshotmanager.cpp:84-105)
    r = p.IndDiameter / 2
    ht = r - p.IndDepth
    assert p.indenter_x == np.floor((x.min() - np.sqrt(r * r - ht * ht)) / p.cellsize) * p.cellsize
    assert p.indenter_y == (y0.max() + 2 * p.cellsize) + ht


def test_h5_reader_errors(built, tmp_path):
    from icempm_multi_b200 import default_params
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file at all" * 10)
    with pytest.raises(RuntimeError, match="not an HDF5 file"):
        load_h5(default_params(), bad)
    with pytest.raises(RuntimeError, match="cannot open"):
        load_h5(default_params(), tmp_path / "missing.h5")
    if os.path.exists(os.path.join(GEOM, "2d_70k.h5")):
        # a truncated copy of a real cloud is refused, not misread
        cut = tmp_path / "cut.h5"
        cut.write_bytes(open(os.path.join(GEOM, "2d_70k.h5"), "rb").read()[:200000])
        with pytest.raises(RuntimeError, match="truncated|inflate"):
            load_h5(default_params(), cut)


def test_scene_place_drops_disabled_points(built):
    from scenarios import params_for
    p = params_for(64, 32, 0.25, 1e-4)
    n = 40
    soa = HostSideSOA(n)
    soa.size = n
    rng = np.random.default_rng(3)
    soa.pos[0][:n] = rng.uniform(0, 5, n)
    soa.pos[1][:n] = rng.uniform(0, 2, n)
    u = soa.utility
    u[:n] = rng.integers(0, 50, n)
    u[[3, 17, 29]] |= STATUS_DISABLED
    x0, y0, g0 = soa.pos[0][:n].copy(), soa.pos[1][:n].copy(), u[:n].copy()
    cnt = C.c_uint(n)
    assert lib().icy_scene_place(C.byref(p), soa.ptr, soa.capacity, C.byref(cnt), 10.0) == 0
    assert cnt.value == n - 3 and p.nPtsTotal == n and p.ParticleVolume == 10.0 / n
    keep = (g0 & STATUS_DISABLED) == 0
    x = x0 + ((p.GridXTotal * p.cellsize) - (x0.max() - x0.min())) / 2
    y = y0 + 2 * p.cellsize
    key = (x * p.cellsize_inv + 0.5).astype(np.int32).astype(np.int64) * p.GridY + \
        (y * p.cellsize_inv + 0.5).astype(np.int32)
    idx = np.nonzero(keep)[0]
    idx = idx[np.argsort(key[idx], kind="stable")]
    m = soa.size = cnt.value
    assert np.array_equal(soa.pos[0][:m], x[idx]) and np.array_equal(soa.utility[:m], g0[idx])


@have_geom
def test_oracle_matches_reference_kernels_on_reference_geometry(built):
    """The oracle against the reference's own kernels (host build, one thread)
    on the 70k-point geometry and parameters of the reference's p1.json."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_host.so")):
        pytest.skip("reference host build absent")
    from oracle.oracle import Oracle, RefHost
    p, _ = parse_file(os.path.join(REF, "build", "p1.json"))
    soa = load_h5(p, os.path.join(GEOM, "2d_70k.h5"))
    a, b = soa.clone(), soa.clone()
    ea, ta, ba = Oracle().run(p, a, 0, 12)
    eb, tb, bb = RefHost().run(p, b, 0, 12, threads=1)
    assert ea == eb == 0 and ta == tb
    assert np.array_equal(comparable_bits(a), comparable_bits(b))
    assert np.array_equal(ba, bb)

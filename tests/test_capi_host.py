"""CPU tests of the C-ABI library: symbols, SimParams / JSON, scene set-up.

No compute call is made here (no GPU); the device path is covered by the
tests marked ``gpu``.
"""
import ctypes as C
import json
import math
import os
import re
import subprocess

import numpy as np
import pytest

from icempm_multi_b200 import default_params, make_block, parse_file, parse_json
from icempm_multi_b200._lib import (EXPORTED, ICY_ERR_CONFIG_MISSING, ICY_ERR_FILE, ICY_ERR_JSON, LIB_PATH,
                                    IcyError, SimParams, lib)
from refpaths import INPUTS as REF_INPUTS
from scenarios import params_for

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "icempm.h")
REF_PARAMS = os.path.join(ROOT, "oracle", "_ref", "libref_params.so")


def header_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(icy_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(built):
    syms = header_symbols()
    assert len(syms) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    defined = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [s for s in syms if s not in defined]
    assert not missing, missing
    L = lib()
    for s in syms:
        assert getattr(L, s) is not None
    assert set(EXPORTED) <= set(syms)


def test_struct_layout_matches_header(built):
    # icy_sim_params field order/size (the reference layout is checked by
    # static_assert when oracle/_ref is built)
    assert C.sizeof(SimParams) == 520 or C.sizeof(SimParams) % 8 == 0
    p = default_params()
    assert p.n_indenter_subdivisions == 100 and p.tpb_P2G == 256 and p.GridHaloSize == 5


def _ref_params():
    from oracle.oracle import RefParams
    return RefParams()


@pytest.mark.skipif(not os.path.exists(REF_PARAMS), reason="reference params build absent")
def test_reset_matches_reference(built):
    ours = default_params().as_dict()
    ref = _ref_params().reset().as_dict()
    for k, v in ref.items():
        assert ours[k] == v or (isinstance(v, float) and math.isnan(v) and math.isnan(ours[k])), k


CONFIGS = [
    {"InputRawPoints": "a.h5", "GridX": 512, "GridY": 256, "GridXDimension": 128.0, "InitialTimeStep": 1e-4,
     "YoungsModulus": 1e9, "DP_phi": 62, "DP_threshold_p": 0, "IndDiameter": 2, "IndVelocity": 1.0,
     "IndDepth": 0.5, "Density": 980, "nPartitions": 1, "GridHaloSize": 8},
    {"InputRawPoints": "b.h5", "GridX": 4096, "GridY": 2048, "GridXDimension": 204.8, "InitialTimeStep": 2e-5,
     "IceCompressiveStrength": 1e8, "IceTensileStrength": 1e7, "IceTensileStrength2": 5e6,
     "IceShearStrength": 7e6, "GrainVariability": 0.6, "tpb_P2G": 128, "SetupType": 1, "PoissonsRatio": 0.25,
     "ExtraSpaceForIncomingPoints": 0.1, "Gravity": 9.8, "SimulationEndTime": 3.5, "ParticleViewSize": 1.5},
    {"InputRawPoints": "cé.h5", "GridX": 1024, "GridY": 440, "GridXDimension": 3.3, "InitialTimeStep": 2.0e-6,
     "DP_phi": 45, "unknown_key": [1, 2, {"x": None}], "nested": {"a": True}},
]


@pytest.mark.skipif(not os.path.exists(REF_PARAMS), reason="reference params build absent")
@pytest.mark.parametrize("cfg", CONFIGS)
def test_parse_matches_reference(built, tmp_path, cfg):
    f = tmp_path / "cfg.json"
    f.write_text(json.dumps(cfg, indent=1))
    ours, raw = parse_file(str(f))
    ref = _ref_params().reset()
    rc, raw_ref, _ = _ref_params().parse_file(ref, str(f))
    assert rc == 0 and raw == raw_ref
    a, b = ours.as_dict(), ref.as_dict()
    for k in a:
        assert a[k] == b[k], (k, a[k], b[k])


@pytest.mark.skipif(not os.path.isdir(REF_INPUTS) or not os.path.exists(REF_PARAMS),
                    reason="reference input files not present")
def test_reference_input_files_parse_identically(built):
    for name in sorted(os.listdir(REF_INPUTS)):
        path = os.path.join(REF_INPUTS, name)
        ours, raw = parse_file(path)
        ref = _ref_params().reset()
        rc, raw_ref, _ = _ref_params().parse_file(ref, path)
        assert rc == 0 and raw == raw_ref, name
        assert bytes(ours) == bytes(ref), name


GOLDEN_PARAMS = os.path.join(ROOT, "tests", "golden", "params_ref.json")


def test_reset_and_parse_match_reference_golden(built, tmp_path):
    """SimParams::Reset and ParseFile against the reference's own parser as
    recorded in tests/golden/params_ref.json (written by
    tests/golden/make_params_golden.py from oracle/_ref/libref_params.so):
    the reference's parameter files and the configurations above, byte for
    byte, where neither the reference tree nor rapidjson is present."""
    g = json.load(open(GOLDEN_PARAMS))
    assert bytes(default_params()) == bytes.fromhex(g["reset"])
    assert len(g["cases"]) >= len(CONFIGS) + 5
    for case in g["cases"]:
        f = tmp_path / "cfg.json"
        f.write_text(case["text"])
        assert case["rc"] == 0, case["name"]
        ours, raw = parse_file(str(f))
        assert raw == case["raw"], case["name"]
        assert bytes(ours) == bytes.fromhex(case["params"]), case["name"]


def test_parse_errors(built, tmp_path):
    with pytest.raises(IcyError) as e:
        parse_json("[1, 2]")
    assert e.value.code == ICY_ERR_JSON
    with pytest.raises(IcyError) as e:
        parse_json('{"GridX": 64,}')          # strict JSON, as rapidjson's default
    assert e.value.code == ICY_ERR_JSON
    with pytest.raises(IcyError) as e:
        parse_json('{"GridX": 64}')
    assert e.value.code == ICY_ERR_CONFIG_MISSING
    with pytest.raises(IcyError) as e:
        parse_file(str(tmp_path / "nope.json"))
    assert e.value.code == ICY_ERR_FILE


def test_parse_missing_key_still_updates_params(built):
    p = default_params()
    rc = lib().icy_params_parse_json(C.byref(p), b'{"GridX": 77, "DP_phi": 30}', None, 0)
    assert rc == ICY_ERR_CONFIG_MISSING and p.GridXTotal == 77
    assert p.DP_tan_phi == math.tan(30 * math.pi / 180)


def test_scene_placement_rules(built):
    h = 0.25
    p = params_for(128, 64, h, 1e-4)
    soa = make_block(p, 16.0, 4.0, ppc=4, seed=9, n_grains=8)
    n = soa.size
    assert n == 64 * 16 * 4 == p.nPtsTotal
    x, y = soa.pos
    # centred in x (snapshotmanager.cpp:71-78): x_offset = (GridX*h - (xmax-xmin))/2 added to raw x
    box = 128 * h
    raw_len = p.xmax - p.xmin
    assert abs((x.min() - p.xmin) - (box - raw_len) / 2) < 1e-12
    assert abs(y.min() - (p.ymin + 2 * h)) < 1e-12
    # sorted by ProxyPoint::getCellIndex
    key = (x / h + 0.5).astype(np.int64) * p.GridY + (y / h + 0.5).astype(np.int64)
    assert np.all(np.diff(key) >= 0)
    # InitializeBlock
    assert np.all(soa.Fe[0] == 1) and np.all(soa.Fe[3] == 1) and np.all(soa.Fe[1:3] == 0)
    assert np.all(soa.Jp_inv == 1) and np.all(soa.vel == 0) and np.all(soa.Bp == 0)
    # indenter start (snapshotmanager.cpp:84-105)
    r = p.IndDiameter / 2
    ht = r - p.IndDepth
    left = (box - raw_len) / 2
    assert p.indenter_x == math.floor((left - math.sqrt(r * r - ht * ht)) / h) * h
    assert p.indenter_y == (p.ymax + 2 * h) + ht
    assert p.ParticleVolume == p.Volume / n and p.ParticleMass == p.ParticleVolume * p.Density
    assert len(np.unique(soa.grains())) > 1
    # 4 points per cell, one per sub-cell quadrant
    cell = (np.floor((x - x.min()) / h).astype(int), np.floor((y - y.min()) / h).astype(int))
    assert np.bincount(cell[0] * 1000 + cell[1]).max() <= 8


def test_scene_is_deterministic(built):
    p1 = params_for(96, 48, 0.25, 1e-4)
    p2 = params_for(96, 48, 0.25, 1e-4)
    a = make_block(p1, 8.0, 2.0, seed=4, n_grains=5)
    b = make_block(p2, 8.0, 2.0, seed=4, n_grains=5)
    c = make_block(params_for(96, 48, 0.25, 1e-4), 8.0, 2.0, seed=5, n_grains=5)
    assert np.array_equal(a.buf, b.buf) and bytes(p1) == bytes(p2)
    assert not np.array_equal(a.pos, c.pos)

"""GPU tests of the C++ host layer through its headless driver icy_cli
(icy::Model / GPU_Implementation5 / SnapshotManager over the C-ABI):
frames, the indenter-force log and the final state against the oracle,
the per-phase loop against the fused one, FP32 split precision, and
checkpoint / resume against a straight run."""
import json
import os
import subprocess

import numpy as np
import pytest

from icempm_multi_b200._lib import CLI_PATH
from icempm_multi_b200.checkpoint import read_checkpoint
from icempm_multi_b200.hssoa import make_block
from scenarios import params_for
from test_gpu_parity import TOL, assert_close, field_errors
from test_gpu_split import POS_TOL

pytestmark = pytest.mark.gpu

H, DT, GRID = 0.25, 1e-4, (96, 48)
BLOCK = (32 * H, 8 * H)
KW = dict(IndVelocity=2.0, IndDepth=0.6)
FORCE_TOL = 1e-9          # relative, frame-averaged indenter force (FP64 atomic order)


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


def config(tmp_path):
    cfg = {"InputRawPoints": "synthetic", "nPartitions": 1, "GridHaloSize": 8, "InitialTimeStep": DT,
           "GridX": GRID[0], "GridY": GRID[1], "GridXDimension": GRID[0] * H, "YoungsModulus": 1e9,
           "PoissonsRatio": 0.3, "Density": 980, "Gravity": 9.81, "DP_phi": 62, "DP_threshold_p": 0,
           "GrainVariability": 0.5, "IndDiameter": 2.0, "IndDepth": KW["IndDepth"],
           "IndVelocity": KW["IndVelocity"], "SetupType": 0, "SimulationEndTime": 10.0}
    path = tmp_path / "cfg.json"
    path.write_text(json.dumps(cfg))
    return str(path)


def cli(tmp_path, *args, check=True):
    cmd = [CLI_PATH, *args]
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=tmp_path, timeout=300)
    if check:
        assert r.returncode == 0, (r.stdout, r.stderr)
    return r


def scene():
    p = params_for(GRID[0], GRID[1], H, DT, **KW)
    soa = make_block(p, BLOCK[0], BLOCK[1], ppc=4, seed=5, n_grains=16)
    return p, soa


def block_args():
    return ["--block", str(BLOCK[0]), str(BLOCK[1]), "--ppc", "4", "--seed", "5", "--grains", "16"]


def test_cli_frames_force_log_and_state_match_oracle(oracle, tmp_path):
    cfg = config(tmp_path)
    cli(tmp_path, cfg, *block_args(), "--frames", "3", "--log", "force.csv", "--checkpoint", "end.ckpt")
    p, soa = scene()
    nf = p.UpdateEveryNthStep
    prm, out, prec = read_checkpoint(tmp_path / "end.ckpt")
    assert prec == 0 and prm.SimulationStep == 3 * nf and out.size == soa.size
    ref = soa.clone()
    t = 0.0
    lines = (tmp_path / "force.csv").read_text().splitlines()
    assert len(lines) == 3
    for k in range(3):
        err, t, bins = oracle.run(p, ref, k * nf, nf, t)
        assert err == 0
        f = np.array([bins[0::2].sum(), bins[1::2].sum()]) / nf
        tt, fn, fx, fy = (float(v) for v in lines[k].split(","))
        assert tt == t
        assert abs(fn - np.hypot(*f)) <= FORCE_TOL * max(np.hypot(*f), 1e-30)
        assert abs(fx - f[0]) <= FORCE_TOL * max(abs(f[0]), np.hypot(*f), 1e-30)
        assert abs(fy - f[1]) <= FORCE_TOL * max(abs(f[1]), np.hypot(*f), 1e-30)
    assert prm.SimulationTime == t
    assert any(float(l.split(",")[1]) > 0 for l in lines)      # the indenter touched the ice
    assert_close(field_errors(out, ref))
    # logs/timings.csv: one line per frame in the reference's column layout (model.cpp:91-95)
    tl = (tmp_path / "logs" / "timings.csv").read_text().splitlines()
    assert len(tl) == 3
    for k, l in enumerate(tl):
        f = [x.strip() for x in l.split(",")]
        assert len(f) == 14 and int(f[0]) == k + 1 and int(f[2]) == soa.size
        assert float(f[7]) > 0 and float(f[13]) >= float(f[7])


def test_cli_per_phase_loop_matches_fused(tmp_path):
    cfg = config(tmp_path)
    cli(tmp_path, cfg, *block_args(), "--frames", "2", "--log", "a.csv", "--checkpoint", "a.ckpt")
    cli(tmp_path, cfg, *block_args(), "--frames", "2", "--log", "b.csv", "--checkpoint", "b.ckpt", "--per-phase")
    _, a, _ = read_checkpoint(tmp_path / "a.ckpt")
    _, b, _ = read_checkpoint(tmp_path / "b.ckpt")
    e = field_errors(a, b)
    assert e["pos"] <= TOL["pos"] and e["vel"] <= TOL["vel"], e


def test_cli_fp32_split_matches_oracle(oracle, tmp_path):
    cfg = config(tmp_path)
    cli(tmp_path, cfg, *block_args(), "--frames", "2", "--precision", "fp32", "--checkpoint", "f.ckpt",
        "--log", "f.csv")
    p, soa = scene()
    _, out, prec = read_checkpoint(tmp_path / "f.ckpt")
    assert prec == 1
    ref = soa.clone()
    assert oracle.run(p, ref, 0, 2 * p.UpdateEveryNthStep)[0] == 0
    assert field_errors(out, ref)["pos"] <= POS_TOL


def test_cli_resume_matches_straight_run(tmp_path):
    cfg = config(tmp_path)
    cli(tmp_path, cfg, *block_args(), "--frames", "3", "--log", "s.csv", "--checkpoint", "straight.ckpt")
    cli(tmp_path, cfg, *block_args(), "--frames", "2", "--log", "r1.csv", "--checkpoint", "mid.ckpt")
    cli(tmp_path, "--resume", "mid.ckpt", "--frames", "1", "--log", "r2.csv", "--checkpoint", "resumed.ckpt")
    ps, s, _ = read_checkpoint(tmp_path / "straight.ckpt")
    pr, r, _ = read_checkpoint(tmp_path / "resumed.ckpt")
    assert pr.SimulationStep == ps.SimulationStep and pr.SimulationTime == ps.SimulationTime
    e = field_errors(r, s)
    assert e["pos"] <= TOL["pos"] and e["vel"] <= TOL["vel"] and e["status"] == 0.0, e
    # the resumed frame logs the same time as the straight run's third frame
    assert (tmp_path / "r2.csv").read_text().split(",")[0] == \
        (tmp_path / "s.csv").read_text().splitlines()[2].split(",")[0]


def test_cli_reports_library_errors(tmp_path):
    cfg = config(tmp_path)
    r = cli(tmp_path, cfg, *block_args(), "--option", "no_such_option=1", "--frames", "1", check=False)
    assert r.returncode == 1 and "set_option" in r.stderr

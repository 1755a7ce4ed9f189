"""Pins the CPU oracle (oracle/oracle.c) to the reference itself.

The reference's own kernel sources (simulation/kernels.cuh, helper_math.cuh,
givens.cuh), compiled unmodified for the host (oracle/_ref/libref_host.so),
run on one thread in the same particle order as the oracle: the two must agree
bit for bit.  Where the reference tree is not available the committed golden
vectors (tests/golden/*.npz, written by tests/golden/make_golden.py from the
same reference build) pin the oracle instead.
"""
import glob
import os

import numpy as np
import pytest

from icempm_multi_b200._lib import STATUS_CRUSHED
from scenarios import comparable_bits, standard, stress

HERE = os.path.dirname(os.path.abspath(__file__))
REF_HOST = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_host.so")
have_ref = pytest.mark.skipif(not os.path.exists(REF_HOST), reason="reference host build absent")


@pytest.fixture(scope="module")
def oracle(built):
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="module")
def ref(built):
    from oracle.oracle import RefHost
    return RefHost()


def _bits(soa):
    return comparable_bits(soa)


@have_ref
@pytest.mark.parametrize("make,steps", [(standard, 120), (stress, 60)])
def test_oracle_bitexact_vs_reference_kernels(oracle, ref, make, steps):
    p, soa = make()
    a, b = soa.clone(), soa.clone()
    ea, ta, ba = oracle.run(p, a, 0, steps)
    eb, tb, bb = ref.run(p, b, 0, steps, threads=1)
    assert ea == eb == 0
    assert ta == tb
    assert np.array_equal(_bits(a), _bits(b))
    assert np.array_equal(ba, bb)


@have_ref
def test_stress_scenario_exercises_every_branch(oracle):
    p, soa = stress()
    pre = soa.crushed().sum()
    oracle.run(p, soa, 0, 60)
    assert soa.crushed().sum() > pre + 20        # new points crushed -> SVD + return map ran
    assert soa.liquid().sum() > 0 and soa.disabled().sum() > 0
    assert np.any(soa.Jp_inv[~soa.liquid()] != 1.0)  # Jp changed by the DP projection


@have_ref
def test_device_math_units_bitexact(oracle, ref):
    """SVD, Kirchhoff stress and the full plasticity step on random matrices."""
    p, _ = stress()
    rng = np.random.default_rng(5)
    for k in range(400):
        F = np.eye(2).ravel() + rng.normal(0, 0.05 if k % 2 else 1e-4, 4)
        if k % 50 == 0:
            F = np.array([1.0 + 1e-3, 0.0, 0.0, 1.0 + 1e-3])   # equal singular values
        Uo, So, Vo = oracle.svd(F)
        Ur, Sr, Vr = ref.svd(F)
        assert np.array_equal(Uo, Ur) and np.array_equal(So, Sr) and np.array_equal(Vo, Vr)
        assert np.array_equal(oracle.kirchhoff(p, F), ref.kirchhoff(p, F))
        util = (k % 30) | (STATUS_CRUSHED if k % 3 == 0 else 0)
        Fr, Jr, ur, pr, qr = ref.plasticity(p, F, 0.98 + 0.04 * rng.random(), util)
        po, qo, Je = oracle.pq(p, F)
        assert (po, qo) == (pr, qr)
        crushed = bool(util & STATUS_CRUSHED) or bool(oracle.failure(p, util & 0xFFFF, po, qo))
        assert crushed == bool(ur & STATUS_CRUSHED)


def test_svd_reconstructs(oracle):
    """U diag(sigma) V^T as the reference forms it reproduces F (to rounding)."""
    rng = np.random.default_rng(11)
    for _ in range(200):
        F = np.eye(2).ravel() + rng.normal(0, 0.3, 4)
        U, S, V = oracle.svd(F)
        U, V = U.reshape(2, 2), V.reshape(2, 2)
        R = U @ np.diag(S) @ V.T
        assert np.allclose(R.ravel(), F, atol=1e-12)
        assert S[0] >= S[1]


def test_golden_vectors(oracle):
    files = sorted(f for f in glob.glob(os.path.join(HERE, "golden", "*.npz"))
                   if not os.path.basename(f).startswith("ref_2d_"))
    assert files, "golden fixtures missing"
    from golden.make_golden import load_case
    for f in files:
        p, soa_in, steps, out, bins, t_end = load_case(f)
        err, t, b = oracle.run(p, soa_in, 0, steps)
        assert err == 0
        assert t == t_end
        ref_out = soa_in.clone()
        ref_out.buf[:, :] = out
        assert np.array_equal(comparable_bits(soa_in), comparable_bits(ref_out)), f
        assert np.array_equal(b, bins), f


def test_oracle_matches_reference_frame_on_70k_geometry(oracle):
    """The oracle against the reference host build's frame (500 sub-steps) on
    the reference's 70,534-point geometry (tests/golden/ref_2d_70k.npz):
    positions, Jp_inv and status words bit for bit, force bins, end time."""
    from golden.make_geometry_golden import load_geometry
    p, soa, steps, ref = load_geometry()
    err, t, bins = oracle.run(p, soa, 0, steps)
    n = soa.size
    assert err == 0 and t == ref["t_end"]
    assert np.array_equal(soa.pos[:, :n], ref["pos_out"])
    assert np.array_equal(soa.Jp_inv[:n], ref["jp_out"])
    assert np.array_equal(soa.utility[:n], ref["util_out"])
    assert np.array_equal(bins, ref["bins"])

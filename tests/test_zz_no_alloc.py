"""icy_step_noalloc: stepping for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: a plug-in inside a host framework that
owns all device memory through its own pool, or code on a latency-critical
path that must not allocate after start-up.  They keep the particle buffer in
their own device memory and call icy_step_noalloc, whose grid and status
scratch live in a fixed-size device array inside the library.  This test
checks, through the C-ABI, that two calls in a row (the second continuing
from the first, reusing the same scratch array) give the same particle state
as the regular instance entry points (icy_mpm_step + icy_mpm_transfer_from_device),
within the FP64 tolerances of the parity tests, and that a grid too large for
the scratch array is refused with a clear error.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from icempm_multi_b200 import GPUImplementation
from icempm_multi_b200._lib import ICY_ERR_CAPACITY, lib
from scenarios import params_for, stress
from test_gpu_parity import assert_close, field_errors

pytestmark = pytest.mark.gpu


def _to_device(soa, torch):
    pitch = (soa.size + 31) // 32 * 32
    d = torch.zeros((16, pitch), dtype=torch.float64, device="cuda")
    d[:, :soa.size] = torch.from_numpy(soa.buf[:, :soa.size].copy()).cuda()
    torch.cuda.synchronize()
    return d, pitch


def _from_device(d, soa, torch):
    out = soa.clone()
    torch.cuda.synchronize()
    out.buf[:, :out.size] = d[:, :out.size].cpu().numpy()
    return out


def test_noalloc_two_calls_match_instance_entry_points(built):
    import torch
    p, soa = stress(seed=12)
    s1, s2 = 30, 25

    # existing entry points: one instance, two icy_mpm_step calls, a download after each
    a = soa.clone()
    g = GPUImplementation(p, a)
    g.update_constants()
    g.transfer_ponts_to_device()
    g.reset_indenter_force_accumulator()
    t = g.run_steps(0, s1, 0.0)
    g.transfer_from_device()
    a1 = a.clone()
    bins1 = g.indenter_bins.copy()
    t = g.run_steps(s1, s2, t)
    g.transfer_from_device()
    a2 = a.clone()
    bins2 = g.indenter_bins.copy()
    g.close()

    # the allocation-free entry point on a caller-owned device buffer
    d, pitch = _to_device(soa, torch)
    dbins = torch.zeros(2 * p.n_indenter_subdivisions, dtype=torch.float64, device="cuda")
    tt = C.c_double(0.0)
    rc = lib().icy_step_noalloc(C.byref(p), C.c_void_p(d.data_ptr()), pitch, soa.size, 0, s1, C.byref(tt),
                                C.c_void_p(dbins.data_ptr()), None)
    assert rc == 0, lib().icy_last_error()
    b1 = _from_device(d, soa, torch)
    nb1 = dbins.cpu().numpy().copy()
    rc = lib().icy_step_noalloc(C.byref(p), C.c_void_p(d.data_ptr()), pitch, soa.size, s1, s2, C.byref(tt),
                                C.c_void_p(dbins.data_ptr()), None)
    assert rc == 0, lib().icy_last_error()
    b2 = _from_device(d, soa, torch)
    nb2 = dbins.cpu().numpy().copy()

    assert tt.value == t
    assert_close(field_errors(b1, a1))
    assert_close(field_errors(b2, a2))
    for mine, ref in ((nb1, bins1), (nb2, bins2)):
        fr, fo = ref.reshape(-1, 2).sum(0), mine.reshape(-1, 2).sum(0)
        assert np.allclose(fo, fr, rtol=1e-6, atol=1e-6 * (np.abs(fr).max() + 1))


def test_noalloc_refuses_grid_beyond_scratch(built):
    import torch
    p = params_for(2048, 1024, 0.1, 1e-4)       # 1024 x 2064 nodes: > ICY_NOALLOC_SCRATCH_BYTES
    d = torch.zeros((16, 32), dtype=torch.float64, device="cuda")
    tt = C.c_double(0.0)
    rc = lib().icy_step_noalloc(C.byref(p), C.c_void_p(d.data_ptr()), 32, 0, 0, 1, C.byref(tt), None, None)
    assert rc == ICY_ERR_CAPACITY
    assert b"scratch" in lib().icy_last_error()
    assert tt.value == 0.0

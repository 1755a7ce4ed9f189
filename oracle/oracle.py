"""ctypes wrapper of the parity oracles.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``   -- liboracle.so, the project's serial FP64 C restatement of the
                  reference hot path (oracle/oracle.c).
* ``RefHost``  -- _ref/libref_host.so, the reference's own kernels
                  (simulation/kernels.cuh) compiled for the host with OpenMP.
* ``RefCuda``  -- _ref/libref_cuda.so, the same kernels built for sm_100a.
* ``RefParams``-- _ref/libref_params.so, the reference's SimParams::ParseFile.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
these, as checkers / the reference arm; the product never imports them.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

from icempm_multi_b200._lib import SimParams  # noqa: E402  (struct layout only)


def build():
    """Build liboracle.so and, where the reference tree exists, _ref/*.so."""
    r = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return C.CDLL(path)


_P = C.POINTER(SimParams)
_vp, _dp = C.c_void_p, C.POINTER(C.c_double)


class Oracle:
    def __init__(self):
        L = _load(os.path.join(HERE, "liboracle.so"))
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [_P, _vp, C.c_uint, C.c_uint, C.c_int, C.c_int, _dp, _vp]
        L.oracle_grid_nodes.restype = C.c_long
        L.oracle_grid_nodes.argtypes = [_P]
        L.oracle_p2g.restype = C.c_int
        L.oracle_p2g.argtypes = [_P, _vp, C.c_uint, C.c_uint, _vp, _vp, _vp]
        L.oracle_update.restype = None
        L.oracle_update.argtypes = [_P, _vp, _vp, _vp, C.c_double, C.c_double, _vp]
        L.oracle_g2p.restype = C.c_int
        L.oracle_g2p.argtypes = [_P, _vp, C.c_uint, C.c_uint, _vp, _vp, C.c_int]
        L.oracle_kirchhoff.argtypes = [_P, _vp, _vp]
        L.oracle_pq.argtypes = [_P, _vp, _dp, _dp, _dp]
        L.oracle_svd.argtypes = [_vp, _vp, _vp, _vp]
        L.oracle_failure.restype = C.c_int
        L.oracle_failure.argtypes = [_P, C.c_int, C.c_double, C.c_double]
        L.oracle_return_map.argtypes = [_P, _vp, _dp, C.c_double, C.c_double, C.c_double]
        self.L = L

    def run(self, params, soa, step0, nsteps, sim_time=0.0):
        """Advance the HostSideSOA ``soa`` in place; returns (err, sim_time, bins)."""
        bins = np.zeros(2 * params.n_indenter_subdivisions)
        t = C.c_double(sim_time)
        err = self.L.oracle_run(C.byref(params), soa.ptr, soa.capacity, soa.size, step0, nsteps, C.byref(t),
                                bins.ctypes.data_as(_vp))
        return err, t.value, bins

    def grid_nodes(self, params):
        return self.L.oracle_grid_nodes(C.byref(params))

    def p2g(self, params, soa):
        nn = self.grid_nodes(params)
        g = np.zeros((3, nn))
        err = self.L.oracle_p2g(C.byref(params), soa.ptr, soa.capacity, soa.size, g[0].ctypes.data_as(_vp),
                                g[1].ctypes.data_as(_vp), g[2].ctypes.data_as(_vp))
        return err, g

    def update(self, params, g, ind_x, ind_y):
        bins = np.zeros(2 * params.n_indenter_subdivisions)
        self.L.oracle_update(C.byref(params), g[0].ctypes.data_as(_vp), g[1].ctypes.data_as(_vp),
                             g[2].ctypes.data_as(_vp), ind_x, ind_y, bins.ctypes.data_as(_vp))
        return bins

    def g2p(self, params, soa, g, record):
        return self.L.oracle_g2p(C.byref(params), soa.ptr, soa.capacity, soa.size, g[1].ctypes.data_as(_vp),
                                 g[2].ctypes.data_as(_vp), int(record))

    def kirchhoff(self, params, F):
        F = np.ascontiguousarray(F, dtype=np.float64)
        out = np.zeros(4)
        self.L.oracle_kirchhoff(C.byref(params), F.ctypes.data_as(_vp), out.ctypes.data_as(_vp))
        return out

    def pq(self, params, F):
        F = np.ascontiguousarray(F, dtype=np.float64)
        p, q, J = C.c_double(), C.c_double(), C.c_double()
        self.L.oracle_pq(C.byref(params), F.ctypes.data_as(_vp), C.byref(p), C.byref(q), C.byref(J))
        return p.value, q.value, J.value

    def svd(self, F):
        F = np.ascontiguousarray(F, dtype=np.float64)
        U, S, V = np.zeros(4), np.zeros(2), np.zeros(4)
        self.L.oracle_svd(F.ctypes.data_as(_vp), U.ctypes.data_as(_vp), S.ctypes.data_as(_vp),
                          V.ctypes.data_as(_vp))
        return U, S, V

    def failure(self, params, grain, p, q):
        return self.L.oracle_failure(C.byref(params), grain, p, q)

    def return_map(self, params, F, Jp, p, q, Je):
        F = np.array(F, dtype=np.float64)
        jp = C.c_double(Jp)
        self.L.oracle_return_map(C.byref(params), F.ctypes.data_as(_vp), C.byref(jp), p, q, Je)
        return F, jp.value


class RefHost:
    """The reference kernels compiled for the host (OpenMP)."""

    def __init__(self):
        L = _load(os.path.join(REF_DIR, "libref_host.so"))
        L.ref_host_run.restype = C.c_int
        L.ref_host_run.argtypes = [_P, _vp, C.c_uint, C.c_uint, C.c_int, C.c_int, _dp, _vp, C.c_int]
        L.ref_host_max_threads.restype = C.c_int
        L.ref_host_svd.argtypes = [_vp, _vp, _vp, _vp]
        L.ref_host_kirchhoff.argtypes = [_P, _vp, _vp]
        L.ref_host_plasticity.argtypes = [_P, _vp, _dp, C.POINTER(C.c_longlong), _dp, _dp]
        self.L = L

    def run(self, params, soa, step0, nsteps, sim_time=0.0, threads=1):
        bins = np.zeros(2 * params.n_indenter_subdivisions)
        t = C.c_double(sim_time)
        err = self.L.ref_host_run(C.byref(params), soa.ptr, soa.capacity, soa.size, step0, nsteps, C.byref(t),
                                  bins.ctypes.data_as(_vp), int(threads))
        return err, t.value, bins

    def max_threads(self):
        return self.L.ref_host_max_threads()

    def svd(self, F):
        F = np.ascontiguousarray(F, dtype=np.float64)
        U, S, V = np.zeros(4), np.zeros(2), np.zeros(4)
        self.L.ref_host_svd(F.ctypes.data_as(_vp), U.ctypes.data_as(_vp), S.ctypes.data_as(_vp),
                            V.ctypes.data_as(_vp))
        return U, S, V

    def kirchhoff(self, params, F):
        F = np.ascontiguousarray(F, dtype=np.float64)
        out = np.zeros(4)
        self.L.ref_host_kirchhoff(C.byref(params), F.ctypes.data_as(_vp), out.ctypes.data_as(_vp))
        return out

    def plasticity(self, params, F, Jp, util):
        F = np.array(F, dtype=np.float64)
        jp, u, p, q = C.c_double(Jp), C.c_longlong(util), C.c_double(), C.c_double()
        self.L.ref_host_plasticity(C.byref(params), F.ctypes.data_as(_vp), C.byref(jp), C.byref(u), C.byref(p),
                                   C.byref(q))
        return F, jp.value, u.value, p.value, q.value


class RefCuda:
    """The reference kernels built for sm_100a, run as one partition."""

    def __init__(self):
        L = _load(os.path.join(REF_DIR, "libref_cuda.so"))
        L.ref_cuda_run.restype = C.c_int
        L.ref_cuda_run.argtypes = [_P, _vp, C.c_uint, C.c_uint, C.c_int, C.c_int, _dp, _vp,
                                   C.POINTER(C.c_float)]
        self.L = L

    def run(self, params, soa, step0, nsteps, sim_time=0.0):
        bins = np.zeros(2 * params.n_indenter_subdivisions)
        t = C.c_double(sim_time)
        ms = C.c_float(0)
        err = self.L.ref_cuda_run(C.byref(params), soa.ptr, soa.capacity, soa.size, step0, nsteps, C.byref(t),
                                  bins.ctypes.data_as(_vp), C.byref(ms))
        return err, t.value, bins, ms.value


class RefParams:
    """The reference's SimParams::Reset / ParseFile."""

    def __init__(self):
        L = _load(os.path.join(REF_DIR, "libref_params.so"))
        L.ref_params_reset.argtypes = [_P]
        L.ref_params_parse_file.restype = C.c_int
        L.ref_params_parse_file.argtypes = [_P, C.c_char_p, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
        L.ref_params_compute_helpers.argtypes = [_P]
        self.L = L

    def reset(self):
        p = SimParams()
        self.L.ref_params_reset(C.byref(p))
        return p

    def parse_file(self, params, path):
        raw = C.create_string_buffer(4096)
        err = C.create_string_buffer(512)
        rc = self.L.ref_params_parse_file(C.byref(params), str(path).encode(), raw, 4096, err, 512)
        return rc, raw.value.decode(), err.value.decode()

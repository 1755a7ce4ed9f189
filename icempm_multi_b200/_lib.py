"""ctypes binding of the C-ABI in ``include/icempm.h`` (libicempm_b200.so).

The library must be built in-tree (``python -m icempm_multi_b200.build``);
importing this module fails loudly if it is missing -- there is no CPU
fallback for the simulation path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libicempm_b200.so")
HOST_LIB_PATH = os.path.join(HERE, "libicempm_host.so")
CLI_PATH = os.path.join(HERE, "icy_cli")

# --- status codes (include/icempm.h) ---
ICY_OK = 0
ICY_ERR_NO_SPACE = 5
ICY_ERR_OUT_OF_GRID = (70, 71, 72, 73)
ICY_ERR_INVALID_ARGUMENT = 100
ICY_ERR_CUDA = 101
ICY_ERR_OUT_OF_MEMORY = 102
ICY_ERR_JSON = 103
ICY_ERR_CONFIG_MISSING = 104
ICY_ERR_FILE = 105
ICY_ERR_CAPACITY = 106
ICY_ERR_POINT_COUNT = 107
ICY_ERR_TIMEOUT = 108
ICY_ERR_NOT_SUPPORTED = 109
ICY_ERR_DRIFT = 110

PRECISION_FP64 = 0
PRECISION_FP32_SPLIT = 1

# HSSOA line indices (simulation/parameters_sim.h:27-35)
IDX_UTILITY, IDX_P, IDX_Q, IDX_JP_INV, POSX, VELX, FE00, BP00, N_PTS_ARRAYS = 0, 1, 2, 3, 4, 6, 8, 12, 16
STATUS_CRUSHED, STATUS_DISABLED, STATUS_LIQUID = 0x10000, 0x20000, 0x40000

_i, _d = C.c_int, C.c_double
# field order of icy::SimParams (simulation/parameters_sim.h:37-85)
SIM_PARAMS_FIELDS = [
    ("n_indenter_subdivisions", _i), ("tpb_P2G", _i), ("tpb_Upd", _i), ("tpb_G2P", _i),
    ("nPtsTotal", _i), ("GridXTotal", _i), ("GridY", _i), ("GridTotal", _i),
    ("GridXDimension", _d), ("InitialTimeStep", _d), ("SimulationEndTime", _d),
    ("UpdateEveryNthStep", _i), ("SimulationStep", _i), ("SimulationTime", _d),
    ("Gravity", _d), ("Density", _d), ("WaterDensity", _d), ("PoissonsRatio", _d), ("YoungsModulus", _d),
    ("lambda_", _d), ("mu", _d), ("kappa", _d),
    ("IceCompressiveStrength", _d), ("IceTensileStrength", _d), ("IceShearStrength", _d),
    ("IceTensileStrength2", _d), ("NACC_beta", _d), ("NACC_M", _d), ("NACC_Msq", _d),
    ("DP_tan_phi", _d), ("DP_threshold_p", _d),
    ("IndDiameter", _d), ("IndRSq", _d), ("IndVelocity", _d), ("IndDepth", _d),
    ("cellsize", _d), ("cellsize_inv", _d), ("Dp_inv", _d),
    ("xmin", _d), ("xmax", _d), ("ymin", _d), ("ymax", _d),
    ("nxmin", _i), ("nxmax", _i), ("nymin", _i), ("nymax", _i),
    ("ParticleVolume", _d), ("ParticleMass", _d), ("WaterParticleMass", _d), ("ParticleViewSize", _d),
    ("indenter_x", _d), ("indenter_x_initial", _d), ("indenter_y", _d), ("indenter_y_initial", _d),
    ("Volume", _d), ("SetupType", _i), ("GrainVariability", _d), ("GridHaloSize", _i),
    ("ExtraSpaceForIncomingPoints", _d), ("PointsTransferBufferFraction", _d),
    ("RebalanceThresholdFreeSpaceRemaining", _d), ("RebalanceThresholdDisabledPercentage", _d),
    ("PointTransferFrequency", _i), ("nPartitions", _i), ("VectorCapacity_transfer", _i),
    ("dt_vol_Dpinv", _d), ("dt_Gravity", _d), ("vmax", _d), ("vmax_squared", _d), ("gbOffset", _i),
]


class SimParams(C.Structure):
    """ctypes mirror of icy_sim_params == icy::SimParams (same layout)."""
    _fields_ = SIM_PARAMS_FIELDS

    def copy(self):
        out = SimParams()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(SimParams))
        return out

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# the symbols include/icempm.h declares (checked by the CPU tests)
EXPORTED = [
    "icy_params_reset", "icy_params_compute_lame", "icy_params_compute_camclay", "icy_params_compute_helpers",
    "icy_params_parse_json", "icy_params_parse_file", "icy_scene_block", "icy_scene_block_count",
    "icy_mpm_create", "icy_mpm_destroy", "icy_mpm_set_stream", "icy_mpm_get_stream", "icy_mpm_update_constants",
    "icy_mpm_transfer_points_to_device", "icy_mpm_transfer_from_device",
    "icy_mpm_reset_indenter_force_accumulator", "icy_mpm_indenter_force", "icy_mpm_reset_grid", "icy_mpm_p2g",
    "icy_mpm_receive_halos", "icy_mpm_update_nodes", "icy_mpm_g2p", "icy_mpm_receive_points", "icy_mpm_step",
    "icy_mpm_synchronize", "icy_mpm_status", "icy_mpm_kernel_launches", "icy_version", "icy_last_error",
    "icy_mpm_profile", "icy_mpm_profile_read", "icy_mpm_set_option", "icy_step_noalloc",
    "icy_batch_create", "icy_batch_destroy", "icy_batch_add", "icy_batch_add_async", "icy_batch_retire",
    "icy_batch_collect", "icy_batch_wait_steps", "icy_batch_remove", "icy_batch_step",
    "icy_batch_download", "icy_batch_synchronize", "icy_batch_set_option", "icy_batch_info",
    "icy_batch_device_bytes", "icy_mpm_device_bytes", "icy_mpm_reserve", "icy_scene_place", "icy_host_alloc", "icy_host_free",
    "icy_batch_set_clock", "icy_mpm_counters",
    "icy_part_plan", "icy_part_create", "icy_part_upload", "icy_part_step", "icy_part_download",
    "icy_part_info", "icy_part_destroy",
]

_lib = None


def lib():
    """Load libicempm_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m icempm_multi_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER(SimParams)
    vp, dp, up = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint)
    sig = {
        "icy_params_reset": (None, [P]),
        "icy_params_compute_lame": (None, [P]),
        "icy_params_compute_camclay": (None, [P]),
        "icy_params_compute_helpers": (None, [P]),
        "icy_params_parse_json": (C.c_int, [P, C.c_char_p, C.c_char_p, C.c_size_t]),
        "icy_params_parse_file": (C.c_int, [P, C.c_char_p, C.c_char_p, C.c_size_t]),
        "icy_scene_block": (C.c_int, [P, C.c_double, C.c_double, C.c_int, C.c_uint64, C.c_int, vp, C.c_uint, up]),
        "icy_scene_block_count": (C.c_uint, [P, C.c_double, C.c_double, C.c_int]),
        "icy_scene_place": (C.c_int, [P, vp, C.c_uint, up, C.c_double]),
        "icy_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(vp)]),
        "icy_host_free": (C.c_int, [vp]),
        "icy_mpm_create": (C.c_int, [P, C.c_int, C.c_uint, C.c_int, C.POINTER(vp)]),
        "icy_mpm_destroy": (C.c_int, [vp]),
        "icy_mpm_set_stream": (C.c_int, [vp, vp]),
        "icy_mpm_get_stream": (vp, [vp]),
        "icy_mpm_update_constants": (C.c_int, [vp, P]),
        "icy_mpm_transfer_points_to_device": (C.c_int, [vp, vp, C.c_uint, C.c_uint]),
        "icy_mpm_transfer_from_device": (C.c_int, [vp, vp, C.c_uint, up, vp]),
        "icy_mpm_reset_indenter_force_accumulator": (C.c_int, [vp]),
        "icy_mpm_indenter_force": (C.c_int, [vp, vp, vp]),
        "icy_mpm_reset_grid": (C.c_int, [vp]),
        "icy_mpm_p2g": (C.c_int, [vp]),
        "icy_mpm_receive_halos": (C.c_int, [vp]),
        "icy_mpm_update_nodes": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
        "icy_mpm_g2p": (C.c_int, [vp, C.c_int, C.c_int]),
        "icy_mpm_receive_points": (C.c_int, [vp]),
        "icy_mpm_step": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "icy_mpm_synchronize": (C.c_int, [vp]),
        "icy_mpm_status": (C.c_int, [vp]),
        "icy_mpm_kernel_launches": (C.c_int64, [vp]),
        "icy_mpm_counters": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "icy_part_plan": (C.c_int, [C.POINTER(SimParams), vp, C.c_uint, C.c_uint, C.c_int, vp, vp, vp, vp]),
        "icy_part_create": (C.c_int, [C.POINTER(SimParams), C.c_int, vp, C.c_uint, C.POINTER(vp)]),
        "icy_part_upload": (C.c_int, [vp, vp, C.c_uint, C.c_uint]),
        "icy_part_step": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_double)]),
        "icy_part_download": (C.c_int, [vp, vp, C.c_uint, C.POINTER(C.c_uint), vp]),
        "icy_part_info": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_uint),
                                    C.POINTER(C.c_int)]),
        "icy_part_destroy": (C.c_int, [vp]),
        "icy_mpm_profile": (C.c_int, [vp, C.c_int]),
        "icy_mpm_set_option": (C.c_int, [vp, C.c_char_p, C.c_double]),
        "icy_mpm_profile_read": (C.c_int, [vp, C.c_int, C.c_char_p, vp, vp, C.POINTER(C.c_int)]),
        "icy_step_noalloc": (C.c_int, [P, vp, C.c_uint, C.c_uint, C.c_int, C.c_int, dp, vp, vp]),
        "icy_batch_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(vp)]),
        "icy_batch_destroy": (C.c_int, [vp]),
        "icy_batch_add": (C.c_int, [vp, P, vp, C.c_uint, C.c_uint, C.POINTER(C.c_int)]),
        "icy_batch_add_async": (C.c_int, [vp, P, vp, C.c_uint, C.c_uint, C.POINTER(C.c_int)]),
        "icy_batch_retire": (C.c_int, [vp, C.c_int, vp, C.c_uint, vp]),
        "icy_batch_collect": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_uint),
                                        C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
        "icy_batch_wait_steps": (C.c_int, [vp, C.c_int]),
        "icy_batch_remove": (C.c_int, [vp, C.c_int]),
        "icy_batch_step": (C.c_int, [vp, C.c_int]),
        "icy_batch_download": (C.c_int, [vp, C.c_int, vp, C.c_uint, up, vp, dp, C.POINTER(C.c_int64)]),
        "icy_batch_synchronize": (C.c_int, [vp]),
        "icy_batch_set_clock": (C.c_int, [vp, C.c_int, C.c_double, C.c_int64]),
        "icy_batch_set_option": (C.c_int, [vp, C.c_char_p, C.c_double]),
        "icy_batch_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.POINTER(vp)]),
        "icy_batch_device_bytes": (C.c_int64, [vp, C.c_int]),
        "icy_mpm_device_bytes": (C.c_int64, [P, C.c_uint, C.c_int]),
        "icy_mpm_reserve": (C.c_int, [C.c_int, C.c_int64]),
        "icy_version": (C.c_char_p, []),
        "icy_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


# the symbols include/icempm_host.h declares
HOST_EXPORTED = ["icy_h5_count", "icy_h5_load", "icy_format_double", "icy_host_last_error"]

_host = None


def host_lib():
    """Load libicempm_host.so, the C++ host layer (raises if it was not built)."""
    global _host
    if _host is not None:
        return _host
    lib()
    if not os.path.exists(HOST_LIB_PATH):
        raise RuntimeError(f"{HOST_LIB_PATH} is missing: build it with `python -m icempm_multi_b200.build`")
    L = C.CDLL(HOST_LIB_PATH)
    P = C.POINTER(SimParams)
    sig = {
        "icy_h5_count": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint)]),
        "icy_h5_load": (C.c_int, [P, C.c_char_p, C.c_void_p, C.c_uint, C.POINTER(C.c_uint)]),
        "icy_format_double": (C.c_int, [C.c_double, C.c_char_p, C.c_size_t]),
        "icy_host_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _host = L
    return L


def format_double(v):
    """The indenter_force.csv number format (fmt's "{}" for a double)."""
    buf = C.create_string_buffer(64)
    check(host_lib().icy_format_double(float(v), buf, 64), "icy_format_double")
    return buf.value.decode()


class IcyError(RuntimeError):
    """A non-zero status from the C-ABI (mirrors the reference's std::runtime_error)."""

    def __init__(self, code, where):
        msg = lib().icy_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code}" + (f": {msg}" if msg else ""))
        self.code = code


def check(code, where):
    if code != ICY_OK:
        raise IcyError(code, where)
    return code


def ptr(a):
    """Address of a C-contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)

"""SimParams helpers: defaults, JSON parsing and the derived constants.

Mirror of ``icy::SimParams`` (simulation/parameters_sim.h:19-105); the work is
done by the C-ABI (``csrc/params.cpp``).
"""
import ctypes as C

from ._lib import SimParams, check, lib


def default_params():
    """SimParams::Reset (simulation/parameters_sim.cpp:5-60)."""
    p = SimParams()
    lib().icy_params_reset(C.byref(p))
    return p


def parse_json(text, params=None):
    """SimParams::ParseFile on JSON text; returns (params, InputRawPoints).

    Raises IcyError (code ICY_ERR_JSON / ICY_ERR_CONFIG_MISSING) like the
    reference throws (simulation/parameters_sim.cpp:75,117-121).
    """
    p = params if params is not None else default_params()
    buf = C.create_string_buffer(4096)
    rc = lib().icy_params_parse_json(C.byref(p), text.encode(), buf, len(buf))
    check(rc, "icy_params_parse_json")
    return p, buf.value.decode()


def parse_file(path, params=None):
    """SimParams::ParseFile (simulation/parameters_sim.cpp:63-126)."""
    p = params if params is not None else default_params()
    buf = C.create_string_buffer(4096)
    rc = lib().icy_params_parse_file(C.byref(p), str(path).encode(), buf, len(buf))
    check(rc, "icy_params_parse_file")
    return p, buf.value.decode()


def compute_helpers(p):
    """SimParams::ComputeHelperVariables (simulation/parameters_sim.cpp:135-153)."""
    lib().icy_params_compute_helpers(C.byref(p))
    return p


def block_params(grid_x, grid_y, h, dt, E=1e9, nu=0.3, rho=980.0, phi_deg=62.0, dp_threshold=0.0,
                 ind_radius=1.0, ind_velocity=1.0, ind_depth=0.5, halo=8, grain_variability=0.5,
                 gravity=9.81):
    """Parameters of a floe-indentation scenario, set through the same JSON keys
    the reference reads (so they pass through SimParams::ParseFile semantics)."""
    import json
    cfg = {
        "InputRawPoints": "synthetic", "nPartitions": 1, "GridHaloSize": halo,
        "InitialTimeStep": dt, "GridX": grid_x, "GridY": grid_y, "GridXDimension": grid_x * h,
        "YoungsModulus": E, "PoissonsRatio": nu, "Density": rho, "Gravity": gravity,
        "DP_phi": phi_deg, "DP_threshold_p": dp_threshold, "GrainVariability": grain_variability,
        "IndDiameter": 2 * ind_radius, "IndVelocity": ind_velocity, "IndDepth": ind_depth,
        "SetupType": 0,
    }
    p, _ = parse_json(json.dumps(cfg))
    return p

"""B200-native MLS-MPM hot path of iceMPM (P2G, grid update, G2P + return mapping).

The compute path is the CUDA library ``libicempm_b200.so`` (sm_100a) behind the
C-ABI of ``include/icempm.h``; this package is the Python mirror of the
reference's host interface (SimParams, HostSideSOA, GPU_Implementation5,
Model) over that C-ABI.
"""
from ._lib import (PRECISION_FP32_SPLIT, PRECISION_FP64, IcyError, SimParams, format_double, host_lib,  # noqa: F401
                   lib)
from .hssoa import HostSideSOA, load_h5, make_block  # noqa: F401
from .model import GPUImplementation, Model  # noqa: F401
from .params import block_params, default_params, parse_file, parse_json  # noqa: F401

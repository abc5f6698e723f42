"""sac_b200 -- B200-native perturbation-MHD hot path of SAC/VAC.

Host side of the drop-in boundary: parameter and snapshot formats (params,
fileio), the ctypes binding of the C-ABI in include/sac_gpu.h (abi), the
time-step driver that mirrors program vac's main loop (vac) and the synthetic
workloads (problems).  The compute path is libsacgpu.so (csrc/).
"""
from .params import SacParams, default_params, make_params  # noqa: F401

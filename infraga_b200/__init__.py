"""infraga_b200: B200-native ray-fan and eigenray path of infraGA/GeoAc.

The compute path is libinfraga_gpu.so (hand-written CUDA for sm_100a behind
the C ABI in include/infraga_gpu.h); this package is a thin host binding.
"""
from ._lib import (ARRIVAL_COLS, CAUSTIC_COLS, FP32C, FP32C_FLAGGED, FP64, GEOM_3D, GEOM_SPH, PATH_COLS, PATH_PROJ, PATH_RAYS,
                   PATH_RESID, PATH_TERRAIN, PROJ_COLS, RAY_AUX_FP64, RAY_FOCUS, RAY_STATUS, Atmosphere, EigParams, FanParams, IgaError, NativeLibraryError, Server, eig_direct,
                   eig_params, eig_run, fan_paths, fan_run, fan_run_device, fan_tune, fan_workspace_bytes, lib,
                   WnlParams, wnl_params, wnl_run)

__all__ = ["ARRIVAL_COLS", "CAUSTIC_COLS", "FP32C", "FP32C_FLAGGED", "FP64", "GEOM_3D", "GEOM_SPH", "PATH_COLS", "PATH_PROJ",
           "PATH_RAYS", "PATH_RESID", "PATH_TERRAIN", "PROJ_COLS", "RAY_AUX_FP64", "RAY_FOCUS", "RAY_STATUS", "Atmosphere", "EigParams", "FanParams", "IgaError", "NativeLibraryError",
           "Server", "eig_direct", "eig_params", "eig_run", "fan_paths", "fan_run", "fan_run_device", "fan_tune",
           "fan_workspace_bytes", "lib", "WnlParams", "wnl_params", "wnl_run"]

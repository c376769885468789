"""arepo_b200: B200 (sm_100a) engine for AREPO's short-range TreePM tree gravity.

The compute path is libarepo_gpugrav.so (arepo_b200/csrc, C ABI in
include/gpugrav.h); this package holds its Python binding and a host-side
interface shaped like the reference's gravity driver.
"""
from ._lib import (  # noqa: F401
    MEM_DEVICE,
    MEM_HOST,
    PREC_FP32,
    PREC_FP64,
    GpuGravError,
    make_params,
)
from .gravity import GravityTree  # noqa: F401

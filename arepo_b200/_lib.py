"""ctypes binding of libarepo_gpugrav (include/gpugrav.h).

The library is built in-tree (arepo_b200/libarepo_gpugrav.so) by
arepo_b200/build.py; loading fails loudly when it is missing: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libarepo_gpugrav.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "gpugrav.h")

ABI_VERSION = 1
MAX_SOFTTYPES = 16
NTAB = 127

OK = 0
ERR_TREE_FULL = -1
ERR_TOPNODES = -2
ERR_OUT_OF_BOX = -3
ERR_INVALID = -10
ERR_OOM = -11
ERR_CUDA = -12
ERR_TIMEOUT = -13
ERR_STATE = -14
ERR_DEEP_TREE = -15
ERR_UNSUPPORTED = -16
ERR_TOO_LARGE = -17

MEM_HOST = 0
MEM_DEVICE = 1
PREC_FP64 = 0
PREC_FP32 = 1
PREC_FP64_GROUP = 2  # the FP32 walk's algorithm in FP64 arithmetic (precision ablation)
FLAG_MULTIPLE_NODE_SOFTENING = 1
FLAG_MINIMUM_OPENING_ANGLE = 2
FLAG_ALLOW_DIRECT_SUMMATION = 4
DIRECT_SUMMATION_THRESHOLD = 3000
DIRECT_FULL = 0
DIRECT_CUT = 1


class Params(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("periodic", C.c_int32),
        ("box_size", C.c_double),
        ("asmth", C.c_double),
        ("rcut", C.c_double),
        ("rcut_cells", C.c_double),
        ("nsofttypes", C.c_int32),
        ("type_of_opening_criterion", C.c_int32),
        ("force_softening", C.c_double * (MAX_SOFTTYPES + 1)),
        ("err_tol_theta", C.c_double),
        ("err_tol_force_acc", C.c_double),
        ("top_node_factor", C.c_double),
        ("multiple_domains", C.c_int32),
        ("precision", C.c_int32),
        ("flags", C.c_int32),
        ("reserved", C.c_int32),
    ]


class TimestepParams(C.Structure):
    """gpugrav_timestep_params: the All.* fields of get_timestep_gravity (timestep.c:284-353)."""
    _fields_ = [
        ("err_tol_int_accuracy", C.c_double),
        ("cf_atime", C.c_double),
        ("cf_a2inv", C.c_double),
        ("cf_hubble_a", C.c_double),
        ("max_size_timestep", C.c_double),
        ("min_size_timestep", C.c_double),
        ("dt_displacement", C.c_double),
        ("timebase_interval", C.c_double),
        ("timebase", C.c_int64),
        ("ti_current", C.c_int64),
        ("nostop_below_min", C.c_int32),
        ("pad", C.c_int32),
        ("synchronized", C.c_uint8 * 64),
    ]


class Domain(C.Structure):
    _fields_ = [
        ("corner", C.c_double * 3),
        ("center", C.c_double * 3),
        ("len", C.c_double),
        ("inverse_len", C.c_double),
        ("big_fac", C.c_double),
    ]


TOPNODE_DTYPE = np.dtype(
    [
        ("start_hi", "<u8"),
        ("start_lo", "<u8"),
        ("size_hi", "<u8"),
        ("size_lo", "<u8"),
        ("daughter", "<i4"),
        ("leaf", "<i4"),
        ("morton_to_peano", "u1", (8,)),
    ]
)


class TreeInfo(C.Structure):
    _fields_ = [
        ("num_particles", C.c_int64),
        ("max_part", C.c_int64),
        ("num_nodes", C.c_int64),
        ("first_non_top", C.c_int64),
        ("num_topnodes", C.c_int32),
        ("num_topleaves", C.c_int32),
        ("max_depth", C.c_int32),
        ("coincident_cells", C.c_int32),
    ]


class ServeConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("max_systems", C.c_int32),
        ("max_particles", C.c_int64),
        ("memory_budget_bytes", C.c_int64),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("admitted", C.c_int64),
        ("completed", C.c_int64),
        ("cancelled", C.c_int64),
        ("waiting", C.c_int64),
        ("running", C.c_int64),
        ("in_flight_particles", C.c_int64),
        ("ticks", C.c_int64),
        ("particle_steps", C.c_int64),
        ("last_tick_s", C.c_double),
        ("last_tick_particles", C.c_int64),
        ("last_tick_systems", C.c_int32),
        ("pad", C.c_int32),
        ("graph_captures", C.c_int64),
        ("graph_replays", C.c_int64),
        ("admit_s", C.c_double),
        ("build_s", C.c_double),
        ("walk_s", C.c_double),
        ("finish_s", C.c_double),
        ("interactions", C.c_int64),
        ("keys_s", C.c_double),
        ("tree_s", C.c_double),
    ]


class Timings(C.Structure):
    _fields_ = [
        ("upload_ms", C.c_double),
        ("domain_ms", C.c_double),
        ("sort_ms", C.c_double),
        ("toptree_ms", C.c_double),
        ("build_ms", C.c_double),
        ("moments_ms", C.c_double),
        ("walk_ms", C.c_double),
        ("download_ms", C.c_double),
        ("interactions", C.c_int64),
        ("walk_kernel_launches", C.c_int32),
        ("build_kernel_launches", C.c_int32),
        ("pm_ms", C.c_double),
    ]


_P = C.c_void_p
_SIGS = {
    "gpugrav_abi_version": (C.c_int32, []),
    "gpugrav_status_string": (C.c_char_p, [C.c_int32]),
    "gpugrav_last_error": (C.c_char_p, [_P]),
    "gpugrav_create": (C.c_int32, [C.POINTER(_P), C.c_int32, C.POINTER(Params)]),
    "gpugrav_destroy": (C.c_int32, [_P]),
    "gpugrav_set_params": (C.c_int32, [_P, C.POINTER(Params)]),
    "gpugrav_set_stream": (C.c_int32, [_P, _P]),
    "gpugrav_synchronize": (C.c_int32, [_P]),
    "gpugrav_load": (C.c_int32, [_P, C.c_int64, _P, _P, _P, C.c_int32, C.POINTER(Domain)]),
    "gpugrav_build": (C.c_int32, [_P, _P, C.c_int32]),
    "gpugrav_walk": (C.c_int32, [_P, _P, _P, _P, _P, C.c_int32]),
    "gpugrav_walk_targets": (C.c_int32, [_P, C.c_int64, _P, _P, _P, _P, _P, C.c_int32]),
    "gpugrav_gravity_direct": (C.c_int32, [_P, C.c_int64, _P, _P, _P, _P, _P, C.c_int32]),
    "gpugrav_direct_split": (C.c_int32, [_P, C.c_int64, _P, _P, _P, _P, _P]),
    "gpugrav_timestep_gravity": (C.c_int32, [_P, _P, C.c_int64, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_int32]),
    "gpugrav_active_particles": (C.c_int32, [_P, C.c_int64, _P, _P, _P, _P, C.c_int32]),
    "gpugrav_set_target_slice": (C.c_int32, [_P, C.c_int32, C.c_int32]),
    "gpugrav_set_target_slice_cost": (C.c_int32, [_P, C.c_int32, C.c_int32, C.c_int64, _P, C.c_int32]),
    "gpugrav_pm_periodic": (C.c_int32, [_P, C.c_int32, C.c_int64, _P, _P, _P, _P, C.c_int32]),
    "gpugrav_set_ewald_table": (C.c_int32, [_P, C.c_int32, _P, _P, _P, _P]),
    "gpugrav_export_mass_per_type": (C.c_int32, [_P, _P]),
    "gpugrav_compute": (C.c_int32, [_P, C.c_int64, _P, _P, _P, _P, C.POINTER(Domain), _P, C.c_int32, _P, _P, _P, C.c_int32]),
    "gpugrav_get_domain": (C.c_int32, [_P, C.POINTER(Domain)]),
    "gpugrav_get_order": (C.c_int32, [_P, _P]),
    "gpugrav_get_keys": (C.c_int32, [_P, _P, _P]),
    "gpugrav_get_topnodes": (C.c_int32, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "gpugrav_get_tree_info": (C.c_int32, [_P, C.POINTER(TreeInfo)]),
    "gpugrav_export_tree": (C.c_int32, [_P] + [_P] * 10),
    "gpugrav_get_timings": (C.c_int32, [_P, C.POINTER(Timings)]),
    "gpugrav_direct": (C.c_int32, [_P, C.c_int64, _P, C.c_int32, _P, _P]),
    "gpugrav_direct_noalloc": (C.c_int32, [C.c_int32, C.POINTER(Params), C.c_int64, _P, _P, _P, C.c_int64, _P, _P,
                                            C.c_int32, _P, _P, _P]),
    "gpugrav_serve_create": (C.c_int32, [C.POINTER(_P), C.c_int32, C.POINTER(Params), C.POINTER(ServeConfig)]),
    "gpugrav_serve_destroy": (C.c_int32, [_P]),
    "gpugrav_serve_last_error": (C.c_char_p, [_P]),
    "gpugrav_serve_submit": (C.c_int32, [_P, C.c_int64, C.c_int64, _P, _P, _P, _P, C.c_int32, C.c_double]),
    "gpugrav_serve_cancel": (C.c_int32, [_P, C.c_int64]),
    "gpugrav_serve_tick": (C.c_int32, [_P, C.POINTER(C.c_int32)]),
    "gpugrav_serve_poll": (C.c_int32, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _P, _P, _P, C.c_int64, _P]),
    "gpugrav_serve_get_stats": (C.c_int32, [_P, C.POINTER(ServeStats)]),
    "gpugrav_measure_fma_peak": (C.c_int32, [C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
}

_lib = None


def header_symbols() -> list[str]:
    """Every entry point declared in include/gpugrav.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|int32_t)\s*\**\s*(gpugrav_\w+)\s*\(", text, re.M)))


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python arepo_b200/build.py` (no CPU fallback exists)"
            )
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.gpugrav_abi_version() != ABI_VERSION:
            raise RuntimeError("libarepo_gpugrav ABI version mismatch")
        _lib = lib
    return _lib


class GpuGravError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gpugrav status {status}: {message}")
        self.status = status


def make_params(
    periodic: bool,
    box_size: float = 1.0,
    asmth: float = 0.0,
    rcut: float = 0.0,
    rcut_cells: float = 4.5,
    softening=(0.01,),
    err_tol_theta: float = 0.7,
    err_tol_force_acc: float = 0.0025,
    type_of_opening_criterion: int = 1,
    top_node_factor: float = 2.5,
    multiple_domains: int = 8,
    precision: int = PREC_FP64,
    multiple_node_softening: bool = False,
    minimum_opening_angle: bool = False,
) -> Params:
    """softening: Plummer-equivalent epsilon per softening type. The spline support is
    ForceSoftening = 2.8 * epsilon with a trailing zero entry (set_softenings,
    src/gravity/grav_softening.c:92-95)."""
    p = Params()
    p.abi_version = ABI_VERSION
    p.periodic = 1 if periodic else 0
    p.box_size = box_size
    p.asmth = asmth
    p.rcut = rcut
    p.rcut_cells = rcut_cells
    p.nsofttypes = len(softening)
    p.type_of_opening_criterion = type_of_opening_criterion
    for i, e in enumerate(softening):
        p.force_softening[i] = 2.8 * e
    p.force_softening[len(softening)] = 0.0
    p.err_tol_theta = err_tol_theta
    p.err_tol_force_acc = err_tol_force_acc
    p.top_node_factor = top_node_factor
    p.multiple_domains = multiple_domains
    p.precision = precision
    p.flags = (FLAG_MULTIPLE_NODE_SOFTENING if multiple_node_softening else 0) | \
        (FLAG_MINIMUM_OPENING_ANGLE if minimum_opening_angle else 0)
    return p


def ptr(a):
    """Address of a numpy array, a torch tensor, or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    raise TypeError(type(a))

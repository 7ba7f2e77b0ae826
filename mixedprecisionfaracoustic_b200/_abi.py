"""ctypes view of include/biot.h and the loader of the in-tree CUDA library.

The library is loaded from ``lib/libbiot_b200.so`` next to this file.  There
is no fallback: if the library is missing the import of anything that needs it
raises, and on a machine without a B200 ``bp_create`` returns BP_ERR_NO_DEVICE.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libbiot_b200.so"

BP_OK = 0
BP_ERR_ARG, BP_ERR_OOM, BP_ERR_CUDA, BP_ERR_CFL, BP_ERR_UNSTABLE = 1, 2, 3, 4, 5
BP_ERR_TIMEOUT, BP_ERR_STATE, BP_ERR_NOT_FOUND, BP_ERR_NO_DEVICE, BP_ERR_BUDGET = 6, 7, 8, 9, 10

PREC = {"fp32": 0, "comp16": 1, "fp64": 2, "cbf16": 3}
FIELDS = ["vux", "vuy", "vuz", "vwx", "vwy", "vwz", "p", "txx", "tyy", "tzz", "txy", "txz", "tyz"]
FIELD = {n: i for i, n in enumerate(FIELDS)}
TRACES = ["txx", "tzz", "vux", "vwx", "p"]          # sisx sisz sisvu sisvw sisp
TRACE = {n: i for i, n in enumerate(TRACES)}
SRC_TAU, SRC_P = 1, 2
ROUND = {"fast": 0, "reference": 1}
MEDIUM = {"auto": 0, "dense": 1}
KERNELS = {"auto": 0, "register": 1, "staged": 2, "march": 3, "fused": 4, "interleaved": 5}
REQ_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}
COEFS = ["rho_x", "rho_y", "rho_z", "rhof", "cc1_x", "cc1_y", "cc1_z", "cc2_x", "cc2_y", "cc2_z",
         "C", "M", "H", "H2u", "mu_xy", "mu_xz", "mu_yz"]
COEF = {n: i for i, n in enumerate(COEFS)}

IntP = C.POINTER(C.c_int)
UIntP = C.POINTER(C.c_uint)
FloatP = C.POINTER(C.c_float)
DoubleP = C.POINTER(C.c_double)


class BpConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("npml", C.c_int),
        ("order", C.c_int), ("precision", C.c_int), ("nt", C.c_int),
        ("dx", C.c_float), ("dt", C.c_float), ("f0", C.c_float), ("t0", C.c_float),
        ("pml_v0", C.c_float), ("pml_r", C.c_float),
        ("src_x", C.c_int), ("src_y", C.c_int), ("src_z", C.c_int), ("src_mask", C.c_int),
        ("nrec", C.c_int), ("rec_x", IntP), ("rec_y", IntP), ("rec_z", IntP),
        ("nsnap", C.c_int), ("snap_steps", IntP), ("snap_fields", C.c_uint), ("snap_masks", UIntP),
        ("snap_y", C.c_int), ("device", C.c_int), ("comp_coef_lo", C.c_int), ("dyn_scale", C.c_int),
        ("check_cfl", C.c_int), ("rounding", C.c_int), ("medium", C.c_int), ("reserved", C.c_int * 2),
    ]


class BpMedium(C.Structure):
    _fields_ = [(n, FloatP) for n in ("rho", "rhof", "M", "C", "H", "H2mu", "mu", "C1", "C2")]


class BpTune(C.Structure):
    _fields_ = [("tile_rows", C.c_int), ("steps_per_sync", C.c_int), ("ctas_per_sm", C.c_int),
                ("tile_segs", C.c_int), ("tile_tz", C.c_int), ("kernel", C.c_int), ("reserved", C.c_int * 2)]


class BpServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("admitted", C.c_longlong), ("completed", C.c_longlong),
        ("failed", C.c_longlong), ("cancelled", C.c_longlong), ("cell_updates", C.c_longlong),
        ("busy_seconds", C.c_double), ("p50_latency_s", C.c_double), ("p99_latency_s", C.c_double),
        ("hbm_in_use", C.c_size_t), ("hbm_budget", C.c_size_t), ("max_resident", C.c_int),
    ]


# (name, restype, argtypes)
_SIGS = [
    ("bp_create", C.c_int, [C.POINTER(BpConfig), C.POINTER(BpMedium), C.POINTER(C.c_void_p)]),
    ("bp_run", C.c_int, [C.c_void_p, C.c_int]),
    ("bp_sync", C.c_int, [C.c_void_p]),
    ("bp_run_timed", C.c_int, [C.c_void_p, C.c_int, FloatP]),
    ("bp_set_graph_steps", C.c_int, [C.c_void_p, C.c_int]),
    ("bp_set_kernel", C.c_int, [C.c_void_p, C.c_int]),
    ("bp_get_kernel", C.c_int, [C.c_void_p, IntP]),
    ("bp_profile_fused", C.c_int, [C.c_void_p, C.c_int, FloatP, DoubleP]),
    ("bp_get_step", C.c_int, [C.c_void_p, IntP]),
    ("bp_get_traces", C.c_int, [C.c_void_p, C.c_int, FloatP, C.c_size_t]),
    ("bp_get_snapshot", C.c_int, [C.c_void_p, C.c_int, C.c_int, FloatP, C.c_size_t]),
    ("bp_snapshot_size", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("bp_get_field", C.c_int, [C.c_void_p, C.c_int, FloatP, C.c_size_t]),
    ("bp_get_field_f64", C.c_int, [C.c_void_p, C.c_int, DoubleP, C.c_size_t]),
    ("bp_get_dims", C.c_int, [C.c_void_p, IntP, IntP, IntP]),
    ("bp_get_coef", C.c_int, [C.c_void_p, C.c_int, FloatP, C.c_size_t]),
    ("bp_field_energy", C.c_int, [C.c_void_p, DoubleP]),
    ("bp_get_scaling", C.c_int, [C.c_void_p, IntP, IntP, FloatP, DoubleP, DoubleP]),
    ("bp_write_reference_outputs", C.c_int, [C.c_void_p, C.c_char_p]),
    ("bp_write_binary_outputs", C.c_int, [C.c_void_p, C.c_char_p]),
    ("bp_receiver_map", C.c_int, [C.c_void_p, IntP, IntP]),
    ("bp_copy_traces_async", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, FloatP]),
    ("bp_checkpoint_size", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("bp_checkpoint", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    ("bp_restore", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    ("bp_profile_phases", C.c_int, [C.c_void_p, C.c_int, FloatP]),
    ("bp_algorithmic_bytes", C.c_int, [C.c_void_p, DoubleP, C.POINTER(C.c_longlong)]),
    ("bp_launches_per_step", C.c_int, [C.c_void_p, IntP]),
    ("bp_get_medium_tuples", C.c_int, [C.c_void_p, IntP]),
    ("bp_set_z_spacing", C.c_int, [C.c_void_p, DoubleP, C.c_int]),
    ("bp_launch_count", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("bp_comp16_encode", C.c_int, [FloatP, C.c_size_t, C.POINTER(C.c_uint16), C.POINTER(C.c_int8)]),
    ("bp_comp16_decode", C.c_int, [C.POINTER(C.c_uint16), C.POINTER(C.c_int8), C.c_size_t, FloatP]),
    ("bp_cbf16_encode", C.c_int, [FloatP, C.c_size_t, C.POINTER(C.c_uint16), C.POINTER(C.c_uint8)]),
    ("bp_cbf16_decode", C.c_int, [C.POINTER(C.c_uint16), C.POINTER(C.c_uint8), C.c_size_t, FloatP]),
    ("bp_rel_l2_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, DoubleP]),
    ("bp_rel_l2_device_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, DoubleP]),
    ("bp_trace_rel_l2", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, DoubleP]),
    ("bp_destroy", None, [C.c_void_p]),
    ("bp_release_cached_memory", C.c_int, [C.c_int]),
    ("bp_debug_fail_allocation", C.c_int, [C.c_int]),
    ("bp_error_string", C.c_char_p, [C.c_int]),
    ("bp_last_error", C.c_char_p, []),
    ("bp_medium_reference_borehole", C.c_int, [C.c_int, C.c_int, C.c_int, FloatP]),
    ("bp_biot_from_moduli", C.c_int, [C.c_double] * 11 + [DoubleP]),
    ("bp_cfl_limit", C.c_int, [C.POINTER(BpConfig), C.POINTER(BpMedium), DoubleP, DoubleP]),
    ("bp_batch_create", C.c_int, [C.POINTER(BpConfig), C.POINTER(BpMedium), C.c_int, C.POINTER(BpTune),
                                  C.POINTER(C.c_void_p)]),
    ("bp_batch_run", C.c_int, [C.c_void_p, C.c_int]),
    ("bp_batch_sync", C.c_int, [C.c_void_p]),
    ("bp_batch_run_timed", C.c_int, [C.c_void_p, C.c_int, FloatP]),
    ("bp_batch_get_traces", C.c_int, [C.c_void_p, C.c_int, C.c_int, FloatP, C.c_size_t]),
    ("bp_batch_get_tune", C.c_int, [C.c_void_p, C.POINTER(BpTune)]),
    ("bp_batch_autotune", C.c_int, [C.c_void_p, C.c_int]),
    ("bp_batch_cell_updates", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("bp_batch_medium_tuples", C.c_int, [C.c_void_p, C.c_int, IntP]),
    ("bp_batch_algorithmic_bytes", C.c_int, [C.c_void_p, DoubleP]),
    ("bp_batch_destroy", None, [C.c_void_p]),
    ("bp_shot_bytes", C.c_int, [C.POINTER(BpConfig), C.POINTER(C.c_size_t)]),
    ("bp_server_create", C.c_int, [C.c_int, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]),
    ("bp_server_submit", C.c_int, [C.c_void_p, C.POINTER(BpConfig), C.POINTER(BpMedium),
                                   C.POINTER(C.c_uint64)]),
    ("bp_server_poll", C.c_int, [C.c_void_p, C.c_uint64, IntP]),
    ("bp_server_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_double]),
    ("bp_server_cancel", C.c_int, [C.c_void_p, C.c_uint64]),
    ("bp_server_get_traces", C.c_int, [C.c_void_p, C.c_uint64, C.c_int, FloatP, C.c_size_t]),
    ("bp_server_release", C.c_int, [C.c_void_p, C.c_uint64]),
    ("bp_server_latency", C.c_int, [C.c_void_p, C.c_uint64, DoubleP]),
    ("bp_server_get_stats", C.c_int, [C.c_void_p, C.POINTER(BpServerStats)]),
    ("bp_server_destroy", None, [C.c_void_p]),
]

_lib = None


def load() -> C.CDLL:
    """Loads the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} missing "
                               "(run python -m mixedprecisionfaracoustic_b200.build)")
        lib = C.CDLL(str(LIB_PATH))
        for name, res, args in _SIGS:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def declared_symbols() -> list[str]:
    return [s[0] for s in _SIGS]


class BiotError(RuntimeError):
    def __init__(self, code: int, where: str):
        lib = load()
        msg = lib.bp_error_string(code).decode()
        detail = (lib.bp_last_error() or b"").decode()
        super().__init__(f"{where}: {msg} ({detail})")
        self.code = code


def check(code: int, where: str) -> None:
    if code != BP_OK:
        raise BiotError(code, where)


def fptr(a):
    return a.ctypes.data_as(FloatP)


def iptr(a):
    return a.ctypes.data_as(IntP)

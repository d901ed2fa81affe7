"""ctypes binding of the C ABI in include/gofish_b200.h (libgofish_b200.so, built in-tree).

The library is the product; this module only declares its entry points.  Loading fails loudly when
the library has not been built -- there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libgofish_b200.so"

MAX_POPULATIONS = 16
MAX_GENERATION = (1 << 24) - 1

GF_OK = 0
STATUS_NAMES = {
    0: "GF_OK",
    1: "GF_ERR_INVALID_ARGUMENT",
    2: "GF_ERR_CUDA",
    3: "GF_ERR_OUT_OF_MEMORY",
    4: "GF_ERR_CAPACITY",
    5: "GF_ERR_STATE",
    6: "GF_ERR_DEVICE",
    7: "GF_ERR_NO_DEVICE",
}

# numpy mirrors of the ABI structs (all members are 4-byte words: no padding)
POP_DTYPE = np.dtype([
    ("Nchrom_e", "<i4"), ("drift", "<i4"), ("alive", "<i4"), ("mutate", "<i4"),
    ("mu", "<f4"), ("F", "<f4"), ("h", "<f4"), ("sel_slope", "<f4"), ("sel_intercept", "<f4"),
])
GEN_DTYPE = np.dtype([
    ("generation", "<i4"), ("compact", "<i4"), ("preserve", "<i4"), ("selection_table", "<i4"),
    ("pop", POP_DTYPE, (MAX_POPULATIONS,)),
    ("migration", "<f4", (MAX_POPULATIONS * MAX_POPULATIONS,)),
])
MSE_DTYPE = np.dtype([
    ("N_ind", "<i4"), ("Nchrom_e", "<i4"), ("mu", "<f4"), ("F", "<f4"), ("h", "<f4"),
    ("sel_slope", "<f4"), ("sel_intercept", "<f4"),
])
assert POP_DTYPE.itemsize == 36 and GEN_DTYPE.itemsize == 16 + 16 * 36 + 1024 and MSE_DTYPE.itemsize == 28


class SimStats(ctypes.Structure):
    _fields_ = [("mutation_generations", ctypes.c_double), ("generations", ctypes.c_int64),
                ("compactions", ctypes.c_int64), ("kernel_launches", ctypes.c_int64)]


class KernelTimes(ctypes.Structure):
    _fields_ = [("drift_ms", ctypes.c_double), ("drift_launches", ctypes.c_int64),
                ("compact_ms", ctypes.c_double), ("compactions", ctypes.c_int64)]


class Tuning(ctypes.Structure):
    _fields_ = [("draw_strategy", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("windows", ctypes.c_int32)]


class Replicate(ctypes.Structure):
    _fields_ = [("seed1", ctypes.c_int32), ("seed2", ctypes.c_int32), ("num_sites", ctypes.c_float),
                ("mu", ctypes.c_float), ("F", ctypes.c_float), ("h", ctypes.c_float),
                ("sel_slope", ctypes.c_float), ("sel_intercept", ctypes.c_float), ("N0", ctypes.c_int32),
                ("growth_rate", ctypes.c_float), ("N_min", ctypes.c_int32), ("N_max", ctypes.c_int32),
                ("num_generations", ctypes.c_int32), ("compact_interval", ctypes.c_int32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("mutation_generations", ctypes.c_double), ("generations", ctypes.c_int64),
                ("super_steps", ctypes.c_int64), ("replicates", ctypes.c_int32), ("active", ctypes.c_int32),
                ("arena_slots", ctypes.c_int64), ("record_wait_ms", ctypes.c_double),
                ("record_producers", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class SimConfig(ctypes.Structure):
    _fields_ = [
        ("seed1", ctypes.c_int32), ("seed2", ctypes.c_int32), ("num_sites", ctypes.c_float),
        ("num_populations", ctypes.c_int32), ("compact_interval", ctypes.c_int32),
        ("reserve_mutations", ctypes.c_int32),
    ]


class MlpConfig(ctypes.Structure):
    _fields_ = [("batch_capacity", ctypes.c_int32), ("lr", ctypes.c_float), ("beta1", ctypes.c_float),
                ("beta2", ctypes.c_float), ("eps", ctypes.c_float), ("weight_decay", ctypes.c_float)]


# every symbol declared in include/*.h, with its ctypes signature
_P = ctypes.c_void_p
_I = ctypes.c_int32
_F = ctypes.c_float
SIGNATURES = {
    "gf_version": (ctypes.c_char_p, []),
    "gf_status_string": (ctypes.c_char_p, [_I]),
    "gf_engine_create": (_I, [_I, _P, ctypes.POINTER(_P)]),
    "gf_engine_destroy": (None, [_P]),
    "gf_engine_last_error": (ctypes.c_char_p, [_P]),
    "gf_engine_device": (_I, [_P]),
    "gf_engine_synchronize": (_I, [_P]),
    "gf_sim_begin_blank": (_I, [_P, ctypes.POINTER(SimConfig), _I]),
    "gf_sim_begin_from_state": (_I, [_P, ctypes.POINTER(SimConfig), _I, _P, _P, _I, _P, _I]),
    "gf_sim_begin_mse": (_I, [_P, ctypes.POINTER(SimConfig), _P, _I]),
    "gf_sim_run": (_I, [_P, _P, _I]),
    "gf_sim_num_mutations": (_I, [_P, ctypes.POINTER(_I)]),
    "gf_sim_read_state": (_I, [_P, _P, _P, _I, ctypes.POINTER(_I)]),
    "gf_sim_sample_begin": (_I, [_P, _P, _P, _I]),
    "gf_sim_sample_wait": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_int64)]),
    "gf_sim_sample_staged": (_I, [_P, ctypes.POINTER(_P)]),
    "gf_sim_device_state": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "gf_sim_selection_view": (_I, [_P, _P]),
    "gf_new_mutation_count": (_I, [_I, _I, _F, _I, _F, _I, _I]),
    "gf_selection_sine_values": (_I, [_P, _F, _F, _F, _F, _I, _I, _P]),
    "gf_population_histogram": (_I, [_P, _P, _I, _I, _F, _P]),
    "gf_site_frequency_spectrum": (_I, [_P, _P, _I, _I, _I, _F, _P]),
    "gf_population_histogram_device": (_I, [_P, _P, _I, _I, _F, _P]),
    "gf_site_frequency_spectrum_device": (_I, [_P, _P, _I, _I, _I, _F, _P]),
    "gf_site_frequency_spectrum_noalloc": (_I, [_P, _I, _I, _I, _F, _P, _P]),
    "gf_sim_stats_read": (_I, [_P, ctypes.POINTER(SimStats)]),
    "gf_joint_site_frequency_spectrum": (_I, [_P, _P, _P, _I, _I, _I, _F, _P]),
    "gf_joint_site_frequency_spectrum_device": (_I, [_P, _P, _P, _I, _I, _I, _F, _P]),
    "gf_joint3_site_frequency_spectrum": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _F, _P]),
    "gf_joint3_site_frequency_spectrum_device": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _F, _P]),
    "gf_replicate_population": (_I, [ctypes.POINTER(Replicate), _I]),
    "gf_replicate_population_table": (None, [ctypes.POINTER(Replicate), _I, _I, _P]),
    "gf_batch_begin": (_I, [_P, _P, _I]),
    "gf_batch_run": (_I, [_P, _I, ctypes.POINTER(_I)]),
    "gf_batch_read_state": (_I, [_P, _I, _P, _P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "gf_batch_sfs": (_I, [_P, _I, _P]),
    "gf_batch_stats_read": (_I, [_P, ctypes.POINTER(BatchStats)]),
    "gf_batch_set_record_budget": (_I, [_P, ctypes.c_int64]),
    "gf_engine_set_profiling": (_I, [_P, _I]),
    "gf_engine_set_tuning": (_I, [_P, ctypes.POINTER(Tuning)]),
    "gf_engine_get_tuning": (_I, [_P, ctypes.POINTER(Tuning)]),
    "gf_engine_read_profile": (_I, [_P, ctypes.POINTER(KernelTimes)]),
    # include/gf_surrogate.h
    "gf_mlp_create": (_I, [_I, _P, ctypes.POINTER(MlpConfig), ctypes.POINTER(_P)]),
    "gf_mlp_destroy": (_I, [_P]),
    "gf_mlp_last_error": (ctypes.c_char_p, [_P]),
    "gf_mlp_param_count": (ctypes.c_int64, []),
    "gf_mlp_set_params": (_I, [_P, _P, ctypes.c_int64]),
    "gf_mlp_get_params": (_I, [_P, _P, ctypes.c_int64]),
    "gf_mlp_set_learning_rate": (_I, [_P, _F]),
    "gf_mlp_forward": (_I, [_P, _P, _I, _P]),
    "gf_mlp_set_fused_inference": (_I, [_P, _I]),
    "gf_mlp_gradients": (_I, [_P, _P, _P, _I, _P, _P]),
    "gf_mlp_train_step": (_I, [_P, _P, _P, _I, _P]),
    "gf_mlp_check": (_I, [_P]),
    "gf_mlp_inject_fault": (_I, [_P, _I]),
    "gf_bf16_gemm": (_I, [_P, _P, _I, _I, _I, _P, _P]),
}

_lib = None


def load(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load libgofish_b200.so and declare every entry point; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is not built; run `python -m parallelpopgen_b200.build` (the CUDA library is required, "
            "there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class GoFishError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data

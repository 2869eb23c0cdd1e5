"""ctypes binding of libmoea_b200.so (declarations in include/moea_b200.h).

The library is the product: this module only loads it and declares the entry
points.  There is no CPU fallback -- if the shared object is missing or a call
fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_LIB_NAME = "libmoea_b200.so"
_lib = None

c_int, c_float, c_double = ctypes.c_int, ctypes.c_float, ctypes.c_double
c_u64, c_u32, c_i64 = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int64
c_size_t, vp = ctypes.c_size_t, ctypes.c_void_p
fp = ctypes.POINTER(ctypes.c_float)
ip = ctypes.POINTER(ctypes.c_int)

EVALUATE_FN = ctypes.CFUNCTYPE(c_int, vp, vp, vp, vp, c_int, c_int, c_int, c_int, c_int, vp)
MATING_FN = ctypes.CFUNCTYPE(c_int, vp, vp, vp, vp, vp, c_int, vp, c_int, c_int, c_int, c_int, vp)
PREPARE_FN = ctypes.CFUNCTYPE(c_int, vp, vp, vp, vp, c_int, c_int, c_int, c_int, c_int, vp, ip)
RESET_FN = ctypes.CFUNCTYPE(None, vp)

class PopulationDesc(ctypes.Structure):
    """moea_population_desc: a borrowed population for the strategy handles."""
    _fields_ = [("d_variables", vp), ("d_objectives", vp), ("d_constraints", vp), ("d_bounds", vp),
                ("size", c_int), ("dimension", c_int), ("objectives", c_int)]


class GenerationDesc(ctypes.Structure):
    """moea_generation_desc: the reference's GenerationContext plus the run seed."""
    _fields_ = [("generation", c_int), ("max_generations", c_int), ("seed", c_u64)]


class NSGA3SelectorConfig(ctypes.Structure):
    """moea_nsga3_selector_config."""
    _fields_ = [("sparse_ratio", c_float), ("cv_bins", c_int), ("cv_clip_upper", c_float),
                ("cv_log_alpha", c_float), ("feasibility_epsilon", c_float), ("association_mode", c_int)]


MOEA_OK = 0
ERROR_NAMES = {1: "invalid argument", 2: "CUDA error", 3: "unsupported", 4: "invalid state",
               5: "device timeout", 6: "out of memory", 7: "callback failed", 8: "load failed"}
MOEA_ERR_INVALID_ARGUMENT = 1


class MoeaError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, 'error')} ({code}): {message}")
        self.code = code


class MoeaValueError(MoeaError, ValueError):
    """MOEA_ERR_INVALID_ARGUMENT: the reference raises ValueError (std::invalid_argument)."""


class AlgorithmConfig(ctypes.Structure):
    """moea_algorithm_config (include/moea_b200.h)."""
    _fields_ = [
        ("algorithm", c_int), ("population_size", c_int), ("max_generations", c_int),
        ("device", c_int), ("seed", c_u64), ("stream", vp),
        ("problem_kind", c_int), ("dimension", c_int), ("objectives", c_int),
        ("constraint_activation_ratio", c_float), ("h_lower", fp), ("h_upper", fp),
        ("evaluate", EVALUATE_FN), ("evaluate_user", vp),
        ("mating", c_int), ("mate", MATING_FN), ("mate_user", vp),
        ("sbx_eta_initial", c_float), ("sbx_eta_final", c_float),
        ("sbx_probability", c_float), ("sbx_copy_probability", c_float),
        ("mutation", c_int), ("pm_eta_initial", c_float), ("pm_eta_final", c_float),
        ("pm_probability", c_float),
        ("directions", c_int), ("partitions", c_int), ("adapt_frequency", c_float),
        ("h_user_directions", fp), ("user_direction_count", c_int),
        ("normalize_user_directions", c_int),
        ("sparse_ratio", c_float), ("cv_bins", c_int), ("cv_clip_upper", c_float),
        ("cv_log_alpha", c_float), ("feasibility_epsilon", c_float),
        ("association_mode", c_int), ("rvea_alpha", c_float),
        ("h_initial_population", fp), ("use_graphs", c_int), ("fused_small", c_int),
        ("save_directory", ctypes.c_char_p), ("save_interval", c_int),
        ("problem_name", ctypes.c_char_p), ("constraint_count", c_int),
        ("prepare", PREPARE_FN), ("problem_reset", RESET_FN),
    ]


class PopulationViewC(ctypes.Structure):
    """moea_population_view (include/moea_b200.h)."""
    _fields_ = [
        ("d_variables", vp), ("d_objectives", vp), ("d_constraints", vp), ("d_auxiliary", vp),
        ("auxiliary_count", c_int), ("size", c_int), ("dimension", c_int), ("objectives", c_int),
        ("active_count", c_int), ("generation", c_int), ("initialized", c_int),
        ("finished", c_int), ("device", c_int), ("total_ms", c_double),
        ("kernels_per_generation", c_int), ("graph_active", c_int),
        ("last_max_front", c_int), ("last_sizes", c_int * 4),
    ]


def library_path() -> Path:
    override = os.environ.get("MOEA_B200_LIBRARY")
    if override:
        return Path(override)
    return Path(__file__).resolve().parent / _LIB_NAME


# (name, restype, argtypes)
_SIGNATURES = [
    ("moea_abi_version", c_int, []),
    ("moea_last_error", ctypes.c_char_p, []),
    ("moea_workspace_create", c_int, [c_int, c_int, c_int, c_int, ctypes.POINTER(vp)]),
    ("moea_workspace_destroy", None, [vp]),
    ("moea_workspace_bytes", c_size_t, [vp]),
    ("moea_workspace_set_peel", c_int, [vp, c_int]),
    ("moea_workspace_set_tiles", c_int, [vp, c_int]),
    ("moea_ndsort", c_int, [vp, vp, vp, c_int, c_int, c_int, vp, ip, vp]),
    ("moea_nds_extract", c_int, [vp, vp, c_int, vp, c_int, vp, vp, vp]),
    ("moea_ideal_point", c_int, [vp, vp, c_int, c_int, vp, vp]),
    ("moea_normalize", c_int, [vp, vp, vp, c_int, c_int, vp, vp, vp]),
    ("moea_associate", c_int, [vp, vp, vp, c_int, c_int, c_int, vp, vp, c_int, vp]),
    ("moea_associate_static", c_int, [vp, vp, c_int, c_int, c_int, vp, vp, vp]),
    ("moea_selftest_wait_timeout", c_int, [vp, c_int, ctypes.c_ulonglong, vp]),
    ("moea_igd", c_int, [vp, vp, c_int, c_int, vp, c_int, c_int, vp, ctypes.POINTER(ctypes.c_double), vp]),
    ("moea_niching", c_int, [vp, c_u64, ctypes.POINTER(c_u64), vp, vp, vp, vp, c_int, c_int, vp, vp]),
    ("moea_nsga3_select", c_int, [vp, vp, vp, c_int, c_int, vp, c_int, c_u64, ctypes.POINTER(c_u64),
                                  vp, vp, vp, vp, c_int, vp]),
    ("moea_quantize_cv", c_int, [vp, vp, c_int, c_float, c_float, c_float, c_int, vp]),
    ("moea_native_open", c_int, [ctypes.c_char_p, ctypes.POINTER(vp)]),
    ("moea_native_close", None, [vp]),
    ("moea_native_schema", c_int, [vp, ctypes.c_char_p, c_size_t, ctypes.POINTER(c_size_t)]),
    ("moea_native_set_int", c_int, [vp, ctypes.c_char_p, ctypes.c_longlong]),
    ("moea_native_set_float", c_int, [vp, ctypes.c_char_p, c_double]),
    ("moea_native_set_bool", c_int, [vp, ctypes.c_char_p, c_int]),
    ("moea_native_set_string", c_int, [vp, ctypes.c_char_p, ctypes.c_char_p]),
    ("moea_native_set_floats", c_int, [vp, ctypes.c_char_p, ctypes.POINTER(c_double), c_int]),
    ("moea_native_create", c_int, [vp, ctypes.c_char_p, c_int, c_int, fp, fp]),
    ("moea_native_constraint_count", c_int, [vp, ip]),
    ("moea_native_evaluate", c_int, [vp, vp, vp, vp, c_int, c_int, c_int, c_int, c_int, vp]),
    ("moea_native_prepare", c_int, [vp, vp, vp, vp, c_int, c_int, c_int, c_int, c_int, vp, ip]),
    ("moea_native_reset", None, [vp]),
    ("moea_rvea_translate", c_int, [vp, vp, c_int, c_int, vp, vp, vp]),
    ("moea_rvea_partition", c_int, [vp, vp, vp, c_int, c_int, c_int, c_int, c_int, vp, vp, vp]),
    ("moea_rvea_gamma", c_int, [vp, vp, c_int, c_int, vp, vp]),
    ("moea_rvea_apd", c_int, [vp, vp, vp, vp, vp, c_int, c_int, c_int, c_int, c_int, c_float, vp, vp]),
    ("moea_rvea_elitism", c_int, [vp, vp, vp, vp, c_int, c_int, c_int, vp, ip, vp]),
    ("moea_rvea_adapt", c_int, [vp, vp, vp, c_int, c_int, c_int, c_int, vp, vp]),
    ("moea_tournament", c_int, [vp, vp, vp, c_int, vp, vp]),
    ("moea_sbx", c_int, [vp, vp, vp, vp, vp, vp, vp, c_float, c_float, c_float, c_int, c_int, vp]),
    ("moea_pm", c_int, [vp, vp, vp, c_float, c_float, c_int, c_int, vp]),
    ("moea_reproduce", c_int, [vp, vp, vp, c_int, vp, vp, vp, c_int, c_int, c_int, c_int, c_float,
                               c_float, c_float, c_int, c_float, c_float, c_u64, c_u32, vp]),
    ("moea_rng_blocks", c_int, [c_u64, c_u32, c_u32, c_i64, vp, vp]),
    ("moea_initialize_population", c_int, [c_u64, c_u32, vp, c_int, c_int, vp, vp]),
    # strategy handles
    ("moea_create_dasdennis", c_int, [c_int, ctypes.POINTER(vp)]),
    ("moea_create_adaptive_directions", c_int, [c_float, ctypes.POINTER(vp)]),
    ("moea_create_user_directions", c_int, [fp, c_int, c_int, c_int, ctypes.POINTER(vp)]),
    ("moea_directions_initialize", c_int, [vp, c_int, c_int, c_int, vp]),
    ("moea_directions_view", c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), ip, ip]),
    ("moea_directions_update", c_int, [vp, ctypes.POINTER(PopulationDesc), vp, ctypes.POINTER(GenerationDesc), vp]),
    ("moea_directions_reset", c_int, [vp, vp]),
    ("moea_directions_destroy", None, [vp]),
    ("moea_create_tournament", c_int, [ctypes.POINTER(vp)]),
    ("moea_create_random_mating", c_int, [ctypes.POINTER(vp)]),
    ("moea_mating_select", c_int, [vp, ctypes.POINTER(PopulationDesc), vp, vp, vp, c_int,
                                   ctypes.POINTER(GenerationDesc), vp]),
    ("moea_mating_destroy", None, [vp]),
    ("moea_create_sbx", c_int, [c_float, c_float, c_float, c_float, ctypes.POINTER(vp)]),
    ("moea_crossover_apply", c_int, [vp, ctypes.POINTER(PopulationDesc), vp, ctypes.POINTER(PopulationDesc),
                                     ctypes.POINTER(GenerationDesc), vp]),
    ("moea_crossover_destroy", None, [vp]),
    ("moea_create_pm", c_int, [c_float, c_float, c_float, ctypes.POINTER(vp)]),
    ("moea_mutation_apply", c_int, [vp, ctypes.POINTER(PopulationDesc), ctypes.POINTER(GenerationDesc), vp]),
    ("moea_mutation_destroy", None, [vp]),
    ("moea_create_nsga3_selector", c_int, [ctypes.POINTER(NSGA3SelectorConfig), ctypes.POINTER(vp)]),
    ("moea_create_rvea_selector", c_int, [c_float, ctypes.POINTER(vp)]),
    ("moea_selector_initialize", c_int, [vp, c_int, c_int, c_int, c_int, vp, c_int, vp]),
    ("moea_selector_prepare", c_int, [vp, ctypes.POINTER(PopulationDesc), ctypes.POINTER(GenerationDesc), vp]),
    ("moea_selector_select", c_int, [vp, ctypes.POINTER(PopulationDesc), ctypes.POINTER(PopulationDesc),
                                     ctypes.POINTER(PopulationDesc), ctypes.POINTER(GenerationDesc), vp]),
    ("moea_selector_mating_state", c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]),
    ("moea_selector_active_count", c_int, [vp, ip, vp]),
    ("moea_selector_finalize", c_int, [vp, ctypes.POINTER(PopulationDesc), vp]),
    ("moea_selector_result_indices", c_int, [vp, ctypes.POINTER(vp), ip]),
    ("moea_selector_reset", c_int, [vp, vp]),
    ("moea_selector_destroy", None, [vp]),
    ("moea_problem_evaluate", c_int, [c_int, vp, c_int, c_int, c_int, vp, vp, vp]),
    ("moea_reference_directions", c_int, [c_int, c_int, c_int, fp, c_size_t, ip]),
    ("moea_algorithm_config_defaults", None, [ctypes.POINTER(AlgorithmConfig), c_int]),
    ("moea_algorithm_create", c_int, [ctypes.POINTER(AlgorithmConfig), ctypes.POINTER(vp)]),
    ("moea_algorithm_destroy", None, [vp]),
    ("moea_algorithm_initialize", c_int, [vp]),
    ("moea_algorithm_step", c_int, [vp]),
    ("moea_algorithm_run", c_int, [vp, ctypes.POINTER(c_double)]),
    ("moea_algorithm_reset", c_int, [vp]),
    ("moea_algorithm_synchronize", c_int, [vp]),
    ("moea_algorithm_finalize", c_int, [vp]),
    ("moea_algorithm_flush_snapshots", c_int, [vp]),
    ("moea_algorithm_load_snapshot", c_int, [vp, ctypes.c_char_p]),
    ("moea_algorithm_view", c_int, [vp, ctypes.POINTER(PopulationViewC)]),
    ("moea_algorithm_directions", c_int, [vp, ctypes.POINTER(vp), ip]),
    ("moea_algorithm_profile_step", c_int, [vp, ctypes.c_char_p, c_size_t, fp, c_int, ip]),
    ("moea_algorithm_selection_stats", c_int, [vp, ip, ip]),
    ("moea_algorithm_device_status", c_int, [vp, ip]),
    ("moea_batch_create", c_int, [ctypes.POINTER(AlgorithmConfig), c_int, vp, c_int, ctypes.POINTER(vp)]),
    ("moea_batch_destroy", None, [vp]),
    ("moea_batch_step", c_int, [vp]),
    ("moea_batch_run", c_int, [vp, c_int, ctypes.POINTER(ctypes.c_double)]),
    ("moea_batch_synchronize", c_int, [vp]),
    ("moea_batch_info", c_int, [vp, ip, ip, ip, ip]),
    ("moea_batch_view", c_int, [vp, c_int, ctypes.POINTER(PopulationViewC)]),
    ("moea_batch_schedule", c_int, [vp, ip, ip, fp, fp, fp, fp, ip]),
    ("moea_batch_tile_shapes", c_int, [vp, ip, c_int]),
]

SYMBOLS = [s[0] for s in _SIGNATURES]


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not path.exists():
            raise ImportError(f"{path} is missing: build it with `python cuda-moea_b200/build.py` "
                              "(the B200 path has no CPU fallback)")
        L = ctypes.CDLL(str(path))
        for name, res, args in _SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.moea_abi_version() != 1:
            raise ImportError("libmoea_b200 ABI mismatch")
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != MOEA_OK:
        msg = lib().moea_last_error()
        cls = MoeaValueError if status == MOEA_ERR_INVALID_ARGUMENT else MoeaError
        raise cls(status, msg.decode() if msg else "")

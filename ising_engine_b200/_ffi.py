"""ctypes bindings of the C ABI in include/ising_b200.h.

The library is loaded from the package's ``_lib`` directory. There is no CPU
fallback: if the library is missing, loading raises, and every call that
fails on the device raises :class:`EngineError` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
import re

from . import _build

_lib = None

IE_OK = 0
STATUS_NAMES = {0: "IE_OK", 1: "IE_ERR_INVALID", 2: "IE_ERR_UNSUPPORTED", 3: "IE_ERR_OOM",
                4: "IE_ERR_CUDA", 5: "IE_ERR_TIMEOUT", 6: "IE_ERR_DEVICE"}


class EngineError(RuntimeError):
    """A non-zero ie_status from the library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class ie_problem(C.Structure):
    _fields_ = [("num_vars", C.c_uint64), ("linear", C.c_void_p), ("row_offsets", C.c_void_p),
                ("col_indices", C.c_void_p), ("values", C.c_void_p), ("energy_offset", C.c_double)]


class ie_config(C.Structure):
    _fields_ = [("temp_max", C.c_double), ("temp_min", C.c_double),
                ("sweeps_per_exchange", C.c_uint64), ("total_exchanges", C.c_uint64),
                ("seed", C.c_uint64), ("num_temps", C.c_uint32), ("num_pops", C.c_uint32),
                ("num_slices", C.c_uint32), ("exchange_interval", C.c_uint32),
                ("force_f64", C.c_int32), ("device", C.c_int32), ("pt_path", C.c_int32),
                ("use_icm", C.c_int32), ("kernel_form", C.c_int32), ("max_cluster", C.c_uint32),
                ("bit_sliced", C.c_int32)]


class ie_problem_device(C.Structure):
    _fields_ = [("num_vars", C.c_uint32), ("nnz", C.c_uint32), ("row_offsets", C.c_void_p),
                ("col_indices", C.c_void_p), ("values", C.c_void_p), ("linear", C.c_void_p)]


class ie_pa_config(C.Structure):
    _fields_ = [("ess_threshold", C.c_double), ("ladder_tuning_iters", C.c_uint32),
                ("ladder_tuning_steps", C.c_uint32), ("post_resample_relaxation", C.c_uint32),
                ("ladder_mode", C.c_int32), ("use_icm", C.c_int32)]


class ie_pa_report(C.Structure):
    _fields_ = [("free_energy", C.c_double), ("resample_events", C.c_uint64), ("n_ess", C.c_uint64),
                ("ess_history", C.c_void_p), ("family_rho", C.c_void_p), ("family_count", C.c_void_p),
                ("capacity", C.c_uint64), ("alphas", C.c_void_p)]


class ie_batch_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("force_f64", C.c_int32),
                ("threads_per_block", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("disable_windows", C.c_int32), ("use_graph", C.c_int32),
                ("kernel_form", C.c_int32), ("item_sites", C.c_uint32), ("tie_shift", C.c_uint32),
                ("bit_sliced", C.c_int32), ("bulk_ring", C.c_int32)]


class ie_serve_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("force_f64", C.c_int32), ("max_requests", C.c_uint32),
                ("site_budget", C.c_uint32), ("max_sites", C.c_uint64), ("max_couplings", C.c_uint64),
                ("max_schedule_steps", C.c_uint64), ("kernel_form", C.c_int32), ("tick_us", C.c_uint32)]


_vp = C.c_void_p
_SIGS = {
    "ie_last_error": ([], C.c_char_p),
    "ie_abi_version": ([], C.c_int),
    "ie_create": ([_vp, _vp, _vp], C.c_int),
    "ie_destroy": ([_vp], C.c_int),
    "ie_set_clamps": ([_vp, _vp, _vp], C.c_int),
    "ie_init_random": ([_vp], C.c_int),
    "ie_set_spins": ([_vp, _vp], C.c_int),
    "ie_step": ([_vp, _vp, C.c_uint32, C.c_uint64], C.c_int),
    "ie_run_schedule": ([_vp, _vp, C.c_uint32, C.c_uint64], C.c_int),
    "ie_run_pt": ([_vp], C.c_int),
    "ie_run_pa": ([_vp, _vp, _vp], C.c_int),
    "ie_presolve": ([_vp, _vp, _vp, C.c_uint64, _vp, _vp, _vp], C.c_int),
    "ie_two_opt": ([_vp, _vp, _vp, _vp], C.c_int),
    "ie_set_init_probs": ([_vp, _vp], C.c_int),
    "ie_warm_start_words": ([C.c_uint64, C.c_uint64, _vp, _vp, _vp, C.c_uint64, C.c_uint64, _vp, _vp], C.c_int),
    "ie_path_relink": ([_vp, _vp, C.c_uint64, _vp, _vp, _vp], C.c_int),
    "ie_connected_components": ([_vp, _vp, _vp, _vp], C.c_int),
    "ie_pa_normalized_weights": ([_vp, C.c_uint64, _vp], C.c_int),
    "ie_pa_effective_sample_size": ([_vp, C.c_uint64, _vp], C.c_int),
    "ie_pa_free_energy_increment": ([_vp, C.c_uint64, _vp], C.c_int),
    "ie_pa_family_entropy": ([_vp, C.c_uint64, _vp, _vp], C.c_int),
    "ie_pa_systematic_resample": ([_vp, C.c_uint64, C.c_double, _vp], C.c_int),
    "ie_pa_adapt_spacings": ([_vp, _vp, C.c_uint64, _vp], C.c_int),
    "ie_pa_feedback_optimized_alphas": ([_vp, _vp, C.c_uint64, C.c_double, _vp], C.c_int),
    "ie_read_spins": ([_vp, _vp], C.c_int),
    "ie_read_energies": ([_vp, _vp], C.c_int),
    "ie_read_swap_stats": ([_vp, _vp, _vp], C.c_int),
    "ie_read_rng_state": ([_vp, _vp, _vp], C.c_int),
    "ie_state_size": ([_vp, _vp], C.c_int),
    "ie_save_state": ([_vp, _vp, C.c_uint64], C.c_int),
    "ie_load_state": ([_vp, _vp, C.c_uint64], C.c_int),
    "ie_state_digest": ([_vp, _vp], C.c_int),
    "ie_fnv1a": ([_vp, C.c_uint64, _vp], C.c_int),
    "ie_read_incumbent": ([_vp, _vp, _vp], C.c_int),
    "ie_read_best": ([_vp, _vp, _vp], C.c_int),
    "ie_one_opt": ([_vp, _vp, _vp, _vp], C.c_int),
    "ie_geometric_temps": ([C.c_double, C.c_double, C.c_uint32, _vp], C.c_int),
    "ie_suggested_temp_range": ([_vp, _vp, _vp], C.c_int),
    "ie_batch_create": ([_vp, C.c_uint32, _vp, _vp, _vp], C.c_int),
    "ie_batch_destroy": ([_vp], C.c_int),
    "ie_batch_init_random": ([_vp], C.c_int),
    "ie_batch_run_schedule": ([_vp, _vp, C.c_uint64], C.c_int),
    "ie_batch_run_schedule_plain": ([_vp, _vp, C.c_uint64, C.c_uint32, C.c_uint32], C.c_int),
    "ie_batch_read_spins": ([_vp, _vp], C.c_int),
    "ie_batch_read_energies": ([_vp, _vp], C.c_int),
    "ie_batch_read_draws": ([_vp, _vp], C.c_int),
    "ie_batch_recompute_energies": ([_vp, _vp], C.c_int),
    "ie_batch_last_run_ms": ([_vp, _vp], C.c_int),
    "ie_batch_autotune": ([_vp, _vp, C.c_uint64, _vp], C.c_int),
    "ie_batch_class_report": ([_vp, C.c_uint32, _vp, _vp, _vp], C.c_int),
    "ie_batch_last_launches": ([_vp, _vp], C.c_int),
    "ie_batch_exact_decisions": ([_vp, _vp], C.c_int),
    "ie_xoshiro_jump_poly": ([C.c_uint64, _vp], C.c_int),
    "ie_probe_peaks": ([C.c_int32, _vp, _vp], C.c_int),
    "ie_sa_run_static": ([_vp, C.c_uint64, _vp, C.c_uint64, _vp, _vp, C.c_int32, _vp], C.c_int),
    "ie_serve_create": ([_vp, _vp], C.c_int),
    "ie_serve_destroy": ([_vp], C.c_int),
    "ie_serve_submit": ([_vp, _vp, C.c_uint64, _vp, C.c_uint64, _vp, _vp, _vp], C.c_int),
    "ie_serve_tick": ([_vp, _vp, _vp, _vp], C.c_int),
    "ie_serve_poll": ([_vp, _vp, C.c_uint32, _vp], C.c_int),
    "ie_serve_result": ([_vp, C.c_uint64, _vp, _vp], C.c_int),
    "ie_serve_footprint": ([_vp, _vp, C.c_uint64, _vp], C.c_int),
    "ie_serve_last_tick": ([_vp, _vp, _vp], C.c_int),
    "ie_v2_create": ([_vp, C.c_uint32, _vp, C.c_int32, _vp], C.c_int),
    "ie_v2_destroy": ([_vp], C.c_int),
    "ie_v2_metropolis": ([_vp, _vp, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, _vp, _vp], C.c_int),
    "ie_v2_exchange": ([_vp, _vp, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, _vp, _vp], C.c_int),
    "ie_v2_gibbs": ([_vp, _vp, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, _vp, _vp], C.c_int),
    "ie_v2_read": ([_vp, _vp, _vp], C.c_int),
    "ie_v2_audit": ([_vp, _vp], C.c_int),
    "ie_v2_coloring": ([_vp, _vp], C.c_int),
}


def header_symbols() -> list[str]:
    """Names of the functions declared in include/ising_b200.h."""
    path = os.path.join(os.path.dirname(_build.HERE), "include", "ising_b200.h")
    text = open(path).read()
    return sorted(set(re.findall(r"\b(ie_[a-z0-9_]+)\s*\(", text)))


def lib(build_if_missing: bool = True):
    """Loads (building first if needed and allowed) the CUDA library."""
    global _lib
    if _lib is None:
        if build_if_missing:
            _build.build()
        if not os.path.exists(_build.LIB_PATH):
            raise ImportError(f"CUDA library not built: {_build.LIB_PATH}")
        L = C.CDLL(_build.LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != IE_OK:
        msg = lib().ie_last_error()
        raise EngineError(status, msg.decode() if msg else "")

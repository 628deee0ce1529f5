"""Population annealing with parallel-tempering equilibration (PA-PT).

Mirrors src/solver/population_annealing.rs: the reweighting / resampling
primitives (``normalized_weights`` :51-56, ``effective_sample_size`` :60-63,
``free_energy_increment`` :70-78, ``family_entropy`` :84-101,
``systematic_resample`` :106-127, ``adapt_spacings`` :141-152,
``feedback_optimized_alphas`` :172-232) computed by the
library's host code, and ``PaDiagnostics`` (:34-45). The annealing driver
(ultimate.rs:576-852) runs on the device through ``Engine.run_pa``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _ffi


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class PaDiagnostics:
    """population_annealing.rs:34-45, plus the frozen ladder shape."""
    free_energy: float = 0.0
    ess_history: list = field(default_factory=list)
    family_entropy_history: list = field(default_factory=list)  # (rho, surviving families)
    resample_events: int = 0
    alphas: np.ndarray | None = None


# LadderMode (ultimate.rs): acceptance uniformization (default) or the
# feedback-optimized ladder of Katzgraber, Trebst, Huse and Troyer
ACCEPTANCE_UNIFORM = 0
FEEDBACK_OPTIMIZED = 1


@dataclass
class PaConfig:
    """The PA knobs of UltimateSolver (ultimate.rs:29-52) with their defaults
    (ultimate.rs:77-86)."""
    ess_threshold: float = 0.5
    ladder_tuning_iters: int = 8
    ladder_tuning_steps: int = 10
    post_resample_relaxation: int = 5
    ladder_mode: int = ACCEPTANCE_UNIFORM
    use_icm: bool = False

    def to_c(self) -> _ffi.ie_pa_config:
        return _ffi.ie_pa_config(float(self.ess_threshold), int(self.ladder_tuning_iters),
                                 int(self.ladder_tuning_steps), int(self.post_resample_relaxation),
                                 int(self.ladder_mode), int(self.use_icm))


def normalized_weights(log_w) -> np.ndarray:
    lw = np.ascontiguousarray(log_w, dtype=np.float64)
    out = np.zeros(len(lw), dtype=np.float64)
    _ffi.check(_ffi.lib().ie_pa_normalized_weights(_p(lw), len(lw), _p(out)))
    return out


def effective_sample_size(w_norm) -> float:
    w = np.ascontiguousarray(w_norm, dtype=np.float64)
    out = C.c_double()
    _ffi.check(_ffi.lib().ie_pa_effective_sample_size(_p(w), len(w), C.byref(out)))
    return out.value


def free_energy_increment(log_w) -> float:
    lw = np.ascontiguousarray(log_w, dtype=np.float64)
    out = C.c_double()
    _ffi.check(_ffi.lib().ie_pa_free_energy_increment(_p(lw), len(lw), C.byref(out)))
    return out.value


def family_entropy(family_ids):
    """(rho, surviving family count); families summed in ascending id order."""
    ids = np.ascontiguousarray(family_ids, dtype=np.uint64)
    rho, fams = C.c_double(), C.c_uint64()
    _ffi.check(_ffi.lib().ie_pa_family_entropy(_p(ids), len(ids), C.byref(rho), C.byref(fams)))
    return rho.value, int(fams.value)


def systematic_resample(w_norm, u: float) -> np.ndarray:
    w = np.ascontiguousarray(w_norm, dtype=np.float64)
    out = np.zeros(len(w), dtype=np.uint64)
    _ffi.check(_ffi.lib().ie_pa_systematic_resample(_p(w), len(w), float(u), _p(out)))
    return out.astype(np.int64)


def adapt_spacings(spacings, acceptance) -> np.ndarray:
    d = np.ascontiguousarray(spacings, dtype=np.float64)
    a = np.ascontiguousarray(acceptance, dtype=np.float64)
    if d.shape != a.shape:
        raise ValueError("spacings and acceptance must have the same length")
    out = np.zeros(len(d), dtype=np.float64)
    _ffi.check(_ffi.lib().ie_pa_adapt_spacings(_p(d), _p(a), len(d), _p(out)))
    return out


def feedback_optimized_alphas(alphas, flow, damping: float) -> np.ndarray:
    """population_annealing.rs:172-232."""
    a = np.ascontiguousarray(alphas, dtype=np.float64)
    f = np.ascontiguousarray(flow, dtype=np.float64)
    if a.shape != f.shape:
        raise ValueError("alphas and flow must have the same length")
    out = np.zeros(len(a), dtype=np.float64)
    _ffi.check(_ffi.lib().ie_pa_feedback_optimized_alphas(_p(a), _p(f), len(a), float(damping), _p(out)))
    return out

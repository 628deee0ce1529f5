"""UltimateSolver's parallel-tempering path on the device.

Mirrors the reference's solver configuration (src/solver/ultimate.rs:18-87)
and its PT path (ultimate.rs:234-387): random init from the master stream,
total_exchanges x sweeps_per_exchange calls of engine::step with energy
resync every 1000 steps, update_incumbent after every exchange block, best
replica extraction, then the 1-opt polish of src/solver/local_search.rs:19-57.

With num_pops > 1 the solve is population annealing with PT equilibration
(ultimate.rs:576-852, run by ``Engine.run_pa``). Presolve and component
decomposition (ultimate.rs:161-218) run first on the host
(``ising_engine_b200.presolve``), as in the reference.
"""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np

from . import _ffi
from .core import QuboModel
from .engine import Engine, _p, _problem

NUM_REPLICAS = 64


def steepest_descent_1opt(model: QuboModel, state, is_clamped=None) -> float:
    """local_search.rs:19-57 (steepest improving flip, lowest index on ties),
    in the same f64 evaluation order, on the host. Polishes ``state`` in
    place. ``UltimateSolver.solve`` runs the device form (``Engine.one_opt``)."""
    n = model.num_vars
    state = np.asarray(state)
    clamped = np.zeros(n, dtype=bool) if is_clamped is None else np.asarray(is_clamped, dtype=bool)
    ro = model.row_offsets.astype(np.int64)
    ci = model.col_indices.astype(np.int64)
    va = model.values
    lin = model.linear
    gains = np.zeros(n)
    for i in range(n):
        field = float(lin[i])
        for k in range(ro[i], ro[i + 1]):
            field += float(va[k]) * float(state[ci[k]])
        gains[i] = (1.0 - 2.0 * float(state[i])) * field
    total = 0.0
    while True:
        best_i, best_g = -1, -1e-12
        for i in range(n):
            if not clamped[i] and gains[i] < best_g:
                best_i, best_g = i, float(gains[i])
        if best_i < 0:
            return total
        total -= best_g
        dirn = 1.0 - 2.0 * float(state[best_i])
        state[best_i] = 1 - state[best_i]
        gains[best_i] = -best_g
        for k in range(ro[best_i], ro[best_i + 1]):
            j = ci[k]
            gains[j] += (1.0 - 2.0 * float(state[j])) * float(va[k]) * dirn


def luby(i: int) -> int:
    """The Luby sequence 1, 1, 2, 1, 1, 2, 4, ... (src/solver/tts.rs:95-112),
    1-indexed."""
    if i < 1:
        raise ValueError("luby is 1-indexed")
    while True:
        k = i.bit_length()  # 2^(k-1) <= i <= 2^k - 1
        if i == (1 << k) - 1:
            return 1 << (k - 1)
        i -= (1 << (k - 1)) - 1


def steepest_descent_2opt_escapes(model: QuboModel, state, is_clamped=None) -> float:
    """local_search.rs:123-143 (the library's host code): polishes ``state``
    (contiguous int8 0/1) in place to a 1-opt minimum with no improving 2-flip
    along a coupling; returns the improvement."""
    if not (isinstance(state, np.ndarray) and state.dtype == np.int8 and state.flags.c_contiguous):
        raise TypeError("state must be a contiguous int8 array")
    keep: list = []
    prob = _problem(model, keep)
    c = None if is_clamped is None else np.ascontiguousarray(is_clamped, dtype=np.uint8)
    imp = C.c_double()
    _ffi.check(_ffi.lib().ie_two_opt(C.byref(prob), _p(state), None if c is None else _p(c), C.byref(imp)))
    return imp.value


def path_relink_finish(model: QuboModel, words, state, is_clamped=None) -> float:
    """ultimate.rs:436-479 (the library's host code): an elite archive of
    ``state`` and every replica of the field ``words`` [cells, n] (bit r =
    replica r, as ``Engine.spins`` returns them), greedy path relinking of
    every elite pair, each polished by 1-opt; the best state replaces
    ``state`` (contiguous int8) when strictly better. Returns its energy."""
    if not (isinstance(state, np.ndarray) and state.dtype == np.int8 and state.flags.c_contiguous):
        raise TypeError("state must be a contiguous int8 array")
    keep: list = []
    prob = _problem(model, keep)
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
    c = None if is_clamped is None else np.ascontiguousarray(is_clamped, dtype=np.uint8)
    e = C.c_double()
    _ffi.check(_ffi.lib().ie_path_relink(C.byref(prob), _p(w), w.size // max(model.num_vars, 1),
                                         None if c is None else _p(c), _p(state), C.byref(e)))
    return e.value


class UltimateSolver:
    """Configuration of the reference's UltimateSolver (ultimate.rs:18-87):
    the PT path (num_pops = 1) and population annealing with PT
    equilibration (num_pops > 1, ultimate.rs:576-852); num_slices = 1."""

    def __init__(self, temp_max: float, temp_min: float, sweeps: int, exchanges: int,
                 seed: int | None, num_temps: int = 10, exchange_interval: int = 1,
                 device: int = 0):
        self.num_replicas = NUM_REPLICAS
        self.temp_max = float(temp_max)
        self.temp_min = float(temp_min)
        self.sweeps_per_exchange = int(sweeps)
        self.total_exchanges = int(exchanges)
        self.seed = int(np.random.SeedSequence().entropy % (1 << 64)) if seed is None else int(seed)
        self.num_slices = 1
        self.num_temps = int(num_temps)
        self.num_pops = 1
        self.exchange_interval = int(exchange_interval)
        self.device = device
        # population-annealing knobs (ultimate.rs:29-52, defaults :77-86)
        self.ess_threshold = 0.5
        self.ladder_tuning_iters = 8
        self.ladder_tuning_steps = 10
        self.post_resample_relaxation = 5
        self.ladder_mode = 0  # 0 acceptance-uniform, 1 feedback-optimized (LadderMode)
        self.use_icm = False  # isoenergetic cluster moves after every exchange block / stage
        self.use_2opt = False  # edge-restricted 2-opt escapes after the 1-opt polish
        self.use_path_relinking = False  # elite path relinking after the polish (PT path)
        self.gnn_heuristic_probs = None  # warm-start probabilities per variable
        # presolve and decomposition before annealing (ultimate.rs:161-218); an
        # extension may switch them off, e.g. where probing's O(n^2 nnz) cost
        # is too high
        self.use_presolve = True

    @staticmethod
    def new(temp_max, temp_min, sweeps, exchanges, seed):
        return UltimateSolver(temp_max, temp_min, sweeps, exchanges, seed)

    def with_quantum_dims(self, slices: int, temps: int, pops: int) -> "UltimateSolver":
        """ultimate.rs:126-131."""
        if slices != 1:
            raise NotImplementedError("only num_slices = 1 is on the device path")
        self.num_temps = int(temps)
        self.num_pops = int(pops)
        return self

    def with_gnn_heuristic(self, probs) -> "UltimateSolver":
        """ultimate.rs:121-124: the initial replicas are drawn with P(x_v = 1) = probs[v]."""
        self.gnn_heuristic_probs = np.asarray(probs, dtype=np.float64).copy()
        return self

    def with_2opt(self, enabled: bool) -> "UltimateSolver":
        """ultimate.rs:133-136."""
        self.use_2opt = bool(enabled)
        return self

    def pa_config(self):
        from .population_annealing import PaConfig
        return PaConfig(self.ess_threshold, self.ladder_tuning_iters, self.ladder_tuning_steps,
                        self.post_resample_relaxation, self.ladder_mode, self.use_icm)

    def engine(self, model: QuboModel, num_pops: int | None = None) -> Engine:
        eng = Engine(model, num_temps=self.num_temps, seed=self.seed,
                     exchange_interval=self.exchange_interval, temp_max=self.temp_max,
                     temp_min=self.temp_min, sweeps_per_exchange=self.sweeps_per_exchange,
                     total_exchanges=self.total_exchanges, device=self.device,
                     num_pops=self.num_pops if num_pops is None else num_pops, use_icm=self.use_icm)
        if self.gnn_heuristic_probs is not None:
            eng.set_init_probs(self.gnn_heuristic_probs)
        return eng

    def _clamps(self, model: QuboModel, clamped):
        n = model.num_vars
        is_clamped = np.zeros(n, dtype=np.uint8)
        cval = np.zeros(n, dtype=np.int8)
        for idx, val in clamped:
            is_clamped[idx] = 1
            cval[idx] = val
        return is_clamped, cval

    def solve_with_luby_restarts(self, model: QuboModel, clamped=(), num_restarts: int = 1) -> np.ndarray:
        """ultimate.rs:95-120: restart i (0-based) solves with total_exchanges *
        luby(i + 1) exchanges and seed + 0x9e3779b97f4a7c15 * (i + 1) (mod 2^64);
        the first state of lowest true energy wins."""
        best_e, best = None, None
        for i in range(max(int(num_restarts), 1)):
            r = copy.copy(self)
            r.total_exchanges = self.total_exchanges * luby(i + 1)
            r.seed = (self.seed + 0x9E3779B97F4A7C15 * (i + 1)) & 0xFFFFFFFFFFFFFFFF
            x = r.solve(model, clamped)
            e = model.calculate_total_energy(x)
            if best_e is None or e < best_e:
                best_e, best = e, x
        return best

    def solve_with_pa_diagnostics(self, model: QuboModel, clamped=()):
        """ultimate.rs:858-890: population annealing with num_pops >= 2 (no
        presolve), then best extraction and 1-opt (ultimate.rs:806-845);
        returns (state, PaDiagnostics)."""
        return self._solve_pa(model, clamped)

    def _solve_pa(self, model: QuboModel, clamped):
        is_clamped, cval = self._clamps(model, clamped)
        with self.engine(model, num_pops=max(self.num_pops, 2)) as eng:
            if len(clamped):
                eng.set_clamps(is_clamped, cval)
            diag = eng.run_pa(self.pa_config())
            _, best = eng.best()
            eng.one_opt(best, is_clamped)
        if self.use_2opt:
            steepest_descent_2opt_escapes(model, best, is_clamped)
        return best, diag

    def solve(self, model: QuboModel, clamped=()) -> np.ndarray:
        """UltimateSolver::solve (ultimate.rs:138-387) for `model` with
        `clamped` fixings: presolve fixings join the clamps; a free-variable
        graph of several components is solved component by component (seed +
        index + 1, ultimate.rs:173-218); otherwise the PT path, or population
        annealing when num_pops > 1 (ultimate.rs:220-232)."""
        clamped = [(int(i), int(v)) for i, v in clamped]
        if self.use_presolve:
            from .presolve import connected_components, extract_component, full_presolve
            clamped = clamped + full_presolve(model, clamped)
            is_clamped, cval = self._clamps(model, clamped)
            comps = connected_components(model, is_clamped == 0)
            if len(comps) > 1:
                result = np.where(is_clamped != 0, cval, 0).astype(np.int8)
                fixed_one = (is_clamped != 0) & (cval == 1)
                for ci, comp in enumerate(comps):
                    sub, gmap = extract_component(model, comp, fixed_one)
                    child = copy.copy(self)
                    child.seed = (self.seed + ci + 1) & 0xFFFFFFFFFFFFFFFF
                    if self.gnn_heuristic_probs is not None:  # ultimate.rs:200-203
                        child.gnn_heuristic_probs = self.gnn_heuristic_probs[gmap]
                    result[gmap] = child.solve(sub)
                return result
        if self.num_pops > 1:
            return self._solve_pa(model, clamped)[0]
        is_clamped, cval = self._clamps(model, clamped)
        with self.engine(model) as eng:
            if len(clamped):
                eng.set_clamps(is_clamped, cval)
            eng.init_random()
            eng.run_pt()
            _, best = eng.best()
            eng.one_opt(best, is_clamped)
            words = eng.spins() if self.use_path_relinking else None
        if self.use_2opt:
            steepest_descent_2opt_escapes(model, best, is_clamped)
        if self.use_path_relinking:  # ultimate.rs:382-385
            path_relink_finish(model, words, best, is_clamped)
        return best

"""Device engines behind the C ABI.

``Engine`` is one problem with ``num_temps`` cells of 64 replicas: the device
counterpart of the reference's ``QuantumField`` + ``StepScratch`` + master
``ChaCha8Rng`` of one solve (src/solver/types.rs:17-58,
src/solver/engine.rs:454-557, src/solver/ultimate.rs:152). ``Engine.step`` is
``engine::step`` (engine.rs:573-819).

``BatchEngine`` is many single-cell problems run together by one persistent
kernel (and, for comparison, one launch per problem: the plain method).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from .core import QuboModel

NUM_REPLICAS = 64


def _problem(model: QuboModel, keep: list) -> _ffi.ie_problem:
    lin = np.ascontiguousarray(model.linear, dtype=np.float64)
    ro = np.ascontiguousarray(model.row_offsets, dtype=np.uint64)
    ci = np.ascontiguousarray(model.col_indices, dtype=np.uint64)
    va = np.ascontiguousarray(model.values, dtype=np.float64)
    keep.extend([lin, ro, ci, va])
    return _ffi.ie_problem(model.num_vars, lin.ctypes.data, ro.ctypes.data, ci.ctypes.data,
                           va.ctypes.data, float(model.energy_offset))


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Engine:
    """One problem, ``num_temps`` x ``num_pops`` cells x 64 replicas, resident
    on the device (cell t + num_temps * p)."""

    def __init__(self, model: QuboModel, num_temps: int = 10, seed: int = 0,
                 exchange_interval: int = 1, temp_max: float = 1.0, temp_min: float = 0.1,
                 sweeps_per_exchange: int = 1, total_exchanges: int = 1, force_f64: bool = False,
                 device: int = 0, pt_path: int = 0, num_pops: int = 1, use_icm: bool = False,
                 kernel_form: int = 0, max_cluster: int = 0, bit_sliced: int = 0):
        self._L = _ffi.lib()
        self.model = model
        self.num_temps = int(num_temps)
        self.num_pops = int(num_pops)
        self.cells = self.num_temps * self.num_pops  # cell t + num_temps * p
        self.n = model.num_vars
        keep: list = []
        prob = _problem(model, keep)
        cfg = _ffi.ie_config(temp_max, temp_min, sweeps_per_exchange, total_exchanges,
                             seed & 0xFFFFFFFFFFFFFFFF, self.num_temps, self.num_pops, 1, exchange_interval,
                             int(force_f64), device, pt_path, int(use_icm), int(kernel_form),
                             int(max_cluster), int(bit_sliced))
        h = C.c_void_p()
        _ffi.check(self._L.ie_create(C.byref(prob), C.byref(cfg), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.ie_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_clamps(self, is_clamped, clamp_val=None) -> None:
        if is_clamped is None:
            _ffi.check(self._L.ie_set_clamps(self._h, None, None))
            return
        f = np.ascontiguousarray(is_clamped, dtype=np.uint8)
        v = np.ascontiguousarray(np.zeros(self.n) if clamp_val is None else clamp_val, dtype=np.int8)
        _ffi.check(self._L.ie_set_clamps(self._h, _p(f), _p(v)))

    def set_init_probs(self, probs) -> None:
        """Warm start (ultimate.rs:121-124, 256-263): later inits draw replica
        r of site v as one with probability probs[v]; None: random init."""
        if probs is None:
            _ffi.check(self._L.ie_set_init_probs(self._h, None))
            return
        p = np.ascontiguousarray(probs, dtype=np.float64)
        if p.shape != (self.n,):
            raise ValueError("probs must have num_vars entries")
        _ffi.check(self._L.ie_set_init_probs(self._h, _p(p)))

    def init_random(self) -> None:
        _ffi.check(self._L.ie_init_random(self._h))

    def set_spins(self, words) -> None:
        w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
        if w.size != self.cells * self.n:
            raise ValueError("words must have num_temps * num_pops * num_vars entries")
        _ffi.check(self._L.ie_set_spins(self._h, _p(w)))

    def step(self, temps, n_steps: int = 1) -> None:
        t = np.ascontiguousarray(temps, dtype=np.float64).reshape(-1)
        _ffi.check(self._L.ie_step(self._h, _p(t), len(t), int(n_steps)))

    def run_schedule(self, temps) -> None:
        t = np.ascontiguousarray(temps, dtype=np.float64)
        if t.ndim == 1:
            t = t[:, None]
        _ffi.check(self._L.ie_run_schedule(self._h, _p(t), t.shape[1], t.shape[0]))

    def run_pt(self) -> None:
        _ffi.check(self._L.ie_run_pt(self._h))

    def run_pa(self, config=None):
        """Population annealing with PT equilibration (ultimate.rs:576-852) on a
        handle with num_pops > 1, from a fresh master stream; returns the
        ``PaDiagnostics``. ``best`` and ``one_opt`` finish the solve."""
        from .population_annealing import PaConfig, PaDiagnostics
        cfg = (config or PaConfig()).to_c()
        cap = 1 << 16
        ess = np.zeros(cap, dtype=np.float64)
        rho = np.zeros(cap, dtype=np.float64)
        fam = np.zeros(cap, dtype=np.uint64)
        alphas = np.zeros(self.num_temps, dtype=np.float64)
        rep = _ffi.ie_pa_report(0.0, 0, 0, ess.ctypes.data, rho.ctypes.data, fam.ctypes.data, cap,
                                alphas.ctypes.data)
        _ffi.check(self._L.ie_run_pa(self._h, C.byref(cfg), C.byref(rep)))
        ne = min(int(rep.n_ess), cap)
        nr = min(int(rep.resample_events), cap)
        return PaDiagnostics(rep.free_energy, ess[:ne].tolist(),
                             [(float(rho[i]), int(fam[i])) for i in range(nr)], int(rep.resample_events), alphas)

    def spins(self) -> np.ndarray:
        w = np.zeros((self.cells, self.n), dtype=np.uint64)
        _ffi.check(self._L.ie_read_spins(self._h, _p(w)))
        return w

    def energies(self) -> np.ndarray:
        e = np.zeros((self.cells, NUM_REPLICAS), dtype=np.float64)
        _ffi.check(self._L.ie_read_energies(self._h, _p(e)))
        return e

    def swap_stats(self):
        k = max(self.num_temps - 1, 1)
        a = np.zeros(k, dtype=np.uint64)
        b = np.zeros(k, dtype=np.uint64)
        _ffi.check(self._L.ie_read_swap_stats(self._h, _p(a), _p(b)))
        return a[: self.num_temps - 1], b[: self.num_temps - 1]

    def swap_acceptance_rates(self) -> np.ndarray:
        a, b = self.swap_stats()
        return np.where(a == 0, 0.0, b / np.maximum(a, 1))

    def rng_state(self):
        d = np.zeros(1, dtype=np.uint64)
        p = np.zeros(1, dtype=np.int32)
        _ffi.check(self._L.ie_read_rng_state(self._h, _p(d), _p(p)))
        return int(d[0]), int(p[0])

    def save_state(self) -> bytes:
        """The device state as one blob (spins, energies, swap statistics,
        stream position, DEO phase, steps run, incumbent)."""
        n = C.c_uint64()
        _ffi.check(self._L.ie_state_size(self._h, C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        _ffi.check(self._L.ie_save_state(self._h, buf, n.value))
        return bytes(buf)

    def load_state(self, blob: bytes) -> None:
        """Restores a blob of save_state into this handle (same problem and
        config); the run continues as the saved one would have."""
        buf = (C.c_uint8 * len(blob)).from_buffer_copy(blob)
        _ffi.check(self._L.ie_load_state(self._h, buf, len(blob)))

    def digest(self) -> int:
        """FNV-1a over the spin words in the reference layout (state.rs:60-67)."""
        d = C.c_uint64()
        _ffi.check(self._L.ie_state_digest(self._h, C.byref(d)))
        return d.value

    def incumbent(self):
        e = np.zeros(1, dtype=np.float64)
        s = np.zeros(self.n, dtype=np.int8)
        _ffi.check(self._L.ie_read_incumbent(self._h, _p(e), _p(s)))
        return float(e[0]), s

    def best(self):
        e = np.zeros(1, dtype=np.float64)
        s = np.zeros(self.n, dtype=np.int8)
        _ffi.check(self._L.ie_read_best(self._h, _p(e), _p(s)))
        return float(e[0]), s

    def one_opt(self, state, is_clamped=None) -> float:
        """local_search.rs:19-57 on the device: polishes ``state`` (int8 0/1)
        in place; returns the total improvement."""
        if not (isinstance(state, np.ndarray) and state.dtype == np.int8 and state.flags.c_contiguous):
            raise TypeError("state must be a contiguous int8 array")
        c = None if is_clamped is None else np.ascontiguousarray(is_clamped, dtype=np.uint8)
        imp = np.zeros(1, dtype=np.float64)
        _ffi.check(self._L.ie_one_opt(self._h, _p(state), None if c is None else _p(c), _p(imp)))
        return float(imp[0])


class BatchEngine:
    """Many single-cell problems (64 replicas each) resident on the device."""

    def __init__(self, models, seeds, device: int = 0, force_f64: bool = False,
                 threads_per_block: int = 0, blocks_per_sm: int = 0, windows: bool = True,
                 graph: bool = False, kernel_form: int = 0, item_sites: int = 0, tie_shift: int = 0,
                 bit_sliced: int = 0, bulk_ring: bool = False):
        self._L = _ffi.lib()
        self.kernel_form = int(kernel_form)
        self.models = list(models)
        self.count = len(self.models)
        keep: list = []
        probs = (_ffi.ie_problem * self.count)(*[_problem(m, keep) for m in self.models])
        self.seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        if self.seeds.shape != (self.count,):
            raise ValueError("one seed per problem")
        cfg = _ffi.ie_batch_config(device, int(force_f64), threads_per_block, blocks_per_sm,
                                   0 if windows else 1, 1 if graph else 0, int(kernel_form),
                                   int(item_sites), int(tie_shift), int(bit_sliced), int(bool(bulk_ring)))
        h = C.c_void_p()
        _ffi.check(self._L.ie_batch_create(probs, self.count, _p(self.seeds), C.byref(cfg),
                                           C.byref(h)))
        self._h = h
        self.ns = np.array([m.num_vars for m in self.models], dtype=np.int64)
        self.offsets = np.zeros(self.count + 1, dtype=np.int64)
        self.offsets[1:] = np.cumsum(self.ns)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.ie_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_random(self) -> None:
        _ffi.check(self._L.ie_batch_init_random(self._h))

    def run_schedule(self, temps) -> float:
        """Runs temps[steps] on every problem; returns device milliseconds."""
        t = np.ascontiguousarray(temps, dtype=np.float64).reshape(-1)
        _ffi.check(self._L.ie_batch_run_schedule(self._h, _p(t), len(t)))
        return self.last_ms()

    def autotune(self, temps, trial_steps: int = 16):
        """Chooses the launch shape by timing short trials of the schedule
        (state restored after each). Level kernel: returns (item_sites,
        threads, 0, 0); per-lane kernels: (n4_int, n2_int, n4_f64, n2_f64)."""
        t = np.ascontiguousarray(temps, dtype=np.float64).reshape(-1)
        out = np.zeros(4, dtype=np.uint32)
        _ffi.check(self._L.ie_batch_autotune(self._h, _p(t), min(int(trial_steps), len(t)), _p(out)))
        return tuple(int(x) for x in out)

    def run_schedule_plain(self, temps, first: int = 0, count: int | None = None) -> float:
        t = np.ascontiguousarray(temps, dtype=np.float64).reshape(-1)
        count = self.count - first if count is None else count
        _ffi.check(self._L.ie_batch_run_schedule_plain(self._h, _p(t), len(t), first, count))
        return self.last_ms()

    def spins(self) -> np.ndarray:
        w = np.zeros(int(self.offsets[-1]), dtype=np.uint64)
        _ffi.check(self._L.ie_batch_read_spins(self._h, _p(w)))
        return w

    def spins_of(self, words: np.ndarray, i: int) -> np.ndarray:
        return words[self.offsets[i]:self.offsets[i + 1]]

    def energies(self) -> np.ndarray:
        e = np.zeros((self.count, NUM_REPLICAS), dtype=np.float64)
        _ffi.check(self._L.ie_batch_read_energies(self._h, _p(e)))
        return e

    def recompute_energies(self) -> np.ndarray:
        e = np.zeros((self.count, NUM_REPLICAS), dtype=np.float64)
        _ffi.check(self._L.ie_batch_recompute_energies(self._h, _p(e)))
        return e

    def draws(self) -> np.ndarray:
        d = np.zeros(self.count, dtype=np.uint64)
        _ffi.check(self._L.ie_batch_read_draws(self._h, _p(d)))
        return d

    def last_ms(self) -> float:
        ms = np.zeros(1, dtype=np.float64)
        _ffi.check(self._L.ie_batch_last_run_ms(self._h, _p(ms)))
        return float(ms[0])

    def class_report(self):
        """Per work class of the last run: (mode, threads per lane, capacity,
        items, device ms); threads per lane 8 marks the windowed kernel, 16 the
        chain kernel, 32 the level kernel (mode "pmj": its bit-sliced +-J
        form; capacity 0: spins in global memory)."""
        n = np.zeros(1, dtype=np.uint32)
        info = np.zeros(5 * 64, dtype=np.uint32)
        ms = np.zeros(64, dtype=np.float64)
        _ffi.check(self._L.ie_batch_class_report(self._h, 64, _p(n), _p(info), _p(ms)))
        k = int(min(n[0], 64))
        return [(("int", "f64", "pmj")[info[5 * i]], int(info[5 * i + 1]), int(info[5 * i + 2]),
                 int(info[5 * i + 3]), float(ms[i])) for i in range(k)]

    def last_launches(self) -> int:
        n = np.zeros(1, dtype=np.uint64)
        _ffi.check(self._L.ie_batch_last_launches(self._h, _p(n)))
        return int(n[0])

    def exact_decisions(self) -> int:
        """Level-kernel decisions taken on the exact path so far."""
        n = np.zeros(1, dtype=np.uint64)
        _ffi.check(self._L.ie_batch_exact_decisions(self._h, _p(n)))
        return int(n[0])


def geometric_temps(temp_max: float, temp_min: float, num_temps: int) -> np.ndarray:
    """ultimate.rs:238-246 (pow then powi), computed by the library."""
    out = np.zeros(num_temps, dtype=np.float64)
    _ffi.check(_ffi.lib().ie_geometric_temps(temp_max, temp_min, num_temps, _p(out)))
    return out


def suggested_temp_range(model: QuboModel):
    """src/solver/schedule.rs:21-43, computed by the library."""
    keep: list = []
    prob = _problem(model, keep)
    a = C.c_double()
    b = C.c_double()
    _ffi.check(_ffi.lib().ie_suggested_temp_range(C.byref(prob), C.byref(a), C.byref(b)))
    return a.value, b.value

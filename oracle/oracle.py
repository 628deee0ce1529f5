"""ctypes wrapper over the CPU oracle (oracle/ie_oracle.cpp).

Test infrastructure only: imported by tests/, by ``__graft_entry__.smoke()`` as
the checker, and by ``bench.py``'s CPU-baseline / ``--impl reference`` leg. The
product package never imports it.

The oracle restates the reference's S1 path (src/solver/engine.rs,
src/solver/ultimate.rs, src/presolve/*, src/solver/local_search.rs) and the
third-party master RNG (rand_chacha 0.3.1 ChaCha8Rng with rand_core 0.6.4
seed_from_u64 and rand 0.8.5 sampling). It is pinned by the reference's
end-to-end golden (tests/test_regression_golden.rs:87-111).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libieoracle.so")
_lib = None

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compiles the oracle shared library with its Makefile; returns its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "ie_oracle.cpp"))
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_chacha8_u64.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _u64p]
        L.or_chacha8_block.argtypes = [_u32p, C.c_uint64, _u32p]
        L.or_xoshiro_x8_f64.argtypes = [C.c_uint64, C.c_uint64, _f64p]
        L.or_fast_exp.argtypes = [C.c_double]
        L.or_fast_exp.restype = C.c_double
        L.or_geometric_temps.argtypes = [C.c_double, C.c_double, C.c_int, _f64p]
        L.or_golden_instance.argtypes = [_i64p, _i64p, _f64p, _f64p]
        L.or_total_energy.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_double, _i8p]
        L.or_total_energy.restype = C.c_double
        L.or_solve.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_double, C.c_double,
                               C.c_double, C.c_int64, C.c_int64, C.c_uint64, C.c_int, _i64p, _i8p,
                               C.c_int64, C.c_int, _i8p, C.c_int]
        L.or_full_presolve.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, _i64p, _i8p,
                                       C.c_int64, _i64p, _i8p]
        L.or_full_presolve.restype = C.c_int64
        L.or_one_opt.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, _i8p, _u8p]
        L.or_one_opt.restype = C.c_double
        L.or_two_opt.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_double, _i8p, _u8p]
        L.or_two_opt.restype = C.c_double
        L.or_warm_start_words.argtypes = [C.c_uint64, C.c_uint64, _f64p, _u8p, _i8p, C.c_int64, C.c_int, _u64p]
        L.or_warm_start_words.restype = C.c_uint64
        L.or_path_relink.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_double, _u64p, C.c_int64, _u8p,
                                     _i8p]
        L.or_path_relink.restype = C.c_double
        L.or_run_schedule.argtypes = [
            C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_int, _f64p, C.c_int64, C.c_uint64,
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int64, C.c_int,
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
            C.c_void_p, C.c_void_p, C.c_int64]
        L.or_replica_energies.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_int, _u64p,
                                          _f64p]
        L.or_run_sa_batch.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                      C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_v2_program.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_double, C.c_int64, _u8p,
                                    C.c_uint64, C.c_uint64, C.c_int64, C.c_void_p, _i64p, _f64p, C.c_int32,
                                    _u64p, _f64p, _i64p, _f64p, _u64p]
        L.or_pa_run.argtypes = [
            C.c_int64, _f64p, _i64p, _i64p, _f64p, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int64,
            C.c_uint64, C.c_int, C.c_int, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int,
            C.c_void_p, C.c_void_p, C.c_int, _u64p, _f64p, _u64p, _f64p, _f64p, _i64p, _f64p, _i64p, _i64p, _f64p, _i8p, _f64p, _i8p]
        L.or_pa_normalized_weights.argtypes = [_f64p, C.c_int64, _f64p]
        L.or_pa_systematic_resample.argtypes = [_f64p, C.c_int64, C.c_double, _i64p]
        L.or_pa_feedback_alphas.argtypes = [_f64p, _f64p, C.c_int64, C.c_double, _f64p]
        L.or_gen_index_inclusive.argtypes = [C.c_uint64, _u64p, C.c_int64, _u64p, _u64p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _csr(model):
    """(n, linear, row, col, val) as contiguous numpy arrays from a model-like
    object with attributes num_vars, linear, row_offsets, col_indices, values."""
    return (int(model.num_vars),
            np.ascontiguousarray(model.linear, dtype=np.float64),
            np.ascontiguousarray(model.row_offsets, dtype=np.int64),
            np.ascontiguousarray(model.col_indices, dtype=np.int64),
            np.ascontiguousarray(model.values, dtype=np.float64))


def chacha8_u64(seed: int, count: int, skip: int = 0) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    lib().or_chacha8_u64(seed, skip, count, out)
    return out


def chacha8_block(key, counter: int) -> np.ndarray:
    out = np.zeros(16, dtype=np.uint32)
    lib().or_chacha8_block(np.ascontiguousarray(key, dtype=np.uint32), counter, out)
    return out


def xoshiro_x8_f64(seed: int, calls: int) -> np.ndarray:
    out = np.zeros(8 * calls, dtype=np.float64)
    lib().or_xoshiro_x8_f64(seed, calls, out)
    return out


def fast_exp(x: float) -> float:
    return lib().or_fast_exp(x)


def geometric_temps(tmax: float, tmin: float, nt: int) -> np.ndarray:
    out = np.zeros(nt, dtype=np.float64)
    lib().or_geometric_temps(tmax, tmin, nt, out)
    return out


def golden_instance():
    """The seeded n=32 instance of tests/test_regression_golden.rs:25-57 as
    (linear, row_offsets, col_indices, values)."""
    row = np.zeros(33, dtype=np.int64)
    col = np.zeros(992, dtype=np.int64)
    val = np.zeros(992, dtype=np.float64)
    lin = np.zeros(32, dtype=np.float64)
    lib().or_golden_instance(row, col, val, lin)
    return lin, row, col, val


def total_energy(model, state, offset: float = 0.0) -> float:
    n, lin, row, col, val = _csr(model)
    return lib().or_total_energy(n, lin, row, col, val, offset,
                                 np.ascontiguousarray(state, dtype=np.int8))


def solve(model, temp_max, temp_min, sweeps, exchanges, seed, num_temps=10, clamped=(),
          threads=1, offset=0.0, use_icm=False) -> np.ndarray:
    """UltimateSolver::new(temp_max, temp_min, sweeps, exchanges, Some(seed))
    with num_temps, then .solve(model, clamped) (ultimate.rs:60-87, 138-387)."""
    n, lin, row, col, val = _csr(model)
    ci = np.array([c[0] for c in clamped], dtype=np.int64)
    cv = np.array([c[1] for c in clamped], dtype=np.int8)
    out = np.zeros(n, dtype=np.int8)
    lib().or_solve(n, lin, row, col, val, offset, temp_max, temp_min, sweeps, exchanges, seed,
                   num_temps, ci, cv, len(clamped), threads, out, int(use_icm))
    return out


def full_presolve(model, clamped=()):
    n, lin, row, col, val = _csr(model)
    ci = np.array([c[0] for c in clamped], dtype=np.int64)
    cv = np.array([c[1] for c in clamped], dtype=np.int8)
    oi = np.zeros(n, dtype=np.int64)
    ov = np.zeros(n, dtype=np.int8)
    k = lib().or_full_presolve(n, lin, row, col, val, ci, cv, len(clamped), oi, ov)
    return [(int(oi[i]), int(ov[i])) for i in range(k)]


def one_opt(model, state, is_clamped=None, with_improvement=False):
    """local_search.rs:19-57 on a copy of state; returns the polished state
    (and the total improvement when asked)."""
    n, lin, row, col, val = _csr(model)
    st = np.ascontiguousarray(state, dtype=np.int8).copy()
    cl = np.zeros(n, dtype=np.uint8) if is_clamped is None else \
        np.ascontiguousarray(is_clamped, dtype=np.uint8)
    imp = lib().or_one_opt(n, lin, row, col, val, st, cl)
    return (st, imp) if with_improvement else st


class RunResult:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def run_schedule(model, temps, seed, init_words=None, clamped=None, clamp_val=None,
                 exchange_interval=1, collect_stats=False, incumbent_every=0, threads=1,
                 want_base_seeds=False, icm_every=0) -> RunResult:
    """The step loop of ultimate.rs:248-336 under temps[steps][nt]."""
    n, lin, row, col, val = _csr(model)
    temps = np.ascontiguousarray(temps, dtype=np.float64)
    if temps.ndim == 1:
        temps = temps[:, None]
    steps, nt = temps.shape
    words = np.zeros((nt, n), dtype=np.uint64)
    en = np.zeros((nt, 64), dtype=np.float64)
    att = np.zeros(max(nt - 1, 1), dtype=np.uint64)
    acc = np.zeros(max(nt - 1, 1), dtype=np.uint64)
    draws = np.zeros(1, dtype=np.uint64)
    bs = np.zeros(steps, dtype=np.uint64) if want_base_seeds else None
    inc_e = np.zeros(1, dtype=np.float64)
    inc_s = np.zeros(n, dtype=np.int8)
    iw = None if init_words is None else np.ascontiguousarray(init_words, dtype=np.uint64)
    cl = None if clamped is None else np.ascontiguousarray(clamped, dtype=np.uint8)
    cv = None if clamp_val is None else np.ascontiguousarray(clamp_val, dtype=np.int8)
    lib().or_run_schedule(n, lin, row, col, val, nt, temps.reshape(-1), steps, seed, _ptr(iw),
                          _ptr(cl), _ptr(cv), exchange_interval, int(collect_stats),
                          incumbent_every, threads, _ptr(words), _ptr(en), _ptr(att), _ptr(acc),
                          _ptr(draws), _ptr(bs), _ptr(inc_e), _ptr(inc_s), int(icm_every))
    return RunResult(words=words, energies=en, swap_attempts=att[:nt - 1],
                     swap_accepts=acc[:nt - 1], draws=int(draws[0]), base_seeds=bs,
                     incumbent_energy=float(inc_e[0]), incumbent_state=inc_s)


def replica_energies(model, words) -> np.ndarray:
    n, lin, row, col, val = _csr(model)
    words = np.ascontiguousarray(words, dtype=np.uint64)
    cells = words.size // max(n, 1)
    out = np.zeros((cells, 64), dtype=np.float64)
    lib().or_replica_energies(n, lin, row, col, val, cells, words.reshape(-1), out)
    return out


def run_sa_batch(models, seeds, temps, threads=1, want_words=True):
    """Independent single-cell SA runs (temps[steps], one temperature per step)
    over many instances, parallel over instances."""
    count = len(models)
    keep = []
    arrs = [_csr(m) for m in models]
    ns = np.array([a[0] for a in arrs], dtype=np.int64)

    def ptrs(idx):
        p = (C.c_void_p * count)(*[a[idx].ctypes.data for a in arrs])
        keep.append(p)
        return C.cast(p, C.c_void_p)

    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    temps = np.ascontiguousarray(temps, dtype=np.float64)
    off = np.zeros(count, dtype=np.int64)
    off[1:] = np.cumsum(ns)[:-1]
    words = np.zeros(int(ns.sum()), dtype=np.uint64) if want_words else None
    en = np.zeros((count, 64), dtype=np.float64)
    lib().or_run_sa_batch(count, ns.ctypes.data_as(C.c_void_p), ptrs(1), ptrs(2), ptrs(3),
                          ptrs(4), seeds.ctypes.data_as(C.c_void_p),
                          temps.ctypes.data_as(C.c_void_p), len(temps), threads, _ptr(words),
                          off.ctypes.data_as(C.c_void_p), en.ctypes.data_as(C.c_void_p))
    return words, off, en


def v2_program(model, r, init, seed, ops, temps, skip_draws=0):
    """S2 operators on one bit-sliced state with one master stream: ops is a
    list of ("metropolis", sweeps) / ("exchange", rounds) / ("gibbs", sweeps), all at per-replica
    temperatures temps (replica k uses temps[k % len]). Returns (planes
    [n, ceil(r/64)], energies [r], [(proposed, accepted)] per op, ledger drift,
    stream position)."""
    n, lin, row, col, val = _csr(model)
    w = (r + 63) // 64
    kinds = np.array([{"metropolis": 0, "exchange": 1, "gibbs": 2}[k] for k, _ in ops], dtype=np.int32)
    counts = np.array([c for _, c in ops], dtype=np.int64)
    temps = np.ascontiguousarray(temps, dtype=np.float64)
    planes = np.zeros(n * w, dtype=np.uint64)
    en = np.zeros(r, dtype=np.float64)
    stats = np.zeros(2 * max(len(ops), 1), dtype=np.int64)
    drift = np.zeros(1, dtype=np.float64)
    draws = np.zeros(1, dtype=np.uint64)
    lib().or_v2_program(n, lin, row, col, val, float(model.energy_offset), r,
                        np.ascontiguousarray(init, dtype=np.uint8), seed, skip_draws, len(ops),
                        kinds.ctypes.data_as(C.c_void_p), counts, temps, len(temps), planes, en, stats,
                        drift, draws)
    return (planes.reshape(n, w), en, [(int(stats[2 * i]), int(stats[2 * i + 1])) for i in range(len(ops))],
            float(drift[0]), int(draws[0]))


def pa_run(model, temp_max, temp_min, sweeps, exchanges, seed, num_temps, num_pops, ess_threshold=0.5,
           tuning_iters=8, tuning_steps=10, relax=5, clamped=None, clamp_val=None, threads=1, offset=0.0,
           ladder_mode=0, use_icm=False):
    """UltimateSolver::new(temp_max, temp_min, sweeps, exchanges, Some(seed)) with
    num_temps, num_pops and the PA knobs, through solve_with_pa_diagnostics
    (ultimate.rs:576-890). Returns a dict: words [nt*pops, n], energies
    [nt*pops, 64], draws, alphas, ess, rho, families, free_energy, resamples,
    best_pre (before 1-opt), incumbent, state."""
    n, lin, row, col, val = _csr(model)
    cells = num_temps * num_pops
    words = np.zeros(cells * n, dtype=np.uint64)
    en = np.zeros(cells * 64, dtype=np.float64)
    draws = np.zeros(1, dtype=np.uint64)
    alphas = np.zeros(num_temps, dtype=np.float64)
    k = max(exchanges, 1)
    ess = np.zeros(k, dtype=np.float64)
    n_ess = np.zeros(1, dtype=np.int64)
    rho = np.zeros(k, dtype=np.float64)
    fam = np.zeros(k, dtype=np.int64)
    n_res = np.zeros(1, dtype=np.int64)
    fe = np.zeros(1, dtype=np.float64)
    best_pre = np.zeros(n, dtype=np.int8)
    inc = np.zeros(1, dtype=np.float64)
    state = np.zeros(n, dtype=np.int8)
    cl = None if clamped is None else np.ascontiguousarray(clamped, dtype=np.uint8)
    cv = None if clamp_val is None else np.ascontiguousarray(clamp_val, dtype=np.int8)
    L = lib()
    L.or_pa_run(n, lin, row, col, val, float(offset), float(temp_max), float(temp_min), int(sweeps), int(exchanges),
                int(seed), int(num_temps), int(num_pops), float(ess_threshold), int(tuning_iters), int(tuning_steps),
                int(relax), int(ladder_mode), int(use_icm), _ptr(cl), _ptr(cv), int(threads), words, en, draws, alphas, ess, n_ess, rho, fam, n_res, fe, best_pre,
                inc, state)
    ne, nr = int(n_ess[0]), int(n_res[0])
    return dict(words=words.reshape(cells, n), energies=en.reshape(cells, 64), draws=int(draws[0]), alphas=alphas,
                ess=ess[:ne], rho=rho[:nr], families=fam[:nr], free_energy=float(fe[0]), resamples=nr,
                best_pre=best_pre, incumbent=float(inc[0]), state=state)


def pa_normalized_weights(log_w) -> np.ndarray:
    lw = np.ascontiguousarray(log_w, dtype=np.float64)
    out = np.zeros(len(lw), dtype=np.float64)
    lib().or_pa_normalized_weights(lw, len(lw), out)
    return out


def pa_systematic_resample(w, u: float) -> np.ndarray:
    w = np.ascontiguousarray(w, dtype=np.float64)
    out = np.zeros(len(w), dtype=np.int64)
    lib().or_pa_systematic_resample(w, len(w), float(u), out)
    return out


def gen_index_inclusive(seed: int, his):
    """gen_range(0..=hi) for each hi in sequence on seed_from_u64(seed);
    returns (values, draws consumed)."""
    hi = np.ascontiguousarray(his, dtype=np.uint64)
    out = np.zeros(len(hi), dtype=np.uint64)
    draws = np.zeros(1, dtype=np.uint64)
    lib().or_gen_index_inclusive(int(seed), hi, len(hi), out, draws)
    return out, int(draws[0])


def pa_feedback_alphas(alphas, flow, damping) -> np.ndarray:
    a = np.ascontiguousarray(alphas, dtype=np.float64)
    f = np.ascontiguousarray(flow, dtype=np.float64)
    out = np.zeros(len(a), dtype=np.float64)
    lib().or_pa_feedback_alphas(a, f, len(a), float(damping), out)
    return out


def two_opt(model, state, clamped=None, offset=0.0):
    """steepest_descent_2opt_escapes (local_search.rs:123-143) on a copy of
    state; returns (state, improvement)."""
    n, lin, row, col, val = _csr(model)
    x = np.array(state, dtype=np.int8)
    cl = np.zeros(n, dtype=np.uint8) if clamped is None else np.ascontiguousarray(clamped, dtype=np.uint8)
    imp = lib().or_two_opt(n, lin, row, col, val, float(offset), x, cl)
    return x, imp


def path_relink_finish(model, words, state, clamped=None, offset=0.0):
    """ultimate.rs:436-479 on a copy of state with the field's words
    [cells, n] (bit r = replica r); returns (state, energy)."""
    n, lin, row, col, val = _csr(model)
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
    x = np.array(state, dtype=np.int8)
    cl = np.zeros(n, dtype=np.uint8) if clamped is None else np.ascontiguousarray(clamped, dtype=np.uint8)
    e = lib().or_path_relink(n, lin, row, col, val, float(offset), w, w.size // max(n, 1), cl, x)
    return x, e


def warm_start_words(seed, skip, probs, cells, clamped=None, clamp_val=None):
    """The warm-start init (ultimate.rs:256-263): words [cells, n] and the
    stream position after them."""
    p = np.ascontiguousarray(probs, dtype=np.float64)
    n = len(p)
    cl = np.zeros(n, np.uint8) if clamped is None else np.ascontiguousarray(clamped, dtype=np.uint8)
    cv = np.zeros(n, np.int8) if clamp_val is None else np.ascontiguousarray(clamp_val, dtype=np.int8)
    out = np.zeros(cells * n, dtype=np.uint64)
    d = lib().or_warm_start_words(int(seed), int(skip), p, cl, cv, n, int(cells), out)
    return out.reshape(cells, n), int(d)

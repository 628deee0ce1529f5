"""Serving: continuous batching of SA solve requests on one GPU.

The reference serves ``POST /api/v1/solve`` (src/bin/server_api.rs): it
validates the request (:70-99), builds the CSR with duplicate edges merged
(:111-156), takes a compute permit (one solve per pool thread, :188-193) and
solves on the Rayon pool. Here the solve is a device-resident request pool
behind ``ie_serve_*`` (include/ising_b200.h): requests are admitted first come
first served as slots and device memory free up, stay resident until their
schedule is done, and every tick advances all resident requests together, so
requests that arrive while others run overlap on the GPU. A request's result
equals the same request solved alone (``BatchEngine`` with one model).

``QuboRequest`` / ``validate`` / ``model_from`` / ``response`` mirror the
reference's JSON schema and checks; ``serve_stream`` drives a timed arrival
stream and reports per-request latency.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from .core import CsrMatrix, QuboModel
from .engine import NUM_REPLICAS, _p, _problem, suggested_temp_range

# server_api.rs:15-17; sweeps here is the SA length (one temperature per
# step), so its maximum is the SA length of the serving stream's largest request.
MAX_NUM_VARS = 50_000
MAX_SWEEPS = 20_000
MAX_EXCHANGES = 10_000


class ServeEngine:
    """The device request pool (``ie_serve_*``)."""

    def __init__(self, device: int = 0, force_f64: bool = False, max_requests: int = 4096,
                 site_budget: int = 65536, max_sites: int = 1 << 24, max_couplings: int = 1 << 27,
                 max_schedule_steps: int = 1 << 25, kernel_form: int = 0, tick_us: int = 0):
        self._L = _ffi.lib()
        cfg = _ffi.ie_serve_config(device, int(force_f64), max_requests, site_budget, max_sites,
                                   max_couplings, max_schedule_steps, int(kernel_form), int(tick_us))
        h = C.c_void_p()
        _ffi.check(self._L.ie_serve_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._n = {}
        self._lock = threading.Lock()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.ie_serve_destroy(self._h)
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

    def submit(self, model: QuboModel, seed: int, temps, is_clamped=None, clamp_val=None) -> int:
        """Queues one SA request (temps: per-step temperatures); returns its id.
        Safe to call from another thread while ``tick`` runs."""
        keep: list = []
        prob = _problem(model, keep)
        t = np.ascontiguousarray(temps, dtype=np.float64).reshape(-1)
        f = v = None
        if is_clamped is not None:
            f = np.ascontiguousarray(is_clamped, dtype=np.uint8)
            v = np.ascontiguousarray(np.zeros(model.num_vars) if clamp_val is None else clamp_val,
                                     dtype=np.int8)
        rid = C.c_uint64()
        _ffi.check(self._L.ie_serve_submit(self._h, C.byref(prob), seed & 0xFFFFFFFFFFFFFFFF, _p(t),
                                           len(t), None if f is None else _p(f),
                                           None if v is None else _p(v), C.byref(rid)))
        with self._lock:
            self._n[rid.value] = model.num_vars
        return rid.value

    def tick(self):
        """Admits queued requests, runs one tick, retires finished ones.
        Returns (active, pending, finished-not-taken)."""
        a, p, f = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _ffi.check(self._L.ie_serve_tick(self._h, C.byref(a), C.byref(p), C.byref(f)))
        return a.value, p.value, f.value

    def poll(self, max_ids: int = 4096) -> list[int]:
        ids = np.zeros(max_ids, dtype=np.uint64)
        n = C.c_uint32()
        _ffi.check(self._L.ie_serve_poll(self._h, _p(ids), max_ids, C.byref(n)))
        return [int(x) for x in ids[: n.value]]

    def result(self, rid: int):
        """(words [N] with bit r = replica r, energies [64]) of a finished request."""
        with self._lock:
            n = self._n.pop(rid)
        w = np.zeros(n, dtype=np.uint64)
        e = np.zeros(NUM_REPLICAS, dtype=np.float64)
        _ffi.check(self._L.ie_serve_result(self._h, rid, _p(w), _p(e)))
        return w, e

    def footprint(self, model: QuboModel, n_steps: int) -> int:
        keep: list = []
        prob = _problem(model, keep)
        b = C.c_uint64()
        _ffi.check(self._L.ie_serve_footprint(self._h, C.byref(prob), n_steps, C.byref(b)))
        return b.value

    def last_tick(self):
        ms = C.c_double()
        n = C.c_uint64()
        _ffi.check(self._L.ie_serve_last_tick(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def run_all(self):
        """Ticks until nothing is resident or queued; returns {id: (words, energies)}."""
        out = {}
        while True:
            a, p, _ = self.tick()
            for rid in self.poll():
                out[rid] = self.result(rid)
            if a == 0 and p == 0:
                return out


@dataclass
class ServeTrace:
    """Per-request timing of a served stream (seconds from stream start)."""
    arrival: np.ndarray
    done: np.ndarray
    results: list = field(default_factory=list)
    tick_ms: list = field(default_factory=list)
    launches: int = 0

    @property
    def latency_ms(self) -> np.ndarray:
        return (self.done - self.arrival) * 1e3

    def summary(self) -> dict:
        lat = self.latency_ms
        span = float(self.done.max()) if len(self.done) else 0.0
        return {"requests": int(len(lat)), "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "makespan_s": span, "ticks": len(self.tick_ms),
                "mean_tick_ms": float(np.mean(self.tick_ms)) if self.tick_ms else 0.0}


def serve_stream(engine: ServeEngine, requests, arrivals, keep_results: bool = True) -> ServeTrace:
    """Serves ``requests`` [(model, seed, temps)] arriving at ``arrivals`` (s
    from now): a submitter thread queues each request at its arrival time
    (its host-side preparation counts toward its latency) while this thread
    ticks the engine; latency = result taken - arrival."""
    count = len(requests)
    arrival = np.asarray(arrivals, dtype=np.float64)
    done = np.full(count, np.nan)
    ids = [None] * count
    id_to_idx = {}
    lock = threading.Lock()
    err = []
    t0 = time.perf_counter()

    def submitter():
        try:
            for i, (m, seed, temps) in enumerate(requests):
                wait = arrival[i] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
                rid = engine.submit(m, seed, temps)
                with lock:
                    ids[i] = rid
                    id_to_idx[rid] = i
        except Exception as e:  # surfaced by the ticking thread
            err.append(e)

    th = threading.Thread(target=submitter, daemon=True)
    th.start()
    results = [None] * count
    trace = ServeTrace(arrival=arrival, done=done)
    finished = 0
    while finished < count:
        if err:
            raise err[0]
        a, p, f = engine.tick()
        ms, nl = engine.last_tick()
        if nl:
            trace.tick_ms.append(ms)
            trace.launches += nl
        for rid in engine.poll():
            r = engine.result(rid)
            now = time.perf_counter() - t0
            with lock:
                i = id_to_idx[rid]
            done[i] = now
            if keep_results:
                results[i] = r
            finished += 1
        if a == 0 and p == 0 and finished < count:
            time.sleep(0.0005)
    th.join()
    trace.results = results
    return trace


# ---- request front-end (server_api.rs:29-48, 70-169) ----

@dataclass
class QuboRequest:
    num_vars: int
    linear: list
    quadratic: list  # (u, v, w) triples
    clamped: list | None = None  # (index, value) pairs
    replicas: int | None = None  # accepted and ignored, as in the reference
    sweeps: int | None = None
    exchanges: int | None = None
    seed: int | None = None

    @staticmethod
    def from_json(d: dict) -> "QuboRequest":
        return QuboRequest(int(d["num_vars"]), list(d["linear"]), [tuple(q) for q in d["quadratic"]],
                           [tuple(c) for c in d["clamped"]] if d.get("clamped") is not None else None,
                           d.get("replicas"), d.get("sweeps"), d.get("exchanges"), d.get("seed"))


def validate(req: QuboRequest) -> None:
    """server_api.rs:70-99; raises ValueError with the reference's message."""
    if req.num_vars == 0:
        raise ValueError("num_vars must be > 0")
    if req.num_vars > MAX_NUM_VARS:
        raise ValueError(f"num_vars exceeds maximum {MAX_NUM_VARS}")
    if len(req.linear) != req.num_vars:
        raise ValueError("linear.len() must equal num_vars")
    for (u, v, _) in req.quadratic:
        if u >= req.num_vars or v >= req.num_vars:
            raise ValueError(f"edge index out of range: ({u}, {v}) for num_vars={req.num_vars}")
    for (idx, val) in req.clamped or []:
        if idx >= req.num_vars:
            raise ValueError(f"clamped index {idx} out of range")
        if val not in (0, 1):
            raise ValueError(f"clamped value must be 0 or 1, got {val}")


def model_from(req: QuboRequest) -> QuboModel:
    """server_api.rs:111-156: both triangles, each row sorted by column,
    duplicates summed, entries with |w| <= 1e-9 dropped, offset 0."""
    rows = [[] for _ in range(req.num_vars)]
    for (u, v, w) in req.quadratic:
        rows[u].append((v, float(w)))
        rows[v].append((u, float(w)))
    ro = [0]
    ci = []
    va = []
    for edges in rows:
        edges.sort(key=lambda e: e[0])  # stable, like sort_by_key
        merged = []
        for (v, w) in edges:
            if merged and merged[-1][0] == v:
                merged[-1][1] += w
            else:
                merged.append([v, w])
        for (v, w) in merged:
            if abs(w) > 1e-9:
                ci.append(v)
                va.append(w)
        ro.append(len(ci))
    q = CsrMatrix(np.array(va, dtype=np.float64), np.array(ci, dtype=np.int64), np.array(ro, dtype=np.int64))
    return QuboModel(req.num_vars, np.array(req.linear, dtype=np.float64), q, 0.0)


def schedule_from(req: QuboRequest, model: QuboModel) -> np.ndarray:
    """Per-step temperatures of the request: the reference's data-driven
    range (schedule.rs:21-43, server_api.rs:161-164), beta linear from
    1/T_max to 1/T_min over ``sweeps`` steps (default 100, clamped to
    [1, MAX_SWEEPS] as server_api.rs:104)."""
    sweeps = min(max(int(req.sweeps if req.sweeps is not None else 100), 1), MAX_SWEEPS)
    t_max, t_min = suggested_temp_range(model)
    k = np.arange(sweeps, dtype=np.float64)
    b0, b1 = 1.0 / t_max, 1.0 / t_min
    betas = b0 + (b1 - b0) * k / max(sweeps - 1, 1)
    return 1.0 / betas


def clamps_from(req: QuboRequest):
    if not req.clamped:
        return None, None
    f = np.zeros(req.num_vars, dtype=np.uint8)
    v = np.zeros(req.num_vars, dtype=np.int8)
    for (i, x) in req.clamped:
        f[i] = 1
        v[i] = x
    return f, v


def best_replica(model: QuboModel, words: np.ndarray, energies: np.ndarray):
    """State (0/1 int8) and model energy of the lowest-energy replica (lowest
    index on ties)."""
    r = int(np.argmin(energies))
    state = ((words >> np.uint64(r)) & np.uint64(1)).astype(np.int8)
    return state, model.calculate_total_energy(state)


def response(status: str, energy: float = 0.0, state=(), compute_time_ms: int = 0) -> dict:
    """QuboResponse (server_api.rs:42-48); errors carry status "error: <msg>"."""
    return {"status": status, "energy": float(energy), "state": [int(x) for x in state],
            "compute_time_ms": int(compute_time_ms)}


def solve_json(engine: ServeEngine, payload: dict) -> dict:
    """One request through the pool, synchronously (validation first, as the
    reference takes no compute capacity for an invalid request)."""
    try:
        req = QuboRequest.from_json(payload)
        validate(req)
    except (ValueError, KeyError, TypeError) as e:
        return response(f"error: {e}")
    t0 = time.perf_counter()
    model = model_from(req)
    temps = schedule_from(req, model)
    f, v = clamps_from(req)
    seed = req.seed if req.seed is not None else int(np.random.SeedSequence().entropy & 0xFFFFFFFFFFFFFFFF)
    rid = engine.submit(model, seed, temps, f, v)
    while True:
        engine.tick()
        if rid in engine.poll():
            break
    words, energies = engine.result(rid)
    state, energy = best_replica(model, words, energies)
    return response("success", energy, state, math.floor((time.perf_counter() - t0) * 1e3))

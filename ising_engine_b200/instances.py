"""Seeded synthetic instances for the measured configurations.

Every generator is deterministic given its seed (numpy PCG64). Ising problems
are lowered to the reference's QUBO form exactly: with s = 2x - 1 and
E_Ising = -sum_<ij> J_ij s_i s_j, the QUBO has coupling q_ij = -4 J_ij (stored
in both triangles), linear term 2 sum_j J_ij and offset -sum_<ij> J_ij, so
E_QUBO(x) = E_Ising(2x - 1).
"""
from __future__ import annotations

import math

import numpy as np

from .core import QuboModel


def ising_to_qubo(n: int, edges_ij: np.ndarray, J: np.ndarray, h: np.ndarray | None = None) -> QuboModel:
    """E = -sum J_ij s_i s_j - sum h_i s_i with s = 2x - 1, as a QuboModel."""
    i = edges_ij[:, 0].astype(np.int64)
    j = edges_ij[:, 1].astype(np.int64)
    J = np.asarray(J, dtype=np.float64)
    lin = np.zeros(n)
    np.add.at(lin, i, 2.0 * J)
    np.add.at(lin, j, 2.0 * J)
    offset = -float(J.sum())
    if h is not None:
        lin -= 2.0 * np.asarray(h, dtype=np.float64)
        offset += float(np.sum(h))
    trip = np.stack([i, j, -4.0 * J], axis=1) if len(J) else np.zeros((0, 3))
    return QuboModel.from_edges(n, lin, trip, offset)


def lattice_edges(L: int, dim: int) -> np.ndarray:
    """Nearest-neighbour bonds of a periodic L^dim lattice, site = x + L*y (+ L^2*z)."""
    idx = np.arange(L ** dim).reshape((L,) * dim)  # axes (z,) y, x
    bonds = []
    for ax in range(dim):
        nb = np.roll(idx, -1, axis=dim - 1 - ax)
        bonds.append(np.stack([idx.reshape(-1), nb.reshape(-1)], axis=1))
    e = np.concatenate(bonds)
    e = np.sort(e, axis=1)
    return e


def pm_j_lattice(L: int, dim: int, seed: int) -> QuboModel:
    """Periodic +-J spin glass on an L^dim lattice (J iid uniform in {-1, +1}, h = 0)."""
    rng = np.random.default_rng(seed)
    e = lattice_edges(L, dim)
    J = rng.choice(np.array([-1.0, 1.0]), size=len(e))
    return ising_to_qubo(L ** dim, e, J)


def maxcut_gnm(n: int, m: int, seed: int) -> QuboModel:
    """Max-Cut of a uniform G(n, m) graph with unit weights, lowered as
    src/bin/gset_official_benchmark.rs:17-28 does: q_ij = 2 w, linear_i =
    -sum_j w_ij, so E(x) = -cut(x)."""
    rng = np.random.default_rng(seed)
    total = n * (n - 1) // 2
    pick = np.sort(rng.choice(total, size=m, replace=False))
    # map linear index over the upper triangle back to (i, j)
    i = (n - 2 - np.floor(np.sqrt(-8 * pick + 4 * n * (n - 1) - 7) / 2.0 - 0.5)).astype(np.int64)
    j = (pick + i + 1 - n * (n - 1) // 2 + (n - i) * ((n - i) - 1) // 2).astype(np.int64)
    lin = np.zeros(n)
    np.add.at(lin, i, -1.0)
    np.add.at(lin, j, -1.0)
    trip = np.stack([i, j, np.full(m, 2.0)], axis=1)
    return QuboModel.from_edges(n, lin, trip, 0.0)


def cut_value(model: QuboModel, state) -> float:
    """Crossing-edge weight (gset_official_benchmark.rs:62-74)."""
    state = np.asarray(state)
    cut = 0.0
    ro, ci, va = model.row_offsets, model.col_indices, model.values
    for a in range(model.num_vars):
        for k in range(int(ro[a]), int(ro[a + 1])):
            b = int(ci[k])
            if a < b and state[a] != state[b]:
                cut += float(va[k]) / 2.0
    return cut


def random_regular_edges(n: int, d: int, rng: np.random.Generator) -> np.ndarray:
    """Simple d-regular graph: configuration-model pairing, then random
    double-edge swaps to remove self-loops and multi-edges."""
    if (n * d) % 2 or d >= n:
        raise ValueError("need n*d even and d < n")
    stubs = np.repeat(np.arange(n, dtype=np.int64), d)
    rng.shuffle(stubs)
    a = stubs[0::2].copy()
    b = stubs[1::2].copy()
    m = len(a)
    key = lambda x, y: min(x, y) * n + max(x, y)
    keys = np.minimum(a, b) * n + np.maximum(a, b)
    uniq, first, cnt = np.unique(keys, return_index=True, return_counts=True)
    bad = set(np.nonzero(a == b)[0].tolist())
    dup_keys = set(uniq[cnt > 1].tolist())
    if dup_keys:
        seen = set()
        for k in np.nonzero(np.isin(keys, list(dup_keys)))[0].tolist():
            if keys[k] in seen:
                bad.add(k)
            else:
                seen.add(int(keys[k]))
    present = {}
    for k in range(m):
        if k in bad:
            continue
        present[int(keys[k])] = present.get(int(keys[k]), 0) + 1
    bad = sorted(bad)
    guard = 0
    while bad:
        guard += 1
        if guard > 200 * m + 1000:
            raise RuntimeError("random regular repair did not converge")
        k = bad[-1]
        o = int(rng.integers(m))
        if o == k or o in bad:
            continue
        x1, y1, x2, y2 = int(a[k]), int(b[k]), int(a[o]), int(b[o])
        if rng.integers(2):
            x2, y2 = y2, x2
        # rewire (x1,y1),(x2,y2) -> (x1,y2),(x2,y1)
        if x1 == y2 or x2 == y1:
            continue
        k1, k2 = key(x1, y2), key(x2, y1)
        if k1 == k2 or present.get(k1, 0) or present.get(k2, 0):
            continue
        ko = key(int(a[o]), int(b[o]))
        present[ko] -= 1
        if present[ko] == 0:
            del present[ko]
        a[k], b[k], a[o], b[o] = x1, y2, x2, y1
        present[k1] = 1
        present[k2] = 1
        bad.pop()
    return np.stack([np.minimum(a, b), np.maximum(a, b)], axis=1)


def random_regular_qubo(n: int, d: int, rng: np.random.Generator, integer: bool) -> QuboModel:
    """Random d-regular QUBO: integer couplings uniform in [-8, 8] without 0
    and linear terms uniform in [-8, 8]; or f32 N(0, 1) couplings and linear
    terms widened exactly to f64."""
    e = random_regular_edges(n, d, rng)
    if integer:
        mag = rng.integers(1, 9, size=len(e))
        sign = rng.choice(np.array([-1, 1]), size=len(e))
        q = (mag * sign).astype(np.float64)
        lin = rng.integers(-8, 9, size=n).astype(np.float64)
    else:
        q = rng.standard_normal(len(e)).astype(np.float32).astype(np.float64)
        lin = rng.standard_normal(n).astype(np.float32).astype(np.float64)
    return QuboModel.from_edges(n, lin, np.concatenate([e.astype(np.float64), q[:, None]], axis=1), 0.0)


def uneven_batch(count: int, seed: int, n_min: int = 64, n_max: int = 4096, d_min: int = 3,
                 d_max: int = 16):
    """The uneven batch: N log-uniform in [n_min, n_max], degree uniform in
    {d_min..d_max} (redrawn until N*d is even), even-indexed instances integer,
    odd-indexed float32. Returns (models, per-instance seeds)."""
    rng = np.random.default_rng(seed)
    models = []
    for i in range(count):
        while True:
            n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
            d = int(rng.integers(d_min, d_max + 1))
            if (n * d) % 2 == 0 and d < n:
                break
        models.append(random_regular_qubo(n, d, rng, integer=(i % 2 == 0)))
    seeds = (np.uint64(seed) * np.uint64(1000003) + np.arange(count, dtype=np.uint64)).astype(np.uint64)
    return models, seeds


def serve_requests(count: int, seed: int, n_min: int = 100, n_max: int = 20000, d_min: int = 4,
                   d_max: int = 32, sweeps_min: int = 1000, sweeps_max: int = 20000):
    """The serving stream's requests: N log-uniform in [n_min, n_max], degree
    uniform in {d_min..d_max} (redrawn until N*d is even), integer couplings
    in [-8, 8] or float32 N(0, 1) with probability 1/2 each, SA length uniform
    in [sweeps_min, sweeps_max]. Returns [(model, seed, sweeps)]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        while True:
            n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
            d = int(rng.integers(d_min, d_max + 1))
            if (n * d) % 2 == 0 and d < n:
                break
        integer = bool(rng.integers(2))
        sweeps = int(rng.integers(sweeps_min, sweeps_max + 1))
        m = random_regular_qubo(n, d, rng, integer=integer)
        out.append((m, int((seed * 7919 + 104729 * i) & 0xFFFFFFFFFFFFFFFF), sweeps))
    return out


def poisson_arrivals(count: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times (s) of a Poisson stream of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def sa_temps(sweeps: int, beta0: float = 0.1, beta1: float = 5.0) -> np.ndarray:
    """Per-step temperatures 1/beta_k with beta linear from beta0 to beta1."""
    k = np.arange(sweeps, dtype=np.float64)
    betas = beta0 + (beta1 - beta0) * k / max(sweeps - 1, 1)
    return 1.0 / betas


def geometric_beta_ladder(nt: int, beta0: float, beta1: float) -> np.ndarray:
    """Temperatures 1/beta for beta geometric from beta0 to beta1 (hot first)."""
    b = beta0 * (beta1 / beta0) ** (np.arange(nt) / max(nt - 1, 1))
    return 1.0 / b

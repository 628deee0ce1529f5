"""The CPU oracle against the reference's own golden vectors and invariants.

The end-to-end golden (tests/test_regression_golden.rs:87-111) pins the master
ChaCha8 stream, rand_core's seed_from_u64 and rand's gen_range through the
seeded instance (its optimum energy matches to every digit) and the whole
UltimateSolver path through the final state. The remaining tests restate the
reference's engine invariants (test_population_annealing.rs:354-420,
test_trotter_correctness.rs:73-143) and cross-check the C++ oracle's step
against an independent pure-Python restatement on small cases.
"""
import json
import os

import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.core import CsrMatrix, QuboModel
from oracle import oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "regression_golden.json")))


def golden_model():
    lin, row, col, val = O.golden_instance()
    return QuboModel(32, lin, CsrMatrix(val, col.astype(np.uint64), row.astype(np.uint64)))


def test_golden_end_to_end():
    m = golden_model()
    s = GOLDEN["solver"]
    state = O.solve(m, s["temp_max"], s["temp_min"], s["sweeps"], s["exchanges"], s["seed"],
                    num_temps=s["num_temps"])
    assert state.tolist() == GOLDEN["golden_state"]
    e = O.total_energy(m, state)
    assert abs(e - GOLDEN["golden_energy"]) < GOLDEN["energy_tolerance"]
    # the product's energy function agrees with the oracle's
    assert m.calculate_total_energy(state) == e


def test_golden_determinism_with_clamps():
    m = golden_model()
    s = GOLDEN["solver"]
    clamps = [(0, 1), (7, 0), (31, 1)]
    a = O.solve(m, s["temp_max"], s["temp_min"], s["sweeps"], s["exchanges"], s["seed"], clamped=clamps)
    b = O.solve(m, s["temp_max"], s["temp_min"], s["sweeps"], s["exchanges"], s["seed"], clamped=clamps)
    assert (a == b).all()
    for i, v in clamps:
        assert a[i] == v


def one_var_model(lin0=10.0):
    return QuboModel(1, np.array([lin0]), CsrMatrix(np.zeros(0), np.zeros(0, np.uint64),
                                                     np.zeros(2, np.uint64)))


@pytest.mark.parametrize("hot,cold,seed,favourable", [(0, 1, 1, True), (1, 0, 2, False)])
def test_swap_statistics_known_answers(hot, cold, seed, favourable):
    """test_population_annealing.rs:354-420: frozen two-level field."""
    m = one_var_model()
    words = np.array([[0xFFFFFFFFFFFFFFFF if hot else 0], [0xFFFFFFFFFFFFFFFF if cold else 0]],
                     dtype=np.uint64)
    r = O.run_schedule(m, np.array([[2.0, 0.5]]), seed, init_words=words, clamped=np.ones(1),
                       clamp_val=np.array([hot]), collect_stats=True)
    rate = r.swap_accepts[0] / r.swap_attempts[0]
    if favourable:
        assert rate == 1.0
        assert r.draws == 1  # base_seed only: no exchange draw when exponent >= 0
    else:
        assert rate < 0.01
        assert r.draws == 1 + 64


def test_single_slice_ground_state_stable():
    """test_trotter_correctness.rs:73-109."""
    n = 16
    m = QuboModel(n, np.full(n, 1.5), CsrMatrix.empty(n))
    r = O.run_schedule(m, np.full((5, 1), 0.01), 3, init_words=np.zeros((1, n), np.uint64))
    assert (r.words == 0).all()


@pytest.mark.parametrize("integer", [True, False])
def test_tracked_energy_matches_recompute(integer):
    """test_trotter_correctness.rs:112-143 (num_slices = 1)."""
    rng = np.random.default_rng(17)
    m = I.random_regular_qubo(40, 5, rng, integer=integer)
    r = O.run_schedule(m, np.tile([2.0, 0.5], (50, 1)), 99)
    rec = O.replica_energies(m, r.words)
    if integer:
        assert (rec == r.energies).all()
    else:
        assert np.max(np.abs(rec - r.energies)) < 1e-6


def test_geometric_temps_match_product():
    from ising_engine_b200.engine import geometric_temps
    for args in [(50.0, 0.05, 10), (1000.0, 0.01, 32), (10.0, 1.0 / 3.0, 32), (3.0, 3.0, 1)]:
        a = O.geometric_temps(*args)
        b = geometric_temps(*args)
        assert a.tobytes() == b.tobytes()


# ---------------------------------------------------------------------------
# Independent pure-Python restatement of engine::step for small cases.
# ---------------------------------------------------------------------------
M64 = (1 << 64) - 1


def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & M64


def _xoshiro_lanes(seed):
    st = seed
    out = []
    for _ in range(32):
        st = (st + 0x9E3779B97F4A7C15) & M64
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        out.append(z ^ (z >> 31))
    return [out[4 * l:4 * l + 4] for l in range(8)]


def _xo_next(s):
    res = (_rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
    t = (s[1] << 17) & M64
    s[2] ^= s[0]
    s[3] ^= s[1]
    s[1] ^= s[2]
    s[0] ^= s[3]
    s[2] ^= t
    s[3] = _rotl(s[3], 45)
    return res


def _fast_exp(x):
    x = max(min(x, 0.0), -20.0)
    r = x * 0.0625
    r2 = r * r
    r3 = r2 * r
    p = 1.0 + r + 0.5 * r2 + (1.0 / 6.0) * r3 + (1.0 / 24.0) * r2 * r2 + (1.0 / 120.0) * r2 * r3 + \
        (1.0 / 720.0) * r3 * r3
    p2 = p * p
    p4 = p2 * p2
    p8 = p4 * p4
    return p8 * p8


def _py_run(m, temps, seed, steps):
    """init + steps of engine::step, exchange every step; returns words, energies, draws."""
    import math
    n, nt = m.num_vars, len(temps)
    draws = O.chacha8_u64(seed, nt * n + steps * (1 + 64 * nt))
    pos = 0

    def nxt():
        nonlocal pos
        v = int(draws[pos])
        pos += 1
        return v

    ro, ci, va, lin = m.row_offsets.astype(int), m.col_indices.astype(int), m.values, m.linear
    x = [[[0] * 64 for _ in range(n)] for _ in range(nt)]
    for t in range(nt):
        for v in range(n):
            w = nxt()
            x[t][v] = [(w >> r) & 1 for r in range(64)]

    def energies(t):
        e = [0.0] * 64
        for v in range(n):
            for r in range(64):
                e[r] += float(lin[v]) * float(x[t][v][r])
            for k in range(ro[v], ro[v + 1]):
                j = ci[k]
                if v < j:
                    for r in range(64):
                        e[r] += float(va[k]) * float(x[t][v][r] & x[t][j][r])
        return e

    E = [energies(t) for t in range(nt)]
    odd = False
    for s in range(steps):
        base = nxt()
        for t in range(nt):
            beta = 1.0 / temps[t]
            lanes = _xoshiro_lanes((base + t) & M64)
            for v in range(n):
                u = [0.0] * 64
                for c in range(8):
                    for l in range(8):
                        u[8 * c + l] = (_xo_next(lanes[l]) >> 12) * 2.0 ** -52
                xv = x[t][v]
                d = [float(lin[v]) * float(1 - 2 * xv[r]) for r in range(64)]
                for k in range(ro[v], ro[v + 1]):
                    xj = x[t][ci[k]]
                    for r in range(64):
                        d[r] += float(va[k]) * float((xj[r] ^ xv[r]) - xv[r])
                for r in range(64):
                    acc = d[r] <= 0.0 or u[r] < _fast_exp(-d[r] * beta)
                    if acc:
                        xv[r] ^= 1
                        E[t][r] += d[r]
        for t in range(1 if odd else 0, nt - 1, 2):
            db = 1.0 / temps[t] - 1.0 / temps[t + 1]
            mask = []
            for r in range(64):
                ex = db * (E[t][r] - E[t + 1][r])
                mask.append(ex >= 0.0 or (nxt() >> 11) * 2.0 ** -53 < math.exp(ex))
            for r in range(64):
                if mask[r]:
                    for v in range(n):
                        x[t][v][r], x[t + 1][v][r] = x[t + 1][v][r], x[t][v][r]
                    E[t][r], E[t + 1][r] = E[t + 1][r], E[t][r]
        odd = not odd
    words = np.array([[sum(x[t][v][r] << r for r in range(64)) for v in range(n)] for t in range(nt)],
                     dtype=np.uint64)
    return words, np.array(E), pos


@pytest.mark.parametrize("integer", [True, False])
def test_oracle_step_matches_python_restatement(integer):
    rng = np.random.default_rng(5 if integer else 6)
    m = I.random_regular_qubo(10, 3, rng, integer=integer)
    temps = [3.0, 1.0, 0.4]
    w, e, draws = _py_run(m, temps, 1234, 4)
    r = O.run_schedule(m, np.tile(temps, (4, 1)), 1234)
    assert (r.words == w).all()
    assert r.energies.tobytes() == e.tobytes()
    assert r.draws == draws

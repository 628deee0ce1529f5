"""engine_v2 (S2) host logic and the oracle's S2 restatement (no GPU).

The oracle's bit-sliced state keeps the reference's i64 field ledger
(sparse_bitslice.rs); the pure-Python restatement here gathers every field
from scratch instead, so agreement checks the ledger and the operators'
stream order independently. Draws come from the oracle's ChaCha8 stream,
which the S1 golden pins."""
import math

import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.v2 import ProblemIR
from oracle import oracle as O


def frustrated():
    """metropolis_sweep.rs:156-172."""
    return ProblemIR.from_pairs(7, -2.0, [1.0, -2.0, 3.0, 0.0, -1.0, 2.0, 1.0],
                                [(0, 1, -1.0), (1, 2, 2.0), (2, 3, -3.0), (0, 3, 1.0), (3, 4, -1.0),
                                 (4, 5, 2.0), (5, 6, -2.0), (2, 6, 1.0)])


def test_from_pairs_merges_and_drops():
    ir = ProblemIR.from_pairs(4, 1.0, [0.0] * 4, [(0, 1, 1.0), (0, 1, 2.0), (2, 3, 1.0), (2, 3, -1.0), (1, 3, 5.0)])
    assert ir.row_ptr.tolist() == [0, 1, 3, 3, 4]
    assert ir.col_idx.tolist() == [1, 0, 3, 1]
    assert ir.weights.tolist() == [3.0, 3.0, 5.0, 5.0]
    assert ir.is_integral()
    assert not ProblemIR.from_pairs(2, 0.5, [0.0, 0.0], [(0, 1, 1.0)]).is_integral()
    f = frustrated()
    assert f.energy(np.array([1, 0, 1, 0, 0, 1, 0])) == -2.0 + 1.0 + 3.0 + 2.0  # no edge among {0, 2, 5}


def py_coloring(ir):
    colors = [None] * ir.n
    for i in range(ir.n):
        used = sorted(colors[int(j)] for j in ir.col_idx[ir.row_ptr[i]:ir.row_ptr[i + 1]] if colors[int(j)] is not None)
        c = 0
        for u in used:
            if u == c:
                c += 1
            elif u > c:
                break
        colors[i] = c
    return colors


@pytest.mark.parametrize("seed", [1, 2])
def test_greedy_coloring(seed):
    m = I.maxcut_gnm(60, 300, seed=seed)
    ir = ProblemIR.from_model(m)
    c = ir.greedy_coloring()
    assert c.tolist() == py_coloring(ir)
    for i in range(ir.n):
        for j in ir.col_idx[ir.row_ptr[i]:ir.row_ptr[i + 1]]:
            assert c[i] != c[int(j)]


def py_program(ir, r, init, seed, ops, temps):
    """S2 restated with fields gathered from scratch (no ledger)."""
    n = ir.n
    ro, ci, wv = ir.row_ptr.astype(int), ir.col_idx.astype(int), ir.weights
    lin = ir.linear
    x = [[int(init[s]) for _ in range(r)] for s in range(n)]
    colors = py_coloring(ir)
    order = [s for c in range(max(colors) + 1) for s in range(n) if colors[s] == c]
    total = sum(c * (r if k == "exchange" else n * r) for k, c in ops)
    draws = O.chacha8_u64(seed, total + 8)
    pos = 0

    def u():
        nonlocal pos
        v = int(draws[pos]) >> 11
        pos += 1
        return v * (1.0 / 9007199254740992.0)

    def field(s, k):
        return int(lin[s]) + sum(int(wv[e]) * x[ci[e]][k] for e in range(ro[s], ro[s + 1]))

    def energy(k):
        l = sum(int(lin[s]) for s in range(n) if x[s][k])
        q = sum(int(wv[e]) for s in range(n) if x[s][k] for e in range(ro[s], ro[s + 1]) if x[ci[e]][k])
        return int(ir.offset) + l + q // 2

    stats = []
    for kind, count in ops:
        p = a = 0
        if kind == "metropolis":
            for _ in range(count):
                for s in order:
                    de = [float(field(s, k) if x[s][k] == 0 else -field(s, k)) for k in range(r)]
                    flips = []
                    for k in range(r):
                        t = temps[k % len(temps)]
                        if de[k] <= 0.0:
                            u()
                            acc = True
                        else:
                            pr = math.exp(-de[k] / t) if t > 0.0 else 0.0
                            acc = u() < pr
                        p += 1
                        if acc:
                            a += 1
                            flips.append(k)
                    for k in flips:
                        x[s][k] ^= 1
        elif kind == "gibbs":
            for _ in range(count):
                for s in order:
                    flips = []
                    for k in range(r):
                        h = float(field(s, k))
                        t = temps[k % len(temps)]
                        bh = h / t if t > 0.0 else (math.inf if h > 0 else (-math.inf if h < 0 else 0.0))
                        try:
                            ex = math.exp(bh)
                        except OverflowError:
                            ex = math.inf
                        one = u() < 1.0 / (1.0 + ex)
                        p += 1
                        if one != bool(x[s][k]):
                            a += 1
                            flips.append(k)
                    for k in flips:
                        x[s][k] ^= 1
        else:
            for rnd in range(count):
                e = [float(energy(k)) for k in range(r)]
                k = rnd & 1
                while k + 1 < r:
                    bi = 1.0 / temps[k % len(temps)]
                    bj = 1.0 / temps[(k + 1) % len(temps)]
                    delta = (bi - bj) * (e[k] - e[k + 1])
                    p += 1
                    uu = u()
                    if delta >= 0.0 or uu < math.exp(delta):
                        for s in range(n):
                            x[s][k], x[s][k + 1] = x[s][k + 1], x[s][k]
                        e[k], e[k + 1] = e[k + 1], e[k]
                        a += 1
                    k += 2
        stats.append((p, a))
    w = (r + 63) // 64
    planes = np.zeros((n, w), dtype=np.uint64)
    for s in range(n):
        for k in range(r):
            if x[s][k]:
                planes[s, k // 64] |= np.uint64(1) << np.uint64(k % 64)
    return planes, np.array([float(energy(k)) for k in range(r)]), stats, pos


@pytest.mark.parametrize("r", [10, 70])
def test_oracle_v2_matches_python_restatement(r):
    ir = frustrated()
    init = np.array([1, 0, 1, 0, 0, 1, 0], np.uint8)
    temps = [0.2 + 0.05 * k for k in range(r)]
    ops = [("metropolis", 3), ("exchange", 2), ("gibbs", 2), ("metropolis", 2), ("exchange", 1), ("gibbs", 1)]
    pl, en, st, drift, draws = O.v2_program(ir.model(), r, init, 11, ops, temps)
    ppl, pen, pst, ppos = py_program(ir, r, init, 11, ops, temps)
    assert (pl == ppl).all()
    assert en.tolist() == pen.tolist()
    assert st == pst
    assert drift == 0.0 and draws == ppos


def test_oracle_gibbs_special_temperatures():
    """T <= 0 and NaN take the greedy limit, T = inf resamples with P = 1/2
    (gibbs_color_sweep.rs:139-149); the fields of this instance reach +-10,
    so T = 0.01 overflows exp for the uphill ones."""
    ir = frustrated()
    init = np.array([0, 1, 1, 0, 1, 0, 1], np.uint8)
    temps = [0.0, -1.0, math.nan, math.inf, 0.01, 1e-300, 3.0]
    r = 21
    pl, en, st, drift, draws = O.v2_program(ir.model(), r, init, 5, [("gibbs", 4)], temps)
    ppl, pen, pst, ppos = py_program(ir, r, init, 5, [("gibbs", 4)], temps)
    assert (pl == ppl).all() and en.tolist() == pen.tolist() and st == pst and draws == ppos


def test_oracle_gibbs_cold_is_monotone_descent():
    """gibbs_color_sweep.rs:255-291: at T = 1e-9 no replica's energy rises."""
    ir = frustrated()
    r = 8
    init = np.zeros(7, np.uint8)
    _, e0, _, _, _ = O.v2_program(ir.model(), r, init, 1, [], [1e-9] * r)
    _, e1, _, drift, _ = O.v2_program(ir.model(), r, init, 1, [("gibbs", 5)], [1e-9] * r)
    assert (e1 <= e0).all() and drift == 0.0

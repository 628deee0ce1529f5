"""The 2-opt escape finisher (host): the library's ie_two_opt equals the
oracle's restatement of local_search.rs:83-143 bit for bit (states and
improvement), never worsens, ends at a 1-opt minimum with no improving
2-flip over ALL pairs (tests/test_local_search.rs:111-175, exhaustively on
small instances), and never moves a clamped variable (:177-195)."""
import itertools

import numpy as np
import pytest

from ising_engine_b200.solver import UltimateSolver, steepest_descent_2opt_escapes
from oracle import oracle as O
from tests.test_pa_host import random_qubo


@pytest.mark.parametrize("seed", range(8))
def test_two_opt_equals_oracle_and_is_2opt(seed):
    m = random_qubo(14, 0.4, 800 + seed, integral=seed % 2 == 0)
    rng = np.random.default_rng(seed)
    for _ in range(3):
        x = rng.integers(0, 2, size=14).astype(np.int8)
        e0 = m.calculate_total_energy(x)
        ref, rimp = O.two_opt(m, x)
        y = x.copy()
        imp = steepest_descent_2opt_escapes(m, y)
        assert y.tolist() == ref.tolist() and imp == rimp
        e1 = m.calculate_total_energy(y)
        assert e1 <= e0 + 1e-12 and abs((e0 - e1) - imp) < 1e-9
        for i in range(14):
            z = y.copy()
            z[i] ^= 1
            assert m.calculate_total_energy(z) >= e1 - 1e-9
        for i, j in itertools.combinations(range(14), 2):
            z = y.copy()
            z[i] ^= 1
            z[j] ^= 1
            assert m.calculate_total_energy(z) >= e1 - 1e-9


def test_two_opt_respects_clamps():
    m = random_qubo(12, 0.5, 5)
    cl = np.zeros(12, np.uint8)
    cl[[0, 3, 7]] = 1
    rng = np.random.default_rng(2)
    for _ in range(5):
        x = rng.integers(0, 2, size=12).astype(np.int8)
        y = x.copy()
        steepest_descent_2opt_escapes(m, y, cl)
        assert (y[[0, 3, 7]] == x[[0, 3, 7]]).all()
        ref, _ = O.two_opt(m, x, cl)
        assert y.tolist() == ref.tolist()


def test_with_2opt_flag():
    s = UltimateSolver(1.0, 0.1, 1, 1, 0)
    assert s.use_2opt is False and s.with_2opt(True) is s and s.use_2opt


@pytest.mark.parametrize("seed", range(6))
def test_path_relink_finisher_equals_oracle(seed):
    """ultimate.rs:436-479: the library's finisher returns the oracle's state
    and energy bit for bit on fields of random and near-duplicate replicas
    (the archive's diversity rule and replacement both fire), never worse
    than the current state."""
    from ising_engine_b200.solver import path_relink_finish
    n = [12, 30, 50][seed % 3]
    m = random_qubo(n, 0.3, 900 + seed, integral=seed % 2 == 1)
    rng = np.random.default_rng(seed)
    cells = 3
    base = rng.integers(0, 2, size=n).astype(np.int8)
    words = np.zeros((cells, n), dtype=np.uint64)
    for c in range(cells):
        for r in range(64):
            x = base.copy() if r % 3 else rng.integers(0, 2, size=n).astype(np.int8)
            x[rng.integers(0, n, size=r % 4)] ^= 1  # near duplicates of the base
            words[c] |= x.astype(np.uint64) << np.uint64(r)
    cl = np.zeros(n, np.uint8)
    cl[[0, n // 2]] = 1
    cur = rng.integers(0, 2, size=n).astype(np.int8)
    ref, re = O.path_relink_finish(m, words, cur, cl)
    got = cur.copy()
    e = path_relink_finish(m, words, got, cl)
    assert got.tolist() == ref.tolist() and e == re
    assert e <= m.calculate_total_energy(cur) and e == m.calculate_total_energy(got)

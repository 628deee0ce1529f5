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

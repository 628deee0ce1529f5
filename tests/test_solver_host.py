"""UltimateSolver host logic (no GPU): the Luby sequence
(tests/test_tts.rs:53-59) and the restart driver of ultimate.rs:95-120 —
budgets, derived seeds and best-by-energy selection — with the device solve
replaced by a recording stand-in."""
import numpy as np

from ising_engine_b200 import solver as S
from ising_engine_b200.core import CsrMatrix, QuboModel


def test_luby_sequence():
    assert [S.luby(i) for i in range(1, 16)] == [1, 1, 2, 1, 1, 2, 4, 1, 1, 2, 1, 1, 2, 4, 8]
    assert S.luby(31) == 16 and S.luby(32) == 1


def test_luby_restart_driver(monkeypatch):
    m = QuboModel(3, np.array([1.0, -2.0, 0.5]), CsrMatrix(np.zeros(0), np.zeros(0, np.uint64),
                                                           np.zeros(4, np.uint64)))
    calls = []
    states = [[1, 0, 0], [0, 1, 0], [0, 1, 1], [0, 1, 0], [1, 1, 1], [0, 0, 0]]

    def fake_solve(self, model, clamped=()):
        calls.append((self.total_exchanges, self.seed, list(clamped)))
        return np.array(states[len(calls) - 1], dtype=np.int8)
    monkeypatch.setattr(S.UltimateSolver, "solve", fake_solve)
    base = S.UltimateSolver(5.0, 0.1, 10, 3, 2 ** 64 - 5)
    x = base.solve_with_luby_restarts(m, [(2, 0)], 6)
    g = 0x9E3779B97F4A7C15
    assert [c[0] for c in calls] == [3 * S.luby(i + 1) for i in range(6)]
    assert [c[1] for c in calls] == [(2 ** 64 - 5 + g * (i + 1)) % 2 ** 64 for i in range(6)]
    assert all(c[2] == [(2, 0)] for c in calls)
    # energies: 1, -2, -1.5, -2, -0.5, 0: the first -2 wins
    assert x.tolist() == [0, 1, 0] and base.total_exchanges == 3 and base.seed == 2 ** 64 - 5

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


def test_warm_start_words_equal_oracle():
    """with_gnn_heuristic's init (ultimate.rs:256-263): the library's host
    generator gives the oracle's words and stream position (clamped sites
    draw nothing; probabilities 0, 1, NaN and out of range included)."""
    import ctypes as C
    from ising_engine_b200 import _ffi
    from oracle import oracle as O
    rng = np.random.default_rng(4)
    n, cells = 37, 5
    probs = rng.random(n)
    probs[[0, 1, 2, 3]] = [0.0, 1.0, np.nan, 1.7]
    cl = np.zeros(n, np.uint8)
    cl[[5, 20]] = 1
    cv = np.zeros(n, np.int8)
    cv[20] = 1
    for seed, skip in ((1, 0), (77, 13)):
        ref, rd = O.warm_start_words(seed, skip, probs, cells, cl, cv)
        w = np.zeros(cells * n, dtype=np.uint64)
        d = C.c_uint64()
        _ffi.check(_ffi.lib().ie_warm_start_words(seed, skip, probs.ctypes.data, cl.ctypes.data, cv.ctypes.data, n,
                                                  cells, w.ctypes.data, C.byref(d)))
        assert np.array_equal(w.reshape(cells, n), ref) and d.value == rd == skip + cells * (n - 2) * 64
        assert (ref[:, 0] == 0).all() and (ref[:, 1] == np.uint64(2 ** 64 - 1)).all() and (ref[:, 2] == 0).all()
        assert (ref[:, 20] == np.uint64(2 ** 64 - 1)).all() and (ref[:, 5] == 0).all()


def test_with_gnn_heuristic_flag():
    s = S.UltimateSolver(1.0, 0.1, 1, 1, 0)
    assert s.with_gnn_heuristic([0.2, 0.8]) is s and s.gnn_heuristic_probs.tolist() == [0.2, 0.8]

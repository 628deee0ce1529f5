"""The solver options around the anneal on the device: the warm start
(with_gnn_heuristic, ultimate.rs:256-263) gives the oracle's initial words,
energies and stream position; the 2-opt and path-relinking finishers inside
UltimateSolver.solve equal the oracle's finishers applied to the device run's
polished state and field."""
import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.engine import Engine
from ising_engine_b200.solver import UltimateSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("num_pops", [1, 2])
def test_warm_start_init(num_pops):
    m = I.maxcut_gnm(90, 400, seed=3)
    probs = np.random.default_rng(1).random(90)
    cl = np.zeros(90, np.uint8)
    cl[[4, 40]] = 1
    cv = np.zeros(90, np.int8)
    cv[40] = 1
    with Engine(m, num_temps=3, num_pops=num_pops, seed=19) as eng:
        eng.set_clamps(cl, cv)
        eng.set_init_probs(probs)
        eng.init_random()
        ref, draws = O.warm_start_words(19, 0, probs, 3 * num_pops, cl, cv)
        assert np.array_equal(eng.spins(), ref)
        assert eng.rng_state()[0] == draws
        assert eng.energies().tobytes() == O.replica_energies(m, ref).tobytes()


def test_finishers_in_solve():
    m = I.maxcut_gnm(60, 200, seed=9)
    s = UltimateSolver(5.0, 0.2, 4, 5, 23, num_temps=4)
    with s.engine(m) as eng:
        eng.init_random()
        eng.run_pt()
        _, best = eng.best()
        eng.one_opt(best)
        words = eng.spins()
    x, _ = O.two_opt(m, best)
    y, _ = O.path_relink_finish(m, words, x)
    s.with_2opt(True)
    s.use_path_relinking = True
    assert s.solve(m).tolist() == y.tolist()

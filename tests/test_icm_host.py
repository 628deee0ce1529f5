"""Isoenergetic cluster moves in the oracle (no GPU), on the reference's
contract (tests/test_icm.rs): after PT blocks with an ICM sweep the tracked
energies still equal a full recomputation, the moves change configurations,
the run is deterministic, and a solve with ICM reaches the exhaustive
optimum."""
import numpy as np

from ising_engine_b200 import instances as I
from oracle import oracle as O
from tests.test_pa_host import brute_force, random_qubo


def test_icm_keeps_energies_synced_and_moves():
    m = I.maxcut_gnm(80, 300, seed=2)
    temps = I.geometric_beta_ladder(4, 0.2, 2.0)
    sched = np.tile(temps, (40, 1))
    a = O.run_schedule(m, sched, 5, icm_every=10)
    b = O.run_schedule(m, sched, 5)
    assert np.array_equal(O.replica_energies(m, a.words), a.energies)
    assert not np.array_equal(a.words, b.words) and a.draws > b.draws
    c = O.run_schedule(m, sched, 5, icm_every=10)
    assert np.array_equal(a.words, c.words) and a.draws == c.draws
    f = random_qubo(60, 0.1, 4)
    r = O.run_schedule(f, np.tile([2.0, 0.7], (30, 1)), 9, icm_every=5)
    rec = O.replica_energies(f, r.words)
    assert np.allclose(rec, r.energies, rtol=0, atol=1e-9)


def test_solve_with_icm_reaches_optimum():
    """test_icm.rs:242-260 on the oracle."""
    for trial in range(3):
        m = random_qubo(12, 0.4, 40 + trial)
        a = O.solve(m, 10.0, 0.05, 5, 15, 300 + trial, use_icm=True)
        assert np.array_equal(a, O.solve(m, 10.0, 0.05, 5, 15, 300 + trial, use_icm=True))
        assert abs(m.calculate_total_energy(a) - brute_force(m)) < 1e-9

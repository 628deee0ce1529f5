"""UltimateSolver.solve end to end on the device with the reference's
presolve and decomposition (ultimate.rs:138-387): the returned state equals
the oracle's restatement of the whole solve bit for bit when presolve fixes
variables, when the free graph splits into components (each solved with
seed + index + 1) and with user clamps; population annealing behind the
same front end keeps the clamps and the fixings."""
import numpy as np
import pytest

from ising_engine_b200.presolve import full_presolve
from ising_engine_b200.solver import UltimateSolver
from oracle import oracle as O
from tests.test_pa_host import random_qubo
from tests.test_presolve_host import block_instance

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,integral", [(0, True), (1, False), (5, True)])
def test_decomposed_solve_equals_oracle(seed, integral):
    m = block_instance(seed, integral)
    for cl in ([], [(3, 1), (17, 0)]):
        ref = O.solve(m, 8.0, 0.1, 12, 10, 900 + seed, num_temps=6, clamped=cl, threads=8)
        s = UltimateSolver(8.0, 0.1, 12, 10, 900 + seed, num_temps=6)
        got = s.solve(m, cl)
        assert got.tolist() == ref.tolist()
        assert all(got[i] == v for i, v in cl)


@pytest.mark.parametrize("seed", [2, 7])
def test_single_component_with_fixings_equals_oracle(seed):
    m = random_qubo(60, 0.08, seed, integral=seed % 2 == 1)
    fix = full_presolve(m)
    ref = O.solve(m, 6.0, 0.05, 10, 12, seed, clamped=[], threads=8)
    got = UltimateSolver(6.0, 0.05, 10, 12, seed).solve(m)
    assert got.tolist() == ref.tolist()
    assert all(got[i] == v for i, v in fix)


def test_population_annealing_behind_presolve():
    m = block_instance(3)
    s = UltimateSolver(8.0, 0.1, 6, 8, 44).with_quantum_dims(1, 4, 2)
    cl = [(0, 1)]
    x = s.solve(m, cl)
    assert x[0] == 1
    for i, v in full_presolve(m, cl):
        assert x[i] == v
    assert x.tolist() == s.solve(m, cl).tolist()

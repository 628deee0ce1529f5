"""Isoenergetic cluster moves on the device against the oracle's
restatement of src/solver/icm.rs, through the C ABI: the PT loop with an ICM
sweep after every exchange block (ultimate.rs:304-336) leaves the same spin
words, tracked energies, swap statistics, stream position and incumbent bit
for bit (integer and f64 couplings, clamps, both PT paths); the whole solve
and population annealing with ICM return the oracle's states."""
import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.engine import Engine, geometric_temps
from ising_engine_b200.population_annealing import PaConfig
from ising_engine_b200.solver import UltimateSolver
from oracle import oracle as O
from tests.test_gpu_parity import assert_same_run
from tests.test_pa_host import random_qubo
from tests.test_presolve_host import block_instance

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", [1, 2])
@pytest.mark.parametrize("integral", [True, False])
def test_pt_loop_with_icm(path, integral):
    rng = np.random.default_rng(3)
    m = I.maxcut_gnm(300, 1500, seed=8) if integral else I.random_regular_qubo(200, 5, rng, integer=False)
    tmax, tmin, sweeps, exchanges, nt = 4.0, 0.2, 7, 9, 6
    temps = geometric_temps(tmax, tmin, nt)
    cl = np.zeros(m.num_vars, np.uint8)
    cl[[1, 50, 99]] = 1
    cv = np.zeros(m.num_vars, np.int8)
    cv[50] = 1
    ref = O.run_schedule(m, np.tile(temps, (sweeps * exchanges, 1)), 61, clamped=cl, clamp_val=cv,
                         incumbent_every=sweeps, icm_every=sweeps, collect_stats=True, threads=8)
    with Engine(m, num_temps=nt, seed=61, temp_max=tmax, temp_min=tmin, sweeps_per_exchange=sweeps,
                total_exchanges=exchanges, pt_path=path, use_icm=True) as eng:
        eng.set_clamps(cl, cv)
        eng.init_random()
        eng.run_pt()
        assert_same_run(eng, ref)
        inc_e, inc_s = eng.incumbent()
        assert inc_e == ref.incumbent_energy and (inc_s == ref.incumbent_state).all()


def test_solve_with_icm_equals_oracle():
    for m, seed in ((block_instance(2), 5), (random_qubo(50, 0.1, 6, integral=True), 6)):
        ref = O.solve(m, 8.0, 0.1, 6, 8, seed, num_temps=5, use_icm=True, threads=8)
        s = UltimateSolver(8.0, 0.1, 6, 8, seed, num_temps=5)
        s.use_icm = True
        assert s.solve(m).tolist() == ref.tolist()


def test_population_annealing_with_icm():
    from tests.test_gpu_pa import check_pa
    m = I.maxcut_gnm(120, 600, seed=12)
    check_pa(m, 4.0, 0.3, 3, 6, 71, 4, 2, PaConfig(ess_threshold=0.9, use_icm=True))

"""Population annealing with PT equilibration on the device (ie_run_pa)
against the oracle's restatement of ultimate.rs:576-852, through the C ABI:
the tuned ladder shape, every population's spin words and tracked energies,
the master-stream position, the ESS and family-entropy histories, the free
energy, the best member (before 1-opt) and the polished solution are equal
bit for bit, for integer and f64 couplings, odd and even ladders, clamps and
resampling at every stage. Then the reference's integration properties
(tests/test_population_annealing.rs:275-321, 595-725) on the device."""
import numpy as np
import pytest

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.engine import Engine
from ising_engine_b200.population_annealing import PaConfig
from ising_engine_b200.solver import UltimateSolver
from oracle import oracle as O
from tests.test_pa_host import brute_force, random_qubo

pytestmark = pytest.mark.gpu


def check_pa(m, tmax, tmin, sweeps, exchanges, seed, nt, pops, cfg, clamped=None, cval=None):
    ref = O.pa_run(m, tmax, tmin, sweeps, exchanges, seed, nt, pops, cfg.ess_threshold, cfg.ladder_tuning_iters,
                   cfg.ladder_tuning_steps, cfg.post_resample_relaxation, clamped=clamped, clamp_val=cval, threads=8,
                   ladder_mode=cfg.ladder_mode, use_icm=cfg.use_icm)
    with Engine(m, num_temps=nt, num_pops=pops, seed=seed, temp_max=tmax, temp_min=tmin,
                sweeps_per_exchange=sweeps, total_exchanges=exchanges) as eng:
        if clamped is not None:
            eng.set_clamps(clamped, cval)
        d = eng.run_pa(cfg)
        assert np.array_equal(d.alphas, ref["alphas"]), "tuned ladder shapes differ"
        w = eng.spins()
        bad = np.nonzero((w != ref["words"]).any(axis=1))[0]
        assert len(bad) == 0, f"spin words differ in cells {bad[:8]}"
        e = eng.energies()
        assert e.tobytes() == ref["energies"].tobytes(), np.argwhere(e != ref["energies"])[:8]
        assert eng.rng_state()[0] == ref["draws"]
        assert d.ess_history == ref["ess"].tolist()
        assert d.resample_events == ref["resamples"]
        assert [r for r, _ in d.family_entropy_history] == ref["rho"].tolist()
        assert [f for _, f in d.family_entropy_history] == ref["families"].tolist()
        assert d.free_energy == ref["free_energy"]
        inc_e, _ = eng.incumbent()
        assert inc_e == ref["incumbent"]
        _, best = eng.best()
        assert np.array_equal(best, ref["best_pre"])
        eng.one_opt(best, clamped)
        assert np.array_equal(best, ref["state"])
    return ref


def test_integer_maxcut_three_populations():
    m = I.maxcut_gnm(300, 2400, seed=21)
    ref = check_pa(m, 5.0, 0.2, 4, 10, 91, 6, 3, PaConfig(ess_threshold=0.9))
    assert ref["resamples"] >= 2


def test_odd_ladder_clamps_resample_every_stage():
    m = I.maxcut_gnm(120, 700, seed=4)
    cl = np.zeros(120, np.uint8)
    cv = np.zeros(120, np.int8)
    cl[[0, 9, 77, 119]] = 1
    cv[[9, 119]] = 1
    ref = check_pa(m, 4.0, 0.3, 3, 7, 5, 5, 2, PaConfig(ess_threshold=1.1, ladder_tuning_iters=3,
                                                         ladder_tuning_steps=4, post_resample_relaxation=2),
                   clamped=cl, cval=cv)
    assert ref["resamples"] == 6


def test_float_couplings_four_populations():
    m = random_qubo(200, 0.05, 8)
    check_pa(m, 6.0, 0.1, 3, 8, 33, 4, 4, PaConfig(ess_threshold=0.6, ladder_tuning_steps=6))


def test_two_level_ladder_without_tuning_and_one_stage():
    m = random_qubo(40, 0.3, 3, integral=True)
    check_pa(m, 3.0, 0.5, 5, 6, 12, 2, 2, PaConfig(ess_threshold=0.95))
    check_pa(m, 3.0, 0.5, 7, 1, 13, 3, 3, PaConfig())


@pytest.mark.parametrize("integral", [True, False])
def test_feedback_optimized_ladder(integral):
    """LadderMode::FeedbackOptimized: round-trip labels travel with the
    replicas through the exchanges, the flow histogram moves the ladder
    (enough tuning steps for round trips) — all bit for bit."""
    m = I.maxcut_gnm(150, 900, seed=6) if integral else random_qubo(100, 0.08, 6)
    ref = check_pa(m, 5.0, 0.5 if integral else 0.1, 3, 6, 17, 7, 2, PaConfig(ess_threshold=0.9, ladder_tuning_iters=4,
                                                         ladder_tuning_steps=120, ladder_mode=1))
    assert not np.allclose(ref["alphas"], np.arange(7) / 6)


def test_feedback_ladder_solver_optimal():
    """test_feedback_ladder.rs:108-131 on the device."""
    for trial in range(2):
        m = random_qubo(14, 0.4, 3 + trial)
        s = UltimateSolver(10.0, 0.05, 5, 15, 700 + trial).with_quantum_dims(1, 8, 2)
        s.ladder_mode = 1
        a = s.solve(m)
        assert np.array_equal(a, s.solve(m))
        assert abs(m.calculate_total_energy(a) - brute_force(m)) < 1e-9


def test_device_pa_finds_optimum_honors_clamps_is_deterministic():
    for trial in range(2):
        m = random_qubo(10, 0.4, 53 + trial)
        s = UltimateSolver(20.0, 0.05, 20, 40, 600 + trial)
        s.num_pops = 2
        x = s.solve(m)
        assert abs(m.calculate_total_energy(x) - brute_force(m)) < 1e-9
    m = random_qubo(12, 0.4, 57)
    s = UltimateSolver(20.0, 0.05, 20, 40, 4242).with_quantum_dims(1, 10, 2)
    a = s.solve(m, [(0, 1), (5, 0)])
    assert a[0] == 1 and a[5] == 0
    assert np.array_equal(a, s.solve(m, [(0, 1), (5, 0)]))


def test_diagnostics_and_relaxation():
    m = random_qubo(16, 0.5, 2001)
    s = UltimateSolver(20.0, 0.05, 5, 20, 555)
    s.num_pops = 3
    s.ess_threshold = 0.8
    x1, d1 = s.solve_with_pa_diagnostics(m)
    x2, d2 = s.solve_with_pa_diagnostics(m)
    assert np.array_equal(x1, x2) and d1.ess_history == d2.ess_history and d1.free_energy == d2.free_energy
    R = 3 * 64
    assert len(d1.ess_history) == 19 and all(1 - 1e-9 <= e <= R + 1e-9 for e in d1.ess_history)
    assert len(d1.family_entropy_history) == d1.resample_events >= 1
    # relaxation as the only equilibration improves on the random init
    m20 = random_qubo(20, 1.0, 223)

    def run(relax):
        s = UltimateSolver(20.0, 0.05, 0, 2, 31337).with_quantum_dims(1, 3, 2)
        s.ess_threshold = 1.1
        s.ladder_tuning_iters = 0
        s.post_resample_relaxation = relax
        return m20.calculate_total_energy(s.solve(m20))
    assert run(8) < run(0)


def test_pa_entry_errors():
    m = I.maxcut_gnm(30, 60, seed=1)
    with Engine(m, num_temps=4, seed=1) as eng:
        with pytest.raises(_ffi.EngineError, match="num_pops > 1"):
            eng.run_pa()
    with Engine(m, num_temps=4, num_pops=2, seed=1) as eng:
        with pytest.raises(_ffi.EngineError, match="ie_run_pa"):
            eng.run_pt()

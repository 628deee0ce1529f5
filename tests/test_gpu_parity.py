"""Parity of the CUDA path with the CPU oracle, through the C ABI.

Integer couplings: spin words, tracked energies, swap statistics, DEO phase
and master-stream position must be bit-identical after k steps. The f64 mode
runs the reference's f64 arithmetic in the reference's order, so the same
bit-identity is asserted there too on these cases; the FP64 recompute check
uses the stated relative tolerance 1e-6.
"""
import json
import os

import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.core import CsrMatrix, QuboModel
from ising_engine_b200.engine import BatchEngine, Engine, geometric_temps
from ising_engine_b200.solver import UltimateSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_REL_TOL = 1e-6
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "regression_golden.json")))


def assert_same_run(eng: Engine, ref, check_stats=True):
    w = eng.spins()
    assert w.shape == ref.words.shape
    bad = np.nonzero((w != ref.words).any(axis=1))[0]
    assert len(bad) == 0, f"spin words differ in cells {bad[:8]}"
    e = eng.energies()
    assert e.tobytes() == ref.energies.tobytes(), np.argwhere(e != ref.energies)[:8]
    draws, _ = eng.rng_state()
    assert draws == ref.draws
    if check_stats and eng.num_temps > 1:
        att, acc = eng.swap_stats()
        assert (att == ref.swap_attempts).all()
        assert (acc == ref.swap_accepts).all()


def assert_batch_energies(b: BatchEngine, models, ref_e, words=None):
    """Energies of a batched run. The level kernel (the default form) reports
    the FP64 recompute of the final state in the reference's order
    (engine.rs:333-368): bit-identical to the oracle's recompute of the same
    words, and within FP64_REL_TOL of the oracle's tracked sum (equal for
    integer couplings). The per-lane forms report the tracked sum itself."""
    e = b.energies()
    ref_e = np.asarray(ref_e).reshape(e.shape)
    if b.kernel_form == 1:
        assert e.tobytes() == ref_e.tobytes(), np.argwhere(e != ref_e)[:8]
        return
    w = b.spins() if words is None else words
    rec = np.stack([O.replica_energies(m, w[b.offsets[i]:b.offsets[i + 1]])[0] for i, m in enumerate(models)])
    assert e.tobytes() == rec.tobytes(), np.argwhere(e != rec)[:8]
    rel = np.abs(e - ref_e) / np.maximum(np.abs(ref_e), 1.0)
    assert rel.max() <= FP64_REL_TOL


def test_lattice_2d_single_cell_1000_sweeps():
    """2D periodic +-J, L=32, one cell at beta=1, random init, 1000 sweeps."""
    m = I.pm_j_lattice(32, 2, seed=2024)
    ref = O.run_schedule(m, np.ones((1000, 1)), 11)
    with Engine(m, num_temps=1, seed=11) as eng:
        eng.init_random()
        eng.step([1.0], 1000)
        assert_same_run(eng, ref)
    b = BatchEngine([m], [11])
    b.init_random()
    b.run_schedule(np.ones(1000))
    assert (b.spins() == ref.words.reshape(-1)).all()
    assert_batch_energies(b, [m], ref.energies)
    assert int(b.draws()[0]) == ref.draws
    b.close()


PT_PATHS = [1, 2]  # one CTA per instance; every cell its own work item


@pytest.mark.parametrize("path", PT_PATHS)
@pytest.mark.parametrize("interval", [1, 3])
def test_pt_maxcut_exchange(interval, path):
    m = I.maxcut_gnm(96, 700, seed=3)
    temps = I.geometric_beta_ladder(8, 0.1, 3.0)
    steps = 61
    ref = O.run_schedule(m, np.tile(temps, (steps, 1)), 77, exchange_interval=interval,
                         collect_stats=True)
    with Engine(m, num_temps=8, seed=77, exchange_interval=interval, pt_path=path) as eng:
        eng.init_random()
        eng.step(temps, 20)
        eng.step(temps, steps - 20)  # split calls continue the same trajectory
        assert_same_run(eng, ref)
        _, deo = eng.rng_state()
        assert deo == (steps // interval) % 2


@pytest.mark.parametrize("path", PT_PATHS)
def test_maxcut_800_pt32_interval10(path):
    """The G(n=800, m=19176) Max-Cut ladder: 32 temperatures, beta geometric
    0.1..3.0, exchange every 10 sweeps, 1000 of the 10^4 sweeps (the level
    kernel's cells; 100 on the one-CTA kernel, 10x slower)."""
    m = I.maxcut_gnm(800, 19176, seed=42)
    temps = I.geometric_beta_ladder(32, 0.1, 3.0)
    steps = 1000 if path == 2 else 100
    ref = O.run_schedule(m, np.tile(temps, (steps, 1)), 1337, exchange_interval=10,
                         collect_stats=True, threads=8)
    with Engine(m, num_temps=32, seed=1337, exchange_interval=10, pt_path=path) as eng:
        eng.init_random()
        eng.step(temps, steps)
        assert_same_run(eng, ref)


@pytest.mark.parametrize("path", PT_PATHS)
def test_clamped_sites_int_and_f64(path):
    rng = np.random.default_rng(9)
    for integer in (True, False):
        m = I.random_regular_qubo(60, 4, rng, integer=integer)
        clamped = np.zeros(60, np.uint8)
        clamped[[0, 7, 31, 59]] = 1
        cval = np.zeros(60, np.int8)
        cval[[0, 31]] = 1
        temps = [2.0, 1.0, 0.5, 0.25]
        ref = O.run_schedule(m, np.tile(temps, (40, 1)), 5, clamped=clamped, clamp_val=cval,
                             collect_stats=True)
        with Engine(m, num_temps=4, seed=5, pt_path=path) as eng:
            eng.set_clamps(clamped, cval)
            eng.init_random()
            eng.step(temps, 40)
            assert_same_run(eng, ref)


@pytest.mark.parametrize("path", PT_PATHS)
@pytest.mark.parametrize("hot,cold,seed,favourable", [(0, 1, 1, True), (1, 0, 2, False)])
def test_swap_statistics_known_answers(hot, cold, seed, favourable, path):
    """test_population_annealing.rs:354-420 on the device."""
    m = QuboModel(1, np.array([10.0]), CsrMatrix(np.zeros(0), np.zeros(0, np.uint64),
                                                 np.zeros(2, np.uint64)))
    with Engine(m, num_temps=2, seed=seed, pt_path=path) as eng:
        eng.set_clamps(np.ones(1, np.uint8), np.array([hot], np.int8))
        eng.set_spins(np.array([[~np.uint64(0) if hot else 0], [~np.uint64(0) if cold else 0]],
                               dtype=np.uint64))
        eng.step([2.0, 0.5], 1)
        rate = eng.swap_acceptance_rates()[0]
        draws, _ = eng.rng_state()
    if favourable:
        assert rate == 1.0 and draws == 1
    else:
        assert rate < 0.01 and draws == 65


@pytest.mark.parametrize("path", PT_PATHS)
def test_pt_float_couplings_resync_across_1000(path):
    """f64 PT with the step-1000 resync falling on an exchange step (interval
    5) and per-step ladders through run_schedule."""
    rng = np.random.default_rng(12)
    m = I.random_regular_qubo(300, 6, rng, integer=False)
    temps = I.geometric_beta_ladder(4, 0.3, 2.0)
    steps = 1003
    ref = O.run_schedule(m, np.tile(temps, (steps, 1)), 4, exchange_interval=5, collect_stats=True)
    with Engine(m, num_temps=4, seed=4, exchange_interval=5, pt_path=path) as eng:
        eng.init_random()
        eng.step(temps, 998)
        eng.step(temps, 5)
        assert_same_run(eng, ref)
    sched = np.stack([temps * (1.0 + 0.01 * k) for k in range(12)])
    ref = O.run_schedule(m, sched, 6, exchange_interval=2, collect_stats=True)
    with Engine(m, num_temps=4, seed=6, exchange_interval=2, pt_path=path) as eng:
        eng.init_random()
        eng.run_schedule(sched)
        assert_same_run(eng, ref)


def test_lattice_3d_cells_in_global_memory():
    """A 3D lattice too large for shared memory (L=32, N=32768): the cells run
    on the windowed kernel with spins in global memory (consecutive sites are
    coupled, so every window level holds one site)."""
    m = I.pm_j_lattice(32, 3, seed=8)
    temps = I.geometric_beta_ladder(4, 0.2, 2.0)
    ref = O.run_schedule(m, np.tile(temps, (7, 1)), 21, exchange_interval=5, collect_stats=True, threads=4)
    with Engine(m, num_temps=4, seed=21, exchange_interval=5, pt_path=2) as eng:
        eng.init_random()
        eng.step(temps, 7)
        assert_same_run(eng, ref)


def test_windowed_global_spins_random_graphs():
    """Single-cell instances beyond shared memory (N = 30000) on the windowed
    kernel with spins in global memory: random graphs (several sites per
    window level, neighbours inside the window and the previous one),
    integer and f64, through the batched entry point."""
    rng = np.random.default_rng(41)
    models = [small_weight_regular(30000, 12, rng), I.random_regular_qubo(26000, 7, rng, integer=False)]
    seeds = np.array([3, 4], dtype=np.uint64)
    temps = I.sa_temps(12, 0.3, 3.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=2)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps[:5])
    b.run_schedule(temps[5:])
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    b.close()


def test_lattice_3d_L64_64_temperatures_full_size():
    """The 3D +-J lattice at full size (L=64, N=262144, 64 temperatures, beta
    geometric 0.2..2.0, exchange every 5 sweeps) for 100 steps: spins,
    energies, swap statistics and stream position equal the oracle's."""
    m = I.pm_j_lattice(64, 3, seed=64)
    temps = I.geometric_beta_ladder(64, 0.2, 2.0)
    ref = O.run_schedule(m, np.tile(temps, (100, 1)), 99, exchange_interval=5, collect_stats=True, threads=16)
    with Engine(m, num_temps=64, seed=99, exchange_interval=5) as eng:
        eng.init_random()
        eng.step(temps, 40)
        eng.step(temps, 60)
        assert_same_run(eng, ref)


@pytest.mark.parametrize("integer", [True, False])
def test_one_opt_and_best_extraction_on_device(integer):
    """local_search.rs:19-57 on the device: the polished state and the total
    improvement equal the oracle's, with and without clamps; the best
    replica extraction returns a configuration whose model energy is the
    reported one."""
    rng = np.random.default_rng(31 if integer else 32)
    m = I.random_regular_qubo(700, 7, rng, integer=integer)
    with Engine(m, num_temps=3, seed=9) as eng:
        for trial in range(3):
            state = (rng.random(m.num_vars) < 0.5).astype(np.int8)
            clamped = (rng.random(m.num_vars) < 0.1).astype(np.uint8) if trial else None
            ref, ref_imp = O.one_opt(m, state, clamped, with_improvement=True)
            imp = eng.one_opt(state, clamped)
            assert (state == ref).all()
            assert imp == ref_imp
        eng.init_random()
        eng.step(I.geometric_beta_ladder(3, 0.5, 2.0), 30)
        e, s = eng.best()
        assert e == m.calculate_total_energy(s)


def test_uneven_batch_bit_exact_and_plain_equal():
    models, seeds = I.uneven_batch(24, seed=7, n_max=600)
    temps = I.sa_temps(60)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps)
    w = b.spins()
    e = b.energies()
    assert (w == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    assert (b.draws() == np.array([m.num_vars + 60 for m in models], np.uint64)).all()
    rec = b.recompute_energies()
    rel = np.abs(rec - e) / np.maximum(np.abs(rec), 1.0)
    assert rel.max() <= FP64_REL_TOL
    b.close()
    p = BatchEngine(models, seeds)
    p.init_random()
    p.run_schedule_plain(temps)
    assert p.last_launches() == len(models)
    assert (p.spins() == w).all()
    assert p.energies().tobytes() == e.tobytes()
    p.close()


def test_f64_resync_across_1000_steps():
    rng = np.random.default_rng(21)
    m = I.random_regular_qubo(48, 6, rng, integer=False)
    temps = I.sa_temps(1003, 0.2, 2.0)
    ref = O.run_schedule(m, temps, 31)
    with Engine(m, num_temps=1, seed=31) as eng:
        eng.init_random()
        eng.run_schedule(temps)
        assert_same_run(eng, ref)
    b = BatchEngine([m], [31])
    b.init_random()
    b.run_schedule(temps)
    assert (b.spins() == ref.words.reshape(-1)).all()
    assert_batch_energies(b, [m], ref.energies)
    b.close()


def test_forced_f64_equals_integer_mode():
    m = I.pm_j_lattice(8, 2, seed=4)
    temps = I.geometric_beta_ladder(4, 0.3, 1.5)
    out = []
    for f in (False, True):
        with Engine(m, num_temps=4, seed=8, force_f64=f) as eng:
            eng.init_random()
            eng.step(temps, 50)
            out.append((eng.spins(), eng.energies(), eng.rng_state(), eng.swap_stats()))
    assert (out[0][0] == out[1][0]).all()
    assert out[0][1].tobytes() == out[1][1].tobytes()
    assert out[0][2] == out[1][2]
    assert all((a == b).all() for a, b in zip(out[0][3], out[1][3]))


def test_golden_pt_trajectory_and_solve():
    """UltimateSolver(50, 0.05, 30, 40, 2024) on the golden n=32 float
    instance: the device PT loop matches the oracle step for step, and the
    full solve returns the reference's golden state."""
    lin, row, col, val = O.golden_instance()
    m = QuboModel(32, lin, CsrMatrix(val, col.astype(np.uint64), row.astype(np.uint64)))
    s = GOLDEN["solver"]
    temps = geometric_temps(s["temp_max"], s["temp_min"], s["num_temps"])
    steps = s["sweeps"] * s["exchanges"]
    ref = O.run_schedule(m, np.tile(temps, (steps, 1)), s["seed"], incumbent_every=s["sweeps"],
                         collect_stats=True)
    solver = UltimateSolver(s["temp_max"], s["temp_min"], s["sweeps"], s["exchanges"], s["seed"])
    with solver.engine(m) as eng:
        eng.init_random()
        eng.run_pt()
        assert_same_run(eng, ref)
        inc_e, inc_s = eng.incumbent()
        assert inc_e == ref.incumbent_energy
        assert (inc_s == ref.incumbent_state).all()
    state = solver.solve(m)
    assert state.tolist() == GOLDEN["golden_state"]
    assert abs(m.calculate_total_energy(state) - GOLDEN["golden_energy"]) < GOLDEN["energy_tolerance"]


def test_batch_long_rows_and_thread_classes():
    """Rows longer than one record (> 16 couplings) and instances of every
    size class (1, 2 and 4 threads per generator lane) in one batch."""
    rng = np.random.default_rng(33)
    models = [I.maxcut_gnm(160, 2600, seed=4),                       # degree ~32, integer
              I.random_regular_qubo(300, 20, rng, integer=False),    # degree 20, f64
              I.random_regular_qubo(260, 18, rng, integer=True)]
    models += [I.random_regular_qubo(int(n), 6, rng, integer=bool(i % 2))
               for i, n in enumerate(rng.integers(40, 200, size=13) * 2)]
    seeds = np.arange(len(models), dtype=np.uint64) * 7 + 3
    temps = I.sa_temps(30, 0.2, 3.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps[:11])
    b.run_schedule(temps[11:])
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    b.close()


@pytest.mark.parametrize("bulk", [False, True])
def test_per_lane_record_ring_forms(bulk):
    """The per-lane kernels (kernel_form 1) with the site-record ring fed by
    16-byte cp.async copies or by 1D bulk copies on mbarriers: spins and
    energies equal the oracle's for rows longer than one record, every thread
    class and lattices (the chain kernel)."""
    rng = np.random.default_rng(35)
    models = [I.maxcut_gnm(160, 2600, seed=5), I.random_regular_qubo(300, 20, rng, integer=False),
              I.pm_j_lattice(32, 2, seed=6), I.pm_j_lattice(12, 3, seed=8)]
    models += [I.random_regular_qubo(int(n), 6, rng, integer=bool(i % 2))
               for i, n in enumerate(rng.integers(40, 700, size=9) * 2)]
    seeds = np.arange(len(models), dtype=np.uint64) * 5 + 1
    temps = I.sa_temps(25, 0.2, 3.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds, kernel_form=1, bulk_ring=bulk)
    b.init_random()
    b.run_schedule(temps[:9])
    b.run_schedule(temps[9:])
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    b.close()


def test_autotune_restores_state():
    """The autotuner's trial runs leave no trace: after tuning, the run equals
    the oracle's from the same initial state."""
    models, seeds = I.uneven_batch(20, seed=99, n_max=900)
    temps = I.sa_temps(24)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds)
    b.init_random()
    chosen = b.autotune(temps, 4)
    assert len(chosen) == 4
    b.run_schedule(temps)
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    assert (b.draws() == np.array([m.num_vars + 24 for m in models], np.uint64)).all()
    b.close()


def test_windowed_kernel_large_instances():
    """Large random-regular instances take the windowed kernel (generator
    phase + level-ordered decisions per window of 8 sites); a large lattice
    (consecutive sites coupled) stays on the per-lane kernel. Both bit-exact."""
    rng = np.random.default_rng(77)
    models = [I.random_regular_qubo(1700, 12, rng, integer=True),
              I.random_regular_qubo(1600, 3, rng, integer=True),
              I.random_regular_qubo(900, 16, rng, integer=False),
              I.random_regular_qubo(2100, 5, rng, integer=False),
              I.pm_j_lattice(48, 2, seed=5)]
    seeds = np.arange(len(models), dtype=np.uint64) + 11
    temps = I.sa_temps(30, 0.2, 4.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps[:13])
    b.run_schedule(temps[13:])
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    b.close()


def small_weight_regular(n, d, rng):
    """Random d-regular QUBO with couplings in {-2, -1, 1, 2}: local fields stay
    within the integer mode's bound at degrees up to 32."""
    e = I.random_regular_edges(n, d, rng)
    q = rng.choice(np.array([-2.0, -1.0, 1.0, 2.0]), size=len(e))
    lin = rng.integers(-4, 5, size=n).astype(np.float64)
    return QuboModel.from_edges(n, lin, np.concatenate([e.astype(np.float64), q[:, None]], axis=1))


def test_windowed_kernel_degree_17_to_32():
    """Sites with 17..32 couplings: the windowed kernel reads its own stream of
    one record per site (the batched kernels split such sites into
    continuation records). Integer and f64 modes, and a clamped instance."""
    rng = np.random.default_rng(79)
    models = [small_weight_regular(2000, 24, rng), small_weight_regular(1800, 32, rng),
              I.random_regular_qubo(1600, 32, rng, integer=False),
              I.random_regular_qubo(1000, 20, rng, integer=False)]
    assert models[0].is_integral()
    seeds = np.arange(len(models), dtype=np.uint64) + 21
    temps = I.sa_temps(25, 0.2, 4.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps)
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    b.close()


def test_batched_runs_replayed_from_cuda_graph():
    """use_graph: the class launches are captured once and replayed; the step
    base comes from device memory, so replays continue the trajectory (the
    f64 resync at step 1000 falls inside the second replay), and a run of a
    different length is captured again."""
    rng = np.random.default_rng(52)
    models = [I.random_regular_qubo(1800, 9, rng, integer=False), I.random_regular_qubo(900, 6, rng, integer=True),
              I.random_regular_qubo(300, 4, rng, integer=False), I.random_regular_qubo(120, 5, rng, integer=True)]
    seeds = np.arange(len(models), dtype=np.uint64) + 61
    temps = I.sa_temps(1250, 0.2, 3.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds, graph=True)
    b.init_random()
    b.run_schedule(temps[:600])
    b.run_schedule(temps[600:1200])
    b.run_schedule(temps[1200:])
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, models, ref_e)
    assert len(b.class_report()) >= 2 and all(c[4] > 0 for c in b.class_report())
    b.close()


def test_windowed_kernel_f64_resync():
    rng = np.random.default_rng(78)
    m = I.random_regular_qubo(800, 9, rng, integer=False)
    temps = I.sa_temps(1002, 0.2, 3.0)
    words_ref, _, ref_e = O.run_sa_batch([m], [5], temps, threads=1)
    b = BatchEngine([m], [5])
    b.init_random()
    b.run_schedule(temps)
    assert (b.spins() == words_ref).all()
    assert_batch_energies(b, [m], ref_e)
    b.close()

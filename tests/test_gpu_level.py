"""The level kernel against the oracle, through the C ABI.

The level kernel generates every lane's stream in segments (GF(2) jumps) and
decides the sites level by level; spins and stream positions must equal the
oracle's site-order sweep bit for bit, energies the FP64 recompute of the
final state (integer couplings: the tracked sum itself).
"""
import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.engine import BatchEngine, Engine
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_REL_TOL = 1e-6


def check_batch(b, models, words_ref, ref_e):
    w = b.spins()
    bad = [i for i in range(len(models)) if (w[b.offsets[i]:b.offsets[i + 1]] !=
                                             words_ref[b.offsets[i]:b.offsets[i + 1]]).any()]
    assert not bad, f"spin words differ in instances {bad[:8]}"
    e = b.energies()
    rec = np.stack([O.replica_energies(m, w[b.offsets[i]:b.offsets[i + 1]])[0] for i, m in enumerate(models)])
    assert e.tobytes() == rec.tobytes()
    rel = np.abs(e - ref_e) / np.maximum(np.abs(ref_e), 1.0)
    assert rel.max() <= FP64_REL_TOL


def log_uniform_batch(count, n_lo, n_hi, seed):
    rng = np.random.default_rng(seed)
    models = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        d = int(rng.integers(3, 17))
        if (n * d) % 2:
            n += 1
        models.append(I.random_regular_qubo(n, d, rng, integer=(i % 2 == 0)))
    seeds = rng.integers(0, 2**63, size=count, dtype=np.int64).astype(np.uint64)
    return models, seeds


def test_log_uniform_batch_100_sweeps():
    """64 instances, N log-uniform in [64, 4096], degree 3..16, integer and
    f32 couplings alternating, SA beta 0.1 -> 5.0 over 100 sweeps."""
    models, seeds = log_uniform_batch(64, 64, 4096, 2031)
    temps = I.sa_temps(100)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=16)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps[:37])
    b.run_schedule(temps[37:])
    check_batch(b, models, words_ref, ref_e)
    assert (b.draws() == np.array([m.num_vars + 100 for m in models], np.uint64)).all()
    b.close()


def test_exact_path_under_forced_ties():
    """tie_shift 24 makes one uphill decision in 256 undecided from the
    stored bits, so the exact path (output recomputed from the lane's seed and
    segment jump) runs thousands of times; the run is still the oracle's."""
    models, seeds = log_uniform_batch(16, 64, 1500, 77)
    temps = I.sa_temps(30, 0.1, 2.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds, tie_shift=24)
    b.init_random()
    b.run_schedule(temps)
    check_batch(b, models, words_ref, ref_e)
    assert b.exact_decisions() > 1000
    b.close()


def test_item_sizes_and_forms_agree():
    """Different item capacities (members per CTA) and the per-lane kernels
    give the same spins."""
    models, seeds = log_uniform_batch(40, 32, 2500, 5)
    temps = I.sa_temps(20, 0.3, 3.0)
    out = []
    for kw in [dict(item_sites=512), dict(item_sites=16384), dict(kernel_form=1)]:
        b = BatchEngine(models, seeds, **kw)
        b.init_random()
        b.run_schedule(temps)
        out.append(b.spins())
        b.close()
    assert (out[0] == out[1]).all()
    assert (out[0] == out[2]).all()


def test_plain_launches_equal_batched():
    models, seeds = log_uniform_batch(10, 64, 3000, 9)
    temps = I.sa_temps(25)
    b = BatchEngine(models, seeds)
    b.init_random()
    b.run_schedule(temps)
    p = BatchEngine(models, seeds)
    p.init_random()
    p.run_schedule_plain(temps)
    assert p.last_launches() == len(models)
    assert (p.spins() == b.spins()).all()
    assert p.energies().tobytes() == b.energies().tobytes()
    b.close()
    p.close()


@pytest.mark.parametrize("L,dim,nt,steps,interval", [(32, 2, 1, 300, 1), (12, 3, 8, 40, 5), (24, 2, 16, 30, 1)])
def test_lattice_ladders_on_level_cells(L, dim, nt, steps, interval):
    """+-J lattices (sequential site chains, depth ~ dim * L levels) as PT
    cells of the level kernel, all in flight and one launch per cell: spins,
    energies, swap statistics and stream position equal the oracle's; the
    per-lane kernels agree."""
    m = I.pm_j_lattice(L, dim, seed=L + dim)
    temps = I.geometric_beta_ladder(nt, 0.3, 1.5) if nt > 1 else np.ones(1)
    ref = O.run_schedule(m, np.tile(temps, (steps, 1)), 5, exchange_interval=interval, collect_stats=True,
                         threads=8)
    for form, path in ((0, 2), (0, 3), (1, 2)):
        with Engine(m, num_temps=nt, seed=5, exchange_interval=interval, pt_path=path, kernel_form=form) as eng:
            eng.init_random()
            eng.step(temps, steps)
            assert (eng.spins() == ref.words).all()
            assert eng.energies().tobytes() == ref.energies.tobytes()
            assert eng.rng_state()[0] == ref.draws
            if nt > 1:
                att, acc = eng.swap_stats()
                assert (att == ref.swap_attempts).all() and (acc == ref.swap_accepts).all()


def pm_j_regular(n, d, c, rng):
    """Random d-regular graph with couplings +-c and lin_v = -sum_j w_vj / 2:
    the Ising lowering of a +-J spin glass, the level kernel's bit-sliced
    form (odd d with even c, or any d)."""
    from ising_engine_b200.core import QuboModel
    e = I.random_regular_edges(n, d, rng)
    w = (c * rng.choice(np.array([-1, 1]), size=len(e))).astype(np.float64)
    lin = np.zeros(n)
    np.add.at(lin, e[:, 0], -w / 2)
    np.add.at(lin, e[:, 1], -w / 2)
    return QuboModel.from_edges(n, lin, np.concatenate([e.astype(np.float64), w[:, None]], axis=1), 0.0)


def test_bit_sliced_pm_j_form_batch():
    """+-J instances (lattices and random regular graphs of degree 3..8, one
    coupling magnitude) run on the bit-sliced form, one thread per site for
    all 64 replicas; spins, energies and stream positions equal the oracle's,
    with clamps too."""
    rng = np.random.default_rng(404)
    models = [I.pm_j_lattice(16, 2, seed=1), I.pm_j_lattice(8, 3, seed=2), I.pm_j_lattice(40, 2, seed=3)]
    models += [pm_j_regular(n, d, 2, rng) for n, d in [(300, 3), (500, 5), (240, 7), (1000, 8), (5000, 4)]]
    seeds = np.arange(len(models), dtype=np.uint64) * 31 + 7
    temps = I.sa_temps(80, 0.2, 3.0)
    words_ref, _, ref_e = O.run_sa_batch(models, seeds, temps, threads=8)
    b = BatchEngine(models, seeds, bit_sliced=1)
    b.init_random()
    b.run_schedule(temps[:33])
    b.run_schedule(temps[33:])
    check_batch(b, models, words_ref, ref_e)
    assert any(c[0] == "pmj" for c in b.class_report())
    b.close()
    m = I.pm_j_lattice(24, 2, seed=9)
    f = np.zeros(m.num_vars, np.uint8)
    f[::7] = 1
    v = (np.arange(m.num_vars) % 3 == 0).astype(np.int8)
    temps = I.geometric_beta_ladder(6, 0.3, 1.5)
    ref = O.run_schedule(m, np.tile(temps, (25, 1)), 3, clamped=f, clamp_val=v, collect_stats=True)
    with Engine(m, num_temps=6, seed=3, pt_path=2, bit_sliced=1) as eng:
        eng.set_clamps(f, v)
        eng.init_random()
        eng.step(temps, 25)
        assert (eng.spins() == ref.words).all()
        assert eng.energies().tobytes() == ref.energies.tobytes()

"""Population annealing host logic (no GPU): the library's reweighting and
resampling primitives against the reference's contract tests
(tests/test_population_annealing.rs:26-138, 326-346, 653-687) and, bit for
bit, against the oracle's restatement; rand 0.8.5's gen_range(0..=k) in the
oracle pinned against raw ChaCha8 draws; the oracle's PA-PT driver
(ultimate.rs:576-852) on the reference's integration properties."""
import itertools
import math

import numpy as np
import pytest

from ising_engine_b200 import population_annealing as P
from ising_engine_b200.core import CsrMatrix, QuboModel
from oracle import oracle as O


def test_weights_follow_boltzmann_ratios():
    w = P.normalized_weights([-0.7 * e for e in (0.0, 1.0, 2.0)])
    assert abs(w.sum() - 1.0) < 1e-12
    assert abs(w[1] / w[0] - math.exp(-0.7)) < 1e-12
    assert abs(w[2] / w[1] - math.exp(-0.7)) < 1e-12


def test_lse_normalization_is_stable_at_extreme_energies():
    w = P.normalized_weights([-2.0e6, -2.0e6 + 1.0, -3.0e6])
    assert np.isfinite(w).all() and abs(w.sum() - 1.0) < 1e-12
    assert w[2] < 1e-300
    assert abs(w[0] / w[1] - math.exp(-1.0)) < 1e-9


def test_ess_bounds_and_exact_values():
    r = 64
    assert abs(P.effective_sample_size(np.full(r, 1.0 / r)) - r) < 1e-9
    d = np.zeros(r)
    d[3] = 1.0
    assert abs(P.effective_sample_size(d) - 1.0) < 1e-12
    two = np.zeros(r)
    two[:2] = 0.5
    assert abs(P.effective_sample_size(two) - 2.0) < 1e-12


def example_weights(r, seed):
    raw = np.random.default_rng(seed).uniform(0.01, 1.0, size=r)
    return raw / raw.sum()


def test_systematic_resample_conserves_size_and_bounds_counts():
    r = 128
    w = example_weights(r, 5)
    for m in range(50):
        c = P.systematic_resample(w, (m + 0.5) / 50)
        assert c.sum() == r
        assert (np.abs(c - r * w) < 1.0 + 1e-9).all()


def test_systematic_resample_is_unbiased_over_the_offset():
    r, grid = 64, 2000
    w = example_weights(r, 9)
    mean = sum(P.systematic_resample(w, (m + 0.5) / grid) for m in range(grid)) / grid
    assert (np.abs(mean - r * w) < 2e-3).all()


def test_adapt_spacings():
    sp = [0.1, 0.3, 0.2, 0.4]
    assert np.allclose(P.adapt_spacings(sp, [0.3] * 4), sp, atol=1e-12, rtol=0)
    out = P.adapt_spacings([0.5, 0.5], [0.9, 0.1])
    assert out[0] > 0.5 and out[1] < 0.5 and abs(out.sum() - 1.0) < 1e-12
    # the 0.02 acceptance floor
    assert np.array_equal(P.adapt_spacings([0.5, 0.5], [0.0, 0.02]), np.array([0.5, 0.5]))


def test_free_energy_and_family_entropy():
    assert abs(P.free_energy_increment([0.7] * 64) - 0.7) < 1e-12
    assert abs(P.free_energy_increment([0.0, math.log(3.0)]) - math.log(2.0)) < 1e-12
    assert abs(P.free_energy_increment([-1.0e6, -1.0e6]) + 1.0e6) < 1e-3
    assert P.free_energy_increment([-math.inf] * 3) == 0.0
    rho, f = P.family_entropy(range(64))
    assert abs(rho - 1.0) < 1e-12 and f == 64
    rho, f = P.family_entropy([7] * 64)
    assert abs(rho - 64.0) < 1e-12 and f == 1
    rho, f = P.family_entropy([i % 2 for i in range(64)])
    assert abs(rho - 32.0) < 1e-12 and f == 2


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_primitives_equal_the_oracle_bitwise(seed):
    rng = np.random.default_rng(seed)
    lw = rng.normal(scale=30.0, size=192)
    w = P.normalized_weights(lw)
    assert np.array_equal(w, O.pa_normalized_weights(lw))
    for u in rng.random(20):
        assert np.array_equal(P.systematic_resample(w, u), O.pa_systematic_resample(w, u))


def test_gen_index_inclusive_pinned_to_raw_draws():
    """rand 0.8.5 sample_single_inclusive(0, hi) for usize, replayed on the raw
    ChaCha8 draws with Python integers: range = hi + 1, zone = (range <<
    leading_zeros(range)) - 1 (2^63 - 1 for a power of two), a draw v is kept
    when (v * range) mod 2^64 <= zone and gives (v * range) >> 64."""
    his = [2 ** k - 1 for k in range(1, 40)] + list(range(1, 300)) + [3 * 2 ** 61, 2 ** 63 + 5]
    vals, draws = O.gen_index_inclusive(5, his)
    assert all(0 <= int(v) <= h for v, h in zip(vals, his))
    raw = O.chacha8_u64(5, draws)
    k = 0
    for h, v in zip(his, vals):
        rng_ = h + 1
        zone = (rng_ << (64 - rng_.bit_length())) - 1
        while True:
            m = int(raw[k]) * rng_
            k += 1
            if m & (2 ** 64 - 1) <= zone:
                assert m >> 64 == int(v)
                break
    assert k == draws > len(his)


def random_qubo(n, density, seed, integral=False):
    rng = np.random.default_rng(seed)
    up = np.triu(rng.uniform(-2, 2, size=(n, n)) * (rng.random((n, n)) < density), 1)
    if integral:
        up = np.round(up * 3)
    q = up + up.T
    ro, ci, va = [0], [], []
    for i in range(n):
        for j in range(n):
            if i != j and q[i, j] != 0:
                ci.append(j)
                va.append(q[i, j])
        ro.append(len(ci))
    lin = rng.uniform(-2, 2, size=n)
    if integral:
        lin = np.round(lin * 3)
    return QuboModel(n, lin, CsrMatrix(np.array(va), np.array(ci, dtype=np.uint64), np.array(ro, dtype=np.uint64)),
                     0.0)


def brute_force(m, fixed=()):
    best = math.inf
    for bits in itertools.product((0, 1), repeat=m.num_vars):
        x = np.array(bits, dtype=np.int8)
        if any(x[i] != v for i, v in fixed):
            continue
        best = min(best, m.calculate_total_energy(x))
    return best


def test_oracle_pa_finds_optimum_honors_clamps_and_is_deterministic():
    """test_population_annealing.rs:275-321 on the oracle (its instances are
    generated here)."""
    for trial in range(3):
        m = random_qubo(10, 0.4, 53 + trial)
        r = O.pa_run(m, 20.0, 0.05, 20, 40, 600 + trial, 10, 2, threads=4)
        assert abs(m.calculate_total_energy(r["state"]) - brute_force(m)) < 1e-9
    m = random_qubo(12, 0.4, 57)
    cl = np.zeros(12, np.uint8)
    cv = np.zeros(12, np.int8)
    cl[[0, 5]] = 1
    cv[0] = 1
    a = O.pa_run(m, 20.0, 0.05, 20, 40, 4242, 10, 2, clamped=cl, clamp_val=cv, threads=4)
    assert a["state"][0] == 1 and a["state"][5] == 0
    b = O.pa_run(m, 20.0, 0.05, 20, 40, 4242, 10, 2, clamped=cl, clamp_val=cv, threads=4)
    assert np.array_equal(a["state"], b["state"]) and a["draws"] == b["draws"]


def test_oracle_pa_diagnostics():
    """test_population_annealing.rs:689-725: ESS per stage after the first,
    in [1, R]; one (rho, families) per resampling event."""
    m = random_qubo(16, 0.5, 2001)
    r = O.pa_run(m, 20.0, 0.05, 5, 20, 555, 10, 3, ess_threshold=0.8, threads=4)
    R = 3 * 64
    assert len(r["ess"]) == 19
    assert ((r["ess"] >= 1 - 1e-9) & (r["ess"] <= R + 1e-9)).all()
    assert r["resamples"] == len(r["rho"]) >= 1
    assert ((r["rho"] >= 1 - 1e-6) & (r["rho"] <= R + 1e-6)).all() and (r["families"] >= 1).all()
    a = r["alphas"]
    assert a[0] == 0.0 and a[-1] == 1.0 and (np.diff(a) > 0).all()


def test_feedback_optimized_alphas():
    """test_feedback_ladder.rs:11-59 on the library's function, and bit for
    bit against the oracle's on random profiles."""
    nt = 8
    a = np.arange(nt) / (nt - 1)
    out = P.feedback_optimized_alphas(a, a.copy(), 1.0)
    assert np.allclose(out, a, atol=1e-9, rtol=0)
    nt = 9
    a = np.arange(nt) / (nt - 1)
    flow = 1.0 / (1.0 + np.exp(-20.0 * (a - 0.5)))
    out = P.feedback_optimized_alphas(a, flow, 1.0)
    c = nt // 2
    assert out[c] - out[c - 1] < out[1] - out[0]
    assert abs(out[0]) < 1e-9 and abs(out[-1] - 1.0) < 1e-9 and (np.diff(out) > 0).all()
    rng = np.random.default_rng(8)
    for k in (2, 3, 5, 12):
        a = np.sort(rng.random(k))
        f = rng.random(k)
        for damp in (0.5, 1.0):
            assert np.array_equal(P.feedback_optimized_alphas(a, f, damp), O.pa_feedback_alphas(a, f, damp))
    assert np.array_equal(P.feedback_optimized_alphas([0, 0.5, 1], [0, 0, 0], 0.5),
                          O.pa_feedback_alphas([0, 0.5, 1], [0, 0, 0], 0.5))


def test_oracle_feedback_ladder_solver():
    """test_feedback_ladder.rs:108-131 on the oracle: deterministic, reaches
    the exhaustive optimum, and the tuned ladder moved off the geometric one."""
    for trial in range(3):
        m = random_qubo(14, 0.4, 3 + trial)
        a = O.pa_run(m, 10.0, 0.05, 5, 15, 700 + trial, 8, 2, ladder_mode=1, threads=4)
        b = O.pa_run(m, 10.0, 0.05, 5, 15, 700 + trial, 8, 2, ladder_mode=1, threads=4)
        assert np.array_equal(a["state"], b["state"]) and a["draws"] == b["draws"]
        assert abs(m.calculate_total_energy(a["state"]) - brute_force(m)) < 1e-9
    # 10 tuning steps per iteration give fewer round trips than levels (the
    # shape stays geometric, ultimate.rs:662-669); 120 steps move it
    assert np.array_equal(a["alphas"], np.arange(8) / 7)
    c = O.pa_run(m, 10.0, 0.05, 5, 15, 9, 8, 2, tuning_steps=120, ladder_mode=1, threads=4)
    assert not np.allclose(c["alphas"], np.arange(8) / 7)
    assert c["alphas"][0] == 0.0 and c["alphas"][-1] == 1.0 and (np.diff(c["alphas"]) > 0).all()

"""engine_v2 (S2) on the device against the oracle's restatement, through
the C ABI: planes, ledger energies, (proposed, accepted) per operator and
stream positions equal after sequences of MetropolisSweep, GibbsColorSweep
and ReplicaExchange applications; the audit finds no drift (integer state)."""
import numpy as np
import pytest

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.v2 import (ChaChaStream, GibbsColorSweep, GpuBitSlice, MetropolisSweep, ProblemIR,
                                  ReplicaExchange)
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def frustrated():
    return ProblemIR.from_pairs(7, -2.0, [1.0, -2.0, 3.0, 0.0, -1.0, 2.0, 1.0],
                                [(0, 1, -1.0), (1, 2, 2.0), (2, 3, -3.0), (0, 3, 1.0), (3, 4, -1.0),
                                 (4, 5, 2.0), (5, 6, -2.0), (2, 6, 1.0)])


def run_gpu(ir, r, init, seed, ops, temps, skip=0):
    st = GpuBitSlice(ir, r, init)
    rng = ChaChaStream(seed, skip)
    stats = []
    for kind, count in ops:
        op = {"metropolis": MetropolisSweep, "exchange": ReplicaExchange, "gibbs": GibbsColorSweep}[kind]()
        rep = op.apply(st, temps, rng, count)
        stats.append((rep.proposed, rep.accepted))
    out = st.planes(), st.energies(), stats, st.audit(), rng.position
    st.close()
    return out


def check(ir, r, init, seed, ops, temps, skip=0):
    pl, en, stt, drift, pos = run_gpu(ir, r, init, seed, ops, temps, skip)
    rpl, ren, rst, rdrift, rpos = O.v2_program(ir.model(), r, init, seed, ops, temps, skip_draws=skip)
    assert (pl == rpl).all(), "planes differ"
    assert en.tolist() == ren.tolist(), "energies differ"
    assert stt == rst and pos == rpos
    assert drift == 0.0 and rdrift == 0.0


def test_reference_identical_on_both_backends_case():
    """metropolis_sweep.rs:174-214: r = 100, temps 0.2 + 0.05 k, 30 sweeps."""
    r = 100
    check(frustrated(), r, np.array([1, 0, 1, 0, 0, 1, 0], np.uint8), 11, [("metropolis", 30)],
          [0.2 + 0.05 * k for k in range(r)])


@pytest.mark.parametrize("r", [64, 130, 33])
def test_metropolis_and_exchange_sequences(r):
    m = I.maxcut_gnm(300, 2400, seed=5)
    ir = ProblemIR.from_model(m)
    assert ir.is_integral()
    init = (np.random.default_rng(r).random(ir.n) < 0.5).astype(np.uint8)
    temps = list(I.geometric_beta_ladder(r, 0.1, 3.0))
    ops = [("metropolis", 12), ("exchange", 3), ("metropolis", 7), ("exchange", 2), ("metropolis", 1)]
    check(ir, r, init, 7, ops, temps, skip=5)


def test_lattice_short_ladder_and_zero_temperature():
    m = I.pm_j_lattice(12, 2, seed=3)
    ir = ProblemIR.from_model(m)
    init = np.zeros(ir.n, np.uint8)
    check(ir, 96, init, 3, [("metropolis", 20), ("exchange", 4)], [2.0, 1.0, 0.5])
    check(ir, 40, init, 4, [("metropolis", 5)], [0.0, 0.7])  # T = 0: pure descent


def test_gibbs_reference_case_and_scorer():
    """gibbs_color_sweep.rs:197-252: r = 100, temps 0.2 + 0.05 k, 30 sweeps,
    seed 7; every replica's ledger energy equals ProblemIR::energy of its
    extracted configuration."""
    ir = frustrated()
    r = 100
    init = np.array([1, 0, 1, 0, 0, 1, 0], np.uint8)
    temps = [0.2 + 0.05 * k for k in range(r)]
    check(ir, r, init, 7, [("gibbs", 30)], temps)
    st = GpuBitSlice(ir, r, init)
    GibbsColorSweep().apply(st, temps, ChaChaStream(7), 30)
    en = st.energies()
    for k in range(r):
        assert ir.energy(st.extract(k)) == en[k]
    st.close()


@pytest.mark.parametrize("r", [64, 97])
def test_gibbs_sequences_and_special_temperatures(r):
    m = I.maxcut_gnm(400, 3000, seed=9)
    ir = ProblemIR.from_model(m)
    init = (np.random.default_rng(r + 1).random(ir.n) < 0.5).astype(np.uint8)
    temps = list(I.geometric_beta_ladder(r - 6, 0.2, 4.0)) + [0.0, -1.0, float("nan"), float("inf"), 1e-300, 0.01]
    ops = [("gibbs", 6), ("exchange", 2), ("metropolis", 3), ("gibbs", 4)]
    check(ir, r, init, 13, [("gibbs", 6)], temps, skip=3)
    finite = [t for t in temps if t > 0.0 and np.isfinite(t)]
    check(ir, r, init, 13, ops, finite)


def test_gibbs_cold_is_monotone_descent():
    """gibbs_color_sweep.rs:255-291."""
    ir = frustrated()
    st = GpuBitSlice(ir, 8, np.zeros(7, np.uint8))
    e0 = st.energies()
    GibbsColorSweep().apply(st, [1e-9] * 8, ChaChaStream(1), 5)
    assert (st.energies() <= e0).all() and st.audit() == 0.0
    st.close()


def test_rejects_non_integral():
    ir = ProblemIR.from_pairs(3, 0.0, [0.5, 0.0, 0.0], [(0, 1, 1.0)])
    with pytest.raises(_ffi.EngineError, match="IE_ERR_INVALID"):
        GpuBitSlice(ir, 8, np.zeros(3, np.uint8))

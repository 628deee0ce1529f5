"""engine_v2 (S2) on the device against the oracle's restatement, through
the C ABI: planes, ledger energies, (proposed, accepted) per operator and
stream positions equal after sequences of MetropolisSweep and
ReplicaExchange applications; the audit finds no drift (integer state)."""
import numpy as np
import pytest

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.v2 import ChaChaStream, GpuBitSlice, MetropolisSweep, ProblemIR, ReplicaExchange
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
        op = MetropolisSweep() if kind == "metropolis" else ReplicaExchange()
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


def test_rejects_non_integral():
    ir = ProblemIR.from_pairs(3, 0.0, [0.5, 0.0, 0.0], [(0, 1, 1.0)])
    with pytest.raises(_ffi.EngineError, match="IE_ERR_INVALID"):
        GpuBitSlice(ir, 8, np.zeros(3, np.uint8))

"""Checkpoint / resume of a handle's device state (the survey's plan for the
reference's replay anchor, src/engine_v2/state.rs:55-67): a blob saved after
k steps and loaded into a fresh handle of the same problem and config
continues the trajectory exactly, and the state digest is FNV-1a over the
spin words in the reference layout."""
import numpy as np
import pytest

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.engine import Engine

pytestmark = pytest.mark.gpu


def fnv1a_words(words: np.ndarray) -> int:
    h = 0xcbf29ce484222325
    for b in np.ascontiguousarray(words, dtype="<u8").tobytes():
        h = ((h ^ b) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h


@pytest.mark.parametrize("integer", [True, False])
def test_checkpoint_resume_continues_the_trajectory(integer):
    rng = np.random.default_rng(8)
    m = I.maxcut_gnm(120, 400, seed=9) if integer else I.random_regular_qubo(150, 6, rng, integer=False)
    temps = I.geometric_beta_ladder(4, 0.3, 2.0)
    with Engine(m, num_temps=4, seed=21, exchange_interval=3) as a:
        a.init_random()
        a.step(temps, 7)
        blob = a.save_state()
        d0 = a.digest()
        assert d0 == fnv1a_words(a.spins())
        a.step(temps, 11)
        want = (a.spins(), a.energies(), a.swap_stats(), a.rng_state(), a.digest())
    with Engine(m, num_temps=4, seed=21, exchange_interval=3) as b:
        b.init_random()
        b.step(temps, 2)  # any prior state: the blob replaces it
        b.load_state(blob)
        assert b.digest() == d0
        b.step(temps, 11)
        assert (b.spins() == want[0]).all()
        assert b.energies().tobytes() == want[1].tobytes()
        att, acc = b.swap_stats()
        assert (att == want[2][0]).all() and (acc == want[2][1]).all()
        assert b.rng_state() == want[3]
        assert b.digest() == want[4]


def test_checkpoint_rejects_a_foreign_or_damaged_blob():
    m = I.maxcut_gnm(80, 240, seed=2)
    temps = I.geometric_beta_ladder(3, 0.3, 2.0)
    with Engine(m, num_temps=3, seed=4) as a:
        a.init_random()
        a.step(temps, 3)
        blob = bytearray(a.save_state())
    with Engine(m, num_temps=3, seed=4) as b:
        bad = bytearray(blob)
        bad[len(bad) // 2] ^= 0xFF  # a spin byte: the digest no longer matches
        with pytest.raises(_ffi.EngineError):
            b.load_state(bytes(bad))
    with Engine(I.maxcut_gnm(81, 240, seed=2), num_temps=3, seed=4) as c:
        with pytest.raises(_ffi.EngineError):
            c.load_state(bytes(blob))

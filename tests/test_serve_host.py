"""Host-side logic of the serving front-end (no GPU): request validation with
the reference's messages (server_api.rs:70-99), CSR construction with
duplicate merging and the 1e-9 drop (:111-156), the per-request schedule from
the data-driven temperature range, and the serving stream's generators."""
import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.serve import (MAX_NUM_VARS, MAX_SWEEPS, QuboRequest, best_replica, clamps_from,
                                     model_from, validate)


def req(**kw):
    d = dict(num_vars=3, linear=[0.0, 1.0, -1.0], quadratic=[(0, 1, 2.0)])
    d.update(kw)
    return QuboRequest(**d)


@pytest.mark.parametrize("kw,msg", [
    (dict(num_vars=0, linear=[]), "num_vars must be > 0"),
    (dict(num_vars=MAX_NUM_VARS + 1, linear=[0.0] * (MAX_NUM_VARS + 1)), f"num_vars exceeds maximum {MAX_NUM_VARS}"),
    (dict(linear=[0.0]), "linear.len() must equal num_vars"),
    (dict(quadratic=[(0, 3, 1.0)]), "edge index out of range: (0, 3) for num_vars=3"),
    (dict(clamped=[(5, 1)]), "clamped index 5 out of range"),
    (dict(clamped=[(1, 2)]), "clamped value must be 0 or 1, got 2"),
])
def test_validate_messages(kw, msg):
    with pytest.raises(ValueError) as e:
        validate(req(**kw))
    assert str(e.value) == msg


def test_validate_accepts():
    validate(req(clamped=[(2, 0)], replicas=99))


def test_model_from_merges_and_drops():
    r = req(num_vars=4, linear=[0.0] * 4,
            quadratic=[(0, 1, 1.0), (1, 0, 2.0), (2, 3, 1e-12), (1, 2, -0.5), (3, 3, 0.25)])
    m = model_from(r)
    # row 0: (1, 3.0); row 1: (0, 3.0), (2, -0.5); row 2: (1, -0.5); row 3: self loop 0.5
    assert m.row_offsets.tolist() == [0, 1, 3, 4, 5]
    assert m.col_indices.tolist() == [1, 0, 2, 1, 3]
    assert m.values.tolist() == [3.0, 3.0, -0.5, -0.5, 0.5]
    assert m.energy_offset == 0.0


def test_schedule_and_clamps():
    from ising_engine_b200.serve import schedule_from
    r = req(sweeps=10 ** 9)
    t = schedule_from(r, model_from(r))
    assert len(t) == MAX_SWEEPS and t[0] > t[-1] > 0
    f, v = clamps_from(req(clamped=[(2, 1), (0, 0)]))
    assert f.tolist() == [1, 0, 1] and v.tolist() == [0, 0, 1]
    assert clamps_from(req()) == (None, None)


def test_best_replica_lowest_index_on_ties():
    m = model_from(req())
    words = np.array([0b10, 0b11, 0b00], dtype=np.uint64)  # replica 0: x=(0,1,0); replica 1: (1,1,0)
    e = np.full(64, 5.0)
    e[0] = e[1] = -1.0
    s, E = best_replica(m, words, e)
    assert s.tolist() == [0, 1, 0] and E == m.calculate_total_energy(s)


def test_serving_stream_generators():
    reqs = I.serve_requests(6, 3, n_min=100, n_max=400, sweeps_min=10, sweeps_max=20)
    for m, seed, sweeps in reqs:
        assert 100 <= m.num_vars <= 400 and 10 <= sweeps <= 20
        deg = np.diff(m.row_offsets.astype(np.int64))
        assert 4 <= deg.min() == deg.max() <= 32
    a = I.poisson_arrivals(2000, 100.0, 1)
    assert np.all(np.diff(a) > 0) and abs(a[-1] / 2000 - 0.01) < 0.002

"""Serving pool (ie_serve_*): every request's result is the same alone and in
the mix, bit for bit (integer and f64 modes both run the reference's
arithmetic, so equality is exact), and agrees with the CPU oracle: spin words
bit for bit, energies equal to the oracle's FP64 recompute of those words
(the level kernel reports the recompute) and within 1e-6 of its tracked sum.

"Alone" is the request solved by itself through the batched entry point
(``BatchEngine`` with one model, ``ie_batch_run_schedule``); "in the mix" is
the request served while requests of other sizes, modes and schedule lengths
arrive, run and leave around it, over many ticks.
"""
import numpy as np
import pytest

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.engine import BatchEngine
from ising_engine_b200.serve import ServeEngine, best_replica, serve_stream, solve_json
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def assert_energies(model, words, e, tracked):
    rec = O.replica_energies(model, words)[0]
    assert e.tobytes() == rec.tobytes()
    assert (np.abs(e - tracked) / np.maximum(np.abs(tracked), 1.0)).max() <= 1e-6


def alone(model, seed, temps):
    b = BatchEngine([model], [seed])
    b.init_random()
    b.run_schedule(temps)
    out = b.spins(), b.energies()[0]
    b.close()
    return out


def mixed_requests():
    """Sizes across every kernel form: 1 and 2 threads per lane (small),
    windowed (large, degree <= 16) and 4 threads per lane (large, degree >
    16), integer and f64, schedules of different lengths."""
    rng = np.random.default_rng(77)
    spec = [(90, 4, True, 37), (300, 6, False, 120), (700, 12, True, 64), (2100, 16, True, 30),
            (2500, 10, False, 25), (1800, 24, True, 18), (2000, 30, False, 22), (160, 5, False, 300),
            (5000, 8, True, 12), (64, 3, True, 900), (1200, 20, False, 40), (3000, 14, False, 16)]
    reqs = []
    for k, (n, d, integer, steps) in enumerate(spec):
        m = I.random_regular_qubo(n, d, rng, integer=integer)
        reqs.append((m, 1000 + 17 * k, I.sa_temps(steps, 0.2, 4.0)))
    return reqs


def test_mix_equals_alone_and_oracle():
    reqs = mixed_requests()
    # a small site budget so that every request spans several ticks and the
    # resident set changes while requests are mid-schedule
    with ServeEngine(site_budget=4096) as srv:
        ids = {}
        results = {}
        order = list(range(len(reqs)))
        first, rest = order[:5], order[5:]
        for i in first:
            m, seed, temps = reqs[i]
            ids[srv.submit(m, seed, temps)] = i
        ticks = 0
        while len(results) < len(reqs):
            a, p, _ = srv.tick()
            ticks += 1
            if rest and ticks % 3 == 0:
                i = rest.pop(0)
                m, seed, temps = reqs[i]
                ids[srv.submit(m, seed, temps)] = i
            for rid in srv.poll():
                results[ids[rid]] = srv.result(rid)
            assert ticks < 10000
        assert ticks > 10
    for i, (m, seed, temps) in enumerate(reqs):
        w, e = results[i]
        wa, ea = alone(m, seed, temps)
        assert (w == wa).all(), f"request {i}: words differ from the request alone"
        assert e.tobytes() == ea.tobytes(), f"request {i}: energies differ from the request alone"
    small = [i for i, r in enumerate(reqs) if r[0].num_vars <= 2100]
    for i in small:
        m, seed, temps = reqs[i]
        wr, _, er = O.run_sa_batch([m], [seed], temps)
        assert (results[i][0] == wr).all(), f"request {i}: words differ from the oracle"
        assert_energies(m, results[i][0], results[i][1], er[0])


def test_admission_by_memory_footprint():
    """A pool too small for all requests at once: later requests wait for
    memory, are admitted as earlier ones leave, and still match alone."""
    rng = np.random.default_rng(5)
    reqs = [(I.random_regular_qubo(n, 8, rng, integer=bool(k % 2)), 50 + k, I.sa_temps(20 + 7 * k))
            for k, n in enumerate([1500, 1200, 1800, 900, 1600, 1000])]
    with ServeEngine(max_sites=4000, max_couplings=40000, site_budget=2048) as srv:
        ids = {srv.submit(m, s, t): k for k, (m, s, t) in enumerate(reqs)}
        saw_wait = False
        results = {}
        while len(results) < len(reqs):
            a, p, _ = srv.tick()
            saw_wait |= p > 0 and a > 0
            for rid in srv.poll():
                results[ids[rid]] = srv.result(rid)
        assert saw_wait, "expected requests to wait for memory"
        assert srv.footprint(reqs[0][0], 20) > 0
    for k, (m, s, t) in enumerate(reqs):
        wa, ea = alone(m, s, t)
        assert (results[k][0] == wa).all() and results[k][1].tobytes() == ea.tobytes()


def test_clamped_request_matches_oracle():
    rng = np.random.default_rng(3)
    for integer in (True, False):
        m = I.random_regular_qubo(80, 5, rng, integer=integer)
        f = np.zeros(80, np.uint8)
        f[[1, 9, 40, 79]] = 1
        v = np.zeros(80, np.int8)
        v[[9, 79]] = 1
        temps = I.sa_temps(60, 0.3, 3.0)
        with ServeEngine(site_budget=512) as srv:
            rid = srv.submit(m, 8, temps, f, v)
            out = srv.run_all()
        ref = O.run_schedule(m, temps[:, None], 8, clamped=f, clamp_val=v)
        assert (out[rid][0] == ref.words[0]).all()
        assert_energies(m, out[rid][0], out[rid][1], ref.energies[0])


def test_stream_and_json_front_end():
    reqs = mixed_requests()[:6]
    arrivals = np.linspace(0.0, 0.05, len(reqs))
    with ServeEngine(site_budget=8192) as srv:
        tr = serve_stream(srv, reqs, arrivals)
        s = tr.summary()
        assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0
        for (m, seed, temps), r in zip(reqs, tr.results):
            wa, ea = alone(m, seed, temps)
            assert (r[0] == wa).all() and r[1].tobytes() == ea.tobytes()
        payload = {"num_vars": 4, "linear": [1.0, -2.0, 0.5, 0.0],
                   "quadratic": [[0, 1, 1.5], [1, 2, -3.0], [1, 0, 0.5], [2, 3, 1.0]],
                   "clamped": [[3, 1]], "sweeps": 200, "seed": 9}
        r = solve_json(srv, payload)
        assert r["status"] == "success" and len(r["state"]) == 4 and r["state"][3] == 1
        from ising_engine_b200.serve import QuboRequest, model_from
        m = model_from(QuboRequest.from_json(payload))
        assert r["energy"] == m.calculate_total_energy(np.array(r["state"]))
        assert solve_json(srv, {"num_vars": 0, "linear": [], "quadratic": []})["status"].startswith("error")


def test_rejects_oversize_requests():
    rng = np.random.default_rng(1)
    with ServeEngine(max_sites=1000, max_couplings=10000) as srv:
        m = I.random_regular_qubo(1200, 4, rng, integer=True)
        with pytest.raises(_ffi.EngineError, match="IE_ERR_OOM"):
            srv.submit(m, 1, I.sa_temps(10))
        with pytest.raises(_ffi.EngineError, match="IE_ERR_INVALID"):
            srv.submit(I.random_regular_qubo(50, 4, rng, integer=True), 1, [1.0, -1.0])


def test_level_and_per_lane_serving_agree():
    """The same stream on the level kernel and on the per-lane kernels: equal
    spin words for every request."""
    reqs = mixed_requests()[:8]
    outs = []
    for form in (0, 1):
        with ServeEngine(site_budget=8192, kernel_form=form) as srv:
            ids = {srv.submit(m, s, t): k for k, (m, s, t) in enumerate(reqs)}
            res = srv.run_all()
            outs.append({ids[r]: res[r][0] for r in res})
    for k in range(len(reqs)):
        assert (outs[0][k] == outs[1][k]).all()

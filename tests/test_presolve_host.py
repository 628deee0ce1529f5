"""Presolve and decomposition host logic (no GPU): the library's
full_presolve equals the oracle's restatement of src/presolve (same fixings,
same order) with and without clamps, its fixings keep an exhaustive optimum
(the reference's contract, tests/test_presolve.rs / test_qpbo.rs style), the
components match a breadth-first search, and a component's sub-model plus its
fixed part reproduces the full energy."""
import itertools

import numpy as np
import pytest

from ising_engine_b200 import instances as I
from ising_engine_b200.core import CsrMatrix, QuboModel
from ising_engine_b200.presolve import connected_components, extract_component, full_presolve
from oracle import oracle as O
from tests.test_pa_host import random_qubo


def block_instance(seed, integral=True):
    """Two random Ising spin-glass blocks and a ferromagnetic chain in QUBO
    form (zero field: symmetric under a global flip, so persistency fixes
    none of them) plus isolated variables with strong fields (fixed): the
    free graph splits into three components."""
    rng = np.random.default_rng(seed)
    n = 26
    J = {}
    for blk in (range(0, 8), range(8, 16)):
        for i, j in itertools.combinations(blk, 2):
            if rng.random() < 0.6:
                J[(i, j)] = float(rng.choice([-1, 1]) * rng.integers(1, 4)) if integral else float(rng.normal())
    for i in range(16, 21):
        J[(i, i + 1)] = -1.0
    lin = np.zeros(n)
    rows = [[] for _ in range(n)]
    for (i, j), v in J.items():  # E = sum J s_i s_j, s = 2x - 1
        lin[i] -= 2 * v
        lin[j] -= 2 * v
        rows[i].append((j, 4 * v))
        rows[j].append((i, 4 * v))
    lin[22:] = [9.0, -9.0, 7.0, -7.0]
    ro, ci, va = [0], [], []
    for r in rows:
        r.sort()
        ci += [j for j, _ in r]
        va += [w for _, w in r]
        ro.append(len(ci))
    return QuboModel(n, lin, CsrMatrix(np.array(va), np.array(ci, dtype=np.uint64), np.array(ro, dtype=np.uint64)),
                     0.0)


@pytest.mark.parametrize("seed", range(12))
def test_presolve_equals_oracle(seed):
    n = [8, 12, 20, 40][seed % 4]
    m = random_qubo(n, [0.1, 0.3, 0.6][seed % 3], seed, integral=seed % 2 == 0)
    for cl in ([], [(0, 1), (n - 1, 0)], [(1, 0)]):
        assert full_presolve(m, cl) == [(int(i), int(v)) for i, v in O.full_presolve(m, cl)]
    b = block_instance(seed, integral=seed % 2 == 0)
    assert full_presolve(b) == [(int(i), int(v)) for i, v in O.full_presolve(b)]


def brute(m, fixed):
    best = np.inf
    for bits in itertools.product((0, 1), repeat=m.num_vars):
        x = np.array(bits, dtype=np.int8)
        if all(x[i] == v for i, v in fixed):
            best = min(best, m.calculate_total_energy(x))
    return best


@pytest.mark.parametrize("seed", range(6))
def test_presolve_keeps_an_optimum(seed):
    m = random_qubo(11, 0.35, 100 + seed, integral=seed % 2 == 1)
    cl = [(3, seed % 2)]
    fix = full_presolve(m, cl)
    assert abs(brute(m, cl + fix) - brute(m, cl)) < 1e-9
    assert all(i != 3 for i, _ in fix)


def bfs_components(m, active):
    seen, out = set(), []
    ro, ci, va = m.row_offsets.astype(int), m.col_indices.astype(int), m.values
    for s in range(m.num_vars):
        if not active[s] or s in seen:
            continue
        comp, todo = [], [s]
        seen.add(s)
        while todo:
            v = todo.pop()
            comp.append(v)
            for e in range(ro[v], ro[v + 1]):
                j = ci[e]
                if va[e] != 0 and active[j] and j not in seen:
                    seen.add(j)
                    todo.append(j)
        out.append(sorted(comp))
    return out


@pytest.mark.parametrize("seed", range(4))
def test_components_and_extraction(seed):
    m = block_instance(seed)
    fix = full_presolve(m)
    fixed = dict(fix)
    active = np.array([i not in fixed for i in range(m.num_vars)])
    comps = connected_components(m, active)
    assert comps == bfs_components(m, active) and len(comps) > 1
    fixed_one = np.array([fixed.get(i, 0) == 1 for i in range(m.num_vars)])
    rng = np.random.default_rng(seed)
    for comp in comps:
        sub, gmap = extract_component(m, comp, fixed_one)
        assert gmap == comp
        for _ in range(5):
            x = np.array([fixed.get(i, 0) for i in range(m.num_vars)], dtype=np.int8)
            y = rng.integers(0, 2, size=len(comp)).astype(np.int8)
            x0 = x.copy()
            x[comp] = y
            # energy difference inside the component = the sub-model's energy
            d = m.calculate_total_energy(x) - m.calculate_total_energy(x0)
            assert abs(d - sub.calculate_total_energy(y)) < 1e-9


def test_large_instance_has_no_fixings_quickly():
    m = I.maxcut_gnm(800, 19176, seed=42)
    assert full_presolve(m) == []

"""Host-side checks of the level kernel's two ideas (no GPU):

1. Stream splitting: the library's jump polynomial x^D mod P(x) moves a
   Xoshiro256 state D steps ahead (engine.rs:115-121 stepped D times).
2. Dependency levels: deciding the sites level by level (level(v) = 1 + max
   level of the unclamped neighbours u < v) reads exactly the neighbour values
   the reference's site order reads, so the sweep's result is the same.
"""
import numpy as np

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I

M64 = (1 << 64) - 1


def xo_step(s):
    s0, s1, s2, s3 = s
    t = (s1 << 17) & M64
    s2 ^= s0
    s3 ^= s1
    s1 ^= s2
    s0 ^= s3
    s2 ^= t
    s3 = ((s3 << 45) | (s3 >> 19)) & M64
    return [s0, s1, s2, s3]


def jump_poly(d):
    out = np.zeros(4, dtype=np.uint64)
    _ffi.check(_ffi.lib().ie_xoshiro_jump_poly(d, out.ctypes.data))
    return [int(x) for x in out]


def xo_jump(s, poly):
    acc = [0, 0, 0, 0]
    for i in range(256):
        if (poly[i >> 6] >> (i & 63)) & 1:
            acc = [a ^ b for a, b in zip(acc, s)]
        s = xo_step(s)
    return acc


def test_jump_polynomial_moves_the_state_ahead():
    rng = np.random.default_rng(5)
    for d in [0, 1, 7, 255, 256, 1024, 8 * 128 * 3, 100003]:
        s = [int(x) for x in rng.integers(0, 2**63, size=4, dtype=np.int64)]
        ref = list(s)
        for _ in range(d):
            ref = xo_step(ref)
        assert xo_jump(s, jump_poly(d)) == ref, d


def levels(rows, cols, clamped):
    n = len(rows) - 1
    lvl = np.zeros(n, dtype=np.int64)
    for v in range(n):
        if clamped[v]:
            continue
        nb = cols[rows[v]:rows[v + 1]]
        lo = [u for u in nb if u < v and not clamped[u]]
        lvl[v] = 1 + max(lvl[u] for u in lo) if lo else 0
    return lvl


def sweep(order, rows, cols, vals, lin, x, u, beta):
    """Metropolis decisions of one replica in the given site order, each
    site's uniform fixed in advance (as the generator phase fixes it)."""
    x = x.copy()
    for v in order:
        de = lin[v] * (1 - 2 * x[v])
        for k in range(rows[v], rows[v + 1]):
            de += vals[k] * ((x[cols[k]] ^ x[v]) - x[v])
        if de <= 0 or u[v] < np.exp(-de * beta):
            x[v] ^= 1
    return x


def test_level_order_reads_the_site_order_values():
    rng = np.random.default_rng(11)
    for n, d, clamp_frac in [(200, 6, 0.0), (300, 12, 0.1), (64, 16, 0.3)]:
        m = I.random_regular_qubo(n, d, rng, integer=True)
        rows = m.row_offsets.astype(np.int64)
        cols = m.col_indices.astype(np.int64)
        clamped = rng.random(n) < clamp_frac
        lvl = levels(rows, cols, clamped)
        # sites of one level are never neighbours; lower neighbours are on
        # lower levels, higher neighbours on higher levels
        for v in range(n):
            if clamped[v]:
                continue
            for u in cols[rows[v]:rows[v + 1]]:
                if clamped[u]:
                    continue
                assert (lvl[u] < lvl[v]) if u < v else (lvl[u] > lvl[v])
        live = [v for v in range(n) if not clamped[v]]
        by_level = sorted(live, key=lambda v: (lvl[v], -v))  # any order inside a level
        for rep in range(3):
            x = rng.integers(0, 2, size=n)
            u = rng.random(n)
            a = sweep(live, rows, cols, m.values, m.linear, x, u, 0.7)
            b = sweep(by_level, rows, cols, m.values, m.linear, x, u, 0.7)
            assert (a == b).all()


def test_lattice_depth_is_about_the_sum_of_the_sides():
    m = I.pm_j_lattice(32, 2, seed=1)
    lvl = levels(m.row_offsets.astype(np.int64), m.col_indices.astype(np.int64), np.zeros(m.num_vars, bool))
    assert 2 * 31 <= lvl.max() <= 2 * 32 + 2

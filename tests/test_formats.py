"""Instance-format readers (host only): the reference's triangle known answer
(frontend.rs:95-103), objective conventions of each family checked against a
direct evaluation of the format's objective on random states, energy equality
of the QuboModel -> ProblemIR bridge, and the readers' errors."""
import numpy as np
import pytest

from ising_engine_b200.formats import (assemble, parse_biqmac_sparse, parse_orlib_bqp, parse_qplib, parse_rudy,
                                       parse_rudy_maxcut, qubo_model_to_ir, rudy_maxcut_ir, tokens)


def test_triangle_cut_lowering():
    ir = rudy_maxcut_ir("3 3\n1 2\n2 3\n1 3\n")
    assert ir.energy([0, 1, 0]) == -2.0
    assert ir.energy([0, 0, 0]) == 0.0


def test_parse_rudy_defaults_and_skips():
    n, edges = parse_rudy("4 5\n1 2\n3 3 7\n2 4 -1.5\n0 1\n5 1\n")
    assert n == 4 and edges == [(0, 1, 1.0), (1, 3, -1.5)]
    with pytest.raises(ValueError, match="empty file"):
        parse_rudy("\n \n")
    with pytest.raises(ValueError, match="bad u"):
        parse_rudy("3 1\n-1 2\n")


def cut_value(n, edges, x):
    return sum(w for (i, j, w) in edges if x[i] != x[j])


def test_maxcut_family_energy_is_minus_cut():
    rng = np.random.default_rng(1)
    n = 12
    lines = [f"{n} 20  % header"]
    edges = []
    while len(edges) < 20:
        i, j = rng.integers(1, n + 1, size=2)
        if i == j:
            continue
        w = int(rng.integers(-3, 4))
        edges.append((i - 1, j - 1, w))
        lines.append(f"{i} {j} {w}  # edge")
    inst = parse_rudy_maxcut("\n".join(lines) + "\n", "g")
    assert inst.maximize and inst.family == "maxcut"
    for _ in range(20):
        x = rng.integers(0, 2, size=n).astype(np.int8)
        assert inst.model.calculate_total_energy(x) == -cut_value(n, edges, x)
    with pytest.raises(ValueError, match="g: vertex out of range"):
        parse_rudy_maxcut("3 1\n1 4 1\n", "g")
    with pytest.raises(ValueError, match="g: bad MaxCut header"):
        parse_rudy_maxcut("3\n1 2 1\n", "g")


def xqx(n, trip, x):
    """x'Qx with Q symmetric and one triangle listed."""
    s = 0.0
    for (i, j, q) in trip:
        if i == j:
            s += q * x[i]
        else:
            s += 2.0 * q * x[i] * x[j]
    return s


def test_orlib_and_biqmac_objectives():
    rng = np.random.default_rng(2)
    probs = []
    text = ["2"]
    for _ in range(2):
        n = 9
        trip = []
        for i in range(n):
            for j in range(i, n):
                if rng.random() < 0.4:
                    trip.append((i, j, int(rng.integers(-20, 21))))
        probs.append((n, trip))
        text.append(f"{n} {len(trip)}")
        text += [f"{i + 1} {j + 1} {q}" for (i, j, q) in trip]
    insts = parse_orlib_bqp("\n".join(text), "bqp")
    assert [i.name for i in insts] == ["bqp.1", "bqp.2"]
    for inst, (n, trip) in zip(insts, probs):
        for _ in range(20):
            x = rng.integers(0, 2, size=n).astype(np.int8)
            assert inst.model.calculate_total_energy(x) == -xqx(n, trip, x)
    n, trip = probs[0]
    bq = parse_biqmac_sparse(f"{n} {len(trip)}\n" + "\n".join(f"{i + 1} {j + 1} {q}" for (i, j, q) in trip), "be")
    assert not bq.maximize
    for _ in range(20):
        x = rng.integers(0, 2, size=n).astype(np.int8)
        assert bq.model.calculate_total_energy(x) == xqx(n, trip, x)
    with pytest.raises(ValueError, match="unexpected EOF in BQP"):
        parse_orlib_bqp("1\n3 2\n1 1 5\n", "bqp")


def test_bridge_preserves_energy_bitwise():
    """frontend.rs:105-140 on a benchmark-style model: integral weights, each
    pair listed once."""
    rng = np.random.default_rng(3)
    n = 30
    pairs = {(min(i, j), max(i, j)) for i, j in rng.integers(0, n, size=(80, 2)) if i != j}
    edges = [(int(i), int(j), float(rng.integers(-9, 10) or 1)) for (i, j) in sorted(pairs)]
    m = assemble(n, edges, rng.integers(-9, 10, size=n).astype(np.float64))
    ir = qubo_model_to_ir(m)
    for _ in range(40):
        x = rng.integers(0, 2, size=n).astype(np.int8)
        assert ir.energy(x) == m.calculate_total_energy(x)


def test_tokens_strip_comments():
    assert tokens("1 2 3 # c") == ["1", "2", "3"]
    assert tokens("% only a comment") == []


def brute(inst):
    n = inst.model.num_vars
    best = min(inst.model.calculate_total_energy(np.array([(b >> v) & 1 for v in range(n)], np.int8))
               for b in range(1 << n))
    return best, -best if inst.maximize else best


def test_qplib_unconstrained_binary():
    """test_benchmark.rs:84-123: pair coefficient -6/2, minimum -1 at (1, 1);
    constrained and continuous types refused."""
    text = ("toy            name\nQBN            type\nminimize       sense\n2              n\n"
            "1              nq\n1 2 -6         q12\n0              b_default\n2              nb\n"
            "1 1            b1\n2 1            b2\n0              c\n")
    inst = parse_qplib(text, "toy")
    assert not inst.maximize and inst.family == "qplib"
    e, native = brute(inst)
    assert abs(e + 1.0) < 1e-9 and abs(native + 1.0) < 1e-9
    with pytest.raises(ValueError, match="is constrained"):
        parse_qplib("c name\nQBL type\nminimize sense\n2 n\n", "c")
    with pytest.raises(ValueError, match="not binary-variable"):
        parse_qplib("c name\nQCN type\nminimize sense\n2 n\n", "c")


def test_qplib_maximize_defaults_and_offset():
    """A maximization: energy = -objective; the diagonal entry and b_default
    reach every variable, listed b entries replace the default, c is the
    offset (and may be missing)."""
    rng = np.random.default_rng(4)
    n = 5
    quad = [(1, 1, 4.0), (1, 3, -2.0), (2, 5, 6.0), (4, 4, -8.0)]
    bdef, blist, c = 1.5, [(2, -3.0), (5, 0.5)], 7.0
    lines = ["q name", "QBN type", "maximize sense", f"{n} n", f"{len(quad)} nq"]
    lines += [f"{i} {j} {q}" for i, j, q in quad] + [f"{bdef} b_default", f"{len(blist)} nb"]
    lines += [f"{i} {v}" for i, v in blist]
    inst = parse_qplib("\n".join(lines + [f"{c} c"]), "q")
    inst2 = parse_qplib("\n".join(lines), "q")
    b = [bdef] * n
    for i, v in blist:
        b[i - 1] = v
    for _ in range(20):
        x = rng.integers(0, 2, size=n).astype(np.int8)
        obj = sum(0.5 * q * x[i - 1] * x[j - 1] for i, j, q in quad) + sum(bi * xi for bi, xi in zip(b, x))
        assert inst.model.calculate_total_energy(x) == pytest.approx(-(obj + c), abs=1e-12)
        assert inst2.model.calculate_total_energy(x) == pytest.approx(-obj, abs=1e-12)
    with pytest.raises(ValueError, match="q: quad index out of range"):
        parse_qplib("q name\nQBN type\nminimize sense\n2 n\n1 nq\n1 3 1\n", "q")
    with pytest.raises(ValueError, match="qplib: missing nb"):
        parse_qplib("q name\nQBN type\nminimize sense\n2 n\n0 nq\n0 b_default\n", "q")

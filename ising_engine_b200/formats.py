"""Instance formats lowered to the solver's problem types (host only).

Restates the reference's readers: the engine_v2 frontend
(src/engine_v2/frontend.rs:11-98: ``qubo_model_to_ir``, ``parse_rudy``,
``maxcut_to_qubo``, ``rudy_maxcut_ir``) and the benchmark family parsers
(src/benchmark/instances.rs:60-231: ``assemble``, ``parse_rudy_maxcut``,
``parse_orlib_bqp``, ``parse_biqmac_sparse``, ``parse_qplib``). Errors raise
``ValueError`` with the reference's message.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .core import CsrMatrix, QuboModel
from .v2 import ProblemIR


@dataclass
class Instance:
    """instances.rs Instance: the model and how its native objective reads
    (maximize: native value = -energy)."""
    name: str
    family: str
    model: QuboModel
    maximize: bool
    best_known: float | None = None


def _uint(tok: str, msg: str) -> int:
    """Rust's usize::from_str: decimal digits with an optional '+'."""
    t = tok[1:] if tok.startswith("+") else tok
    if not t.isdigit():
        raise ValueError(msg)
    return int(t)


def _float(tok: str, msg: str) -> float:
    try:
        return float(tok)
    except ValueError:
        raise ValueError(msg) from None


def tokens(line: str) -> list[str]:
    """instances.rs:88-95: the part before '#' or '%', whitespace-split."""
    for c in "#%":
        line = line.split(c, 1)[0]
    return line.split()


def assemble(n: int, edges, linear) -> QuboModel:
    """instances.rs:60-86: both triangles, each row stable-sorted by column,
    no merging, offset 0."""
    rows = [[] for _ in range(n)]
    for (i, j, w) in edges:
        rows[i].append((j, w))
        rows[j].append((i, w))
    vals, cols, ro = [], [], [0]
    for r in rows:
        r.sort(key=lambda e: e[0])
        for (j, w) in r:
            cols.append(j)
            vals.append(w)
        ro.append(len(cols))
    return QuboModel(n, np.asarray(linear, dtype=np.float64),
                     CsrMatrix(np.asarray(vals, dtype=np.float64), np.asarray(cols, dtype=np.uint64),
                               np.asarray(ro, dtype=np.uint64)), 0.0)


def parse_rudy(text: str):
    """frontend.rs:38-72: header `n m`, then lines `i j [w]` (1-indexed,
    weight 1 when missing); self-loops and out-of-range lines skipped.
    Returns (n, [(a, b, w)] with a < b)."""
    lines = [l.split() for l in text.splitlines()]
    lines = [t for t in lines if t]
    if not lines:
        raise ValueError("empty file")
    header = lines[0]
    n = _uint(header[0], "bad n")
    edges = []
    for t in lines[1:]:
        if len(t) < 2:
            continue
        u = _uint(t[0], "bad u")
        v = _uint(t[1], "bad v")
        w = _float(t[2], "bad w") if len(t) > 2 else 1.0
        if u == v or u < 1 or v < 1 or u > n or v > n:
            continue
        edges.append((min(u, v) - 1, max(u, v) - 1, w))
    return n, edges


def maxcut_to_qubo(n: int, edges) -> ProblemIR:
    """frontend.rs:76-85: per edge (u, v, w): linear[u] -= w, linear[v] -= w,
    pair (u, v) += 2w; the lowest energy is minus the largest cut."""
    linear = [0.0] * n
    pairs = []
    for (u, v, w) in edges:
        linear[u] -= w
        linear[v] -= w
        pairs.append((u, v, 2.0 * w))
    return ProblemIR.from_pairs(n, 0.0, linear, pairs)


def rudy_maxcut_ir(text: str) -> ProblemIR:
    n, edges = parse_rudy(text)
    return maxcut_to_qubo(n, edges)


def qubo_model_to_ir(m: QuboModel) -> ProblemIR:
    """frontend.rs:20-33: upper-triangle extraction (a self-loop folds half of
    its weight into the linear term)."""
    linear = np.array(m.linear, dtype=np.float64)
    pairs = []
    for i in range(m.num_vars):
        for (j, w) in m.quadratic.get_row(i):
            if j > i:
                pairs.append((i, j, w))
            elif j == i:
                linear[i] += 0.5 * w
    return ProblemIR.from_pairs(m.num_vars, m.energy_offset, linear, pairs)


def parse_rudy_maxcut(text: str, name: str) -> Instance:
    """instances.rs:103-141 (G-Set / Biq Mac MaxCut): header `n m`, then lines
    `i j w`; a vertex out of range is an error, self-loops are skipped."""
    lines = [tokens(l) for l in text.splitlines()]
    lines = [t for t in lines if t]
    if not lines:
        raise ValueError("empty MaxCut file")
    ht = lines[0]
    if len(ht) < 2:
        raise ValueError(f"{name}: bad MaxCut header")
    n = _uint(ht[0], "bad n")
    _uint(ht[1], "bad m")
    edges, linear = [], [0.0] * n
    for t in lines[1:]:
        if len(t) < 3:
            continue
        i = _uint(t[0], "bad edge i")
        j = _uint(t[1], "bad edge j")
        w = _float(t[2], "bad edge w")
        if i == 0 or j == 0 or i > n or j > n:
            raise ValueError(f"{name}: vertex out of range")
        i, j = i - 1, j - 1
        if i == j:
            continue
        edges.append((i, j, 2.0 * w))
        linear[i] -= w
        linear[j] -= w
    return Instance(name, "maxcut", assemble(n, edges, linear), True)


def _stream(text: str, eof: str):
    toks = text.split()
    pos = 0

    def nxt() -> str:
        nonlocal pos
        if pos >= len(toks):
            raise ValueError(eof)
        pos += 1
        return toks[pos - 1]
    return nxt


def parse_orlib_bqp(text: str, name: str) -> list[Instance]:
    """instances.rs:150-188 (OR-Library BQP, maximisation): problem count, then
    per problem `n nnz` and `nnz` triples `i j q` of one triangle of the
    symmetric Q; energy = -objective (diagonal into linear, off-diagonal
    pairs counted twice)."""
    nxt = _stream(text, "unexpected EOF in BQP")
    p = _uint(nxt(), "bad problem count")
    out = []
    for k in range(p):
        n = _uint(nxt(), "bad n")
        nnz = _uint(nxt(), "bad nnz")
        edges, linear = [], [0.0] * n
        for _ in range(nnz):
            i = _uint(nxt(), "bad i")
            j = _uint(nxt(), "bad j")
            v = _float(nxt(), "bad q")
            if i == 0 or j == 0 or i > n or j > n:
                raise ValueError(f"{name}: index out of range")
            i, j = i - 1, j - 1
            if i == j:
                linear[i] -= v
            else:
                edges.append((i, j, -2.0 * v))
        out.append(Instance(f"{name}.{k + 1}", "orlib_bqp", assemble(n, edges, linear), True))
    return out


def parse_biqmac_sparse(text: str, name: str) -> Instance:
    """instances.rs:196-231 (Biq Mac sparse BQP, minimisation of x'Qx): `n nnz`
    then `nnz` triples `i j q` of one triangle of the symmetric Q."""
    nxt = _stream(text, "unexpected EOF in Biq Mac sparse")
    n = _uint(nxt(), "bad n")
    nnz = _uint(nxt(), "bad nnz")
    edges, linear = [], [0.0] * n
    for _ in range(nnz):
        i = _uint(nxt(), "bad i")
        j = _uint(nxt(), "bad j")
        v = _float(nxt(), "bad q")
        if i == 0 or j == 0 or i > n or j > n:
            raise ValueError(f"{name}: index out of range")
        i, j = i - 1, j - 1
        if i == j:
            linear[i] += v
        else:
            edges.append((i, j, 2.0 * v))
    return Instance(name, "biqmac_sparse", assemble(n, edges, linear), False)


def _as_usize(x: float) -> int:
    """Rust's saturating `f64 as usize`: NaN and negatives give 0, toward zero."""
    if x != x or x <= 0.0:
        return 0
    return int(min(x, 2.0 ** 64 - 1))


def parse_qplib(text: str, name: str) -> Instance:
    """instances.rs:227-345 (QPLIB, the unconstrained binary subset): one
    logical line per field, numeric fields first and free text after; type
    code `?B N` only; objective 1/2 sum of the listed q_ij x_i x_j (each listed
    entry once, diagonal into the linear term) + b'x + c, negated for a
    maximization so that the energy is always minimized."""
    lines = [l.split() for l in text.splitlines()]
    lines = iter([t for t in lines if t])

    def next_line(what: str):
        t = next(lines, None)
        if t is None:
            raise ValueError(f"qplib: missing {what}")
        return t

    def parse1(t, w: str) -> float:
        if not t:
            raise ValueError(f"qplib: empty {w}")
        try:
            return float(t[0])
        except ValueError:
            raise ValueError(f"qplib: bad {w}") from None

    next_line("name")
    ptype = next_line("type")[0]
    if len(ptype) < 2 or ptype[1].upper() != "B":
        raise ValueError(f"{name}: QPLIB type {ptype} not binary-variable (unsupported)")
    if len(ptype) < 3 or ptype[2].upper() != "N":
        raise ValueError(f"{name}: QPLIB type {ptype} is constrained; only unconstrained instances supported")
    maximize = next_line("sense")[0].lower() == "maximize"
    n = _as_usize(parse1(next_line("n"), "n"))
    sign = -1.0 if maximize else 1.0
    nq = _as_usize(parse1(next_line("nq"), "nq"))
    edges, linear = [], [0.0] * n
    for _ in range(nq):
        t = next_line("quad term")
        if len(t) < 3:
            raise ValueError(f"{name}: short quad line")
        i = _as_usize(parse1(t[0:1], "qi"))
        j = _as_usize(parse1(t[1:2], "qj"))
        q = parse1(t[2:3], "qv")
        if i == 0 or j == 0 or i > n or j > n:
            raise ValueError(f"{name}: quad index out of range")
        i, j = i - 1, j - 1
        if i == j:
            linear[i] += sign * 0.5 * q
        else:
            edges.append((i, j, sign * 0.5 * q))
    b_default = parse1(next_line("b_default"), "b_default")
    linear = [v + sign * b_default for v in linear]
    nb = _as_usize(parse1(next_line("nb"), "nb"))
    for _ in range(nb):
        t = next_line("linear term")
        if len(t) < 2:
            raise ValueError(f"{name}: short linear line")
        i = _as_usize(parse1(t[0:1], "bi"))
        v = parse1(t[1:2], "bv")
        if i == 0 or i > n:
            raise ValueError(f"{name}: linear index out of range")
        linear[i - 1] += sign * (v - b_default)
    try:
        c = parse1(next_line("c"), "c")
    except ValueError:
        c = 0.0
    m = assemble(n, edges, linear)
    m.energy_offset = sign * c
    return Instance(name, "qplib", m, maximize)

"""Presolve and decomposition (host only), as UltimateSolver::solve applies
them before annealing (src/solver/ultimate.rs:161-218).

``full_presolve`` (src/presolve/mod.rs:279-324: roof-duality strong
persistencies on the clamp-reduced model unioned with probing weak
persistencies) and ``connected_components`` (mod.rs:189-218) are computed by
the library's host code; ``extract_component`` (mod.rs:229-270) builds a
component's sub-model here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from .core import CsrMatrix, QuboModel
from .engine import _p, _problem


def full_presolve(model: QuboModel, clamped=()) -> list:
    """Provably optimum-preserving fixings [(index, value)] beyond the user's
    clamps, in the reference's order."""
    keep: list = []
    prob = _problem(model, keep)
    ci = np.ascontiguousarray([c[0] for c in clamped], dtype=np.uint64)
    cv = np.ascontiguousarray([c[1] for c in clamped], dtype=np.int8)
    out_i = np.zeros(max(model.num_vars, 1), dtype=np.uint64)
    out_v = np.zeros(max(model.num_vars, 1), dtype=np.int8)
    k = C.c_uint64()
    _ffi.check(_ffi.lib().ie_presolve(C.byref(prob), _p(ci), _p(cv), len(ci), _p(out_i), _p(out_v), C.byref(k)))
    return [(int(out_i[i]), int(out_v[i])) for i in range(k.value)]


def connected_components(model: QuboModel, active) -> list:
    """Components of the graph of nonzero couplings among active variables,
    in ascending order of their smallest vertex, each sorted."""
    keep: list = []
    prob = _problem(model, keep)
    act = np.ascontiguousarray(active, dtype=np.uint8)
    comp = np.zeros(max(model.num_vars, 1), dtype=np.uint64)
    k = C.c_uint64()
    _ffi.check(_ffi.lib().ie_connected_components(C.byref(prob), _p(act), _p(comp), C.byref(k)))
    out = [[] for _ in range(k.value)]
    for v in range(model.num_vars):
        if comp[v] != np.uint64(0xFFFFFFFFFFFFFFFF):
            out[int(comp[v])].append(v)
    return out


def extract_component(model: QuboModel, comp, fixed_one):
    """mod.rs:229-270: the sub-model of one component (couplings to members
    kept in row order, couplings to variables fixed at 1 folded into the
    linear term, offset 0) and its local -> global map."""
    g2l = {g: l for l, g in enumerate(comp)}
    ro, ci, va = model.row_offsets.astype(np.int64), model.col_indices.astype(np.int64), model.values
    lin, rows, cols, vals = [], [0], [], []
    for g in comp:
        h = float(model.linear[g])
        for e in range(ro[g], ro[g + 1]):
            j = int(ci[e])
            if j in g2l:
                cols.append(g2l[j])
                vals.append(float(va[e]))
            elif fixed_one[j]:
                h += float(va[e])
        lin.append(h)
        rows.append(len(cols))
    sub = QuboModel(len(comp), np.array(lin, dtype=np.float64),
                    CsrMatrix(np.array(vals, dtype=np.float64), np.array(cols, dtype=np.uint64),
                              np.array(rows, dtype=np.uint64)), 0.0)
    return sub, list(comp)

"""Problem types mirroring the reference's QuboModel and CsrMatrix.

``QuboModel`` / ``CsrMatrix`` follow src/core/hubo.rs:165-189 and
src/core/csr_matrix.rs:6-30: both triangles of the coupling matrix are stored,
and the model energy is ``offset + sum_i lin_i x_i + 1/2 sum_csr w x_i x_j``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CsrMatrix:
    values: np.ndarray
    col_indices: np.ndarray
    row_offsets: np.ndarray

    def get_row(self, row: int):
        s, e = int(self.row_offsets[row]), int(self.row_offsets[row + 1])
        return zip(self.col_indices[s:e].tolist(), self.values[s:e].tolist())

    @staticmethod
    def empty(num_vars: int) -> "CsrMatrix":
        return CsrMatrix(np.zeros(0), np.zeros(0, dtype=np.uint64),
                         np.zeros(num_vars + 1, dtype=np.uint64))


class QuboModel:
    """QUBO over x in {0,1}^n (src/core/hubo.rs:165-173)."""

    def __init__(self, num_vars: int, linear, quadratic: CsrMatrix, energy_offset: float = 0.0):
        self.num_vars = int(num_vars)
        self.linear = np.ascontiguousarray(linear, dtype=np.float64)
        self.quadratic = CsrMatrix(
            np.ascontiguousarray(quadratic.values, dtype=np.float64),
            np.ascontiguousarray(quadratic.col_indices, dtype=np.uint64),
            np.ascontiguousarray(quadratic.row_offsets, dtype=np.uint64))
        self.energy_offset = float(energy_offset)
        if self.linear.shape != (self.num_vars,):
            raise ValueError("linear must have num_vars entries")
        if self.quadratic.row_offsets.shape != (self.num_vars + 1,):
            raise ValueError("row_offsets must have num_vars + 1 entries")

    # accessors used by the oracle wrapper and the FFI
    @property
    def row_offsets(self):
        return self.quadratic.row_offsets

    @property
    def col_indices(self):
        return self.quadratic.col_indices

    @property
    def values(self):
        return self.quadratic.values

    @property
    def nnz(self) -> int:
        return int(self.quadratic.row_offsets[-1]) if self.num_vars else 0

    def calculate_total_energy(self, state) -> float:
        """hubo.rs:176-189, in the same summation order."""
        state = np.asarray(state)
        e = self.energy_offset
        ro = self.quadratic.row_offsets
        ci = self.quadratic.col_indices
        va = self.quadratic.values
        for i in range(self.num_vars):
            if state[i] == 1:
                e += float(self.linear[i])
                for k in range(int(ro[i]), int(ro[i + 1])):
                    if state[int(ci[k])] == 1:
                        e += float(va[k]) * 0.5
        return e

    def is_integral(self) -> bool:
        return bool(np.all(self.linear == np.trunc(self.linear)) and
                    np.all(self.quadratic.values == np.trunc(self.quadratic.values)))

    @staticmethod
    def from_edges(num_vars: int, linear, edges, energy_offset: float = 0.0) -> "QuboModel":
        """Builds the two-triangle CSR from upper-triangle (i, j, w) triples,
        each row sorted by column (the layout the reference's builders make)."""
        edges = np.asarray(edges, dtype=np.float64).reshape(-1, 3) if len(edges) else np.zeros((0, 3))
        i = edges[:, 0].astype(np.int64)
        j = edges[:, 1].astype(np.int64)
        w = edges[:, 2]
        rows = np.concatenate([i, j])
        cols = np.concatenate([j, i])
        vals = np.concatenate([w, w])
        order = np.lexsort((cols, rows))
        rows, cols, vals = rows[order], cols[order], vals[order]
        counts = np.bincount(rows, minlength=num_vars)
        ro = np.zeros(num_vars + 1, dtype=np.uint64)
        ro[1:] = np.cumsum(counts)
        return QuboModel(num_vars, linear, CsrMatrix(vals, cols.astype(np.uint64), ro), energy_offset)

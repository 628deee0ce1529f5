"""engine_v2 (S2) on the device: the integral bit-sliced state and the
MetropolisSweep / ReplicaExchange operators behind ``ie_v2_*``.

Mirrors the reference's S2 seam: ``ProblemIR`` (src/engine_v2/ir.rs:14-148),
the ``SpinState`` queries of the bit-sliced backend
(src/engine_v2/backends/sparse_bitslice.rs:238-347) and ``Operator::apply``
(src/engine_v2/operator.rs:72-86) of ``MetropolisSweep``
(src/engine_v2/operators/metropolis_sweep.rs:95-146), ``GibbsColorSweep``
(src/engine_v2/operators/gibbs_color_sweep.rs:119-165) and ``ReplicaExchange``
(src/engine_v2/operators/replica_exchange.rs:61-110). The operators' shared
``ChaCha8Rng`` is a ``ChaChaStream``: its seed and the number of 64-bit draws
consumed so far; each apply advances it by exactly the draws the reference's
operator takes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _ffi
from .core import CsrMatrix, QuboModel
from .engine import _p, _problem


class ProblemIR:
    """src/engine_v2/ir.rs:14-148: both triangles, rows sorted by column,
    duplicate pairs summed, zero weights dropped."""

    def __init__(self, n: int, offset: float, linear, row_ptr, col_idx, weights):
        self.n = int(n)
        self.offset = float(offset)
        self.linear = np.ascontiguousarray(linear, dtype=np.float64)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        self.col_idx = np.ascontiguousarray(col_idx, dtype=np.uint64)
        self.weights = np.ascontiguousarray(weights, dtype=np.float64)

    @staticmethod
    def from_pairs(n: int, offset: float, linear, pairs) -> "ProblemIR":
        """ir.rs:30-69; pairs are (i, j, q) with i < j < n."""
        adj = [[] for _ in range(n)]
        for (i, j, q) in pairs:
            if not (i < j < n):
                raise ValueError("pairs must satisfy i < j < n")
            adj[i].append((j, float(q)))
            adj[j].append((i, float(q)))
        row, col, wts = [0], [], []
        for r in adj:
            r.sort(key=lambda e: e[0])
            k = 0
            while k < len(r):
                j, q = r[k][0], 0.0
                while k < len(r) and r[k][0] == j:
                    q += r[k][1]
                    k += 1
                if q != 0.0:
                    col.append(j)
                    wts.append(q)
            row.append(len(col))
        return ProblemIR(n, offset, linear, row, col, wts)

    @staticmethod
    def from_model(m: QuboModel) -> "ProblemIR":
        return ProblemIR(m.num_vars, m.energy_offset, m.linear, m.row_offsets, m.col_indices, m.values)

    def model(self) -> QuboModel:
        return QuboModel(self.n, self.linear, CsrMatrix(self.weights, self.col_idx, self.row_ptr), self.offset)

    def is_integral(self) -> bool:
        """ir.rs:143-148."""
        f = lambda a: bool(np.all(np.asarray(a) == np.trunc(a)))
        return f(self.offset) and f(self.linear) and f(self.weights)

    def energy(self, x) -> float:
        """ir.rs:85-103: offset, then per set site its linear term and half of
        the sum of its set neighbours' weights."""
        x = np.asarray(x)
        e = self.offset
        for i in range(self.n):
            if x[i] == 0:
                continue
            e += float(self.linear[i])
            pair = 0.0
            for k in range(int(self.row_ptr[i]), int(self.row_ptr[i + 1])):
                if x[int(self.col_idx[k])] != 0:
                    pair += float(self.weights[k])
            e += 0.5 * pair
        return e

    def greedy_coloring(self) -> np.ndarray:
        """ir.rs:114-139, computed by the library."""
        keep: list = []
        prob = _problem(self.model(), keep)
        out = np.zeros(self.n, dtype=np.uint32)
        _ffi.check(_ffi.lib().ie_v2_coloring(C.byref(prob), _p(out)))
        return out


@dataclass
class ChaChaStream:
    """The operators' ChaCha8Rng: seed_from_u64(seed) after `position` draws."""
    seed: int
    position: int = 0


@dataclass
class Report:
    """operator.rs Report: moves proposed / accepted and the work estimate."""
    proposed: int = 0
    accepted: int = 0
    work: float = 0.0


class GpuBitSlice:
    """The bit-sliced state (sparse_bitslice.rs) resident on the device."""

    def __init__(self, ir: ProblemIR, num_replicas: int, init, device: int = 0):
        self._L = _ffi.lib()
        self.ir = ir
        self.r = int(num_replicas)
        self.w = (self.r + 63) // 64
        keep: list = []
        prob = _problem(ir.model(), keep)
        x = np.ascontiguousarray(init, dtype=np.uint8)
        if x.shape != (ir.n,):
            raise ValueError("init must have n entries")
        h = C.c_void_p()
        _ffi.check(self._L.ie_v2_create(C.byref(prob), self.r, _p(x), device, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.ie_v2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_vars(self) -> int:
        return self.ir.n

    def num_replicas(self) -> int:
        return self.r

    def planes(self) -> np.ndarray:
        """[n, ceil(r/64)] u64: bit b of word q of a site = replica 64q + b."""
        out = np.zeros(self.ir.n * self.w, dtype=np.uint64)
        _ffi.check(self._L.ie_v2_read(self._h, _p(out), None))
        return out.reshape(self.ir.n, self.w)

    def energies(self) -> np.ndarray:
        e = np.zeros(self.r, dtype=np.float64)
        _ffi.check(self._L.ie_v2_read(self._h, None, _p(e)))
        return e

    def extract(self, replica: int) -> np.ndarray:
        p = self.planes()
        return ((p[:, replica // 64] >> np.uint64(replica % 64)) & np.uint64(1)).astype(np.uint8)

    def overlap(self, a: int, b: int) -> float:
        """sparse_bitslice.rs:291-303."""
        xa, xb = self.extract(a), self.extract(b)
        return float(np.sum(np.where(xa == xb, 1, -1))) / self.ir.n if self.ir.n else 1.0

    def digest(self) -> int:
        """FNV-1a over the planes' little-endian bytes (state.rs:60-67, sparse_bitslice.rs:313-315)."""
        h = 0xcbf29ce484222325
        for b in self.planes().reshape(-1).astype("<u8").tobytes():
            h ^= b
            h = (h * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
        return h

    def audit(self) -> float:
        d = C.c_double()
        _ffi.check(self._L.ie_v2_audit(self._h, C.byref(d)))
        return d.value


class MetropolisSweep:
    """metropolis_sweep.rs:95-146 on the device."""
    NAME = "metropolis_sweep"

    def apply(self, state: GpuBitSlice, temperatures, rng: ChaChaStream, sweeps: int) -> Report:
        t = np.ascontiguousarray(temperatures, dtype=np.float64)
        p, a = C.c_uint64(), C.c_uint64()
        _ffi.check(state._L.ie_v2_metropolis(state._h, _p(t), len(t), int(sweeps), rng.seed & 0xFFFFFFFFFFFFFFFF,
                                             rng.position, C.byref(p), C.byref(a)))
        rng.position += p.value
        return Report(p.value, a.value, float(state.ir.n * state.r * sweeps))


class GibbsColorSweep:
    """gibbs_color_sweep.rs:119-165 on the device: heat-bath resampling, one
    draw per (site, replica) in chromatic order; T <= 0 is the greedy limit."""
    NAME = "gibbs_color_sweep"

    def apply(self, state: GpuBitSlice, temperatures, rng: ChaChaStream, sweeps: int) -> Report:
        t = np.ascontiguousarray(temperatures, dtype=np.float64)
        p, a = C.c_uint64(), C.c_uint64()
        _ffi.check(state._L.ie_v2_gibbs(state._h, _p(t), len(t), int(sweeps), rng.seed & 0xFFFFFFFFFFFFFFFF,
                                        rng.position, C.byref(p), C.byref(a)))
        rng.position += p.value
        return Report(p.value, a.value, float(state.ir.n * state.r * sweeps))


class ReplicaExchange:
    """replica_exchange.rs:61-110 on the device."""
    NAME = "replica_exchange"

    def apply(self, state: GpuBitSlice, temperatures, rng: ChaChaStream, sweeps: int) -> Report:
        t = np.ascontiguousarray(temperatures, dtype=np.float64)
        if state.r < 2 or len(t) == 0:
            return Report()
        p, a = C.c_uint64(), C.c_uint64()
        _ffi.check(state._L.ie_v2_exchange(state._h, _p(t), len(t), int(sweeps), rng.seed & 0xFFFFFFFFFFFFFFFF,
                                           rng.position, C.byref(p), C.byref(a)))
        rng.position += p.value
        return Report(p.value, a.value, float(sweeps) * state.ir.n * state.r)

"""ie_sa_run_static: one SA run that allocates no device memory.

It exists for callers that cannot call cudaMalloc (hosts whose framework owns
a fixed device pool and forbids other allocators, services that must not
block or fail on an allocation mid-request). The problem and the outputs live
in device memory the caller owns (here: torch tensors); all scratch lives in
the library's fixed static device array. The results must equal the regular
batched entry point's, bit for bit, on two calls in a row.
This file is collected last so a failure here stops a -x run only after every
other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from ising_engine_b200 import _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.engine import BatchEngine

pytestmark = pytest.mark.gpu


def run_static(model, seed, temps, stream=None, cols_override=None):
    import torch
    dev = torch.device("cuda:0")
    rows = torch.tensor(np.asarray(model.row_offsets, dtype=np.uint32).view(np.int32), device=dev)
    c = np.asarray(model.col_indices if cols_override is None else cols_override, dtype=np.uint32)
    cols = torch.tensor(c.view(np.int32), device=dev)
    vals = torch.tensor(np.asarray(model.values, dtype=np.float64), device=dev)
    lin = torch.tensor(np.asarray(model.linear, dtype=np.float64), device=dev)
    words = torch.zeros(model.num_vars, dtype=torch.int64, device=dev)
    energies = torch.zeros(64, dtype=torch.float64, device=dev)
    prob = _ffi.ie_problem_device(model.num_vars, model.nnz, rows.data_ptr(), cols.data_ptr(),
                                  vals.data_ptr(), lin.data_ptr())
    t = np.ascontiguousarray(temps, dtype=np.float64)
    handle = None if stream is None else C.c_void_p(stream.cuda_stream)
    torch.cuda.synchronize()
    st = _ffi.lib().ie_sa_run_static(C.byref(prob), seed, t.ctypes.data_as(C.c_void_p), len(t),
                                     words.data_ptr(), energies.data_ptr(), 0, handle)
    _ffi.check(st)
    torch.cuda.synchronize()
    return words.cpu().numpy().view(np.uint64), energies.cpu().numpy()


def run_regular(model, seed, temps):
    b = BatchEngine([model], [seed])
    b.init_random()
    b.run_schedule(temps)
    w, e = b.spins(), b.energies()[0]
    b.close()
    return w, e


def test_static_run_matches_batched_entry_point_twice():
    rng = np.random.default_rng(2027)
    cases = [(I.random_regular_qubo(700, 12, rng, integer=True), 41, I.sa_temps(40, 0.1, 3.0)),
             (I.random_regular_qubo(333, 18, rng, integer=False), 42, I.sa_temps(25, 0.2, 4.0))]
    for model, seed, temps in cases:  # two calls in a row through the shared scratch
        ws, es = run_static(model, seed, temps)
        wr, er = run_regular(model, seed, temps)
        assert (ws == wr).all()
        assert es.tobytes() == er.tobytes()


def test_static_run_rejects_oversized_input():
    model = I.random_regular_qubo(20000, 3, np.random.default_rng(1), integer=True)
    with pytest.raises(_ffi.EngineError) as ei:
        run_static(model, 1, I.sa_temps(2))
    assert ei.value.status == 1
    assert "16384" in str(ei.value)


def test_static_run_reports_a_bad_csr_then_runs_on_a_stream():
    """A column index >= num_vars is found on the device before any use of the
    CSR and returns IE_ERR_INVALID; the next call, on a non-default stream,
    still equals the batched entry point."""
    import torch
    rng = np.random.default_rng(77)
    model = I.random_regular_qubo(256, 6, rng, integer=True)
    bad = np.asarray(model.col_indices, dtype=np.uint32).copy()
    bad[len(bad) // 2] = model.num_vars + 5
    with pytest.raises(_ffi.EngineError) as ei:
        run_static(model, 3, I.sa_temps(5), cols_override=bad)
    assert ei.value.status == 1
    assert "invalid CSR" in str(ei.value)
    temps = I.sa_temps(12, 0.2, 2.0)
    s = torch.cuda.Stream()
    ws, es = run_static(model, 9, temps, stream=s)
    wr, er = run_regular(model, 9, temps)
    assert (ws == wr).all()
    assert es.tobytes() == er.tobytes()

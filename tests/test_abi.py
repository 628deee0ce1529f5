"""The C-ABI library builds, loads and exports every function the header
declares; host-only entry points behave without a GPU."""
import ctypes as C

import numpy as np

from ising_engine_b200 import _build, _ffi
from ising_engine_b200 import instances as I
from ising_engine_b200.engine import _problem


def test_library_exports_every_header_symbol():
    L = _ffi.lib()
    syms = _ffi.header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) == set(_ffi._SIGS), "bindings and header disagree"
    assert L.ie_abi_version() == 1


def test_library_is_in_tree():
    assert _build.LIB_PATH.startswith(_build.HERE)


def test_invalid_arguments_return_status_not_abort():
    L = _ffi.lib()
    assert L.ie_create(None, None, None) == 1  # IE_ERR_INVALID
    assert b"NULL" in L.ie_last_error()
    assert L.ie_geometric_temps(1.0, 0.1, 0, None) == 1


def test_suggested_temp_range_matches_definition():
    """src/solver/schedule.rs:21-43."""
    m = I.maxcut_gnm(50, 200, 3)
    from ising_engine_b200.engine import suggested_temp_range
    tmax, tmin = suggested_temp_range(m)
    ro, va, lin = m.row_offsets.astype(int), m.values, m.linear
    ml = max(abs(lin[i]) + np.abs(va[ro[i]:ro[i + 1]]).sum() for i in range(m.num_vars))
    mn = min(np.abs(lin[lin != 0]).min(), np.abs(va[va != 0]).min())
    assert tmax == ml / np.log(2.0)
    assert tmin == min(mn / np.log(100.0), tmax * 0.5)


def _header_struct_fields(name):
    """Field names, in order, of `typedef struct name { ... } name;` in the header."""
    import os
    import re
    txt = open(os.path.join(os.path.dirname(_build.HERE), "include", "ising_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), txt, flags=re.S)
    assert m, name
    fields = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if decl:
            fields += [v.strip().lstrip("*") for v in decl.split()[-1].split(",")]
    return fields


def test_config_structs_match_the_header():
    """The ctypes mirrors of the config structs list the header's fields in
    the header's order (callers zero-initialise and set fields by name, so a
    field out of place would shift every later one)."""
    for name in ["ie_config", "ie_batch_config", "ie_serve_config", "ie_pa_config", "ie_problem"]:
        ours = [f[0] for f in getattr(_ffi, name)._fields_]
        assert ours == _header_struct_fields(name), name


def test_fnv1a_matches_the_reference_definition():
    """ie_fnv1a is FNV-1a 64 (src/engine_v2/state.rs:60-67): offset basis
    0xcbf29ce484222325, prime 0x100000001b3, xor then multiply per byte."""
    rng = np.random.default_rng(5)
    for n in (0, 1, 7, 64, 1000):
        data = rng.integers(0, 256, size=n, dtype=np.uint8)
        h = 0xcbf29ce484222325
        for b in data.tobytes():
            h = ((h ^ b) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
        out = C.c_uint64()
        buf = data.ctypes.data if n else None
        assert _ffi.lib().ie_fnv1a(buf, n, C.byref(out)) == 0
        assert out.value == h
    assert _ffi.lib().ie_fnv1a(None, 0, C.byref(out)) == 0 and out.value == 0xcbf29ce484222325

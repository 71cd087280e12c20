"""The C ABI on the host side (no GPU work): the library loads and exports
every function include/minisweep_b200.h declares, and the host parts of the
reference API behave as the reference's (flags, sizes, built-in Quantities,
state initialisation and norms, Sweeper flag validation)."""
import ctypes
import os
import re

import numpy as np
import pytest

import minisweep_b200 as msb
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "minisweep_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M):
        line_start = src.rfind("\n", 0, m.start()) + 1
        line = src[line_start:m.end()]
        if line.lstrip().startswith(("static", "#", "typedef", "enum", "return")):
            continue
        names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_function():
    L = msb.lib()
    names = declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_mirror_headers_resolve_to_the_abi():
    for h in ["env.h", "arguments.h", "pointer.h", "dimensions.h", "quantities.h", "sweeper.h",
              "array_operations.h", "definitions.h", "types.h"]:
        txt = open(os.path.join(ROOT, "include", h)).read()
        assert '#include "minisweep_b200.h"' in txt


def _args(s):
    a = msb.Arguments()
    msb.lib().Arguments_create_from_string(ctypes.byref(a), s.encode())
    return a


def test_arguments_read_once():
    L = msb.lib()
    a = _args("--ncell_x 7 --ne 3 --bogus 1")
    g = lambda n, d: L.Arguments_consume_int_or_default(ctypes.byref(a), n.encode(), d)
    assert g("--ncell_x", 5) == 7
    assert g("--ncell_x", 5) == 5  # consumed: default now
    assert g("--na", 33) == 33
    assert g("--ne", 30) == 3
    assert not L.Arguments_are_all_consumed(ctypes.byref(a))
    assert g("--bogus", 0) == 1
    assert L.Arguments_are_all_consumed(ctypes.byref(a))
    L.Arguments_destroy(ctypes.byref(a))


def test_dimensions_sizes():
    L = msb.lib()
    L.Dimensions_size_state.argtypes = [msb.Dimensions, ctypes.c_int]
    L.Dimensions_size_state.restype = ctypes.c_size_t
    L.Dimensions_size_state_angles.argtypes = [msb.Dimensions, ctypes.c_int]
    L.Dimensions_size_state_angles.restype = ctypes.c_size_t
    d = msb.Dimensions(3, 4, 5, 6, 16, 7)
    assert L.Dimensions_size_state(d, 4) == 3 * 4 * 5 * 6 * 16 * 4
    assert L.Dimensions_size_state_angles(d, 4) == 3 * 4 * 5 * 6 * 7 * 4 * 8


@pytest.mark.parametrize("nm,na", [(16, 32), (4, 7), (16, 33), (8, 100)])
def test_builtin_quantities_match_oracle(nm, na):
    L = msb.lib()
    env = msb.Env()
    q = msb.Quantities()
    d = msb.Dimensions(3, 4, 5, 2, nm, na)
    L.Quantities_create(ctypes.byref(q), d, ctypes.byref(env))
    n = nm * na * 8
    a = np.ctypeslib.as_array(ctypes.cast(q.a_from_m.h_, ctypes.POINTER(ctypes.c_double)), (n,)).copy()
    m = np.ctypeslib.as_array(ctypes.cast(q.m_from_a.h_, ctypes.POINTER(ctypes.c_double)), (n,)).copy()
    ra, rm = oracle.am_matrices(nm, na)
    assert np.array_equal(a, ra) and np.array_equal(m, rm)
    v = np.zeros(3 * 4 * 5 * 2 * nm * 4)
    L.initialize_state(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d, 4, ctypes.byref(q))
    assert np.array_equal(v, oracle.init_state(3, 4, 5, 2, nm))
    s, dd = ctypes.c_double(), ctypes.c_double()
    w = v.copy()
    w[7] += 0.5
    L.get_state_norms(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                      w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d, 4, ctypes.byref(s), ctypes.byref(dd),
                      ctypes.byref(env))
    assert dd.value == 0.25 and s.value == float(np.sum(w * w))
    L.Quantities_destroy(ctypes.byref(q))


@pytest.mark.parametrize("flags,msg", [
    ("--nblock_z 3", "same z dimension"),        # ncell_z % nblock_z != 0 (sweeper_kba_c.h:71-72)
    ("--nblock_z 0", "blocking factor"),
    ("--nthread_octant 3", "thread count"),       # power of two in [1, 8]
    ("--nsemiblock 16", "semiblock count"),
    ("--nthread_octant 8 --nsemiblock 2", "atomic vo update"),
    ("--ncell_x_per_subblock 0", "subblock size"),
    ("--nthread_e 0", "thread count"),
])
def test_sweeper_rejects_invalid_flags(flags, msg):
    L = msb.lib()
    env = msb.Env()
    a = _args(flags)
    q = msb.Quantities()
    d = msb.Dimensions(4, 4, 4, 2, 16, 8)
    L.Quantities_create(ctypes.byref(q), d, ctypes.byref(env))
    sw = msb.Sweeper()
    rc = L.Sweeper_create_status(ctypes.byref(sw), d, ctypes.byref(q), ctypes.byref(env), ctypes.byref(a))
    assert rc == msb.MSB_ERR_ARG
    assert msg in msb.last_error()
    L.Quantities_destroy(ctypes.byref(q))
    L.Arguments_destroy(ctypes.byref(a))


def test_unsupported_sizes_are_reported():
    L = msb.lib()
    env = msb.Env()
    a = _args("")
    q = msb.Quantities()
    d = msb.Dimensions(4, 4, 4, 2, 12, 8)  # NM = 12 has no kernel variant
    L.Quantities_create(ctypes.byref(q), d, ctypes.byref(env))
    sw = msb.Sweeper()
    rc = L.Sweeper_create_status(ctypes.byref(sw), d, ctypes.byref(q), ctypes.byref(env), ctypes.byref(a))
    assert rc in (msb.MSB_ERR_UNSUPPORTED, msb.MSB_ERR_CUDA)
    L.Quantities_destroy(ctypes.byref(q))
    L.Arguments_destroy(ctypes.byref(a))


@pytest.mark.parametrize("flags,d,code", [
    ("--precision 3", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_ARG),          # no such precision
    ("--precision -1", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_ARG),
    ("--precision 1", (4, 4, 4, 2, 16, 129), msb.MSB_ERR_UNSUPPORTED),  # na <= 128 (four 32-angle passes)
    ("--precision 2", (4, 4, 4, 2, 12, 32), msb.MSB_ERR_UNSUPPORTED),  # NM 12
    ("--tile 33", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_ARG),              # tile shapes: 0, 42, 24
    ("--autotune 2", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_ARG),
    ("--tile 24 --precision 1", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_UNSUPPORTED),  # mixed: one 4 x 4 tile
    ("--tile 24", (4, 4, 4, 2, 16, 129), msb.MSB_ERR_UNSUPPORTED),     # na <= 128
    ("--autotune 1 --precision 1", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_UNSUPPORTED),  # FP64 only
    ("--ie_base -2", (4, 4, 4, 2, 16, 32), msb.MSB_ERR_ARG),           # first global group of a slice
])
def test_precision_flag_checks(flags, d, code):
    L = msb.lib()
    env = msb.Env()
    a = _args(flags)
    q = msb.Quantities()
    dims = msb.Dimensions(*d)
    L.Quantities_create(ctypes.byref(q), dims, ctypes.byref(env))
    sw = msb.Sweeper()
    rc = L.Sweeper_create_status(ctypes.byref(sw), dims, ctypes.byref(q), ctypes.byref(env), ctypes.byref(a))
    assert rc == code, msb.last_error()
    L.Quantities_destroy(ctypes.byref(q))
    L.Arguments_destroy(ctypes.byref(a))

"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU checkers.

* ``liboracle.so`` -- the repository's plain-C FP64 restatement of the reference
  sweep (``oracle/sweep_oracle.c``), compiled by ``make -C oracle``.
* ``_ref/libref_nm{4,16}.so`` -- the reference's own serial KBA sweeper compiled
  from its sources together with ``oracle/ref_dump.c`` (``make -C oracle ref``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package; the product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NOCTANT = 8
_dp = ctypes.POINTER(ctypes.c_double)


def reference_tree() -> str:
    """The reference's source tree: $MINISWEEP_REF when set, else a checkout
    named ``reference`` beside this repository (the Makefile's default too)."""
    return os.environ.get("MINISWEEP_REF") or os.path.abspath(os.path.join(HERE, "..", "..", "reference"))


def build(with_reference: bool | None = None) -> None:
    """Compile the C restatement (and the reference build when its tree exists)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    if with_reference is None:
        with_reference = os.path.isdir(os.path.join(reference_tree(), "src"))
    if with_reference:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])
        # the reference's own CUDA sweep for sm_100a (a timing comparator)
        subprocess.check_call(["make", "-s", "-C", HERE, "ref_cuda"], stdout=subprocess.DEVNULL,
                              stderr=subprocess.DEVNULL)
        # the reference's driver programs linked with the product library
        if os.path.exists(os.path.join(os.path.dirname(HERE), "minisweep_b200", "libminisweep_b200.so")):
            subprocess.check_call(["make", "-s", "-C", HERE, "dropin"])


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(with_reference=False)
        L = ctypes.CDLL(path)
        L.oracle_init_am_matrices.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.oracle_init_state.argtypes = [ctypes.c_int] * 6 + [_dp]
        L.oracle_sweep.argtypes = [ctypes.c_int] * 7 + [_dp, _dp, _dp, _dp]
        L.oracle_sweep_groups.argtypes = [ctypes.c_int] * 9 + [_dp, _dp, _dp, _dp]
        L.oracle_state_norms.argtypes = [ctypes.c_size_t, _dp, _dp, _dp, _dp]
        L.oracle_normsq_closed_form.argtypes = [ctypes.c_int] * 6
        L.oracle_normsq_closed_form.restype = ctypes.c_double
        L.oracle_scalefactor_space.argtypes = [ctypes.c_int] * 3
        L.oracle_scalefactor_energy.argtypes = [ctypes.c_int]
        L.oracle_scalefactor_unknown.argtypes = [ctypes.c_int]
        L.oracle_init_face.argtypes = [ctypes.c_int] * 7
        L.oracle_init_face.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def state_size(nx, ny, nz, ne, nm, nu=4) -> int:
    return nx * ny * nz * ne * nm * nu


def am_matrices(nm: int, na: int):
    a = np.zeros(nm * na * NOCTANT)
    m = np.zeros(nm * na * NOCTANT)
    lib().oracle_init_am_matrices(nm, na, _p(a), _p(m))
    return a, m


def init_state(nx, ny, nz, ne, nm, nu=4) -> np.ndarray:
    v = np.zeros(state_size(nx, ny, nz, ne, nm, nu))
    lib().oracle_init_state(nx, ny, nz, ne, nm, nu, _p(v))
    return v


def sweep(nx, ny, nz, ne, nm, na, a_from_m, m_from_a, vi, nu=4, groups=None) -> np.ndarray:
    vi = np.ascontiguousarray(vi, dtype=np.float64)
    vo = np.zeros_like(vi)
    a_from_m = np.ascontiguousarray(a_from_m, dtype=np.float64)
    m_from_a = np.ascontiguousarray(m_from_a, dtype=np.float64)
    if groups is None:
        lib().oracle_sweep(nx, ny, nz, ne, nm, nu, na, _p(a_from_m), _p(m_from_a), _p(vi), _p(vo))
    else:
        lib().oracle_sweep_groups(nx, ny, nz, ne, nm, nu, na, groups[0], groups[1],
                                  _p(a_from_m), _p(m_from_a), _p(vi), _p(vo))
    return vo


def norms(vi: np.ndarray, vo: np.ndarray):
    s, d = ctypes.c_double(), ctypes.c_double()
    lib().oracle_state_norms(vi.size, _p(vi), _p(vo), ctypes.byref(s), ctypes.byref(d))
    return s.value, d.value


def normsq_closed_form(nx, ny, nz, ne, nm, nu=4) -> float:
    return lib().oracle_normsq_closed_form(nx, ny, nz, ne, nm, nu)


def random_problem(nx, ny, nz, ne, nm, na, seed=1234, nu=4):
    """Random-input variant: vi ~ U[0,1), a_from_m ~ N(0, 1/nm) per octant and
    m_from_a = pinv(a_from_m) per octant in FP64 (numpy PCG64 + SVD pinv).
    Layouts are the reference's (see sweep_oracle.h)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    vi = rng.random(state_size(nx, ny, nz, ne, nm, nu))
    a = np.zeros((NOCTANT, nm, na))
    m = np.zeros((NOCTANT, na, nm))
    for o in range(NOCTANT):
        A = rng.normal(0.0, 1.0 / np.sqrt(nm), size=(na, nm))  # [ia][im]
        a[o] = A.T                                             # stored [im][ia]
        m[o] = np.linalg.pinv(A).T                             # pinv is [im][ia]; stored [ia][im]
    return a.reshape(-1), m.reshape(-1), vi


# ---------------------------------------------------------------- reference
_ref = {}


def ref_lib(nm: int):
    if nm not in _ref:
        path = os.path.join(HERE, "_ref", f"libref_nm{nm}.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        L.ref_run.argtypes = [ctypes.c_char_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_run.restype = ctypes.c_int
        _ref[nm] = L
    return _ref[nm]


def ref_run(argstring: str, nx, ny, nz, ne, nm, a_from_m=None, m_from_a=None, vi=None, nu=4):
    """Run the reference's own serial KBA sweeper (oracle/_ref). Returns
    (vo, vi, normsq, normsqdiff) as the reference's runner leaves them."""
    L = ref_lib(nm)
    if L is None:
        raise FileNotFoundError("reference build missing (make -C oracle ref)")
    n = state_size(nx, ny, nz, ne, nm, nu)
    vo_out = np.zeros(n)
    vi_out = np.zeros(n)
    s, d = ctypes.c_double(), ctypes.c_double()
    keep = []

    def opt(x):
        if x is None:
            return None
        x = np.ascontiguousarray(x, dtype=np.float64)
        keep.append(x)
        return _p(x)

    rc = L.ref_run(argstring.encode(), opt(a_from_m), opt(m_from_a), opt(vi),
                   _p(vo_out), _p(vi_out), ctypes.byref(s), ctypes.byref(d))
    if rc != 0:
        raise ValueError(f"reference rejected flags: {argstring}")
    return vo_out, vi_out, s.value, d.value

"""minisweep_b200 -- B200-native KBA sweep behind the minisweep C API.

The product is ``libminisweep_b200.so`` (C ABI declared in
``include/minisweep_b200.h``).  This module is a thin ctypes binding used by
the tests and the benchmark: it mirrors the reference's C structs and calls
the library's entry points.  There is no Python or CPU compute path; if the
library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libminisweep_b200.so")
NU = 4
NOCTANT = 8
TASK_INTS = 16

MSB_OK, MSB_ERR_ARG, MSB_ERR_CUDA, MSB_ERR_TIMEOUT, MSB_ERR_UNSUPPORTED = 0, -1, -2, -3, -4


def build() -> None:
    """Compile the CUDA library in-tree for sm_100a."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "csrc"), "-j8"])


class Dimensions(ctypes.Structure):
    _fields_ = [("ncell_x", ctypes.c_int), ("ncell_y", ctypes.c_int), ("ncell_z", ctypes.c_int),
                ("ne", ctypes.c_int), ("nm", ctypes.c_int), ("na", ctypes.c_int)]


class Arguments(ctypes.Structure):
    _fields_ = [("argc", ctypes.c_int), ("argv_unconsumed", ctypes.POINTER(ctypes.c_char_p)),
                ("argstring", ctypes.c_char_p)]


class Env(ctypes.Structure):
    _fields_ = [("nproc_x_", ctypes.c_int), ("nproc_y_", ctypes.c_int), ("tag_", ctypes.c_int),
                ("is_proc_active_", ctypes.c_int), ("is_using_device_", ctypes.c_int),
                ("stream_kernel_faces_", ctypes.c_void_p), ("device_", ctypes.c_int), ("proc_", ctypes.c_int),
                ("nproc_world_", ctypes.c_int), ("flags_", ctypes.c_int), ("comm_", ctypes.c_void_p)]


class KbaMsg(ctypes.Structure):
    """msb_kba_msg: one face slab crossing between neighbouring processes."""
    _fields_ = [("peer", ctypes.c_int), ("is_send", ctypes.c_int), ("axis", ctypes.c_int), ("side", ctypes.c_int),
                ("bytes", ctypes.c_size_t), ("buf", ctypes.c_void_p)]


EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(KbaMsg), ctypes.c_int)
SUM_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double))
ALLGATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_int))
BARRIER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int)


class Comm(ctypes.Structure):
    """msb_comm: the process group's transport, as C callbacks."""
    _fields_ = [("ctx", ctypes.c_void_p), ("exchange", EXCHANGE_FN), ("sum_double", SUM_FN),
                ("allgather_int", ALLGATHER_FN), ("barrier", BARRIER_FN)]


class Pointer(ctypes.Structure):
    _fields_ = [("n_", ctypes.c_size_t), ("h_", ctypes.c_void_p), ("d_", ctypes.c_void_p),
                ("is_using_device_", ctypes.c_int), ("is_pinned_", ctypes.c_int), ("is_alias_", ctypes.c_int)]


class Quantities(ctypes.Structure):
    _fields_ = [("a_from_m", Pointer), ("m_from_a", Pointer), ("ix_base_vals", ctypes.c_void_p),
                ("iy_base_vals", ctypes.c_void_p), ("ix_base", ctypes.c_int), ("iy_base", ctypes.c_int),
                ("ncell_x_g", ctypes.c_int), ("ncell_y_g", ctypes.c_int), ("ncell_z_g", ctypes.c_int)]


class Sweeper(ctypes.Structure):
    _fields_ = [("dims", Dimensions), ("dims_b", Dimensions), ("dims_g", Dimensions)] + [
        (n, ctypes.c_int) for n in (
            "nblock_z", "nblock_octant", "noctant_per_block", "nsemiblock", "ncell_x_per_subblock",
            "ncell_y_per_subblock", "ncell_z_per_subblock", "nthread_e", "nthread_octant", "nthread_x",
            "nthread_y", "nthread_z", "is_face_comm_async", "precision")] + [("impl_", ctypes.c_void_p)]


class ProblemDesc(ctypes.Structure):
    """msb_problem: one problem of a batch (sizes + device arrays)."""
    _fields_ = [("ncell_x", ctypes.c_int), ("ncell_y", ctypes.c_int), ("ncell_z", ctypes.c_int),
                ("ne", ctypes.c_int), ("na", ctypes.c_int), ("nm", ctypes.c_int),
                ("vi", ctypes.c_void_p), ("vo", ctypes.c_void_p),
                ("a_from_m", ctypes.c_void_p), ("m_from_a", ctypes.c_void_p)]


MAX_CLASSES = 16


class BatchInfo(ctypes.Structure):
    _fields_ = [("nproblem", ctypes.c_int), ("nclass", ctypes.c_int), ("npred", ctypes.c_int),
                ("nsm", ctypes.c_int), ("ntask", ctypes.c_longlong), ("scratch_bytes", ctypes.c_size_t),
                ("scratch_needed_all", ctypes.c_size_t), ("sim_makespan", ctypes.c_double),
                ("sim_busy", ctypes.c_double), ("tune_ms", ctypes.c_double),
                ("class_nm", ctypes.c_int * MAX_CLASSES), ("class_nch", ctypes.c_int * MAX_CLASSES),
                ("class_tx", ctypes.c_int * MAX_CLASSES), ("class_ty", ctypes.c_int * MAX_CLASSES),
                ("class_ntask", ctypes.c_longlong * MAX_CLASSES)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() (CUDA library not built)")
        L = ctypes.CDLL(LIB_PATH)
        P, D = ctypes.POINTER, ctypes.c_double
        L.msb_last_error.restype = ctypes.c_char_p
        L.Env_initialize.argtypes = [P(Env), ctypes.c_int, ctypes.c_void_p]
        L.Env_set_values.argtypes = [P(Env), P(Arguments)]
        L.Env_finalize.argtypes = [P(Env)]
        L.Arguments_create_from_string.argtypes = [P(Arguments), ctypes.c_char_p]
        L.Arguments_destroy.argtypes = [P(Arguments)]
        L.Arguments_consume_int_or_default.argtypes = [P(Arguments), ctypes.c_char_p, ctypes.c_int]
        L.Arguments_are_all_consumed.argtypes = [P(Arguments)]
        L.Quantities_create.argtypes = [P(Quantities), Dimensions, P(Env)]
        L.Quantities_destroy.argtypes = [P(Quantities)]
        L.Sweeper_create_status.argtypes = [P(Sweeper), Dimensions, P(Quantities), P(Env), P(Arguments)]
        L.Sweeper_destroy.argtypes = [P(Sweeper), P(Env)]
        L.Sweeper_sweep_status.argtypes = [P(Sweeper), P(Pointer), P(Pointer), P(Quantities), P(Env)]
        L.Sweeper_sweep_device.argtypes = [P(Sweeper), ctypes.c_void_p, ctypes.c_void_p, P(Quantities), P(Env)]
        L.Sweeper_sync_status.argtypes = [P(Sweeper), P(Env)]
        L.Sweeper_sweep_iterations.argtypes = [P(Sweeper), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               P(Quantities), P(Env)]
        L.msb_measure_fp64_peak.argtypes = [P(D), P(D), ctypes.c_int]
        L.Sweeper_last_stats.argtypes = [P(Sweeper), P(ctypes.c_longlong), P(ctypes.c_int)]
        L.msb_iterations_slices.argtypes = [P(Sweeper)]
        L.Sweeper_debug_tasks.argtypes = [P(Sweeper), P(ctypes.c_int), ctypes.c_longlong]
        L.Sweeper_debug_tasks.restype = ctypes.c_longlong
        L.Sweeper_set_spin_limit.argtypes = [P(Sweeper), ctypes.c_longlong]
        L.Sweeper_tile.argtypes = [P(Sweeper), P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_float),
                                   P(ctypes.c_float)]
        L.Sweeper_plan.argtypes = [P(Sweeper)] + [P(ctypes.c_int)] * 5
        L.msb_state_norms_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, P(D), P(D), P(Env)]
        L.msb_initialize_state_device.argtypes = [ctypes.c_void_p, Dimensions, P(Env)]
        L.msb_initialize_state_slice_device.argtypes = [ctypes.c_void_p, Dimensions, ctypes.c_int, P(Env)]
        L.msb_schedule_tasks.argtypes = [ctypes.c_int] * 7 + [P(ctypes.c_int), ctypes.c_longlong]
        L.msb_schedule_tasks.restype = ctypes.c_longlong
        L.msb_batch_create.argtypes = [P(ctypes.c_void_p), P(ProblemDesc), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_size_t, ctypes.c_int]
        L.msb_batch_plan.argtypes = [P(ctypes.c_void_p), P(ProblemDesc), ctypes.c_int, ctypes.c_int,
                                     ctypes.c_size_t, ctypes.c_int]
        L.msb_batch_destroy.argtypes = [ctypes.c_void_p]
        L.msb_batch_destroy.restype = None
        L.msb_batch_sweep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.msb_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.msb_batch_sync.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.msb_batch_problem_ms.argtypes = [ctypes.c_void_p, P(D), ctypes.c_int]
        L.msb_batch_info.argtypes = [ctypes.c_void_p, P(BatchInfo)]
        L.msb_batch_tasks.argtypes = [ctypes.c_void_p, P(ctypes.c_int), P(ctypes.c_int), ctypes.c_longlong]
        L.msb_batch_tasks.restype = ctypes.c_longlong
        L.msb_batch_entries.argtypes = [ctypes.c_void_p, P(ctypes.c_int), P(ctypes.c_int), ctypes.c_int]
        L.msb_batch_scratch.argtypes = [ctypes.c_void_p, P(ctypes.c_longlong), P(ctypes.c_longlong),
                                        P(ctypes.c_int), P(ctypes.c_int), ctypes.c_int]
        L.msb_batch_set_spin_limit.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        L.msb_builtin_matrices.argtypes = [ctypes.c_int, ctypes.c_int, P(D), P(D)]
        L.msb_env_set_comm.argtypes = [P(Env), ctypes.c_int, ctypes.c_int, P(Comm)]
        IP = P(ctypes.c_int)
        L.msb_kba_plan.argtypes = [ctypes.c_int] * 3 + [IP] * 4
        L.msb_kba_plan_messages.argtypes = [ctypes.c_int] * 5 + [IP, ctypes.c_int]
        L.msb_kba_info.argtypes = [P(Sweeper), IP, P(ctypes.c_size_t), P(ctypes.c_size_t)]
        L.msb_kba_set_buffers.argtypes = [P(Sweeper)] + [ctypes.c_void_p] * 6
        L.msb_kba_begin.argtypes = [P(Sweeper), ctypes.c_void_p, ctypes.c_void_p, P(Quantities), P(Env)]
        L.msb_kba_step.argtypes = [P(Sweeper), ctypes.c_int, P(Env)]
        L.msb_kba_messages.argtypes = [P(Sweeper), ctypes.c_int, P(KbaMsg), ctypes.c_int]
        L.msb_kba_unpack.argtypes = [P(Sweeper), ctypes.c_int, P(Env)]
        L.msb_kba_end.argtypes = [P(Sweeper), P(Env)]
        L.initialize_state.argtypes = [P(D), Dimensions, ctypes.c_int, P(Quantities)]
        L.get_state_norms.argtypes = [P(D), P(D), Dimensions, ctypes.c_int, P(D), P(D), P(Env)]
        _lib = L
    return _lib


class SweepError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check(rc: int) -> None:
    if rc != MSB_OK:
        raise SweepError(rc, lib().msb_last_error().decode())


def last_error() -> str:
    return lib().msb_last_error().decode()


def schedule(nx, ny, nz, ne, tx=4, ty=2, gp_block=1) -> np.ndarray:
    """Task table (ntask x 16 ints) the sweeper builds; no GPU needed."""
    L = lib()
    n = L.msb_schedule_tasks(nx, ny, nz, ne, tx, ty, gp_block, None, 0)
    if n < 0:
        raise SweepError(int(n), last_error())
    out = np.zeros((n, TASK_INTS), dtype=np.int32)
    L.msb_schedule_tasks(nx, ny, nz, ne, tx, ty, gp_block, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
    return out


def kba_plan(nproc_x: int, nproc_y: int, nblock_z: int):
    """Step plan of a decomposed sweep (host only): (nstep, unit_oct, unit_zb,
    start[proc, unit]).  Unit k is octant unit_oct[k] on z-block unit_zb[k]."""
    L = lib()
    IP = ctypes.POINTER(ctypes.c_int)
    nunit = NOCTANT * nblock_z
    nstep = ctypes.c_int()
    oct_ = np.zeros(nunit, dtype=np.int32)
    zb = np.zeros(nunit, dtype=np.int32)
    start = np.zeros((nproc_x * nproc_y, nunit), dtype=np.int32)
    _check(L.msb_kba_plan(nproc_x, nproc_y, nblock_z, ctypes.byref(nstep), oct_.ctypes.data_as(IP),
                          zb.ctypes.data_as(IP), start.ctypes.data_as(IP)))
    return nstep.value, oct_, zb, start


def kba_plan_messages(nproc_x: int, nproc_y: int, nblock_z: int, proc: int, step: int):
    """Messages of process `proc` after step `step` (host only): a list of
    dicts peer / is_send / axis / side / unit."""
    out = np.zeros(5 * 8, dtype=np.int32)
    n = lib().msb_kba_plan_messages(nproc_x, nproc_y, nblock_z, proc, step,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 8)
    if n < 0:
        raise SweepError(n, last_error())
    keys = ("peer", "is_send", "axis", "side", "unit")
    return [dict(zip(keys, (int(v) for v in out[5 * i:5 * i + 5]))) for i in range(n)]


def local_extent(n_global: int, nproc: int, proc: int):
    """(offset, size) of process `proc`'s share of n_global cells along one
    axis, as the reference's driver splits it (runner.c:95-106)."""
    lo, hi = (proc * n_global) // nproc, ((proc + 1) * n_global) // nproc
    return lo, hi - lo


def make_comm(exchange, sum_double, allgather_int, barrier) -> Comm:
    """msb_comm from Python callables: exchange(nactive, msgs) with msgs a
    list of KbaMsg; sum_double(nactive, x) -> float; allgather_int(nactive, v) ->
    list of ints; barrier(nactive) -- the collectives over the active
    processes 0 .. nactive - 1.  A callable that raises makes the call return
    -1.  Keep the result alive as long as an Env uses it (it holds the
    callbacks)."""
    import traceback

    def guard(fn):
        def call(*a):
            try:
                return fn(*a)
            except Exception:  # the C caller only sees the status
                traceback.print_exc()
                return -1
        return call

    def ex(_ctx, nactive, msgs, n):
        exchange(nactive, [msgs[i] for i in range(n)])
        return 0

    def sm(_ctx, nactive, v):
        v[0] = float(sum_double(nactive, v[0]))
        return 0

    def ag(_ctx, nactive, value, out):
        vals = allgather_int(nactive, int(value))
        for i, x in enumerate(vals):
            out[i] = int(x)
        return 0

    def br(_ctx, nactive):
        barrier(nactive)
        return 0

    c = Comm(None, EXCHANGE_FN(guard(ex)), SUM_FN(guard(sm)), ALLGATHER_FN(guard(ag)), BARRIER_FN(guard(br)))
    return c


def fp64_peak(reps: int = 5):
    """Measured FP64 throughput of this GPU (TFLOP/s): (tensor-core mma, FMA pipe)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(lib().msb_measure_fp64_peak(ctypes.byref(a), ctypes.byref(b), reps))
    return a.value, b.value


def random_matrices(nm: int, na: int, seed: int = 1234):
    """Transform matrices of the random-input precision study, in the
    reference layouts: a_from_m[oct][im][ia] drawn N(0, 1/nm) (numpy PCG64),
    m_from_a[oct][ia][im] = its least-squares pseudo-inverse in FP64 (SVD).
    The state of that study is drawn U[0, 1) by the caller."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = np.zeros((NOCTANT, nm, na))
    m = np.zeros((NOCTANT, na, nm))
    for o in range(NOCTANT):
        A = rng.normal(0.0, 1.0 / np.sqrt(nm), size=(na, nm))  # [ia][im]
        a[o] = A.T
        m[o] = np.linalg.pinv(A).T
    return a.reshape(-1), m.reshape(-1)


class Problem:
    """One sweep problem driven through the reference-compatible C API:
    Env + Quantities (built-in) + Sweeper created from a reference flag string."""

    def __init__(self, argstring: str, nm: int = 16, proc: int = 0, nproc: int = 1, comm: Comm = None):
        """proc / nproc / comm: this process's place in a process group (the
        counterpart of the reference's MPI world); with --nproc_x / --nproc_y
        the problem is then this process's subdomain of the global one
        (runner.c:95-106)."""
        L = lib()
        self.env = Env()
        L.Env_initialize(ctypes.byref(self.env), 0, None)
        self._comm = comm
        if nproc > 1 or comm is not None:
            _check(L.msb_env_set_comm(ctypes.byref(self.env), proc, nproc,
                                      ctypes.byref(comm) if comm is not None else None))
        self.args = Arguments()
        L.Arguments_create_from_string(ctypes.byref(self.args), argstring.encode())
        L.Env_set_values(ctypes.byref(self.env), ctypes.byref(self.args))
        g = lambda name, d: L.Arguments_consume_int_or_default(ctypes.byref(self.args), name.encode(), d)
        gx, gy = g("--ncell_x", 5), g("--ncell_y", 5)
        npx, npy = self.env.nproc_x_, self.env.nproc_y_
        self.x0, nx = local_extent(gx, npx, proc % npx)
        self.y0, ny = local_extent(gy, npy, proc // npx)
        self.dims = Dimensions(nx, ny, g("--ncell_z", 5), g("--ne", 30), nm, g("--na", 33))
        self.dims_global = Dimensions(gx, gy, self.dims.ncell_z, self.dims.ne, nm, self.dims.na)
        self.niterations = g("--niterations", 1)
        self.quan = Quantities()
        L.Quantities_create(ctypes.byref(self.quan), self.dims, ctypes.byref(self.env))
        self.sweeper = Sweeper()
        rc = L.Sweeper_create_status(ctypes.byref(self.sweeper), self.dims, ctypes.byref(self.quan),
                                     ctypes.byref(self.env), ctypes.byref(self.args))
        if rc != MSB_OK:
            msg = last_error()
            L.Quantities_destroy(ctypes.byref(self.quan))
            L.Arguments_destroy(ctypes.byref(self.args))
            L.Env_finalize(ctypes.byref(self.env))
            raise SweepError(rc, msg)
        if not L.Arguments_are_all_consumed(ctypes.byref(self.args)):
            self.close()
            raise SweepError(MSB_ERR_ARG, "Invalid argument detected.")
        self.nstate = (self.dims.ncell_x * self.dims.ncell_y * self.dims.ncell_z * self.dims.ne * nm * NU)
        self._closed = False

    # ---------------------------------------------------------------- data
    def matrices(self):
        """Host copies of a_from_m and m_from_a (reference layouts)."""
        n = self.dims.nm * self.dims.na * NOCTANT
        a = np.ctypeslib.as_array(ctypes.cast(self.quan.a_from_m.h_, ctypes.POINTER(ctypes.c_double)), (n,))
        m = np.ctypeslib.as_array(ctypes.cast(self.quan.m_from_a.h_, ctypes.POINTER(ctypes.c_double)), (n,))
        return a, m

    def set_matrices(self, a_from_m: np.ndarray, m_from_a: np.ndarray) -> None:
        a, m = self.matrices()
        a[:] = a_from_m
        m[:] = m_from_a

    def init_state(self) -> np.ndarray:
        v = np.zeros(self.nstate)
        lib().initialize_state(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.dims, NU,
                               ctypes.byref(self.quan))
        return v

    # ---------------------------------------------------------------- runs
    def sweep_host(self, vi: np.ndarray) -> np.ndarray:
        """vo = sweep(vi) through Sweeper_sweep's reference semantics (host in, host out)."""
        vi = np.ascontiguousarray(vi, dtype=np.float64)
        vo = np.zeros_like(vi)
        pvi = Pointer(vi.size, vi.ctypes.data, None, 0, 0, 0)
        pvo = Pointer(vo.size, vo.ctypes.data, None, 0, 0, 0)
        _check(lib().Sweeper_sweep_status(ctypes.byref(self.sweeper), ctypes.byref(pvo), ctypes.byref(pvi),
                                          ctypes.byref(self.quan), ctypes.byref(self.env)))
        return vo

    def sweep_host_ptr(self, vo_ptr: int, vi_ptr: int) -> None:
        """Sweeper_sweep on host buffers given by address (e.g. pinned torch
        tensors): the reference driver's call, host vi in, host vo out."""
        n = self.nstate
        pvi = Pointer(n, vi_ptr, None, 0, 1, 0)
        pvo = Pointer(n, vo_ptr, None, 0, 1, 0)
        _check(lib().Sweeper_sweep_status(ctypes.byref(self.sweeper), ctypes.byref(pvo), ctypes.byref(pvi),
                                          ctypes.byref(self.quan), ctypes.byref(self.env)))

    def sweep_device(self, vo_ptr: int, vi_ptr: int) -> None:
        """Enqueue vo = sweep(vi) on device arrays (async on self.stream)."""
        _check(lib().Sweeper_sweep_device(ctypes.byref(self.sweeper), ctypes.c_void_p(vo_ptr),
                                          ctypes.c_void_p(vi_ptr), ctypes.byref(self.quan), ctypes.byref(self.env)))

    def sweep_iterations_host(self, out_ptr: int, in_ptr: int, niterations: int) -> None:
        """Host buffers in and out, niterations device-resident sweeps (one C call)."""
        _check(lib().Sweeper_sweep_iterations(ctypes.byref(self.sweeper), ctypes.c_void_p(out_ptr),
                                              ctypes.c_void_p(in_ptr), niterations, ctypes.byref(self.quan),
                                              ctypes.byref(self.env)))

    def iterations_slices(self) -> int:
        """Group-pair slices the last sweep_host / sweep_iterations_host call ran in (1: whole)."""
        r = lib().msb_iterations_slices(ctypes.byref(self.sweeper))
        if r < 0:
            _check(r)
        return r

    def sync(self) -> None:
        _check(lib().Sweeper_sync_status(ctypes.byref(self.sweeper), ctypes.byref(self.env)))

    def state_norms(self, vi: np.ndarray, vo: np.ndarray):
        """(normsq, normsqdiff) of host arrays by the library's get_state_norms
        (the reference's loop order, array_operations.c:69-110)."""
        s, d = ctypes.c_double(), ctypes.c_double()
        DP = ctypes.POINTER(ctypes.c_double)
        lib().get_state_norms(vi.ctypes.data_as(DP), vo.ctypes.data_as(DP), self.dims, NU, ctypes.byref(s),
                              ctypes.byref(d), ctypes.byref(self.env))
        return s.value, d.value

    def norms_device(self, vi_ptr: int, vo_ptr: int):
        s, d = ctypes.c_double(), ctypes.c_double()
        _check(lib().msb_state_norms_device(ctypes.c_void_p(vi_ptr), ctypes.c_void_p(vo_ptr), self.nstate,
                                            ctypes.byref(s), ctypes.byref(d), ctypes.byref(self.env)))
        return s.value, d.value

    def init_state_device(self, v_ptr: int, ie_base: int = 0) -> None:
        """Built-in initial state on the device; with ie_base, of the energy-group
        slice whose group 0 is global group ie_base."""
        _check(lib().msb_initialize_state_slice_device(ctypes.c_void_p(v_ptr), self.dims, ie_base,
                                                       ctypes.byref(self.env)))

    @property
    def stream(self) -> int:
        return self.env.stream_kernel_faces_ or 0

    def tasks(self) -> np.ndarray:
        L = lib()
        n = L.Sweeper_debug_tasks(ctypes.byref(self.sweeper), None, 0)
        out = np.zeros((n, TASK_INTS), dtype=np.int32)
        L.Sweeper_debug_tasks(ctypes.byref(self.sweeper), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
        return out

    def tile(self) -> dict:
        """Tile shape in use and, with --autotune 1, the first sweep's times of
        the chosen and the other shape (ms)."""
        tx, ty = ctypes.c_int(), ctypes.c_int()
        a, b = ctypes.c_float(), ctypes.c_float()
        _check(lib().Sweeper_tile(ctypes.byref(self.sweeper), ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(a),
                                  ctypes.byref(b)))
        out = {"tx": tx.value, "ty": ty.value, "ms_chosen": a.value, "ms_other": b.value}
        k, w, h, n, ap = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().Sweeper_plan(ctypes.byref(self.sweeper), ctypes.byref(k), ctypes.byref(w), ctypes.byref(h),
                                  ctypes.byref(n), ctypes.byref(ap)))
        out.update(fp64_kernel=k.value, task_window=w.value, l2_hints=h.value, candidates=n.value,
                   angle_pass=ap.value)
        return out

    def set_timeout_ns(self, ns: int) -> None:
        _check(lib().Sweeper_set_spin_limit(ctypes.byref(self.sweeper), ns))

    # ---------------------------------------------- decomposed sweep by steps
    def kba_info(self):
        """(steps per sweep, bytes of an x-face message, of a y-face message)."""
        n, bx, by = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib().msb_kba_info(ctypes.byref(self.sweeper), ctypes.byref(n), ctypes.byref(bx), ctypes.byref(by)))
        return n.value, bx.value, by.value

    def kba_set_buffers(self, send_x, send_y, recv_x_lo, recv_x_hi, recv_y_lo, recv_y_hi) -> None:
        """Device addresses of the message buffers (None: the sweeper's own)."""
        b = [ctypes.c_void_p(p) if p else None for p in (send_x, send_y, recv_x_lo, recv_x_hi, recv_y_lo,
                                                          recv_y_hi)]
        _check(lib().msb_kba_set_buffers(ctypes.byref(self.sweeper), *b))

    def kba_begin(self, vo_ptr: int, vi_ptr: int) -> None:
        _check(lib().msb_kba_begin(ctypes.byref(self.sweeper), ctypes.c_void_p(vo_ptr), ctypes.c_void_p(vi_ptr),
                                   ctypes.byref(self.quan), ctypes.byref(self.env)))

    def kba_step(self, step: int) -> None:
        _check(lib().msb_kba_step(ctypes.byref(self.sweeper), step, ctypes.byref(self.env)))

    def kba_messages(self, step: int):
        msgs = (KbaMsg * 8)()
        n = lib().msb_kba_messages(ctypes.byref(self.sweeper), step, msgs, 8)
        if n < 0:
            raise SweepError(n, last_error())
        return [msgs[i] for i in range(n)]

    def kba_unpack(self, step: int) -> None:
        _check(lib().msb_kba_unpack(ctypes.byref(self.sweeper), step, ctypes.byref(self.env)))

    def kba_end(self) -> None:
        _check(lib().msb_kba_end(ctypes.byref(self.sweeper), ctypes.byref(self.env)))

    def close(self) -> None:
        if getattr(self, "_closed", True):
            return
        L = lib()
        L.Sweeper_destroy(ctypes.byref(self.sweeper), ctypes.byref(self.env))
        L.Quantities_destroy(ctypes.byref(self.quan))
        L.Arguments_destroy(ctypes.byref(self.args))
        L.Env_finalize(ctypes.byref(self.env))
        self._closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_case(argstring: str, nm: int = 16):
    """One run of the reference driver's Runner_run_case (runner.c:51-183) on
    this library: the built-in initial state, --niterations sweeps through
    Sweeper_sweep's host-in / host-out semantics with the vi/vo swap, then the
    norms of the two host arrays.  Returns (normsq, normsqdiff)."""
    with Problem(argstring, nm=nm) as pb:
        vi = pb.init_state()
        vo = np.zeros_like(vi)
        for it in range(pb.niterations):
            if it % 2 == 0:
                vo = pb.sweep_host(vi)
            else:
                vi = pb.sweep_host(vo)
        return pb.state_norms(vi, vo)


def compare_runs(argstring1: str, argstring2: str, nm: int = 16) -> bool:
    """The reference's compare_runs (runner.c:187-241): both runs must have
    normsqdiff == 0 and the same normsq."""
    n1, d1 = run_case(argstring1, nm)
    n2, d2 = run_case(argstring2, nm)
    return d1 == 0.0 and d2 == 0.0 and n1 == n2


# ------------------------------------------------------------------ batches
def batch_workload(n: int = 256, seed: int = 7) -> list:
    """The batched serving workload: n independent problems drawn with numpy's
    PCG64 from `seed`, in this order per field: ncell_x and ncell_y uniform in
    {8..48}, ncell_z in {8..64}, ne from {8, 16, 32, 64}, na from {16, 32, 64},
    nm from {4, 16} (NU = 4, built-in Quantities)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nx = rng.integers(8, 49, n)
    ny = rng.integers(8, 49, n)
    nz = rng.integers(8, 65, n)
    ne = rng.choice([8, 16, 32, 64], n)
    na = rng.choice([16, 32, 64], n)
    nm = rng.choice([4, 16], n)
    return [dict(ncell_x=int(nx[i]), ncell_y=int(ny[i]), ncell_z=int(nz[i]), ne=int(ne[i]), na=int(na[i]),
                 nm=int(nm[i])) for i in range(n)]


def small_batch_workload(n: int = 256, seed: int = 11) -> list:
    """Many small problems, the case batching is for (each alone leaves most
    SMs idle): drawn with numpy's PCG64 from `seed`, per problem in this
    order: ncell_x, ncell_y uniform in {4..12}, ncell_z in {4..16}, ne from
    {2, 4, 8}, na from {16, 32}, nm from {4, 16} (NU = 4, built-in
    Quantities)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        nx, ny, nz = int(rng.integers(4, 13)), int(rng.integers(4, 13)), int(rng.integers(4, 17))
        ne, na, nm = int(rng.choice([2, 4, 8])), int(rng.choice([16, 32])), int(rng.choice([4, 16]))
        out.append(dict(ncell_x=nx, ncell_y=ny, ncell_z=nz, ne=ne, na=na, nm=nm))
    return out


def state_size(p: dict) -> int:
    return p["ncell_x"] * p["ncell_y"] * p["ncell_z"] * p["ne"] * p["nm"] * NU


def init_state_device(v_ptr: int, p: dict) -> None:
    """Built-in initial state of problem p into a device array (default stream)."""
    d = Dimensions(p["ncell_x"], p["ncell_y"], p["ncell_z"], p["ne"], p["nm"], p["na"])
    _check(lib().msb_initialize_state_device(ctypes.c_void_p(v_ptr), d, None))


def builtin_matrices(nm: int, na: int):
    """Built-in a_from_m / m_from_a (reference layouts) for nm moments, na angles."""
    n = nm * na * NOCTANT
    a, m = np.zeros(n), np.zeros(n)
    DP = ctypes.POINTER(ctypes.c_double)
    _check(lib().msb_builtin_matrices(nm, na, a.ctypes.data_as(DP), m.ctypes.data_as(DP)))
    return a, m


def _descs(problems: list):
    arr = (ProblemDesc * len(problems))()
    for i, p in enumerate(problems):
        arr[i] = ProblemDesc(p["ncell_x"], p["ncell_y"], p["ncell_z"], p["ne"], p["na"], p["nm"],
                             p.get("vi", 0) or None, p.get("vo", 0) or None, p.get("a_from_m", 0) or None,
                             p.get("m_from_a", 0) or None)
    return arr


class Batch:
    """Many problems swept by one persistent kernel launch (msb_batch_*).

    `problems`: dicts with the sizes (ncell_x, ncell_y, ncell_z, ne, na, nm)
    and device pointers (vi, vo, a_from_m, m_from_a).  With `plan_nsm` set,
    only the host-side plan is built (no GPU; pointers may be absent)."""

    def __init__(self, problems: list, precision: int = 0, scratch_bytes: int = 0, autotune: bool = False,
                 plan_nsm: int = 0, tile24_mask: int = 0):
        L = lib()
        self.n = len(problems)
        self._h = ctypes.c_void_p()
        d = _descs(problems)
        if plan_nsm:
            rc = L.msb_batch_plan(ctypes.byref(self._h), d, self.n, plan_nsm, scratch_bytes, tile24_mask)
        else:
            rc = L.msb_batch_create(ctypes.byref(self._h), d, self.n, precision, scratch_bytes, int(autotune))
        _check(rc)

    def sweep(self, direction: int = 0, stream: int = 0) -> None:
        _check(lib().msb_batch_sweep(self._h, direction, ctypes.c_void_p(stream)))

    def run(self, niterations: int, stream: int = 0) -> None:
        _check(lib().msb_batch_run(self._h, niterations, ctypes.c_void_p(stream)))

    def sync(self, stream: int = 0) -> None:
        _check(lib().msb_batch_sync(self._h, ctypes.c_void_p(stream)))

    def problem_ms(self) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().msb_batch_problem_ms(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.n))
        return out

    def info(self) -> dict:
        i = BatchInfo()
        _check(lib().msb_batch_info(self._h, ctypes.byref(i)))
        nc = i.nclass
        return dict(nproblem=i.nproblem, nclass=nc, npred=i.npred, nsm=i.nsm, ntask=i.ntask,
                    scratch_bytes=i.scratch_bytes, scratch_needed_all=i.scratch_needed_all,
                    sim_makespan=i.sim_makespan, sim_busy=i.sim_busy, tune_ms=i.tune_ms,
                    classes=[dict(nm=i.class_nm[c], nch=i.class_nch[c], tile=(i.class_tx[c], i.class_ty[c]),
                                  ntask=i.class_ntask[c]) for c in range(nc)])

    def entries(self):
        """(problem, first angle) of every entry: the batch sweeps each problem
        in entries of 32 angles, as a Sweeper sweeps it in passes."""
        L = lib()
        n = L.msb_batch_entries(self._h, None, None, 0)
        if n < 0:
            raise SweepError(n, last_error())
        prob = np.zeros(n, dtype=np.int32)
        a0 = np.zeros(n, dtype=np.int32)
        IP = ctypes.POINTER(ctypes.c_int)
        L.msb_batch_entries(self._h, prob.ctypes.data_as(IP), a0.ctypes.data_as(IP), n)
        return prob, a0

    def tasks(self):
        """(table: ntask x 16 ints with global dependency ids, entry of each task)."""
        L = lib()
        n = L.msb_batch_tasks(self._h, None, None, 0)
        rec = np.zeros((n, TASK_INTS), dtype=np.int32)
        prob = np.zeros(n, dtype=np.int32)
        IP = ctypes.POINTER(ctypes.c_int)
        L.msb_batch_tasks(self._h, rec.ctypes.data_as(IP), prob.ctypes.data_as(IP), n)
        return rec, prob

    def scratch(self):
        """(offset, bytes, pred_off, pred) of the face-scratch arena placement, per entry."""
        L = lib()
        ne = L.msb_batch_entries(self._h, None, None, 0)
        off = np.zeros(ne, dtype=np.int64)
        nb = np.zeros(ne, dtype=np.int64)
        po = np.zeros(ne + 1, dtype=np.int32)
        LP, IP = ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)
        npred = L.msb_batch_scratch(self._h, off.ctypes.data_as(LP), nb.ctypes.data_as(LP), po.ctypes.data_as(IP),
                                    None, 0)
        if npred < 0:
            raise SweepError(npred, last_error())
        pred = np.zeros(max(npred, 1), dtype=np.int32)
        _check(min(0, L.msb_batch_scratch(self._h, None, None, None, pred.ctypes.data_as(IP), len(pred))))
        return off, nb, po, pred[:npred]

    def set_timeout_ns(self, ns: int) -> None:
        _check(lib().msb_batch_set_spin_limit(self._h, ns))

    def close(self) -> None:
        if self._h:
            lib().msb_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

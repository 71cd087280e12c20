"""Start a program as a process group on this node.

    python -m minisweep_b200.launch -n N [--timeout S] -- PROGRAM [ARGS...]

The counterpart of `mpirun -n N` for programs that use the library through
the reference's C API (its sweep and tester drivers, built against this
library): every process gets MSB_NPROC=N, MSB_PROC=i and MSB_GROUP=<id> in its
environment, and its Env_initialize joins the group and selects GPU
i % (GPUs visible).  The exit status is the first non-zero status of the
processes (0 when all succeed); when one fails or the time limit passes, the
others are stopped.
"""
from __future__ import annotations

import argparse
import os
import signal
import subprocess
import sys
import time
import uuid


def run(nproc: int, cmd: list[str], timeout: float | None = None, env: dict | None = None) -> int:
    if nproc < 1:
        raise ValueError("nproc must be >= 1")
    group = f"{os.getpid()}_{uuid.uuid4().hex[:12]}"
    base = dict(os.environ if env is None else env)
    procs = []
    for i in range(nproc):
        e = dict(base, MSB_NPROC=str(nproc), MSB_PROC=str(i), MSB_GROUP=group)
        procs.append(subprocess.Popen(cmd, env=e, start_new_session=True))
    deadline = None if timeout is None else time.monotonic() + timeout
    status = 0
    try:
        while True:
            codes = [p.poll() for p in procs]
            failed = [c for c in codes if c not in (None, 0)]
            if failed and status == 0:
                status = failed[0]
                break
            if all(c is not None for c in codes):
                break
            if deadline is not None and time.monotonic() > deadline:
                status = 124
                print(f"launch: time limit of {timeout} s reached", file=sys.stderr)
                break
            time.sleep(0.05)
    finally:
        for p in procs:
            if p.poll() is None:
                os.killpg(p.pid, signal.SIGTERM)  # each process leads its own session
        for p in procs:
            try:
                p.wait(timeout=30)
            except subprocess.TimeoutExpired:
                os.killpg(p.pid, signal.SIGKILL)
                p.wait()
        try:  # normally removed by process 0 once everybody attached
            os.unlink(f"/dev/shm/msb_{group}")
        except OSError:
            pass
    return status


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("-n", type=int, required=True, help="number of processes")
    ap.add_argument("--timeout", type=float, default=None, help="seconds before every process is stopped")
    ap.add_argument("cmd", nargs=argparse.REMAINDER, help="-- PROGRAM [ARGS...]")
    a = ap.parse_args(argv)
    cmd = a.cmd[1:] if a.cmd and a.cmd[0] == "--" else a.cmd
    if not cmd:
        ap.error("no program given")
    return run(a.n, cmd, a.timeout)


if __name__ == "__main__":
    sys.exit(main())

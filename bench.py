#!/usr/bin/env python
"""Benchmark of the B200 KBA sweep (minisweep's Sweeper_sweep hot path).

Workload: 64^3 cells, ne 64, na 32 angles per octant, NM 16 moments, NU 4,
nblock_z 8, niterations 10, the built-in deterministic Quantities, FP64 plain.
One step = one run of the reference driver's iteration loop (runner.c:148-155):
10 sweeps with the vi/vo swap.  Metric: cell-angle-group updates per second,
one update = one (cell, angle, group, octant) solve, 64^3 * 32 * 64 * 8 per
sweep.  The FP64 sweep is the headline `value`; the mixed-precision sweeps
(--precision 1: FP16 halves, 2: BF16 halves) are timed the same way and
reported beside it in `mixed`, each with its error against the FP64 sweep on
the built-in problem and on the random-input study (state U[0,1) from
torch's generator seeded 1234, a_from_m N(0, 1/nm) from PCG64 seed 1234,
m_from_a its pseudo-inverse).

`batched` reports the batched serving workload beside them: 256 independent
problems of uneven sizes (seed 7) swept by one persistent launch per sweep,
with problems/s and the per-problem completion latency (p50 / p99).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun rank r sweeps groups [64 r, 64 r + 64) of a 64 N-group problem
(`--ie_base 64 r`: its own arrays, global group indices in the initial state
and boundary fluxes); energy groups are independent, so the only exchange is
the all-reduce of the two FP64 checksums (and the max of the timings).  The
per-GPU work is fixed, so scaling is weak.
The reference arm times the reference's own OpenMP CPU sweep (built from its
sources into oracle/_ref) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NX = NY = NZ = 64
NE, NA, NM, NU, NBLOCK_Z, NITER = 64, 32, 16, 4, 8, 10
IE_BASE = 0  # under torchrun: global index of this rank's first energy group
METRIC = "cell-angle-group updates/s, FP64 plain vs mixed-precision at stated error"
UNIT = "updates/s"
WORKLOAD = (f"minisweep KBA sweep, {NX}x{NY}x{NZ} cells, ne {NE}, na {NA}, NM {NM}, NU {NU}, "
            f"nblock_z {NBLOCK_Z}, niterations {NITER}, built-in Quantities, FP64 plain")


# Sizes default to the module's workload at call time (--case small changes it).
def updates_per_sweep(nx=None, ny=None, nz=None, ne=None, na=None) -> int:
    nx, ny, nz, ne, na = (NX if nx is None else nx, NY if ny is None else ny, NZ if nz is None else nz,
                          NE if ne is None else ne, NA if na is None else na)
    return nx * ny * nz * ne * na * 8


def flops_per_sweep(nx=None, ny=None, nz=None, ne=None, na=None, nm=None) -> float:
    # the reference's flop model (runner.c:162-166): two transforms + 12 per solve
    nx, ny, nz, ne, na, nm = (NX if nx is None else nx, NY if ny is None else ny, NZ if nz is None else nz,
                              NE if ne is None else ne, NA if na is None else na, NM if nm is None else nm)
    state = nx * ny * nz * ne * nm * NU
    return state * 8 * 2.0 * na * 2 + nx * ny * nz * ne * na * NU * 8 * 12.0


def config_dict(ne=None) -> dict:
    gb = NX * NY * NZ * NE * NM * NU * 8 / 1e9
    return {"workload": WORKLOAD, "ncell": [NX, NY, NZ], "ne_per_gpu": NE if ne is None else ne, "na": NA,
            "nm": NM, "nu": NU, "nblock_z": NBLOCK_Z, "niterations": NITER,
            "l2": f"state arrays of {gb:.2f} GB each, far above the 126 MB L2: no flush needed between steps"}


# ------------------------------------------------------------------ helpers
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out = self.proc.communicate()[0]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    """HBM copy bandwidth and BF16 GEMM peaks measured on this GPU pool
    (MEASURED_PEAKS.json), else an earlier measurement of the same pool's
    B200s (6.65 TB/s, 1.59 PFLOP/s), marked as the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        d["source"] = "measured (MEASURED_PEAKS.json)"
        return d
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback (earlier measurement on this pool)"}


def profile_traffic(kernel: str = "sweep_fp64_kernel") -> float | None:
    """DRAM bytes per 64^3 sweep of a kernel from its committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", kernel + ".md")) as f:
            m = re.search(r"traffic_bytes_per_sweep_64cubed:\s*([0-9.eE+]+)", f.read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def reference_binary() -> str | None:
    p = os.path.join(ROOT, "oracle", "_ref", f"sweep_omp_nm{NM}")
    return p if os.access(p, os.X_OK) else None


def cpu_sample(ne_sample: int | None = None):
    """One run of the reference OpenMP sweep on the host cores: one sweep of
    the benchmark problem (all NE groups, --nthread_e = the host cores), or of
    its first ne_sample groups.  Returns (updates/s, seconds, threads,
    description) or None."""
    binp = reference_binary()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    ne = ne_sample or NE
    nthr = max(1, min(ne, cores or 1))
    if binp is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(nthr), OMP_PROC_BIND="true")
    args = [binp, "--ncell_x", str(NX), "--ncell_y", str(NY), "--ncell_z", str(NZ), "--ne", str(ne),
            "--na", str(NA), "--nblock_z", str(NBLOCK_Z), "--nthread_e", str(nthr), "--nthread_octant", "1",
            "--niterations", "1"]
    out = subprocess.run(args, env=env, capture_output=True, text=True, timeout=1500).stdout
    m = re.search(r"time:\s*([0-9.]+)", out)
    ok = "PASS" in out
    if not m or not ok:
        return None
    sec = float(m.group(1))
    u = updates_per_sweep(ne=ne)
    desc = (f"reference OpenMP sweep (oracle/_ref/sweep_omp_nm{NM}, --nthread_e {nthr} --nthread_octant 1, "
            f"OMP_PROC_BIND=true), {NX}^3 cells x ne {ne} x na {NA} x NM {NM}, nblock_z {NBLOCK_Z}, "
            f"one sweep ({u:.3g} updates, {sec:.2f} s)")
    return u / sec, sec, nthr, desc


def cpu_sample_port():
    """Fallback when the reference build is absent: the oracle port, 1 thread."""
    import numpy as np

    import oracle
    nx = ny = nz = 16
    ne = 8
    a, m = oracle.am_matrices(NM, NA)
    vi = oracle.init_state(nx, ny, nz, ne, NM)
    t0 = time.perf_counter()
    oracle.sweep(nx, ny, nz, ne, NM, NA, a, m, vi)
    sec = time.perf_counter() - t0
    u = updates_per_sweep(nx, ny, nz, ne, NA)
    del np
    return u / sec, sec, 1, f"oracle port (oracle/sweep_oracle.c), {nx}^3 x ne {ne} x na {NA}, 1 thread"


# ------------------------------------------------------------------ arms
def run_reference(args, rank: int) -> int:
    """The reference arm: the reference's own OpenMP sweep on the host cores,
    on the GPU arm's problem (same config).  A timed step is one sweep of the
    whole 64^3 x ne 64 problem (about 20 s on 16 cores; the metric is a rate
    per sweep, the GPU arm's step runs the problem's 10 sweeps).  A CPU binary
    has nothing to warm up beyond what every fresh process pays, so the warm-up
    steps sweep a quarter of the groups."""
    if rank != 0:
        return 0
    vals, secs = [], []
    kind = "reference"
    desc, nthr = "", 1
    for i in range(args.warmup + args.steps):
        timed = i >= args.warmup
        r = cpu_sample(None if timed else max(1, NE // 4))
        if r is None:
            kind = "port"
            r = cpu_sample_port()
        if timed:
            vals.append(r[0])
            secs.append(r[1])
            nthr, desc = r[2], r[3]
    v = sorted(vals)[len(vals) // 2]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the reference's built-in deterministic Quantities", "config": config_dict(),
            "step": "one sweep of the configured problem (its niterations are repeats of that sweep; "
                    "value is the median per-step rate)",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthr, "kind": kind,
                             "sample": desc + "; warm-up steps: ne %d" % max(1, NE // 4)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def measure_mixed(args, pb64, flags, va, vb, stream, dev, world, ms_fp64=None) -> list:
    """Time the mixed-precision sweeps (a step is NITER device-resident sweeps,
    like the FP64 step) and measure their error against the FP64 sweep.

    Each sweep of a mixed step sweeps the same initial state: fed back into
    itself, the built-in problem amplifies any rounding by about 1e8 per sweep
    (the FP64 oracle turns a 1e-7 perturbation of its state into an O(10)
    error in one sweep; the exact-integer FP64 sweep is a fixed point only
    because it rounds nothing), so only the error of one sweep from the same
    input is meaningful.  va / vb are reused: they hold no result needed
    afterwards."""
    import torch

    import minisweep_b200 as msb
    from minisweep_b200.parallel import max_over_ranks

    n = pb64.nstate
    out = []
    peaks = measured_peaks()
    fmt = {1: "FP16 hi+lo halves", 2: "BF16 hi+lo halves"}
    for prec in (1, 2):
        pb = msb.Problem(flags + f" --precision {prec}", nm=NM)
        st = torch.cuda.ExternalStream(pb.stream)

        def step(evs=None):
            for _ in range(NITER):
                if evs is not None:
                    e = torch.cuda.Event(enable_timing=True)
                    e.record(st)
                    evs.append(e)
                pb.sweep_device(vb.data_ptr(), va.data_ptr())
            if evs is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record(st)
                evs.append(e)

        pb.init_state_device(va.data_ptr(), IE_BASE)
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            step()
        pb.sync()
        pb.init_state_device(va.data_ptr(), IE_BASE)
        torch.cuda.synchronize()
        clocks = Clocks(torch.cuda.current_device())
        clocks.start()
        evs = []
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(st)
        for _ in range(args.steps):
            step(evs)
        t1.record(st)
        pb.sync()
        torch.cuda.synchronize()
        clk = clocks.stop()
        elapsed = max_over_ranks(t0.elapsed_time(t1) / 1e3)
        sweep_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(len(evs) - 1) if (i + 1) % (NITER + 1) != 0]
        ms_sweep = sum(sweep_ms) / len(sweep_ms)
        value = updates_per_sweep() * NITER * args.steps * world / elapsed
        # ---- error on the built-in problem: FP64 leaves the state unchanged
        # (vo == vi exactly), so the reference result is the initial state
        pb.init_state_device(va.data_ptr(), IE_BASE)
        pb.sweep_device(vb.data_ptr(), va.data_ptr())
        pb.sync()
        torch.cuda.synchronize()
        f64 = va
        one_max = (torch.max(torch.abs(vb - f64)) / torch.max(torch.abs(f64))).item()
        nf = torch.sum(f64 * f64)
        one_nsq = abs((torch.sum(vb * vb) - nf) / nf).item()
        # ---- random-input study: the same draws through the FP64 and the mixed sweep
        am, mm = msb.random_matrices(NM, NA, seed=1234)
        gen = torch.Generator(device=dev)
        gen.manual_seed(1234)
        vr = torch.rand(n, dtype=torch.float64, device=dev, generator=gen)
        torch.cuda.synchronize()  # the library's stream does not wait for torch's
        a0, m0 = (x.copy() for x in pb64.matrices())
        pb64.set_matrices(am, mm)
        pb.set_matrices(am, mm)
        pb64.sweep_device(va.data_ptr(), vr.data_ptr())
        pb64.sync()
        pb.sweep_device(vb.data_ptr(), vr.data_ptr())
        pb.sync()
        torch.cuda.synchronize()
        r_max = (torch.max(torch.abs(vb - va)) / torch.max(torch.abs(va))).item()
        nr = torch.sum(va * va)
        r_nsq = abs((torch.sum(vb * vb) - nr) / nr).item()
        del vr
        torch.cuda.empty_cache()
        pb64.set_matrices(a0, m0)
        hbm = 16.0 * NX * NY * NZ * NE * NM * NU / (ms_sweep * 1e-3) / 1e9
        out.append({"precision": prec, "format": fmt[prec], "value": value, "unit": UNIT,
                    "ms_per_step": 1e3 * elapsed / args.steps, "ms_per_sweep_kernel": ms_sweep,
                    "dtype": "fp16/bf16 split products, fp32 accumulate and faces, f64 vo",
                    "gpu_launches": 3 * args.steps * NITER, "clocks": clk,
                    "launches_per_sweep": "3: vi converted to FP16/BF16 hi+lo operand blocks, the sweep kernel, "
                                          "and the FP64 sum of the eight octant partials",
                    "step": "%d sweeps of the initial state (not fed back: see error_note)" % NITER,
                    "error_builtin": {"max_rel": one_max, "normsq_rel": one_nsq},
                    "error_note": "errors of one sweep against the FP64 sweep of the same input; fed back, "
                                  "the built-in problem amplifies any rounding ~1e8x per sweep (measured with "
                                  "the FP64 oracle on a 1e-7 perturbation)",
                    "error_random_seed1234": {"max_rel": r_max, "normsq_rel": r_nsq},
                    "roofline": {"bound": "hbm", "achieved": hbm, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                                 "peak_source": peaks.get("source"),
                                 "frac": hbm / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
                                 "traffic": profile_traffic("sweep_mixed_kernel"),
                                 "traffic_source": "constant read from profiles/sweep_mixed_kernel.md: ncu DRAM "
                                                   "bytes of one 32^3 x ne 32 sweep scaled x16; not measured in "
                                                   "this run",
                                 "algorithmic": "16 x state bytes per sweep (vi read + vo write) / mean sweep "
                                                "kernel time"}})
        pb.close()
    return out


def measure_dense(args, dev, world: int, local_rank: int) -> dict | None:
    """The angle/group-heavy case: 32x32x96 cells, ne 128, na 128, NM 16,
    nblock_z 12, built-in Quantities.  One FP64 sweep (kernel, tile shape,
    task window and angle passes autotuned by the untimed first sweep) against one sweep of each
    mixed precision (four 32-angle passes), each timed after one untimed
    sweep; under torchrun each rank sweeps its own 128-group slice.  The FP64
    sweep of the built-in problem returns its input exactly, so the mixed
    errors are measured against the initial state."""
    if args.no_dense:
        return None
    import torch

    import minisweep_b200 as msb
    from minisweep_b200.parallel import max_over_ranks

    nx, ny, nz, ne, na, nm, nbz = 32, 32, 96, 128, 128, 16, 12
    ie_base = ne * int(os.environ.get("RANK", "0"))  # this rank's energy-group slice
    fl = f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na} --nblock_z {nbz} --ie_base {ie_base}"
    upd = nx * ny * nz * ne * na * 8
    flops = flops_per_sweep(nx, ny, nz, ne, na, nm)
    out = {"workload": f"{nx}x{ny}x{nz} cells, ne {ne}, na {na}, NM {nm}, NU {NU}, nblock_z {nbz}, built-in "
                       f"Quantities, one sweep per timing (after one untimed sweep)",
           "updates_per_sweep": upd, "flops_per_sweep": flops, "runs": []}
    va = vb = None
    clocks = Clocks(local_rank)
    clocks.start()
    for prec in (0, 1, 2):
        with msb.Problem(fl + (" --autotune 1" if prec == 0 else f" --precision {prec}"), nm=nm) as pb:
            if va is None:
                va = torch.empty(pb.nstate, dtype=torch.float64, device=dev)
                vb = torch.empty_like(va)
            pb.init_state_device(va.data_ptr(), ie_base)
            torch.cuda.synchronize()
            st = torch.cuda.ExternalStream(pb.stream) if pb.stream else torch.cuda.current_stream()
            pb.sweep_device(vb.data_ptr(), va.data_ptr())
            pb.sync()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            pb.sweep_device(vb.data_ptr(), va.data_ptr())
            e1.record(st)
            pb.sync()
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1) / 1e3) * 1e3
            r = {"precision": prec, "ms_per_sweep": ms, "updates_per_s": upd * world / (ms * 1e-3),
                 "launches_per_sweep": (na + 63) // 64 if prec == 0 else 1 + 2 * ((na + 31) // 32)}
            if prec == 0:
                r["exact"] = bool(torch.equal(va, vb))
                r["tflops"] = flops / (ms * 1e-3) / 1e12
                r["tile"] = pb.tile()
                r["launches_per_sweep"] = (na + r["tile"]["angle_pass"] - 1) // r["tile"]["angle_pass"]
            else:
                r["max_rel"] = (torch.max(torch.abs(vb - va)) / torch.max(torch.abs(va))).item()
                nf = torch.sum(va * va)
                r["normsq_rel"] = abs((torch.sum(vb * vb) - nf) / nf).item()
            out["runs"].append(r)
    out["clocks"] = clocks.stop()
    f64 = out["runs"][0]["ms_per_sweep"]
    for r in out["runs"][1:]:
        r["speedup_vs_fp64"] = f64 / r["ms_per_sweep"]
    del va, vb
    torch.cuda.empty_cache()
    return out


def measure_batched(args, dev, world: int, rank: int, local_rank: int) -> dict | None:
    """The batched serving workload: 256 independent problems (seed 7, sizes in
    msb.batch_workload), every one swept by ONE persistent launch per sweep;
    under torchrun each rank takes every world-th problem (no exchange).
    Reports problems/s, the per-problem completion latency inside the launch
    (p50 / p99), the CUDA-graph iteration loop, and the same problems swept
    one Sweeper at a time for comparison."""
    if args.no_batch:
        return None
    import numpy as np
    import torch

    import minisweep_b200 as msb
    from minisweep_b200.parallel import max_over_ranks

    W = msb.batch_workload()
    mine = [i for i in range(len(W)) if i % world == rank]
    probs = [W[i] for i in mine]
    vis, vos, mats, descs = [], [], {}, []
    for q in probs:
        n = msb.state_size(q)
        vi = torch.empty(n, dtype=torch.float64, device=dev)
        vo = torch.empty_like(vi)
        msb.init_state_device(vi.data_ptr(), q)
        key = (q["nm"], q["na"])
        if key not in mats:
            a, m = msb.builtin_matrices(*key)
            mats[key] = (torch.from_numpy(a).to(dev), torch.from_numpy(m).to(dev))
        vis.append(vi)
        vos.append(vo)
        descs.append(dict(q, vi=vi.data_ptr(), vo=vo.data_ptr(), a_from_m=mats[key][0].data_ptr(),
                          m_from_a=mats[key][1].data_ptr()))
    torch.cuda.synchronize()
    t0 = time.time()
    b = msb.Batch(descs, autotune=True)
    create_s = time.time() - t0
    info = b.info()
    # the planner's list-scheduling simulation (one worker per SM): SM time
    # busy when the problems share one launch, and when each runs alone
    singles_ms, singles_busy = [], []
    for q in probs:
        with msb.Batch([q], plan_nsm=info["nsm"]) as b1:
            i1 = b1.info()
        singles_ms.append(i1["sim_makespan"])
        singles_busy.append(i1["sim_busy"])
    sm_, sb_ = np.array(singles_ms), np.array(singles_busy)
    sim = {"busy_batched": info["sim_busy"], "busy_one_at_a_time_work_weighted": float((sm_ * sb_).sum() / sm_.sum()),
           "busy_one_at_a_time_min": float(sb_.min()),
           "predicted_speedup_vs_unbatched": float(sm_.sum() / info["sim_makespan"]),
           "note": "host-side list-scheduling simulation of the planner (task durations from their wavefront "
                   "steps): one problem alone already keeps the SMs this busy, so a shared launch can recover "
                   "at most the difference"}
    s = torch.cuda.Stream(device=dev)
    sh = s.cuda_stream

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        b.sync(sh)
        return e0.elapsed_time(e1)

    for _ in range(max(1, args.batch_warmup)):
        b.sweep(0, sh)
        b.sync(sh)
    clocks = Clocks(local_rank)
    clocks.start()
    ms = [timed(lambda: b.sweep(0, sh)) for _ in range(max(1, args.batch_steps))]
    clk = clocks.stop()
    done_ms = b.problem_ms()
    graph_ms = timed(lambda: b.run(2, sh))  # vi -> vo -> vi as one captured graph
    b.sweep(0, sh)
    b.sync(sh)
    b.close()
    # the same problems, one Sweeper (one launch) after another
    seq_ms = 0.0
    exact = True
    for i, q in enumerate(probs):
        fl = f"--ncell_x {q['ncell_x']} --ncell_y {q['ncell_y']} --ncell_z {q['ncell_z']} --ne {q['ne']} --na {q['na']}"
        with msb.Problem(fl, nm=q["nm"]) as pb1:
            ref = torch.empty_like(vos[i]) if i < 8 else vos[i]
            st1 = torch.cuda.ExternalStream(pb1.stream) if pb1.stream else torch.cuda.current_stream()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st1)
            pb1.sweep_device(ref.data_ptr(), vis[i].data_ptr())
            e1.record(st1)
            pb1.sync()
            seq_ms += e0.elapsed_time(e1)
            if i < 8:  # the batched result equals the problem's own Sweeper bit for bit
                exact = exact and bool(torch.equal(ref, vos[i]))
    # mixed precision on the same problems: one mixed Sweeper per problem, one
    # after another (the persistent batched kernel sweeps in FP64 only); the
    # FP64 sweep of the built-in problem returns its input, so the error of
    # each mixed result is measured against vi
    mix_ms, mix_done, mix_rel, mix_nsq = [], [], 0.0, 0.0
    for i, q in enumerate(probs):
        fl = f"--ncell_x {q['ncell_x']} --ncell_y {q['ncell_y']} --ncell_z {q['ncell_z']} --ne {q['ne']} --na {q['na']}"
        with msb.Problem(fl + " --precision 1", nm=q["nm"]) as pb1:
            out = torch.empty_like(vis[i])
            st1 = torch.cuda.ExternalStream(pb1.stream) if pb1.stream else torch.cuda.current_stream()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st1)
            pb1.sweep_device(out.data_ptr(), vis[i].data_ptr())
            e1.record(st1)
            pb1.sync()
            mix_ms.append(e0.elapsed_time(e1))
            mix_done.append(sum(mix_ms))
            ref = vis[i]
            mix_rel = max(mix_rel, (torch.max(torch.abs(out - ref)) / torch.max(torch.abs(ref))).item())
            nr = torch.sum(ref * ref)
            mix_nsq = max(mix_nsq, abs((torch.sum(out * out) - nr) / nr).item())
            del out
    mix_total = max_over_ranks(sum(mix_ms) / 1e3) * 1e3
    batch_ms = max_over_ranks(min(ms) / 1e3) * 1e3
    seq_ms = max_over_ranks(seq_ms / 1e3) * 1e3
    upd = sum(q["ncell_x"] * q["ncell_y"] * q["ncell_z"] * q["ne"] * q["na"] * 8 for q in W)
    del vis, vos, descs, mats
    torch.cuda.empty_cache()
    return {"workload": "batched serving: 256 independent problems from seed 7 (numpy PCG64), ncell_x,y in "
                        "{8..48}, ncell_z in {8..64}, ne in {8,16,32,64}, na in {16,32,64}, NM in {4,16}, NU 4, "
                        "built-in Quantities, FP64",
            "metric": "problems/s", "value": len(W) / (batch_ms / 1e3), "unit": "problems/s",
            "updates_per_s": upd / (batch_ms / 1e3),
            "ms_per_batch_sweep": batch_ms, "launches_per_sweep": 1,
            "latency_ms": {"p50": float(np.percentile(done_ms, 50)), "p99": float(np.percentile(done_ms, 99)),
                           "max": float(done_ms.max()),
                           "definition": "device time from the start of the batched launch to the completion "
                                         "of each problem's last task (rank 0's share)"},
            "graph_2_iterations_ms": graph_ms,
            "unbatched_ms": seq_ms,
            "speedup_vs_unbatched": seq_ms / batch_ms,
            "exact_vs_sweeper": exact,
            "mixed_sequential": {
                "precision": 1, "format": "FP16 hi+lo halves", "value": len(W) / (mix_total / 1e3),
                "unit": "problems/s", "ms_total": mix_total,
                "latency_ms": {"p50": float(np.percentile(mix_done, 50)), "p99": float(np.percentile(mix_done, 99)),
                               "definition": "completion time of each problem counted from the start of the "
                                             "sequence (rank 0's share)"},
                "error_vs_fp64_max_over_problems": {"max_rel": mix_rel, "normsq_rel": mix_nsq},
                "launches_per_problem": "1 (vi conversion) + 2 per 32-angle pass (sweep kernel + partial sum)",
                "note": "one mixed-precision Sweeper per problem, swept one after another: the persistent "
                        "batched kernel sweeps in FP64 only"},
            "problems_per_rank": len(probs), "ntask": info["ntask"],
            "classes": [{"nm": c["nm"], "angle_chunks": c["nch"], "tile": list(c["tile"]), "ntask": c["ntask"]}
                        for c in info["classes"]],
            "scratch_gb": info["scratch_bytes"] / 1e9, "scratch_needed_all_gb": info["scratch_needed_all"] / 1e9,
            "scratch_waits": info["npred"], "create_s": create_s, "autotune_ms": info["tune_ms"],
            "sm_utilisation_simulated": sim,
            "small_problems": measure_small_batch(dev, world, rank),
            "clocks": clk,
            "note": "one persistent launch sweeps every problem; the face scratch of all problems at once "
                    "does not fit beside the state, so problems reuse the scratch of completed ones (device-side "
                    "waits on per-problem completion counters)"}


def measure_small_batch(dev, world: int, rank: int) -> dict:
    """Many small problems (msb.small_batch_workload: 256 problems from seed
    11, 4..12 cells a side, 2..8 groups), the serving case batching is for:
    one persistent launch per sweep against the same problems swept one
    Sweeper (one launch) after another, each after one untimed sweep."""
    import numpy as np
    import torch

    import minisweep_b200 as msb
    from minisweep_b200.parallel import max_over_ranks

    W = msb.small_batch_workload()
    probs = [W[i] for i in range(len(W)) if i % world == rank]
    vis, vos, mats, descs = [], [], {}, []
    for q in probs:
        vi = torch.empty(msb.state_size(q), dtype=torch.float64, device=dev)
        msb.init_state_device(vi.data_ptr(), q)
        key = (q["nm"], q["na"])
        if key not in mats:
            a, m = msb.builtin_matrices(*key)
            mats[key] = (torch.from_numpy(a).to(dev), torch.from_numpy(m).to(dev))
        vis.append(vi)
        vos.append(torch.empty_like(vi))
        descs.append(dict(q, vi=vi.data_ptr(), vo=vos[-1].data_ptr(), a_from_m=mats[key][0].data_ptr(),
                          m_from_a=mats[key][1].data_ptr()))
    torch.cuda.synchronize()
    s = torch.cuda.Stream(device=dev)
    sh = s.cuda_stream
    with msb.Batch(descs, autotune=True) as b:
        def timed(fn):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            b.sync(sh)
            return e0.elapsed_time(e1)

        for _ in range(2):
            b.sweep(0, sh)
            b.sync(sh)
        batch_ms = min(timed(lambda: b.sweep(0, sh)) for _ in range(3))
        done_ms = b.problem_ms()
    seq_ms, exact = 0.0, True
    for i, q in enumerate(probs):
        fl = f"--ncell_x {q['ncell_x']} --ncell_y {q['ncell_y']} --ncell_z {q['ncell_z']} --ne {q['ne']} --na {q['na']}"
        with msb.Problem(fl, nm=q["nm"]) as pb1:
            out = torch.empty_like(vis[i])
            st1 = torch.cuda.ExternalStream(pb1.stream) if pb1.stream else torch.cuda.current_stream()
            pb1.sweep_device(out.data_ptr(), vis[i].data_ptr())
            pb1.sync()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st1)
            pb1.sweep_device(out.data_ptr(), vis[i].data_ptr())
            e1.record(st1)
            pb1.sync()
            seq_ms += e0.elapsed_time(e1)
            exact = exact and bool(torch.equal(out, vos[i]))
    batch_ms = max_over_ranks(batch_ms / 1e3) * 1e3
    seq_ms = max_over_ranks(seq_ms / 1e3) * 1e3
    del vis, vos, descs, mats
    torch.cuda.empty_cache()
    return {"workload": "256 small problems from seed 11 (numpy PCG64): ncell_x,y in {4..12}, ncell_z in "
                        "{4..16}, ne in {2,4,8}, na in {16,32}, NM in {4,16}, NU 4, built-in Quantities, FP64",
            "value": len(W) / (batch_ms / 1e3), "unit": "problems/s", "ms_per_batch_sweep": batch_ms,
            "unbatched_ms": seq_ms, "speedup_vs_unbatched": seq_ms / batch_ms, "exact_vs_sweeper": exact,
            "latency_ms": {"p50": float(np.percentile(done_ms, 50)), "p99": float(np.percentile(done_ms, 99))},
            "note": "each of these problems alone leaves most SMs idle; one launch sweeps them all side by "
                    "side (unbatched: one Sweeper per problem, default plan, timed after one untimed sweep)"}


def run_ours(args, rank: int, world: int, local_rank: int) -> int:
    import torch

    import minisweep_b200 as msb
    from minisweep_b200.parallel import max_over_ranks, sum_norms

    # this rank's GPU first: the NCCL communicator binds to the current device
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # rank r sweeps groups [64 r, 64 r + 64) of a 64 N-group problem: its own
    # arrays, the global group index in the initial state and boundary fluxes
    global IE_BASE
    IE_BASE = NE * rank
    flags = (f"--ncell_x {NX} --ncell_y {NY} --ncell_z {NZ} --ne {NE} --na {NA} --nblock_z {NBLOCK_Z} "
             f"--niterations {NITER} --ie_base {IE_BASE}")
    # --autotune 1: the first (warm-up) sweep times every candidate plan
    # (both FP64 kernels x both tile shapes x task windows) and keeps the
    # fastest for every later sweep; --fp64-flags fixes the plan instead
    pb = msb.Problem(flags + " " + (args.fp64_flags or "--autotune 1"), nm=NM)
    n = pb.nstate
    va = torch.empty(n, dtype=torch.float64, device=dev)
    vb = torch.empty(n, dtype=torch.float64, device=dev)
    pb.init_state_device(va.data_ptr(), IE_BASE)
    stream = torch.cuda.ExternalStream(pb.stream)
    torch.cuda.synchronize()
    peak_dmma, peak_dfma = msb.fp64_peak(5)

    def one_step(evs=None):
        a, b = va, vb
        for _ in range(NITER):
            if evs is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record(stream)
                evs.append(e)
            pb.sweep_device(b.data_ptr(), a.data_ptr())
            a, b = b, a
        if evs is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record(stream)
            evs.append(e)

    for _ in range(args.warmup):
        one_step()
    pb.sync()
    tile = pb.tile()
    barrier()
    clocks = Clocks(local_rank)
    clocks.start()
    evs = []
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        one_step(evs)
    t_end.record(stream)
    pb.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed = t_start.elapsed_time(t_end) / 1e3
    sweep_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(len(evs) - 1) if (i + 1) % (NITER + 1) != 0]
    elapsed = max_over_ranks(elapsed)
    barrier()

    # correctness of the timed result (built-in Quantities: vo == vi exactly)
    normsq, normsqdiff = sum_norms(*pb.norms_device(va.data_ptr(), vb.data_ptr()))
    mixed = [] if args.no_mixed else measure_mixed(args, pb, flags, va, vb, stream, dev, world, ms_fp64=None)
    closed = None
    try:
        import oracle
        closed = oracle.normsq_closed_form(NX, NY, NZ, NE * world, NM)
    except Exception:  # the oracle is only the checker; the number stands without it
        pass

    def finish(e2e):
        pb.close()
        batched = measure_batched(args, dev, world, rank, local_rank)
        dense = measure_dense(args, dev, world, local_rank)
        upd = updates_per_sweep() * NITER
        value = upd * args.steps * world / elapsed
        ms_sweep = sum(sweep_ms) / len(sweep_ms)
        for mx in mixed:
            mx["speedup_vs_fp64"] = mx["value"] / value
        tf = flops_per_sweep() / (ms_sweep * 1e-3) / 1e12
        hbm_bytes = 16.0 * NX * NY * NZ * NE * NM * NU  # read vi once, write vo once
        peaks = measured_peaks()
        traffic = profile_traffic()
        roofline = {"bound": "tensor", "achieved": tf, "peak": peak_dmma, "unit": "TFLOP/s",
                    "frac": tf / peak_dmma if peak_dmma else None,
                    "traffic": traffic,
                    "traffic_source": "constant read from profiles/sweep_fp64_kernel.md: ncu DRAM bytes of one "
                                      "32^3 x ne 32 sweep scaled x16 to this workload; not measured in this run",
                    "peak_source": "FP64 mma.sync peak measured live by msb_measure_fp64_peak (MEASURED_PEAKS.json "
                                   "has no FP64 figure); FMA-pipe FP64 peak %.2f TF/s" % peak_dfma,
                    "algorithmic": "reference flop model (runner.c:162-166) %.4g flop per sweep / mean sweep "
                                   "kernel time %.2f ms" % (flops_per_sweep(), ms_sweep),
                    "hbm_view": {"achieved_gbs": hbm_bytes / (ms_sweep * 1e-3) / 1e9,
                                 "peak_gbs": peaks.get("hbm_gbs"), "peak_source": peaks.get("source"),
                                 "note": "algorithmic bytes 16 x state (vi read + vo write); the FP64 path is "
                                         "FP64-compute-bound, not HBM-bound"}}
        if rank == 0:
            cpu = None
            if world == 1 and not args.no_cpu:
                # a bounded sample for the GPU arm's own line: a quarter of the
                # groups (the full problem is the reference arm's step)
                r = cpu_sample(ne_sample=max(1, NE // 4))
                kind = "reference"
                if r is None:
                    r = cpu_sample_port()
                    kind = "port"
                cpu = {"value": r[0], "unit": UNIT, "cores": r[2], "kind": kind, "sample": r[3]}
            line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic: the reference's built-in deterministic Quantities (index-derived state, "
                            "faces and transform matrices)",
                    "config": config_dict(),
                    "step": f"one run of the configured problem: its {NITER} sweeps with the vi/vo swap",
                    "parallelism": f"{world} GPU(s), each an energy-group slice of {NE} groups of a "
                                   f"{NE * world}-group problem; checksums all-reduced (2 FP64 scalars), no other "
                                   "exchange",
                    "tile": {"cells_per_cta": [tile["tx"], tile["ty"]],
                             "autotune_first_sweep_ms": {"chosen": tile["ms_chosen"],
                                                         "best_other_tile": tile["ms_other"]}},
                    "plan": {"fp64_kernel": "chained wavefront" if tile["fp64_kernel"] else "staged",
                             "task_window_x_sms": tile["task_window"], "l2_hints": tile["l2_hints"],
                             "angles_per_pass": tile["angle_pass"], "plans_timed": tile["candidates"]},
                    "roofline": roofline, "cpu_baseline": cpu,
                    "e2e": e2e,
                    "clocks": clk, "gpu_launches": args.steps * NITER,
                    "mixed": mixed,
                    "mixed_target": "mixed precision >= 2x the FP64 sweep at <= 1e-5 relative normsq error "
                                    "against it",
                    "check": {"normsq": normsq, "normsqdiff": normsqdiff, "normsq_closed_form": closed,
                              "pass": normsqdiff == 0.0 and (closed is None or (
                                  normsq == closed if world == 1 else abs(normsq - closed) <= 1e-12 * closed)),
                              "scope": f"all {NE * world} groups: per-rank checksums all-reduced (SUM)"},
                    "ms_per_sweep_kernel": ms_sweep,
                    "batched": batched,
                    "dense_case": dense}
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # end to end through the C ABI: host vi in, 10 sweeps, host result out
    if args.no_e2e:
        return finish(None)
    host_in = torch.empty(n, dtype=torch.float64, pin_memory=True)
    host_out = torch.empty(n, dtype=torch.float64, pin_memory=True)
    pb.init_state_device(va.data_ptr(), IE_BASE)
    torch.cuda.synchronize()
    host_in.copy_(va)
    del va, vb
    torch.cuda.empty_cache()
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        pb.sweep_iterations_host(host_out.data_ptr(), host_in.data_ptr(), NITER)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = e0.elapsed_time(e1) / 1e3
    e2e_s = max_over_ranks(e2e_s)
    e2e_ok = bool(torch.equal(host_out, host_in))
    e2e_slices = pb.iterations_slices()
    # the reference driver's own loop (runner.c:148-155): one Sweeper_sweep
    # per iteration on host buffers, each call copying vi in and vo out
    barrier()
    e0.record(stream)
    a_h, b_h = host_in, host_out
    for _ in range(NITER):
        pb.sweep_host_ptr(b_h.data_ptr(), a_h.data_ptr())
        a_h, b_h = b_h, a_h
    e1.record(stream)
    torch.cuda.synchronize()
    loop_s = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    # the built-in state is a fixed point of the sweep: the last output equals its input
    loop_ok = bool(torch.equal(a_h, b_h))
    return finish({"value": updates_per_sweep() * NITER * e2e_steps * world / e2e_s, "unit": UNIT,
                   "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                   "path": "Sweeper_sweep_iterations (host vi in, 10 device sweeps, host result out)",
                   "group_slices": e2e_slices,
                   "reference_driver_loop": {
                       "value": updates_per_sweep() * NITER * world / loop_s, "unit": UNIT,
                       "h2d_bytes_per_step": 8 * n * NITER, "d2h_bytes_per_step": 8 * n * NITER,
                       "path": "Sweeper_sweep on pinned host Pointers, once per iteration (runner.c's loop: "
                               "every call copies vi in and vo out, in group slices)",
                       "result_matches": loop_ok},
                   "overlap": "the groups are swept in slices of group pairs, each through all 10 sweeps; a "
                              "slice's host copies overlap the other slices' sweeps (same results)",
                   "result_matches": e2e_ok})


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched serving workload")
    ap.add_argument("--no-dense", action="store_true", help="skip the 32x32x96 / ne 128 / na 128 case")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision sweeps")
    ap.add_argument("--fp64-flags", default="", help="sweeper flags of the FP64 step instead of --autotune 1 "
                                                     "(e.g. '--fp64_kernel 1 --tile 42 --task_window 8')")
    ap.add_argument("--batch-steps", type=int, default=2, help="timed batched sweeps")
    ap.add_argument("--batch-warmup", type=int, default=1, help="untimed batched sweeps")
    ap.add_argument("--case", choices=["config2", "small"], default="config2",
                    help="small: 32^3 cells, ne 32, one sweep per step, no e2e / CPU legs (profiling runs)")
    args = ap.parse_args()
    if args.case == "small":
        global NX, NY, NZ, NE, NITER, WORKLOAD
        NX = NY = NZ = 32
        NE, NITER = 32, 1
        args.no_cpu = True
        args.no_e2e = True
        args.no_batch = True
        args.no_dense = True
        WORKLOAD = WORKLOAD.replace("64x64x64", "32x32x32").replace("ne 64", "ne 32").replace(
            "niterations 10", "niterations 1")
    else:
        args.no_e2e = False
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())

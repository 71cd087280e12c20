"""GPU checks of batched sweeps (msb_batch_*): many problems in one
persistent launch must give, for every problem, exactly the result of that
problem's own Sweeper (FP64, bit for bit), whatever the class mix, the
scratch arena size (problems reusing the face scratch of completed ones), the
tile chosen by the autotuner, or the iteration loop run as a CUDA graph.
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import minisweep_b200 as msb  # noqa: E402

PROBLEMS = [
    dict(ncell_x=5, ncell_y=4, ncell_z=6, ne=3, na=7, nm=16),
    dict(ncell_x=9, ncell_y=7, ncell_z=3, ne=8, na=40, nm=4),
    dict(ncell_x=3, ncell_y=11, ncell_z=5, ne=1, na=32, nm=8),
    dict(ncell_x=12, ncell_y=6, ncell_z=4, ne=5, na=64, nm=16),
    dict(ncell_x=1, ncell_y=1, ncell_z=1, ne=2, na=16, nm=4),
    dict(ncell_x=8, ncell_y=8, ncell_z=8, ne=4, na=33, nm=16),
    dict(ncell_x=6, ncell_y=10, ncell_z=7, ne=6, na=20, nm=4),
    dict(ncell_x=16, ncell_y=12, ncell_z=10, ne=7, na=32, nm=16),
    dict(ncell_x=7, ncell_y=5, ncell_z=4, ne=3, na=100, nm=8),  # four passes, the last ragged
]


def flags(p):
    return f"--ncell_x {p['ncell_x']} --ncell_y {p['ncell_y']} --ncell_z {p['ncell_z']} --ne {p['ne']} --na {p['na']}"


def single(p, vi, a=None, m=None, niter=1):
    # the problem's own Sweeper with the kernel the batch uses (the staged
    # FP64 kernel, 32-angle passes): same summation order, same bits
    with msb.Problem(flags(p) + " --fp64_kernel 0 --angle_pass 32", nm=p["nm"]) as pb:
        if a is not None:
            pb.set_matrices(a, m)
        v = vi
        for _ in range(niter):
            v = pb.sweep_host(v)
    return v


class Device:
    """Device arrays of a list of problems (built-in state and matrices unless given)."""

    def __init__(self, problems, mats=None, states=None):
        dev = torch.device("cuda:0")
        self.vi, self.vo, self.a, self.m, self.host_vi = [], [], [], [], []
        self.descs = []
        for i, p in enumerate(problems):
            if states is not None and states[i] is not None:
                vi_h = states[i]
            else:
                with msb.Problem(flags(p), nm=p["nm"]) as pb:
                    vi_h = pb.init_state()
            a_h, m_h = mats[i] if mats is not None and mats[i] is not None else msb.builtin_matrices(p["nm"], p["na"])
            vi = torch.from_numpy(vi_h).to(dev)
            vo = torch.full_like(vi, float("nan"))
            a = torch.from_numpy(np.ascontiguousarray(a_h)).to(dev)
            m = torch.from_numpy(np.ascontiguousarray(m_h)).to(dev)
            self.vi.append(vi), self.vo.append(vo), self.a.append(a), self.m.append(m), self.host_vi.append(vi_h)
            d = dict(p)
            d.update(vi=vi.data_ptr(), vo=vo.data_ptr(), a_from_m=a.data_ptr(), m_from_a=m.data_ptr())
            self.descs.append(d)
        torch.cuda.synchronize()


def test_batch_matches_single_sweepers():
    D = Device(PROBLEMS)
    with msb.Batch(D.descs) as b:
        b.sweep(0)
        b.sync()
        info = b.info()
    assert info["nclass"] == 3  # one class per NM: every entry sweeps one 32-angle chunk
    for i, p in enumerate(PROBLEMS):
        ref = single(p, D.host_vi[i])
        got = D.vo[i].cpu().numpy()
        assert np.array_equal(got, ref), (i, p)


def test_batch_small_problem_workload():
    """The first 48 problems of the small-problem serving workload (many
    problems that each leave most SMs idle), against their own Sweepers."""
    W = msb.small_batch_workload()[:48]
    D = Device(W)
    with msb.Batch(D.descs, autotune=True) as b:
        b.sweep(0)
        b.sync()
    for i, p in enumerate(W):
        assert np.array_equal(D.vo[i].cpu().numpy(), single(p, D.host_vi[i])), (i, p)


def test_batch_matches_oracle():
    probs = PROBLEMS[:3]
    D = Device(probs)
    with msb.Batch(D.descs) as b:
        b.sweep(0)
        b.sync()
    for i, p in enumerate(probs):
        a, m = oracle.am_matrices(p["nm"], p["na"])
        ref = oracle.sweep(p["ncell_x"], p["ncell_y"], p["ncell_z"], p["ne"], p["nm"], p["na"], a, m, D.host_vi[i])
        assert np.array_equal(D.vo[i].cpu().numpy(), ref)


def test_batch_scratch_reuse():
    # arena of the largest problem's face scratch: problems wait for the
    # completion of those whose bytes they reuse
    probe = msb.Batch(PROBLEMS, plan_nsm=148)
    _, nb, _, _ = probe.scratch()
    probe.close()
    D = Device(PROBLEMS)
    with msb.Batch(D.descs, scratch_bytes=int(nb.max())) as b:
        assert b.info()["npred"] > 0
        b.sweep(0)
        b.sync()
        ms = b.problem_ms()
    assert np.all(ms > 0)
    for i, p in enumerate(PROBLEMS):
        assert np.array_equal(D.vo[i].cpu().numpy(), single(p, D.host_vi[i])), i


@pytest.mark.parametrize("niter", [1, 2, 3])
def test_batch_graph_iterations(niter):
    probs = PROBLEMS[:4]
    D = Device(probs)
    s = torch.cuda.Stream()
    with msb.Batch(D.descs) as b:
        b.run(niter, s.cuda_stream)
        b.sync(s.cuda_stream)
        b.run(niter, s.cuda_stream)  # the cached graph again
        b.sync(s.cuda_stream)
    # an odd count leaves its result in vo and the next run starts again from
    # vi; an even count leaves it in vi, where the next run continues
    total = 2 * niter if niter % 2 == 0 else niter
    for i, p in enumerate(probs):
        ref = single(p, D.host_vi[i], niter=total)
        got = (D.vi[i] if niter % 2 == 0 else D.vo[i]).cpu().numpy()
        assert np.array_equal(got, ref), (i, niter)


def test_batch_caller_matrices_and_state():
    probs = [PROBLEMS[0], PROBLEMS[3], PROBLEMS[6]]
    mats, states = [], []
    for k, p in enumerate(probs):
        a, m, vi = oracle.random_problem(p["ncell_x"], p["ncell_y"], p["ncell_z"], p["ne"], p["nm"], p["na"],
                                         seed=20 + k)
        mats.append((a, m))
        states.append(vi)
    D = Device(probs, mats=mats, states=states)
    with msb.Batch(D.descs) as b:
        b.sweep(0)
        b.sync()
    for i, p in enumerate(probs):
        ref = single(p, states[i], a=mats[i][0], m=mats[i][1])
        assert np.array_equal(D.vo[i].cpu().numpy(), ref), i


def test_batch_autotune():
    D = Device(PROBLEMS)
    with msb.Batch(D.descs, autotune=True) as b:
        info = b.info()
        assert info["tune_ms"] > 0
        for i in range(len(PROBLEMS)):
            D.vo[i].fill_(float("nan"))
        torch.cuda.synchronize()
        b.sweep(0)
        b.sync()
    tiles = {c["tile"] for c in info["classes"]}
    assert tiles <= {(4, 2), (2, 4)}
    for i, p in enumerate(PROBLEMS):
        assert np.array_equal(D.vo[i].cpu().numpy(), single(p, D.host_vi[i])), i


def test_batch_timeout_reports_and_recovers():
    # a wait budget of 1 ns: a task whose dependency is not yet complete gives
    # up at once; the launch ends with MSB_ERR_TIMEOUT and the context stays
    # usable
    probs = [dict(ncell_x=16, ncell_y=16, ncell_z=16, ne=8, na=32, nm=16)]
    D = Device(probs)
    with msb.Batch(D.descs) as b:
        b.set_timeout_ns(1)
        b.sweep(0)
        with pytest.raises(msb.SweepError) as e:
            b.sync()
        assert e.value.code == msb.MSB_ERR_TIMEOUT
        b.set_timeout_ns(0)
        b.sweep(0)
        b.sync()
    assert np.array_equal(D.vo[0].cpu().numpy(), single(probs[0], D.host_vi[0]))

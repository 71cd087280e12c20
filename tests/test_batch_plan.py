"""Host-side checks of the batch planner (msb_batch_plan: no GPU).

A batch sweeps many problems in one persistent launch.  Its task table must
be safe for the kernel's protocol:

* every problem is swept in entries of 32 angles (its angle passes), in
  pass order: each later pass shares the first pass's scratch and waits for
  the pass before it;
* topological: every dependency of a task precedes it in the table, and
  belongs to the same entry;
* one contiguous range per class (the CTAs work through classes in order);
* every entry's tasks are exactly the schedule its problem's own Sweeper
  would build for the same tile (the records, dependencies renumbered);
* face scratch: two entries whose arena ranges overlap are ordered -- all
  tasks of the earlier one precede all tasks of the later one in the table,
  and the later one waits (transitively) for the earlier one's completion.
"""
import numpy as np
import pytest

import minisweep_b200 as msb

TK_OCT, TK_PHASE, TK_GP, TK_X0, TK_X1, TK_Y0, TK_Y1, TK_Z0, TK_Z1 = range(9)
TK_FLAGS, TK_DEP_X, TK_DEP_Y, TK_DEP_Z, TK_DEP_VO, TK_DEP_MODE, TK_LEVEL = range(9, 16)
DEPS = [TK_DEP_X, TK_DEP_Y, TK_DEP_Z, TK_DEP_VO]

SMALL = [
    dict(ncell_x=5, ncell_y=4, ncell_z=6, ne=3, na=7, nm=16),
    dict(ncell_x=9, ncell_y=7, ncell_z=3, ne=8, na=40, nm=4),
    dict(ncell_x=3, ncell_y=11, ncell_z=5, ne=1, na=32, nm=8),
    dict(ncell_x=12, ncell_y=6, ncell_z=4, ne=5, na=64, nm=16),
    dict(ncell_x=1, ncell_y=1, ncell_z=1, ne=2, na=16, nm=4),
    dict(ncell_x=8, ncell_y=8, ncell_z=8, ne=4, na=33, nm=16),
    dict(ncell_x=6, ncell_y=10, ncell_z=7, ne=6, na=20, nm=4),
]


def plan(problems, nsm=8, scratch=0, mask=0):
    return msb.Batch(problems, plan_nsm=nsm, scratch_bytes=scratch, tile24_mask=mask)


def check_plan(b, problems, mask=0):
    rec, prob = b.tasks()
    n = len(rec)
    info = b.info()
    assert info["ntask"] == n and info["nproblem"] == len(problems)
    eprob, ea0 = b.entries()
    # entries: every problem's 32-angle passes, in order
    for p, pr in enumerate(problems):
        mine = np.nonzero(eprob == p)[0]
        assert list(ea0[mine]) == list(range(0, pr["na"], 32))
        assert np.all(np.diff(mine) == 1)
    idx = np.arange(n)
    # topological, same-problem dependencies
    for d in DEPS:
        dep = rec[:, d]
        has = dep >= 0
        assert np.all(dep[has] < idx[has])
        assert np.all(prob[dep[has]] == prob[has])
    # contiguous classes
    total = 0
    for c in info["classes"]:
        total += c["ntask"]
    assert total == n
    change = np.count_nonzero(np.diff([_class_of(problems[eprob[e]], info) for e in prob]))
    assert change <= info["nclass"] - 1
    # each entry's records = its problem's own schedule (dependencies renumbered)
    for e in range(len(eprob)):
        pr = problems[eprob[e]]
        mine = np.nonzero(prob == e)[0]
        k = {4: 0, 8: 1, 16: 2}[pr["nm"]]
        t24 = (mask >> k) & 1
        tx, ty = (2, 4) if t24 else (4, 2)
        own = msb.schedule(pr["ncell_x"], pr["ncell_y"], pr["ncell_z"], pr["ne"], tx, ty, 1)
        assert len(own) == len(mine)
        got = rec[mine][:, :TK_FLAGS + 1]
        key = lambda a: np.lexsort(a.T[::-1])
        assert np.array_equal(got[key(got)], own[:, :TK_FLAGS + 1][key(own[:, :TK_FLAGS + 1])])
        # dependency structure: same (phase, oct, gp, tile) targets
        pos = {tuple(r[:TK_Z1 + 1]): i for i, r in enumerate(rec[mine])}
        ident = {tuple(r[:TK_Z1 + 1]): r for r in own}
        for i, r in enumerate(rec[mine]):
            o = ident[tuple(r[:TK_Z1 + 1])]
            for d in DEPS:
                if o[d] < 0:
                    assert r[d] < 0
                else:
                    tgt = tuple(own[o[d]][:TK_Z1 + 1])
                    assert r[d] == mine[pos[tgt]]
    return rec, prob


def _class_of(p, info):
    for c, cl in enumerate(info["classes"]):
        if cl["nm"] == p["nm"] and cl["nch"] == 1:
            return c
    raise AssertionError("no class")


def test_plan_all_resident():
    b = plan(SMALL)
    check_plan(b, SMALL)
    off, nb, po, pred = b.scratch()
    eprob, ea0 = b.entries()
    # enough scratch for all at once: an entry waits only for its problem's
    # previous pass, whose scratch it shares
    for e in range(len(eprob)):
        ps = list(pred[po[e]:po[e + 1]])
        if ea0[e] == 0:
            assert ps == []
        else:
            assert ps == [e - 1] and eprob[e - 1] == eprob[e] and off[e] == off[e - 1]
    # the problems' placements are disjoint
    first = ea0 == 0
    order = np.argsort(off[first])
    o, b_ = off[first][order], (off + nb)[first][order]
    assert np.all(o[1:] >= b_[:-1])


@pytest.mark.parametrize("mask", [0, 0b111111, 0b101010])
def test_plan_tiles(mask):
    check_plan(plan(SMALL, mask=mask), SMALL, mask=mask)


@pytest.mark.parametrize("nsm", [1, 3, 148])
def test_plan_reuse_is_ordered(nsm):
    # scratch for the largest problem only: problems run one after another
    # in the arena, and every overlap is ordered
    probe = plan(SMALL, nsm=nsm)
    _, nb, _, _ = probe.scratch()
    b = plan(SMALL, nsm=nsm, scratch=int(nb.max()))
    rec, prob = check_plan(b, SMALL)
    off, nb, po, pred = b.scratch()
    n = len(off)  # entries
    first = np.array([np.min(np.nonzero(prob == p)[0]) for p in range(n)])
    last = np.array([np.max(np.nonzero(prob == p)[0]) for p in range(n)])
    preds = [set(pred[po[p]:po[p + 1]]) for p in range(n)]

    def waits_for(q, p):  # q waits (transitively) for p
        seen, todo = set(), [q]
        while todo:
            x = todo.pop()
            for y in preds[x]:
                if y == p:
                    return True
                if y not in seen:
                    seen.add(y)
                    todo.append(y)
        return False

    overlaps = 0
    for p in range(n):
        for q in range(n):
            if p == q:
                continue
            if off[p] < off[q] + nb[q] and off[q] < off[p] + nb[p] and first[p] < first[q]:
                overlaps += 1
                assert last[p] < first[q]
                assert waits_for(q, p)
    assert overlaps > 0
    # the waits only point to problems placed earlier in the table
    for q in range(n):
        for p in preds[q]:
            assert last[p] < first[q]


def test_plan_scratch_too_small():
    with pytest.raises(msb.SweepError):
        plan(SMALL, scratch=1024)


def test_plan_rejects_unsupported():
    with pytest.raises(msb.SweepError):
        plan([dict(ncell_x=2, ncell_y=2, ncell_z=2, ne=2, na=129, nm=16)])
    with pytest.raises(msb.SweepError):
        plan([dict(ncell_x=2, ncell_y=2, ncell_z=2, ne=2, na=16, nm=12)])
    with pytest.raises(msb.SweepError):
        plan([dict(ncell_x=0, ncell_y=2, ncell_z=2, ne=2, na=16, nm=4)])


def test_workload_generator():
    w = msb.batch_workload()
    assert len(w) == 256
    assert w == msb.batch_workload()
    for p in w:
        assert 8 <= p["ncell_x"] <= 48 and 8 <= p["ncell_y"] <= 48 and 8 <= p["ncell_z"] <= 64
        assert p["ne"] in (8, 16, 32, 64) and p["na"] in (16, 32, 64) and p["nm"] in (4, 16)
    assert {p["nm"] for p in w} == {4, 16} and {p["na"] for p in w} == {16, 32, 64}


def test_plan_workload_subset_with_reuse():
    # 24 problems of the serving workload, arena of twice the largest
    w = msb.batch_workload()[:24]
    probe = plan(w, nsm=148)
    _, nb, _, _ = probe.scratch()
    b = plan(w, nsm=148, scratch=int(2 * nb.max()))
    rec, prob = b.tasks()
    for d in DEPS:
        dep = rec[:, d]
        has = dep >= 0
        assert np.all(dep[has] < np.arange(len(rec))[has])
        assert np.all(prob[dep[has]] == prob[has])
    assert b.info()["npred"] > 0

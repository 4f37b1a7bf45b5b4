"""The request server (lbm_server_*): continuous batching of solves.

Solves of different sizes, methods and step counts are submitted at
different times into a server whose arena holds only a few of them, so
they queue, join and leave the resident set at different step boundaries
and the arena gets compacted.  Each result must equal the same solve run
alone in a batch of one (same precision, same tile shape) bit for bit,
and a failing or cancelled solve must not disturb the others.
"""
import numpy as np
import pytest

from uq_b200 import native as N
from uq_b200 import workloads as W
from uq_b200.solver import Batch, Server

from golden_util import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("rho", "ux", "uy", "T", "p")
BYTES_PER_NODE = {"f32": 3 * 26 * 4 + 4 + 1, "f64": 3 * 26 * 8 + 8 + 1}


def _mix():
    return [
        W.couette(nx=48, ny=40, steps=30, seed=1, fmethod=1, rkmethod=1),
        W.couette(nx=64, ny=64, steps=45, seed=2, fmethod=0, rkmethod=0, u_w=0.15),
        W.riemann(nx=64, ny=48, steps=25, fmethod=0, rkmethod=1),
        W.couette(nx=33, ny=37, steps=20, seed=3, fmethod=1, rkmethod=0, tau=0.08),
        W.riemann(nx=40, ny=40, steps=35, fmethod=1, rkmethod=0),
        W.couette(nx=96, ny=24, steps=15, seed=4, fmethod=1, rkmethod=1, Pr=0.9),
        W.random_state(37, 29, seed=3, bc="mirror", solid_frac=0.1, steps=12, du=0.02, drho=0.02, dT=0.02),
    ]


def _alone(case, precision):
    b = Batch([case], precision=precision)
    b.step(int(case["steps"]))
    st = int(b.status()[0])
    out = b.macro(0)
    b.close()
    return st, out


def _case_slots(c):
    """Node slots a solve takes in the arena: ny rows of its pitch, which
    holds 4 ghost columns on each side when the solve is periodic in x."""
    nx, ny = c["bnd"].shape
    ghosts = 8 if c.get("periodicX") and nx >= 8 else 0
    return ny * (-(-(nx + ghosts) // 32) * 32)


def _arena_for(cases, precision, resident):
    """An arena that holds about `resident` of the largest solves."""
    slots = max(_case_slots(c) for c in cases)
    return int(resident * slots * BYTES_PER_NODE[precision]) + 4096


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_results_identical_alone_and_in_the_mix(cuda_device, precision):
    cases = _mix()
    srv = Server(precision=precision, arena_bytes=_arena_for(cases, precision, 2.5), status_poll_steps=4)
    ids = {}
    # the first four at once (they queue for the arena), the rest one by one
    # as earlier solves finish, so they join a running batch
    for k in range(4):
        ids[srv.submit(cases[k])] = k
    nxt, done = 4, []
    while len(done) < len(cases):
        rid = srv.wait_any(timeout=120.0)
        assert rid is not None, "server made no progress"
        done.append(rid)
        if nxt < len(cases):
            ids[srv.submit(cases[nxt])] = nxt
            nxt += 1
    infos = {rid: srv.info(rid) for rid in ids}
    for rid, k in ids.items():
        code, got = srv.result(rid)
        st, ref = _alone(cases[k], precision)
        assert code == st == N.LBM_OK, (k, code, st)
        assert infos[rid]["steps_done"] == cases[k]["steps"]
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), (k, f, np.max(np.abs(got[f] - ref[f])))
    stats = srv.stats()
    assert stats["completed"] == len(cases) and stats["failed"] == 0
    assert stats["repacks"] >= len(cases)
    # solves overlapped on the device: some pair was resident at the same step
    spans = sorted((i["step_admit"], i["step_done"]) for i in infos.values())
    assert any(spans[j + 1][0] < spans[j][1] for j in range(len(spans) - 1))
    # and the arena was too small for all of them at once
    assert any(i["t_admit"] > i["t_submit"] + 1e-4 for i in infos.values()) or stats["compactions"] > 0
    srv.close()


def test_mixed_precision_server_within_tolerance_of_fp64(cuda_device):
    # short horizon: these flows amplify any perturbation (FP64 round-off
    # included) by orders of magnitude within tens of steps
    cases = [dict(c, steps=10) for c in _mix()[:3]]
    srv = Server(precision="f32")
    ids = [srv.submit(c) for c in cases]
    for rid, case in zip(ids, cases):
        assert srv.wait(rid, timeout=120.0)
        code, got = srv.result(rid)
        assert code == N.LBM_OK
        st, ref = _alone(case, "f64")
        assert st == N.LBM_OK
        for f in ("rho", "T"):
            assert rel_l2(got[f], ref[f]) <= 1e-5, (f, rel_l2(got[f], ref[f]))
        u = np.hypot(got["ux"], got["uy"])
        uref = np.hypot(ref["ux"], ref["uy"])
        assert np.sqrt(np.sum((u - uref) ** 2) / max(np.sum(uref ** 2), 1e-300)) <= 1e-5
    srv.close()


def test_failing_solve_is_evicted_without_disturbing_others(cuda_device):
    good = _mix()[:2]
    bad = W.couette(nx=40, ny=32, steps=200, seed=9)
    bad["density"] = np.asarray(bad["density"], dtype=np.float64).copy()
    bad["density"][2:] = -1.0  # non-physical state: the device checks flag it
    srv = Server(precision="f32", status_poll_steps=2)
    ids = [srv.submit(good[0]), srv.submit(bad), srv.submit(good[1])]
    for rid in ids:
        assert srv.wait(rid, timeout=120.0)
    code_bad, _ = srv.result(ids[1])
    assert code_bad in (N.LBM_ERR_NONFINITE, N.LBM_ERR_EQUILIBRIUM)
    assert srv.info(ids[1])["steps_done"] < 200  # removed early
    for rid, case in ((ids[0], good[0]), (ids[2], good[1])):
        code, got = srv.result(rid)
        st, ref = _alone(case, "f32")
        assert code == st == N.LBM_OK
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f])
    assert srv.stats()["failed"] == 1
    srv.close()


def test_cancel_release_and_errors(cuda_device):
    srv = Server(precision="f32")
    long_case = W.couette(nx=64, ny=64, steps=10 ** 7, seed=5)
    short_case = _mix()[0]
    rid_long = srv.submit(long_case)
    rid_short = srv.submit(short_case)
    assert srv.wait(rid_short, timeout=120.0)
    assert srv.info(rid_long)["state"] == N.LBM_REQ_RESIDENT
    assert not srv.wait(rid_long, timeout=0.05)
    srv.cancel(rid_long)
    assert srv.wait(rid_long, timeout=60.0)
    code, _ = srv.result(rid_long)
    assert code == N.LBM_ERR_CANCELLED
    code, got = srv.result(rid_short)
    st, ref = _alone(short_case, "f32")
    assert code == st == N.LBM_OK
    assert np.array_equal(got["rho"], ref["rho"])
    srv.release(rid_long)
    with pytest.raises(N.LbmError) as e:
        srv.info(rid_long)
    assert e.value.code == N.LBM_ERR_NOT_FOUND
    # a solve that can never fit the arena and one without a step count
    small = Server(precision="f32", arena_bytes=2 * 1024 * 1024)
    with pytest.raises(N.LbmError) as e:
        small.submit(W.couette(nx=256, ny=256, steps=10))
    assert e.value.code == N.LBM_ERR_NOMEM
    no_steps = dict(short_case, steps=0, tol=1e-6)
    with pytest.raises(N.LbmError) as e:
        small.submit(no_steps)
    assert e.value.code == N.LBM_ERR_INVALID
    small.close()
    srv.close()


def test_fragmented_arena_is_compacted(cuda_device):
    # three 64 x 64 solves (64 x 96 node slots each) fill an arena of ~3.6 of
    # them; the middle one finishes first and leaves a hole too small for a
    # 96 x 64 solve (64 x 128 slots), although the free total is large enough
    a = W.couette(nx=64, ny=64, steps=3000, seed=11)
    b = W.couette(nx=64, ny=64, steps=5, seed=12)
    c = W.couette(nx=64, ny=64, steps=3000, seed=13, fmethod=0)
    d = W.couette(nx=96, ny=64, steps=20, seed=14, rkmethod=0)
    slots, slots_d = _case_slots(a), _case_slots(d)
    assert slots_d > 0.6 * slots  # the hole b leaves, and the free end, are each too small for d
    srv = Server(precision="f32", arena_bytes=int(3.6 * slots * BYTES_PER_NODE["f32"]), use_graph=False)
    ids = [srv.submit(a), srv.submit(b), srv.submit(c)]
    assert srv.wait(ids[1], timeout=120.0)
    assert srv.info(ids[0])["state"] == N.LBM_REQ_RESIDENT
    ids.append(srv.submit(d))
    for rid in ids:
        assert srv.wait(rid, timeout=120.0)
    stats = srv.stats()
    assert stats["compactions"] >= 1
    # d was admitted while a and c were still resident
    info_d, info_a = srv.info(ids[3]), srv.info(ids[0])
    assert info_d["step_admit"] < info_a["step_done"]
    for rid, case in zip(ids, (a, b, c, d)):
        code, got = srv.result(rid)
        st, ref = _alone(case, "f32")
        assert code == st == N.LBM_OK
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), (rid, f)
    srv.close()


def test_fast_lane_small_solves_take_several_steps(cuda_device):
    # one large solve paces the batch; the small ones (each < 1/16 of the
    # resident nodes) take 4 steps per server step and still end exactly
    # on their step counts with the results they have alone
    big = W.couette(nx=256, ny=256, steps=600, seed=21)
    small = [W.couette(nx=32, ny=32, steps=97 + 10 * k, seed=22 + k, fmethod=k % 2, rkmethod=(k // 2) % 2)
             for k in range(4)]
    srv = Server(precision="f32", use_graph=True)
    ids = [srv.submit(big)] + [srv.submit(c) for c in small]
    for rid in ids:
        assert srv.wait(rid, timeout=120.0)
    for rid, case in zip(ids[1:], small):
        info = srv.info(rid)
        assert info["steps_done"] == case["steps"]
        server_steps = info["step_done"] - info["step_admit"]
        assert server_steps < case["steps"] / 2, (server_steps, case["steps"])
        code, got = srv.result(rid)
        st, ref = _alone(case, "f32")
        assert code == st == N.LBM_OK
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), f
    code, got = srv.result(ids[0])
    st, ref = _alone(big, "f32")
    assert code == st == N.LBM_OK and np.array_equal(got["rho"], ref["rho"])
    srv.close()

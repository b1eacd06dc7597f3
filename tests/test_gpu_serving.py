"""Continuous-batching server: every result the same alone and in the mix
(bit-exact), admission by HBM budget, refusals, and host-injected failures.
No GPU fault is provoked: failures are made on the host."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def M():
    from impeller_b200 import build
    build.build()
    from impeller_b200 import msm
    msm._lib.load()
    return msm


@pytest.fixture(scope="module")
def srs():
    return O.gen_points(1 << 15, seed=31)


def test_results_same_alone_and_in_the_mix(M, srs):
    ctx = M.MsmContext(srs)
    ctx.precompute(16)  # some jobs use the resident table set, the rest plain windows
    rng = np.random.default_rng(5)
    sizes = [int(2 ** rng.uniform(0, 15)) for _ in range(48)] + [1 << 15, 1, 2]
    scal = [O.gen_scalars(n, seed=31, stream=i) for i, n in enumerate(sizes)]
    srv = M.MsmServer(ctx, max_batch=6, max_inflight=3)
    ids = [srv.submit(s) for s in scal]
    res = [srv.wait(j) for j in ids]
    st = srv.stats()
    srv.close()
    for i, (n, s) in enumerate(zip(sizes, scal)):
        alone = ctx.msm_host(s)
        assert (res[i][0] == alone).all(), (i, n)
        if n <= 4096:
            assert (res[i][0] == O.msm(srs[:n], s)).all(), (i, n)
    assert st["completed"] == len(sizes) and st["failed"] == 0
    assert st["batches"] < len(sizes) and st["mean_batch"] > 1.0
    assert st["max_concurrent"] >= 2  # batches overlapped on the device
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    ctx.close()


def test_admission_by_hbm_budget(M, srs):
    ctx = M.MsmContext(srs)
    srv = M.MsmServer(ctx, max_batch=8, max_inflight=2, hbm_budget=2 << 20)
    with pytest.raises(M._lib.ImpellerError, match="budget"):
        srv.submit(O.gen_scalars(1 << 15, seed=1, stream=1))
    small = [O.gen_scalars(64, seed=1, stream=10 + i) for i in range(12)]
    ids = [srv.submit(s) for s in small]
    for j, s in zip(ids, small):
        out, _ = srv.wait(j)
        assert (out == O.msm(srs[:64], s)).all()
    st = srv.stats()
    assert st["rejected"] == 1 and st["completed"] == 12
    assert st["peak_bytes"] <= st["budget_bytes"]
    srv.close()
    ctx.close()


def test_refuses_invalid_jobs(M, srs):
    ctx = M.MsmContext(srs[:100])
    srv = M.MsmServer(ctx)
    L = M._lib.load()
    import ctypes
    jid = ctypes.c_uint64()
    sc = O.gen_scalars(200, seed=2, stream=2)
    assert L.impeller_server_submit(srv.handle, sc.ctypes.data, 0, ctypes.byref(jid)) != 0    # n == 0
    assert L.impeller_server_submit(srv.handle, sc.ctypes.data, 101, ctypes.byref(jid)) != 0  # n > SRS
    assert L.impeller_server_submit(srv.handle, None, 10, ctypes.byref(jid)) != 0             # no scalars
    assert srv.stats()["rejected"] == 3
    ok = srv.submit(sc[:100])
    assert (srv.wait(ok)[0] == O.msm(srs[:100], sc[:100])).all()
    srv.close()
    ctx.close()


def test_injected_failure_then_recovery(M, srs):
    ctx = M.MsmContext(srs[:1000])
    srv = M.MsmServer(ctx, max_batch=4, max_inflight=1)
    srv.inject_failures(1)
    sc = O.gen_scalars(1000, seed=3, stream=3)
    bad = srv.submit(sc)
    with pytest.raises(M._lib.ImpellerError, match="failed"):
        srv.wait(bad)
    good = srv.submit(sc)
    assert (srv.wait(good)[0] == O.msm(srs[:1000], sc)).all()
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
    srv.close()
    ctx.close()


def test_second_wait_on_a_taken_job_returns_an_error(M, srs):
    # two threads wait on one job id: one takes the result, the other gets
    # an error instead of blocking
    import threading
    ctx = M.MsmContext(srs[:2000])
    srv = M.MsmServer(ctx, max_batch=4, max_inflight=1)
    sc = O.gen_scalars(2000, seed=4, stream=4)
    jid = srv.submit(sc)
    outcomes = []

    def waiter():
        try:
            outcomes.append(("ok", srv.wait(jid)[0]))
        except M._lib.ImpellerError as e:
            outcomes.append(("err", str(e)))

    ts = [threading.Thread(target=waiter) for _ in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert not any(t.is_alive() for t in ts)
    oks = [o for o in outcomes if o[0] == "ok"]
    errs = [o for o in outcomes if o[0] == "err"]
    assert len(oks) == 1 and len(errs) == 1, outcomes
    assert (oks[0][1] == O.msm(srs[:2000], sc)).all()
    # and a later wait on the taken id is refused at once
    with pytest.raises(M._lib.ImpellerError):
        srv.wait(jid)
    srv.close()
    ctx.close()


@pytest.mark.parametrize("step,what", [(1, "memory pool"), (2, "stream"), (3, "pinned result buffer"),
                                       (4, "pool reserve")])
def test_server_setup_failure_releases_and_recovers(M, srs, step, what):
    # a failure injected on the host at each setup step: create returns the
    # error with the step in the message, and a later create works
    ctx = M.MsmContext(srs[:500])
    L = M._lib.load()
    M._lib.check(L.impeller_server_fail_setup_step(step), "fail_setup_step")
    with pytest.raises(M._lib.ImpellerError, match=f"impeller_server_create: {what}: "):
        M.MsmServer(ctx, max_batch=4, max_inflight=2, hbm_budget=64 << 20)
    srv = M.MsmServer(ctx, max_batch=4, max_inflight=2, hbm_budget=64 << 20)
    sc = O.gen_scalars(500, seed=5, stream=step)
    assert (srv.wait(srv.submit(sc))[0] == O.msm(srs[:500], sc)).all()
    srv.close()
    ctx.close()


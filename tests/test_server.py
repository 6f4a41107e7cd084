"""Serving loop (mb_server_*): requests submitted while others are on the device are admitted as
arena memory and ring slots free up, and each result equals the same problem solved alone by
mb_batch_solve (same kernel code per instance: bitwise, checked here within 1e-12 relative)."""
import time

import numpy as np
import pytest

from helpers import SDP, SMALL, TDC, TDC_TOL, product_problem
from mumblebee_b200 import _lib
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMSettings, Server, batch_solve

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.status == b.status and a.niter == b.niter
    assert abs(a.pobj - b.pobj) <= 1e-12 * max(1.0, abs(b.pobj))
    for x, y in ((a.p, b.p), (a.d, b.d), (a.y, b.y)):
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-14)


def _mix(ctx):
    pbs = [f() for f in SMALL.values()] + [f() for f in SDP.values()]
    pbs += [G.portfolio(n, seed=s) for n, s in ((120, 1), (260, 2), (400, 3))]
    return [product_problem(pb, ctx=ctx) for pb in pbs]


def test_results_in_the_mix_equal_alone():
    ctx = Context.default(0)
    probs = _mix(ctx)
    alone = [batch_solve([p])[0] for p in probs]
    srv = Server(IPMSettings(), arena_bytes=1 << 30, capacity=64, ctx=ctx)
    tickets = []
    for i, p in enumerate(probs):            # staggered arrivals: later requests join running ones
        tickets.append(srv.submit(p))
        if i % 3 == 2:
            time.sleep(0.002)
    for t in tickets:
        assert srv.wait(t, 120.0) == Server.DONE
    for t, a in zip(tickets, alone):
        r, times, dev = srv.result(t)
        _same(r, a)
        assert times[0] <= times[1] <= times[2] and dev[1] > dev[0]
    st = srv.stats()
    assert st["completed"] == len(probs) and st["failed"] == 0 and st["arena_used"] == 0
    srv.close()


def test_admission_waits_for_arena_memory():
    ctx = Context.default(0)
    probs = [product_problem(G.portfolio(300, seed=s), ctx=ctx) for s in range(6)]
    one = max(p.footprint() for p in probs)
    srv = Server(IPMSettings(), arena_bytes=int(2.5 * one) + (1 << 20), capacity=16, ctx=ctx)   # two at a time
    tickets = [srv.submit(p) for p in probs]
    seen_queue = False
    for _ in range(2000):
        st = srv.stats()
        seen_queue |= st["running"] <= 2 and st["planned"] + st["queued"] > 0
        if st["completed"] == len(probs):
            break
        time.sleep(0.005)
    alone = batch_solve(probs)
    for t, a in zip(tickets, alone):
        assert srv.wait(t, 120.0) == Server.DONE
        _same(srv.result(t)[0], a)
    assert seen_queue
    srv.close()


def test_oversize_request_fails_and_server_goes_on():
    ctx = Context.default(0)
    small = product_problem(SMALL["port_small"](), ctx=ctx)
    big = product_problem(G.portfolio(400, seed=0), ctx=ctx)
    srv = Server(IPMSettings(), arena_bytes=small.footprint() * 3, capacity=8, ctx=ctx)
    tb, ts = srv.submit(big), srv.submit(small)
    assert srv.wait(tb, 60.0) == Server.FAILED
    with pytest.raises(_lib.MBError, match="arena"):
        srv.result(tb)
    assert srv.wait(ts, 60.0) == Server.DONE
    _same(srv.result(ts)[0], batch_solve([small])[0])
    srv.close()


def test_requests_after_a_lull_are_served():
    ctx = Context.default(0)
    p = product_problem(TDC["exp_small"](), ctx=ctx)
    s = IPMSettings(**TDC_TOL)
    srv = Server(s, arena_bytes=64 << 20, capacity=8, ctx=ctx)
    t1 = srv.submit(p)
    assert srv.wait(t1, 60.0) == Server.DONE
    r1 = srv.result(t1)[0]
    time.sleep(0.2)                           # nothing on the device in between
    t2 = srv.submit(p)
    assert srv.wait(t2, 60.0) == Server.DONE
    r2 = srv.result(t2)[0]
    _same(r2, r1)
    assert srv.stats()["launches"] >= 2
    srv.close()

"""Serving: continuous batching gives every request the result it gets alone.

A stream of requests with different sizes and methods goes through the server
with a small batch cap and an HBM budget that forces several batches to run at
the same time on separate streams.  Each request is then solved alone (its own
batch); energies must agree to 1e-12 Ha.  The budget is never exceeded.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone():
    from uegccd_b200 import Batch, serve

    reqs = serve.poisson_stream(14, rate=1e9, seed=3, nelectrons=(14, 54), ratios=(4, 8))
    srv = serve.Server(hbm_budget=600 << 20, max_batch=3, tol=1e-9)
    peak = {"b": 0}
    orig = srv._run_batch

    def spy(group, t0):
        with srv.lock:
            peak["b"] = max(peak["b"], srv.in_use)
        orig(group, t0)

    srv._run_batch = spy
    wall = srv.run(reqs, realtime=False)
    assert all(r.status >= 0 for r in reqs)
    assert srv.batches_started >= 3
    assert peak["b"] <= srv.budget
    for r in reqs:
        b = Batch([r.system])
        if r.method == "MP2":
            rc, e2, res = b.solve(max_iter=1)
            assert abs(e2[0] - r.ecorr) < 1e-12
        else:
            rc, e2, res = b.solve(drpa=(r.method == "dRPA"), **srv.opts)
            assert abs(res[0]["ecorr"] - r.ecorr) < 1e-12, (r.rid, r.method, res[0]["ecorr"], r.ecorr)
            assert res[0]["niter"] == r.niter
        b.close()
    s = serve.summarize(reqs, wall)
    assert s["completed"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0


def test_budget_admission_queues_requests():
    from uegccd_b200 import _capi, serve

    reqs = serve.poisson_stream(6, rate=1e9, seed=11, nelectrons=(54,), ratios=(8,), weights=(0.0, 0.0, 1.0))
    one = _capi.footprint(serve.build_system(reqs[0]), 6)[0]
    srv = serve.Server(hbm_budget=int(one * 1.5), max_batch=8, tol=1e-8)
    srv.run(reqs, realtime=False)
    # only one request fits at a time: six batches, never two at once
    assert srv.batches_started == 6
    assert srv.max_concurrent == 1
    assert all(r.status >= 0 for r in reqs)

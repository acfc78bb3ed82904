"""Serving: continuous batching gives every request the result it gets alone.

A stream of requests with different sizes and methods goes through the server
with a small batch cap and an HBM budget that forces several cohorts to run at
the same time on separate streams.  Each request is then solved alone (its own
batch); energies must agree to 1e-12 Ha.  The budget is never exceeded.  The
incremental solve (uegccd_batch_start / _advance) gives every solve the result of
uegccd_batch_solve, and releases a solve's result when it stops, before its
cohort's slowest solve ends.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone():
    from uegccd_b200 import Batch, serve

    reqs = serve.poisson_stream(14, rate=1e9, seed=3, nelectrons=(14, 54), ratios=(4, 8))
    srv = serve.Server(hbm_budget=600 << 20, max_batch=3, tol=1e-9)
    peak = {"b": 0}
    orig = srv._run_cohort

    def spy(group, t0):
        with srv.lock:
            peak["b"] = max(peak["b"], srv.in_use)
        orig(group, t0)

    srv._run_cohort = spy
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


def _systems(specs):
    from oracle.oracle import Oracle, parse_input_text

    out = []
    for n, cut, rs, tw in specs:
        vals = parse_input_text("")
        vals.update({"# Electrons": n, "Momentum Cutoff": cut, "rSMin": rs, "rSMax": rs, "NTwist": tw})
        o = Oracle(vals)
        sc = o.scalars()
        out.append((o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec()))
    return out


@pytest.mark.parametrize("drpa", [False, True])
def test_incremental_solve_matches_batch_solve(drpa):
    """Solves that stop at different rounds: each is released once, with the iteration
    count, energy and MaxRes of the one-call solve."""
    from uegccd_b200 import Batch

    systems = _systems([("14", "5", "1.0", "0 0 0"), ("24", "10", "5.0", "0.1 0.2 0.45"),
                        ("24", "10", "0.7", "-0.3 0.1 0.2"), ("54", "24", "2.0", "0.2 0.1 -0.4")])
    opts = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-10)
    rc, e2, ref = Batch(systems).solve(drpa=drpa, **opts)
    b = Batch(systems)
    e2i = b.start(drpa=drpa, **opts)
    np.testing.assert_array_equal(e2, e2i)
    got, rounds, order = {}, 0, []
    active = len(systems)
    while active:
        active, done = b.advance(1)
        rounds += 1
        for s, r in done:
            assert s not in got
            got[s] = r
            order.append(s)
    assert sorted(got) == list(range(len(systems)))
    assert len({ref[s]["niter"] for s in range(len(systems))}) > 1   # they stop at different rounds
    assert order == sorted(order, key=lambda s: (ref[s]["niter"] + 3) // 4)
    for s, r in got.items():
        assert r["niter"] == ref[s]["niter"]
        assert abs(r["ecorr"] - ref[s]["ecorr"]) < 1e-12
        assert abs(r["max_res"] - ref[s]["max_res"]) <= 1e-12 * max(1.0, abs(ref[s]["max_res"]))
        assert r["status"] == ref[s]["status"] == 0
        if drpa:
            assert abs(r["ecorr_sosex"] - ref[s]["ecorr_sosex"]) < 1e-12


def test_served_solves_retire_before_their_cohort_ends():
    """One cohort with a fast and a slow solve: the fast one's result comes back first."""
    from uegccd_b200 import serve

    fast = serve.Request(0, 14, 1.0, 4, (0.0, 0.0, 0.0), "CCD")
    slow = serve.Request(1, 54, 5.0, 16, (0.1, 0.2, 0.3), "CCD")
    srv = serve.Server(hbm_budget=8 << 30, max_batch=8, tol=1e-10, batch_window=2.0)
    srv.run([fast, slow], realtime=False)
    assert srv.batches_started == 1
    assert fast.status == 0 and slow.status == 0
    assert fast.niter < slow.niter
    assert fast.t_done < slow.t_done

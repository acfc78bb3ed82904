"""Failure paths of the solve calls, made on the host (no GPU fault is ever provoked).

* A NaN planted in one system's host-prepared eigenvalues: that solve ends with
  UEGCCD_ERR_NUMERIC in its own status, the call returns UEGCCD_ERR_NUMERIC, and the
  other solves of the batch finish exactly as they do without it.
* MaxIter reached: max_iter=2 returns UEGCCD_NOT_CONVERGED with fail set, the outcome
  the reference prints as "DID NOT CONVERGE" (CCD.f90:103-114).
* Device memory: a library memory cap below a batch's needs makes uegccd_batch_create
  return UEGCCD_ERR_ALLOC and leaves the library's memory as it was; a cap that holds only
  part of the DIIS history makes the solve take fewer vectors, as SetUpDIISCC steps its
  depth down until Allocate succeeds (DIISCC.f90:22-29).
* The two-channel form: a NaN ends its solve with UEGCCD_ERR_NUMERIC too.
* Devices: a batch created on one host thread and solved from another gives the same
  energies, and every call leaves the calling thread's current device as it was.
"""
import ctypes as C
import threading

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text

pytestmark = pytest.mark.gpu

ERR_ALLOC, ERR_NUMERIC, NOT_CONVERGED = -3, -5, 1


def _sys(n="24", cut="10", rs="2.0", twist="0.1 0.2 0.3"):
    vals = parse_input_text("")
    vals.update({"# Electrons": n, "Momentum Cutoff": cut, "rSMin": rs, "rSMax": rs, "NTwist": twist})
    o = Oracle(vals)
    sc = o.scalars()
    return (o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())


def _twist_systems(k):
    import bench

    return bench.build_systems(bench.twists(k))


def test_nan_in_one_system_is_reported_per_solve():
    from uegccd_b200 import Batch

    good = [_sys(twist="0.1 0.2 0.3"), _sys(twist="-0.2 0.05 0.4")]
    bad = list(_sys(twist="0.3 -0.1 0.0"))
    eig = bad[3].copy()
    eig[bad[0] + 2] = np.nan          # a virtual orbital energy
    bad[3] = eig
    opts = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-9)
    b = Batch([good[0], tuple(bad), good[1]])
    rc, e2, res = b.solve(raise_on_error=False, **opts)
    assert rc == ERR_NUMERIC
    assert res[1]["status"] == ERR_NUMERIC
    assert res[0]["status"] == 0 and res[2]["status"] == 0
    rc2, e2g, ref = Batch(good).solve(**opts)
    assert rc2 == 0
    for a, c in zip((res[0], res[2]), ref):
        assert abs(a["ecorr"] - c["ecorr"]) < 1e-12 and a["niter"] == c["niter"]


def test_max_iter_reports_not_converged():
    from uegccd_b200 import Batch, Context

    s = _sys()
    rc, e2, res = Batch([s]).solve(max_iter=2)
    assert rc == NOT_CONVERGED
    assert res[0]["niter"] == 2 and res[0]["fail"] == 1 and res[0]["status"] == NOT_CONVERGED
    ctx = Context(*s)
    e2c, ta, tb, tc = ctx.mp2()
    rc, r, en, dts = ctx.ccd(ta, tb, tc, max_iter=2)
    assert rc == NOT_CONVERGED and r["fail"] == 1 and len(en) == 2


def test_memory_cap_refuses_create_and_keeps_the_library_consistent():
    from uegccd_b200 import Batch, _capi

    systems = _twist_systems(4)
    _capi.trim_cache()
    held0, cached0 = _capi.memory_info()
    try:
        _capi.set_memory_limit(held0 + (16 << 20))   # far below one 64 MB chunk
        with pytest.raises(_capi.UegccdError) as exc:
            Batch(systems)
        assert exc.value.code == ERR_ALLOC
        held1, _ = _capi.memory_info()
        assert held1 <= held0 + (16 << 20)            # nothing beyond the cap was kept
    finally:
        _capi.set_memory_limit(0)
    rc, e2, res = Batch(systems).solve(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-9)
    assert rc == 0 and all(r["ndiis"] == 6 for r in res)


def test_memory_cap_steps_the_diis_depth_down():
    from uegccd_b200 import Batch, _capi

    systems = _twist_systems(16)
    namp = sum(_capi.footprint(s, 0)[1] for s in systems)
    hist_bytes = lambda k: -(-k * namp * 8 // 256) * 256 + -(-k * namp * 4 // 256) * 256
    _capi.trim_cache()
    b = Batch(systems)
    rc, _, ref = b.solve()          # replay first: control buffers, no history
    assert rc == 0
    _capi.trim_cache()
    held, _ = _capi.memory_info()
    try:
        _capi.set_memory_limit(held + hist_bytes(3) + (1 << 20))
        rc, e2, res = b.solve(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-9)
    finally:
        _capi.set_memory_limit(0)
    assert rc == 0
    assert all(r["ndiis"] == 3 for r in res), [r["ndiis"] for r in res]
    # the same solve with three vectors asked for outright
    rc, e2b, res3 = Batch(systems).solve(scheme=1, ndiis=3, denom_factor=1.0, tol=1e-9)
    for a, c in zip(res, res3):
        assert abs(a["ecorr"] - c["ecorr"]) < 1e-12 and a["niter"] == c["niter"]


def _current_device():
    rt = C.CDLL("libcudart.so.12")
    d = C.c_int(-7)
    assert rt.cudaGetDevice(C.byref(d)) == 0
    return d.value


def test_batch_created_on_one_thread_solves_on_another():
    from uegccd_b200 import Batch

    systems = [_sys(twist="0.1 0.2 0.3"), _sys(n="14", cut="5", rs="1.0", twist="0 0 0")]
    opts = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-9)
    ref = Batch(systems).solve(**opts)[2]
    box = {}
    t = threading.Thread(target=lambda: box.update(b=Batch(systems, device=0)))
    t.start()
    t.join()

    def solve():
        box["dev_before"] = _current_device()
        box["res"] = box["b"].solve(**opts)[2]
        box["dev_after"] = _current_device()

    t = threading.Thread(target=solve)
    t.start()
    t.join()
    assert box["dev_before"] == box["dev_after"]
    for a, c in zip(box["res"], ref):
        assert abs(a["ecorr"] - c["ecorr"]) < 1e-12 and a["niter"] == c["niter"]


def test_nan_in_a_two_channel_solve_is_reported():
    """The two-channel form (Do XRings F) with a NaN planted in the eigenvalues: the solve
    stops with UEGCCD_ERR_NUMERIC instead of iterating to MaxIter, and the context stays
    usable: the same solve on clean eigenvalues then converges."""
    from uegccd_b200 import Context, _capi

    nocc, L, mad, eig, nvec = _sys()
    ctx = Context(nocc, L, mad, eig, nvec)
    _, ta, tb, tc = ctx.mp2()
    bad = eig.copy()
    bad[nocc + 2] = np.nan
    ctx.set_eigen(bad)
    with pytest.raises(_capi.UegccdError) as err:
        ctx.ccd(ta.copy(), tb.copy(), tc.copy(), do_ring=1, do_xring=0)
    assert err.value.code == ERR_NUMERIC
    ctx.set_eigen(eig)
    rc, r, _, _ = ctx.ccd(ta.copy(), tb.copy(), tc.copy(), do_ring=1, do_xring=0)
    assert rc == 0 and r["status"] == 0 and np.isfinite(r["ecorr"])

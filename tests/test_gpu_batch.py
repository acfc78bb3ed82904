"""Batched solves: many systems (different NOcc, NAO, twists, rs) in one launch per
residual term give the same results as each system alone.

The batch shares every kernel launch, so a solve must not see another solve's
data: this is checked with systems of different sizes, where any offset error
would show.  Tolerance: 1e-12 Ha between alone and in the mix (same iteration).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text

pytestmark = pytest.mark.gpu


def _systems(goldens):
    out = []
    g5 = parse_input_text("")
    g5.update(goldens["G5"]["keys"])
    out.append(Oracle(g5))                                  # N=24, 34 orbitals, rs=5, twisted
    out.append(Oracle(goldens["G1"]["input_text"]))         # N=14, 57 orbitals, rs=1
    v = parse_input_text("")
    v.update({"# Electrons": "54", "Momentum Cutoff": "24", "rSMin": "2.0", "rSMax": "2.0",
              "NTwist": "0.31 -0.12 0.07"})
    out.append(Oracle(v))                                   # N=54, 485 orbitals, twisted
    v = parse_input_text("")
    v.update({"# Electrons": "14", "Momentum Cutoff": "2", "rSMin": "1.0", "rSMax": "1.0",
              "NTwist": "0.1 0.1 0.1"})
    out.append(Oracle(v))                                   # N=14, 19 orbitals
    return out


def _tuple(o):
    sc = o.scalars()
    return (o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())


def test_batch_equals_alone_ccd(goldens):
    from uegccd_b200 import Batch, Context

    systems = _systems(goldens)
    b = Batch([_tuple(o) for o in systems])
    rc, e2, res = b.solve(max_iter=12)
    for s, o in enumerate(systems):
        ctx = Context(*_tuple(o))
        e2a, ta, tb, tc = ctx.mp2()
        rca, ra, en, _ = ctx.ccd(ta, tb, tc, max_iter=12)
        assert abs(e2[s] - e2a) < 1e-13
        assert res[s]["niter"] == ra["niter"]
        assert abs(res[s]["ecorr"] - ra["ecorr"]) < 1e-12, (s, res[s]["ecorr"], ra["ecorr"])
        np.testing.assert_allclose(b.amplitudes(s), tb, atol=1e-13, rtol=0)


def test_batch_converged_g5_member(goldens):
    """A converged member reproduces its golden energy while other members keep iterating."""
    from uegccd_b200 import Batch

    systems = _systems(goldens)
    b = Batch([_tuple(o) for o in systems])
    rc, e2, res = b.solve()
    assert res[0]["niter"] == goldens["G5"]["niter"]
    assert abs(res[0]["ecorr"] - goldens["G5"]["ec_ccd"]) < 1e-9
    assert all(r["fail"] == 0 for r in res)


def test_batch_drpa_equals_alone(goldens):
    from uegccd_b200 import Batch, Context

    systems = _systems(goldens)
    b = Batch([_tuple(o) for o in systems])
    rc, e2, res = b.solve(drpa=True, do_mosaic=0)
    g1 = res[1]
    assert g1["niter"] == goldens["G1"]["niter"]
    assert abs(g1["ecorr"] - goldens["G1"]["ec_drpa"]) < 1e-11
    assert abs(g1["ecorr_sosex"] - goldens["G1"]["ec_sosex"]) < 1e-11
    for s, o in enumerate(systems):
        ctx = Context(*_tuple(o))
        e2a, ta, tb, tc = ctx.mp2()
        rca, ra, en, _ = ctx.drpa(ta.copy(), do_mosaic=0)
        assert abs(res[s]["ecorr"] - ra["ecorr"]) < 1e-12


def test_all_amplitudes_and_reused_memory(goldens):
    """The batch-wide download equals the per-solve one, and a batch built on device
    memory that a destroyed batch left in the cache gives bitwise the same solves."""
    from uegccd_b200 import Batch, _capi

    systems = [_tuple(o) for o in _systems(goldens)]
    runs = []
    for rep in range(3):
        b = Batch(systems)
        rc, e2, res = b.solve(max_iter=6)
        allt = b.all_amplitudes()
        for s in range(b.n):
            np.testing.assert_array_equal(allt[s], b.amplitudes(s))
        runs.append(([r["ecorr"] for r in res], [a.copy() for a in allt]))
        b.close()
        if rep == 1:
            _capi.lib().uegccd_trim_cache()
    for e, amps in runs[1:]:
        assert e == runs[0][0]
        for a, c in zip(amps, runs[0][1]):
            np.testing.assert_array_equal(a, c)


def test_ring_cta_tuning_and_pinned_download(goldens):
    """The launch-shape tuner leaves a CTA size from its candidate set in every ring pair
    class, and a page-locked destination receives the same amplitudes as a pageable one."""
    import ctypes as C

    from uegccd_b200 import Batch

    systems = [_tuple(o) for o in _systems(goldens)]
    b = Batch(systems)
    b.solve(max_iter=4)
    th = b.ring_threads()
    assert len(th) == 4 and all(t in (32, 64, 128, 256) for t in th)
    shapes = b.launch_shapes()
    assert shapes["ring_threads"] == th and shapes["stage_threads"] in (64, 128, 256)
    assert shapes["ladder_order"] in ("block", "longest first") and shapes["hh_chunk"] in (32, 64)
    n = b.amplitude_count()
    rt = C.CDLL("libcudart.so.12")
    p = C.c_void_p()
    assert rt.cudaHostAlloc(C.byref(p), C.c_size_t(8 * n), C.c_uint(0)) == 0
    try:
        pinned = np.ctypeslib.as_array((C.c_double * n).from_address(p.value))
        a = [x.copy() for x in b.all_amplitudes(out=pinned)]
        c = b.all_amplitudes()
        for x, y in zip(a, c):
            np.testing.assert_array_equal(x, y)
    finally:
        rt.cudaFreeHost(p)


def test_fp64_peak_probe():
    """The register-only FP64 MMA probe (the bench's FP64 roofline denominator, bench_peak.cu)
    reports a B200-sized figure: its datasheet FP64 tensor peak is about 37-40 TFLOP/s."""
    import bench

    v = bench.probe_fp64_peak()
    assert v is not None and 20.0 < v < 60.0, v


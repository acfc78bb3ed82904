"""The two-channel form (two_channel.cu) against the oracle: per-term range flags
(CCD.f90:620-937, CasedERI HEG.f90:689-774), Do Rings without Do XRings and the reverse
(CCD.f90:174-175), and range-separated dRPA.  In these cases T2abba(i,j,a) = -T2abab(i,j,b)
no longer holds, so the GPU iterates both channels as the reference does.

Tolerances as in test_gpu_parity.py: each term 1e-12 of its largest element, the replay solve
the same iteration count and every printed energy within 1e-11 Ha."""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import Context
from uegccd_b200 import _capi as capi

pytestmark = pytest.mark.gpu

KEYS = ["Rings Range", "XRings Range", "Ladders Range", "Mosaics Range", "DriverDir Range",
        "DriverEx Range", "Energy Range", "LinRings Range", "QuadRings Range", "DRings Range",
        "ExRings Range", "LinLadd Range", "QuadLadd Range", "DLadders Range", "ExLadders Range"]
assert len(KEYS) == len(capi.RANGE_TERMS)

# per-term flags under Safe ERI: direct and exchange integrals of the same term differ
MIXED = dict(ring=1, xring=2, ladder=0, mosaic=2, driver_direct=1, driver_exchange=0, energy=2, lin_rings=0,
             quad_rings=1, direct_rings=0, exchange_rings=2, lin_ladders=1, quad_ladders=0, direct_ladders=2,
             exchange_ladders=0)
NONE_TERMS = dict(ring=3, ladder=1, driver_exchange=3, exchange_rings=1, quad_ladders=2)


def _screening(nel, L):
    """HEGData%ScreeningDistance after change_rs (HEG.f90:510-512)."""
    density = nel / L ** 3.0
    kf = (3.0 * math.pi ** 2.0 * density) ** (1.0 / 3.0)
    return (4.0 / math.pi * kf) ** 0.5


def _setup(flags=None, safe=False, extra=None, twist=(0.1, 0.2, 0.3)):
    v = parse_input_text("")
    if extra:
        v.update(extra)
    for k, name in zip(KEYS, capi.RANGE_TERMS):
        v[k] = str((flags or {}).get(name, 0))
    v["Safe ERI"] = "T" if safe else "F"
    o = Oracle(v)
    o.change_twist(twist)
    sc = o.scalars()
    ctx = Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())
    if flags is not None:
        ctx.set_eri(flags, safe_eri=safe, screening=_screening(2 * o.nocc, sc["L"]))
    return o, ctx


def _two_channel_amplitudes(o, seed=5):
    """MP2 amplitudes with noise on each channel apart, so that the spin relation fails."""
    rng = np.random.default_rng(seed)
    _, ta, tb, tc, _ = o.mp2()
    tb = tb + 1e-3 * rng.standard_normal(tb.shape) * (tb != 0)
    tc = tc + 1e-3 * rng.standard_normal(tc.shape) * (tc != 0)
    return tb, tc


@pytest.mark.parametrize("case", ["plain", "mixed flags", "flags 3", "core+gap flags"])
def test_two_channel_terms_match_oracle(case):
    extra, flags, safe = None, None, False
    if case == "mixed flags":
        flags, safe = MIXED, True
    elif case == "flags 3":
        flags, safe = NONE_TERMS, True
    elif case == "core+gap flags":
        # flags, GapII and CoreN all set: SetPointers picks CasedERI without Safe ERI
        extra = {"CoreFactor": "0.3", "GapII": "0.05", "rSMin": "2.0", "rSMax": "2.0"}
        flags = dict(ring=1, ladder=2, energy=1, exchange_rings=2)
    o, ctx = _setup(flags, safe, extra)
    if case == "core+gap flags":
        ctx.set_integrals(core_n=int(o.nocc * 0.3), gapii=0.05)
        _, ta, tb, tc, _ = o.mp2()
        o.ccd(ta, tb, tc, max_iter=3)          # core pairs stay zero, as the reference keeps them
    else:
        tb, tc = _two_channel_amplitudes(o)
    for mask in (1, 2, 4, 8, 16, 31):
        ga, gb = o.ccd_g2(tb, tc, mask)
        ha, hb = ctx.ccd_g2_2ch(tb, tc, mask)
        scale = max(np.abs(ga).max(), np.abs(gb).max())
        # flag 3 ("none") zeroes whole terms: the rings of "flags 3" vanish
        assert scale > 0 or (case == "flags 3" and mask == 8)
        assert np.abs(ha - ga).max() <= 1e-12 * scale, (case, mask, "abab")
        assert np.abs(hb - gb).max() <= 1e-12 * scale, (case, mask, "abba")
    for mask in (1, 2, 8, 11):
        g = o.drpa_g2(tb, mask)
        h = ctx.drpa_g2(tb, mask)
        assert np.abs(h - g).max() <= 1e-12 * np.abs(g).max(), (case, mask, "dRPA")
        assert np.abs(g).max() > 0 or (case == "flags 3" and mask == 8)


@pytest.mark.parametrize("rings", [(1, 0), (0, 1)])
def test_rings_without_xrings_ccd_matches_oracle(rings):
    """Do Rings T / Do XRings F and the reverse: the replay solve of both channels."""
    ring, xring = rings
    o, ctx = _setup(extra={"Do Rings": "T" if ring else "F", "Do XRings": "T" if xring else "F"})
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, dts = ctx.ccd(ta, tb, tc, do_ring=ring, do_xring=xring)
    _, ta2, tb2, tc2, _ = o.mp2()
    st, en_o, dts_o = o.ccd(ta2, tb2, tc2)
    assert rc == 0 and not r["fail"]
    assert r["niter"] == st.niter
    np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)
    np.testing.assert_allclose(dts, dts_o, atol=1e-11, rtol=0)
    assert abs(r["ecorr"] - st.ecorr) < 1e-11
    assert abs(r["max_res"] - st.max_res) < 1e-11
    for x, y in ((ta, ta2), (tb, tb2), (tc, tc2)):
        assert np.abs(x - y).max() < 1e-10
    # the spin relation T2abba(i,j,a) = -T2abab(i,j,b), a permutation within each pair (i,j),
    # would keep the two channels' norms equal: here it fails
    assert abs(np.linalg.norm(tc2) - np.linalg.norm(tb2)) > 1e-6


@pytest.mark.parametrize("case", ["mixed flags", "flags 3"])
def test_per_term_flags_ccd_matches_oracle(case):
    flags = MIXED if case == "mixed flags" else NONE_TERMS
    o, ctx = _setup(flags, safe=True)
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, _ = ctx.ccd(ta, tb, tc)
    _, ta2, tb2, tc2, _ = o.mp2()
    st, en_o, _ = o.ccd(ta2, tb2, tc2)
    assert rc == 0 and not r["fail"]
    assert r["niter"] == st.niter
    np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)
    assert abs(r["ecorr"] - st.ecorr) < 1e-11
    assert np.abs(tb - tb2).max() < 1e-10 and np.abs(tc - tc2).max() < 1e-10
    # the flags change the answer: the plain CCD differs
    plain = Oracle(parse_input_text(""))
    plain.change_twist((0.1, 0.2, 0.3))
    _, pa, pb, pc, _ = plain.mp2()
    st_p, _, _ = plain.ccd(pa, pb, pc)
    assert abs(st_p.ecorr - st.ecorr) > 1e-6


def test_range_separated_drpa_matches_oracle():
    """dRPA with per-term flags: the terms take their flags, the energy flag 0
    (dRPA.f90:206-207, 363-529)."""
    flags = dict(ring=1, mosaic=2, driver_direct=1, quad_rings=2, direct_rings=0)
    o, ctx = _setup(flags, safe=True, extra={"Do Mosaics": "T"})
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, _ = ctx.drpa(ta.copy(), do_mosaic=1)
    _, ta2, _, _, _ = o.mp2()
    st, en_o, _ = o.drpa(ta2.copy())
    assert r["niter"] == st.niter
    np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)
    assert abs(r["ecorr"] - st.ecorr) < 1e-11
    assert abs(r["ecorr_sosex"] - st.ecorr_sosex) < 1e-11
    assert r["fail"] == st.fail


def test_two_channel_diis_reaches_the_replay_answer():
    """The Pulay scheme on both channels (one set of coefficients) converges to the energy of
    the replay iteration, in fewer iterations."""
    o, ctx = _setup(extra={"Do XRings": "F"})
    _, ta, tb, tc = ctx.mp2()
    args = [x.copy() for x in (ta, tb, tc)]
    rc, r_rep, _, _ = ctx.ccd(*args, do_ring=1, do_xring=0, tol=1e-10)
    args = [x.copy() for x in (ta, tb, tc)]
    rc2, r_diis, _, _ = ctx.ccd(*args, do_ring=1, do_xring=0, tol=1e-10, scheme=1, ndiis=6)
    assert rc == 0 and rc2 == 0
    assert r_diis["ndiis"] == 6
    assert r_diis["niter"] < r_rep["niter"]
    assert abs(r_diis["ecorr"] - r_rep["ecorr"]) < 1e-9
    # again on the same context: the history left by the first solve changes nothing
    args = [x.copy() for x in (ta, tb, tc)]
    rc3, r_again, _, _ = ctx.ccd(*args, do_ring=1, do_xring=0, tol=1e-10, scheme=1, ndiis=6)
    assert rc3 == 0 and r_again["niter"] == r_diis["niter"] and r_again["ecorr"] == r_diis["ecorr"]


def test_two_channel_refusals():
    o, ctx = _setup()
    _, ta, tb, tc = ctx.mp2()
    with pytest.raises(capi.UegccdError):      # FP64 only
        ctx.ccd(ta, tb, tc, do_ring=1, do_xring=0, precision=1)
    with pytest.raises(capi.UegccdError):      # flags outside 0..3
        ctx.set_eri({"ring": 4}, safe_eri=True, screening=1.0)
    with pytest.raises(capi.UegccdError):      # a screened flag needs the screening distance
        ctx.set_eri({"ring": 1}, safe_eri=True, screening=0.0)
    # clearing the selection returns to the spin-adapted kernels
    ctx.set_eri({"ring": 1}, safe_eri=True, screening=1.0)
    ctx.set_eri(None)
    rc, r, _, _ = ctx.ccd(ta, tb, tc)
    _, ta2, tb2, tc2, _ = o.mp2()
    st, _, _ = o.ccd(ta2, tb2, tc2)
    assert rc == 0 and abs(r["ecorr"] - st.ecorr) < 1e-11


def test_two_channel_n54_iterations_match_oracle():
    """N=54, 485 plane waves (the GPU-vs-reference configuration), rs=1, per-term flags under
    Safe ERI: three two-channel iterations on the GPU and in the oracle agree term for term."""
    flags = dict(ring=1, exchange_rings=2, ladder=1, driver_exchange=3, energy=2)
    o, ctx = _setup(flags, safe=True, extra={"# Electrons": "54", "Momentum Cutoff": "24"}, twist=(0.0, 0.0, 0.0))
    assert (o.nocc, o.nao) == (27, 485)
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, dts = ctx.ccd(ta, tb, tc, max_iter=4)
    _, ta2, tb2, tc2, _ = o.mp2()
    st, en_o, dts_o = o.ccd(ta2, tb2, tc2, max_iter=4)
    assert r["niter"] == st.niter == 4
    np.testing.assert_allclose(en, en_o, atol=1e-12, rtol=0)
    np.testing.assert_allclose(dts, dts_o, atol=1e-13, rtol=0)
    assert np.abs(tb - tb2).max() < 1e-13 and np.abs(tc - tc2).max() < 1e-13
    print(f"two-channel N=54: {r['gpu_ms'] / 4:.3f} ms per iteration (4 residuals + start), "
          f"{r['kernel_launches']} launches")


def test_batch_two_channel_matches_oracle():
    """A batch CCD solve with Do XRings F runs each system in the two-channel form: the
    oracle's iteration count and energies per twist, T2abab back from the batch, each solve's
    iteration table; the structure factor (spin-adapted amplitudes only) is refused."""
    from uegccd_b200 import Batch

    systems, refs = [], []
    for tw in ((0.1, 0.2, 0.3), (-0.2, 0.05, 0.4)):
        o, _ = _setup(extra={"Do XRings": "F"}, twist=tw)
        sc = o.scalars()
        systems.append((o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec()))
        _, ta2, tb2, tc2, _ = o.mp2()
        st, en_o, _ = o.ccd(ta2, tb2, tc2)
        refs.append((st, en_o, tb2))
    b = Batch(systems)
    rc, e2, res = b.solve(do_ring=1, do_xring=0)
    assert rc == 0
    for s, (st, en_o, tb2) in enumerate(refs):
        assert res[s]["niter"] == st.niter
        assert abs(res[s]["ecorr"] - st.ecorr) < 1e-11
        en, _ = b.history(s)
        np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)
        assert np.abs(b.amplitudes(s) - tb2).max() < 1e-10
    with pytest.raises(capi.UegccdError):
        b.structure_factor(0)
    # an incremental solve stays spin-adapted: refused
    with pytest.raises(capi.UegccdError):
        b.start(do_ring=1, do_xring=0)


def test_batch_two_channel_with_a_uniform_range_flag():
    """A batch solve with Do XRings F on the batch's uniform range flag (uegccd_batch_set_range,
    every term on flag 1 under Safe ERI) in the two-channel form, against the oracle."""
    from uegccd_b200 import Batch

    flags = {name: 1 for name in capi.RANGE_TERMS}
    o, _ = _setup(flags, safe=True, extra={"Do XRings": "F"})
    sc = o.scalars()
    b = Batch([(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())])
    b.set_range(1, _screening(2 * o.nocc, sc["L"]))
    rc, e2, res = b.solve(do_ring=1, do_xring=0, range_flags=len(KEYS))
    _, ta2, tb2, tc2, _ = o.mp2()
    st, en_o, _ = o.ccd(ta2, tb2, tc2)
    assert rc == 0
    assert res[0]["niter"] == st.niter
    assert abs(res[0]["ecorr"] - st.ecorr) < 1e-11
    en, _ = b.history(0)
    np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)


def test_two_channel_solve_with_core_and_gap():
    """Do XRings F with CoreN and GapII (NoCaseERI, HEG.f90:776-833): the replay solve of both
    channels against the oracle; the core pairs stay zero in both channels."""
    o, ctx = _setup(extra={"Do XRings": "F", "CoreFactor": "0.3", "GapII": "0.05"})
    core = int(o.nocc * 0.3)
    ctx.set_integrals(core_n=core, gapii=0.05)
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, _ = ctx.ccd(ta, tb, tc, do_ring=1, do_xring=0, core_n=core, gapii=0.05)
    _, ta2, tb2, tc2, _ = o.mp2()
    st, en_o, _ = o.ccd(ta2, tb2, tc2)
    assert rc == 0 and r["niter"] == st.niter
    np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)
    assert np.abs(tb - tb2).max() < 1e-10 and np.abs(tc - tc2).max() < 1e-10
    assert np.all(tb[:, :core, :] == 0) and np.all(tc[:, :, :core] == 0)


def test_general_drpa_diis_reaches_the_replay_answer():
    """dRPA with per-term flags under the Pulay scheme converges to the replay energy."""
    flags = dict(ring=1, driver_direct=1)
    o, ctx = _setup(flags, safe=True)
    _, ta, _, _ = ctx.mp2()
    rc, r_rep, _, _ = ctx.drpa(ta.copy(), tol=1e-10)
    rc2, r_diis, _, _ = ctx.drpa(ta.copy(), tol=1e-10, scheme=1, ndiis=6)
    assert rc == 0 and rc2 == 0 and r_diis["ndiis"] == 6
    assert r_diis["niter"] <= r_rep["niter"]
    assert abs(r_diis["ecorr"] - r_rep["ecorr"]) < 1e-9
    assert abs(r_diis["ecorr_sosex"] - r_rep["ecorr_sosex"]) < 1e-9

"""The CAS-core and gap integral options on the GPU against the oracle: CoreN
(CoreERI, HEG.f90:835-888), GapII (GapERI, HEG.f90:890-942), both (NoCaseERI,
HEG.f90:776-833) and both under 'Safe ERI' (CasedERI, HEG.f90:689-774), as
SetPointers (Main.f90:274-318) selects them.

The oracle evaluates the masked integrals inside every loop, as the reference does;
the GPU filters the |q|^2 table (GapII) and holds the core pairs at zero (CoreN).
Tolerances as in test_gpu_parity.py: terms 1e-12 of the largest term, energies on
the same iteration count 1e-11 Ha.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import Batch, Context

pytestmark = pytest.mark.gpu

CASES = {   # CoreFactor, GapII, Safe ERI -- for N=14 (7 occupied) CoreFactor 0.3 gives CoreN = 2
    "core": ("0.3", "-0.01", "F"),
    "gap": ("0.0", "0.05", "F"),
    "core+gap": ("0.3", "0.05", "F"),
    "core+gap safe": ("0.3", "0.05", "T"),
}


def _oracle(case, **over):
    cf, gap, safe = CASES[case]
    v = parse_input_text("")
    v.update({"CoreFactor": cf, "GapII": gap, "Safe ERI": safe})
    v.update(over)
    return Oracle(v)


def _opts(o, case):
    """CoreN = NElectron/2 * CoreFactor, truncated (as the reference sets it), and GapII."""
    cf, gap, _ = CASES[case]
    return dict(core_n=int(o.nocc * float(cf)), gapii=float(gap))


def _ctx(o, case):
    sc = o.scalars()
    ctx = Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())
    ctx.set_integrals(**_opts(o, case))
    return ctx


@pytest.mark.parametrize("case", list(CASES))
def test_mp2_matches_oracle(case):
    o = _oracle(case)
    e_ref, ta, tb, tc, _ = o.mp2()
    e2, ga, gb, gc = _ctx(o, case).mp2()
    assert abs(e2 - e_ref) < 1e-13
    for x, y in ((ga, ta), (gb, tb), (gc, tc)):
        assert np.abs(x - y).max() < 1e-15
    core = _opts(o, case)["core_n"]
    if core:
        assert np.all(gb[:, :core, :] == 0) and np.all(gb[:, :, :core] == 0)


@pytest.mark.parametrize("mask", [1, 2, 4, 24, 31])
@pytest.mark.parametrize("case", ["core+gap", "core+gap safe"])
def test_residual_terms_match_oracle(case, mask):
    """G2 of the MP2 amplitudes after two CCD iterations (core pairs zero, as every
    amplitude the reference produces under CoreN)."""
    o = _oracle(case, **{"rSMin": "2.0", "rSMax": "2.0"})
    _, ta, tb, tc, _ = o.mp2()
    o.ccd(ta, tb, tc, max_iter=3)
    ga, _ = o.ccd_g2(tb, tc, mask)
    g = _ctx(o, case).ccd_g2(tb, mask)
    scale = np.abs(ga).max()
    assert scale > 0
    assert np.abs(g - ga).max() <= 1e-12 * scale, (mask, np.abs(g - ga).max(), scale)


@pytest.mark.parametrize("case", list(CASES))
def test_ccd_replay_matches_oracle(case):
    o = _oracle(case)
    ctx = _ctx(o, case)
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, dts = ctx.ccd(ta, tb, tc, **_opts(o, case))
    assert rc == 0 and not r["fail"]
    _, ta2, tb2, tc2, _ = o.mp2()
    st, en_o, dts_o = o.ccd(ta2, tb2, tc2)
    assert r["niter"] == st.niter
    np.testing.assert_allclose(en, en_o, atol=1e-11, rtol=0)
    assert abs(r["ecorr"] - st.ecorr) < 1e-11
    assert np.abs(tb - tb2).max() < 1e-10


@pytest.mark.parametrize("case", ["core", "core+gap"])
def test_drpa_matches_oracle(case):
    o = _oracle(case, **{"DodRPASOSEX": "T"})
    ctx = _ctx(o, case)
    _, ta, tb, tc = ctx.mp2()
    rc, r, en, _ = ctx.drpa(ta.copy(), **_opts(o, case))
    _, ta2, _, _, _ = o.mp2()
    st, en_o, _ = o.drpa(ta2.copy())
    assert r["niter"] == st.niter
    np.testing.assert_allclose(en, en_o, atol=1e-12, rtol=0)
    assert abs(r["ecorr_sosex"] - st.ecorr_sosex) < 1e-12


@pytest.mark.parametrize("case", ["core", "core+gap"])
def test_structure_factor_matches_oracle(case):
    """SfV keeps the integral of the last contribution in the reference's loop order:
    0 where that is a core pair."""
    o = _oracle(case)
    _, ta, tb, tc, _ = o.mp2()
    ref = o.structure_factor(ta, tb, tc)
    ctx = _ctx(o, case)
    _, _, tb_g, _ = ctx.mp2()
    ours = ctx.structure_factor(tb_g)
    np.testing.assert_array_equal(ours["g"], ref["g"])
    np.testing.assert_array_equal(ours["v"], ref["v"])
    assert np.any((ref["g"] > 0) & (ref["v"] == 0))   # core pairs do decide some points
    scale = np.abs(ref["sum"]).max()
    for k in ("sum", "dsum", "xsum"):
        assert np.abs(ours[k] - ref[k]).max() <= 1e-13 * scale


def test_batch_solve_with_integral_options():
    """A batch of two twists under CoreN and GapII (Pulay DIIS, tight) against the
    contexts of the same systems, and the options reset to the plain integrals."""
    systems, oracles = [], []
    for tw in ((0.1, 0.2, 0.3), (-0.25, 0.05, 0.4)):
        o = _oracle("core+gap")
        o.change_twist(tw)
        sc = o.scalars()
        systems.append((o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec()))
        oracles.append(o)
    opts = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-11, **_opts(oracles[0], "core+gap"))
    b = Batch(systems)
    rc, e2, res = b.solve(**opts)
    assert rc == 0
    for s, o in enumerate(oracles):
        e_ref, ta, tb, tc, _ = o.mp2()
        assert abs(e2[s] - e_ref) < 1e-13
        ctx = _ctx(o, "core+gap")
        _, ta, tb, tc = ctx.mp2()
        rc1, r1, _, _ = ctx.ccd(ta, tb, tc, **opts)
        assert rc1 == 0 and abs(res[s]["ecorr"] - r1["ecorr"]) < 1e-11
    # back to the plain integrals: the same batch gives the default MP2 energies
    b.set_integrals(0, 0.0)
    e_plain = b.mp2()
    for s, o in enumerate(oracles):
        v = parse_input_text("")
        p = Oracle(v)
        p.change_twist((0.1, 0.2, 0.3) if s == 0 else (-0.25, 0.05, 0.4))
        assert abs(e_plain[s] - p.mp2()[0]) < 1e-13

"""Range-separated integrals with one flag for every CCD term (CasedERI, HEG.f90:689-774),
the case in which direct and exchange integrals share the flag and the spin adaptation
holds: the GPU against the oracle's CasedERI, with all fifteen "... Range" Input values set
to the flag under Safe ERI.  The MP2 start keeps the plain integrals (MP2.f90:61-62); every
CCD term and the energy take the flag.  Replay iteration: the same iteration count, every
printed energy within 1e-11 Ha."""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import Context

pytestmark = pytest.mark.gpu

RANGE_KEYS = ["Rings Range", "XRings Range", "Ladders Range", "Mosaics Range", "DriverDir Range",
              "DriverEx Range", "Energy Range", "LinRings Range", "QuadRings Range", "DRings Range",
              "ExRings Range", "LinLadd Range", "QuadLadd Range", "DLadders Range", "ExLadders Range"]


def _screening(nel, L):
    """HEGData%ScreeningDistance after change_rs (HEG.f90:510-512)."""
    density = nel / L ** 3.0
    kf = (3.0 * math.pi ** 2.0 * density) ** (1.0 / 3.0)
    return (4.0 / math.pi * kf) ** 0.5


@pytest.mark.parametrize("flag", [1, 2])
def test_uniform_range_flag_ccd_matches_oracle(flag):
    v = parse_input_text("")
    v.update({k: str(flag) for k in RANGE_KEYS})
    v["Safe ERI"] = "T"
    o = Oracle(v)
    o.change_twist((0.1, 0.2, 0.3))
    sc = o.scalars()
    ctx = Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())
    e2, ta, tb, tc = ctx.mp2()
    e2_ref, ta2, tb2, tc2, _ = o.mp2()
    assert abs(e2 - e2_ref) < 1e-13          # MP2 on the plain integrals
    ctx.set_range(flag, _screening(2 * o.nocc, sc["L"]))
    rc, r, en, _ = ctx.ccd(ta, tb, tc, range_flags=flag * len(RANGE_KEYS))
    assert rc == 0 and not r["fail"]
    st, en_o, _ = o.ccd(ta2, tb2, tc2)
    assert r["niter"] == st.niter
    np.testing.assert_allclose(en[: r["niter"]], en_o[: st.niter], atol=1e-11, rtol=0)
    assert abs(r["ecorr"] - st.ecorr) < 1e-11
    assert np.abs(tb - tb2).max() < 1e-10
    # the flag really changes the answer, and clearing it gives the plain CCD back
    plain = Oracle(parse_input_text(""))
    plain.change_twist((0.1, 0.2, 0.3))
    _, pa, pb, pc, _ = plain.mp2()
    st_p, _, _ = plain.ccd(pa, pb, pc)
    assert abs(st_p.ecorr - st.ecorr) > 1e-6
    ctx.set_range(0)
    _, ta, tb, tc = ctx.mp2()
    rc, r0, _, _ = ctx.ccd(ta, tb, tc)
    assert rc == 0 and abs(r0["ecorr"] - st_p.ecorr) < 1e-11


def test_range_flags_need_a_uniform_flag():
    """range_flags without a flag set (terms with different flags), or for dRPA: refused."""
    o = Oracle(parse_input_text(""))
    sc = o.scalars()
    ctx = Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())
    _, ta, tb, tc = ctx.mp2()
    with pytest.raises(Exception):
        ctx.ccd(ta, tb, tc, range_flags=3)
    ctx.set_range(1, 1.0)
    with pytest.raises(Exception):
        ctx.drpa(ta.copy(), range_flags=15)

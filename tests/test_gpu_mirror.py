"""The kernels form G on the amplitudes i <= j and write each value to its mirror (j,i,b),
so the GPU's amplitudes and G keep the pair symmetry t(ij,a) = t(ji,b) exactly (bitwise) for
i != j, where the reference's two halves agree to rounding.  On a diagonal pair (i,i) both
t(ii,a) and t(ii,b) are formed, each on its own: they agree to rounding."""
import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import Context

pytestmark = pytest.mark.gpu


def _pairs(o):
    O, M = o.nocc, o.nao
    nv = o.nvec()
    idx = {tuple(nv[p]): p for p in range(M)}
    out = []
    for i in range(O):
        for j in range(O):
            for a in range(O, M):
                b = idx.get(tuple(nv[i] + nv[j] - nv[a]), -1)
                if b >= O:
                    out.append((i, j, a, b))
    return out


def _ctx(o):
    sc = o.scalars()
    return Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())


@pytest.mark.parametrize("twist", [(0.0, 0.0, 0.0), (0.1, 0.2, 0.3)])
def test_ccd_amplitudes_and_terms_are_mirror_exact(twist):
    o = Oracle(parse_input_text(""))
    o.change_twist(twist)
    O = o.nocc
    ctx = _ctx(o)
    _, ta, tb, tc = ctx.mp2()
    rc, r, _, _ = ctx.ccd(ta, tb, tc, scheme=1, ndiis=6, denom_factor=1.0, tol=1e-11)
    assert rc == 0 and not r["fail"]
    pairs = _pairs(o)
    assert len(pairs) > 0
    scale = np.abs(tb).max()
    for i, j, a, b in pairs:
        if i != j:
            assert tb[a - O, j, i] == tb[b - O, i, j]
        else:
            assert abs(tb[a - O, j, i] - tb[b - O, i, j]) <= 1e-14 * scale
    g = ctx.ccd_g2(tb, 31)
    gscale = np.abs(g).max()
    for i, j, a, b in pairs:
        if i != j:
            assert g[a - O, j, i] == g[b - O, i, j]
        else:
            assert abs(g[a - O, j, i] - g[b - O, i, j]) <= 1e-14 * gscale
    # and the result is the reference's fixed point
    _, ta2, tb2, tc2, _ = o.mp2()
    st, _, _ = o.ccd(ta2, tb2, tc2, tol=1e-11)
    assert abs(r["ecorr"] - st.ecorr) < 1e-10

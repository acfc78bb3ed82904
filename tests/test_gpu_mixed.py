"""Mixed precision: the particle-particle ladder on the 5th-generation tensor cores
(tcgen05, FP16 operands, FP32 accumulation in tensor memory).

1. Term level: the tensor-core ladder of t against the FP64 ladder, on the
   reference's N=24 system and on N=54 with 485 plane waves.  Tolerance 4e-3 of
   the largest ladder element (FP16 rounding of both operands, sums of a few hundred
   terms in FP32).
2. Solve level: the defect-correction iteration (tensor cores on t - t_ref, FP64
   refresh of t_ref every few iterations, FP64 sweeps at the end) converges to the
   FP64 fixed point: energies agree to 1e-9 Ha, far inside 1 microHartree per electron.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text

pytestmark = pytest.mark.gpu


def _ctx(o):
    from uegccd_b200 import Context

    sc = o.scalars()
    return Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())


@pytest.mark.parametrize("which", ["G5", "N54"])
def test_tensor_core_ladder_term(goldens, which):
    vals = parse_input_text("")
    if which == "G5":
        vals.update(goldens["G5"]["keys"])
    else:
        vals.update({"# Electrons": "54", "Momentum Cutoff": "24", "NTwist": "0.2 -0.1 0.3"})
    o = Oracle(vals)
    ctx = _ctx(o)
    e2, ta, tb, tc = ctx.mp2()
    g64 = ctx.ccd_g2(tb, mask=4, precision=0)
    g16 = ctx.ccd_g2(tb, mask=4, precision=1)
    scale = np.abs(g64).max()
    err = np.abs(g16 - g64).max()
    assert scale > 0
    assert err < 4e-3 * scale, (err, scale)
    assert err > 0.0  # it really ran in reduced precision


def test_mixed_solve_matches_fp64(goldens):
    vals = parse_input_text("")
    vals.update(goldens["G5"]["keys"])
    o = Oracle(vals)
    ctx = _ctx(o)
    e2, ta, tb, tc = ctx.mp2()
    diis = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-10)
    rc1, r64, _, _ = ctx.ccd(ta.copy(), tb.copy(), tc.copy(), **diis)
    rc2, r16, _, _ = ctx.ccd(ta.copy(), tb.copy(), tc.copy(), precision=1, **diis)
    assert rc1 == 0 and rc2 == 0
    assert abs(r64["ecorr"] - r16["ecorr"]) < 1e-9, (r64["ecorr"], r16["ecorr"])


def test_mixed_batch_twists_match_fp64():
    from uegccd_b200 import Batch, heg

    inp = heg.default_input(nelectron=54, maxkpoint=30, rsmin=1.0, rsmax=1.0, fcut=6.857)
    h = heg.Heg(inp)
    rng = np.random.default_rng(5)
    systems = []
    for tw in rng.random((6, 3)) - 0.5:
        h.change_twist(tw)
        systems.append(h.system())
    b = Batch(systems)
    diis = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-9)
    rc1, _, r64 = b.solve(**diis)
    rc2, _, r16 = b.solve(precision=1, **diis)
    for a, c in zip(r64, r16):
        assert abs(a["ecorr"] - c["ecorr"]) < 54 * 1e-6  # 1 microHartree per electron
        assert abs(a["ecorr"] - c["ecorr"]) < 1e-8

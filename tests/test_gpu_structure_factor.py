"""Structure factors on the GPU (k_sf) against the oracle's restatement of
CCEnergyAndSF and DrvMBPT (CCD.f90:240-351, MP2.f90:86-117), and the fort.80,
fort.81 and fort.82 files of the ZCode drop-in.

Tolerances: the support of the grid (the transfers q that an allowed amplitude
reaches) is compared exactly, SfG and SfV bit for bit (host expressions of q
alone), the three sums within 1e-13 of the largest |SfSum| (the device sums each
grid point in a fixed tree order, the oracle in the reference's loop order).
"""
import re

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import Batch, Context, zcode

pytestmark = pytest.mark.gpu

FLOAT = re.compile(r"-?\d+\.\d+(?:E[+-]\d+)?")


def _tuple(o):
    sc = o.scalars()
    return (o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())


def _check(ours, ref):
    assert ours["S"] == ref["S"]
    np.testing.assert_array_equal(ours["g"] > 0, ref["g"] > 0)
    np.testing.assert_array_equal(ours["g"], ref["g"])
    np.testing.assert_array_equal(ours["v"], ref["v"])
    scale = np.abs(ref["sum"]).max()
    assert scale > 0
    for k in ("sum", "dsum", "xsum"):
        assert np.abs(ours[k] - ref[k]).max() <= 1e-13 * scale, k


def _g5_vals(goldens):
    v = parse_input_text("")
    v.update(goldens["G5"]["keys"])
    return v


@pytest.mark.parametrize("case", ["n14", "g5"])
def test_mp2_structure_factor_matches_oracle(goldens, case):
    o = Oracle(parse_input_text("") if case == "n14" else _g5_vals(goldens))
    e2, ta, tb, tc, _ = o.mp2()
    ref = o.structure_factor(ta, tb, tc)
    ctx = Context(*_tuple(o))
    _, _, tb_g, _ = ctx.mp2()
    ours = ctx.structure_factor(tb_g)
    _check(ours, ref)
    assert 0.5 * float((ours["sum"] * ours["v"]).sum()) == pytest.approx(e2, rel=1e-12)


def test_ccd_structure_factor_matches_oracle():
    """Converged CCD amplitudes (N=14, rs=1, Pulay DIIS to 1e-12) through the context."""
    o = Oracle(parse_input_text(""))
    _, ta, tb, tc, _ = o.mp2()
    ctx = Context(*_tuple(o))
    rc, r, _, _ = ctx.ccd(ta, tb, tc, scheme=1, ndiis=6, denom_factor=1.0, tol=1e-12)
    assert rc == 0
    ref = o.structure_factor(ta, tb, tc)   # the same (converged) arrays
    ours = ctx.structure_factor(tb)
    _check(ours, ref)
    assert 0.5 * float((ours["sum"] * ours["v"]).sum()) == pytest.approx(r["ecorr"], rel=1e-12)


def test_batch_mp2_structure_factors_n54(goldens):
    """Four twists of N=54 (485 plane waves) in one batch: uegccd_batch_mp2, then the
    structure factor of every solve against the oracle's MP2 of that twist."""
    vals = parse_input_text("")
    vals.update({"# Electrons": "54", "Momentum Cutoff": "24"})
    twists = [(0.0, 0.0, 0.0), (0.1, 0.2, 0.45), (-0.3, 0.25, 0.05), (0.45, -0.45, 0.2)]
    oracles, systems = [], []
    for tw in twists:
        o = Oracle(vals)
        o.change_twist(tw)
        oracles.append(o)
        systems.append(_tuple(o))
    assert oracles[0].nao == 485
    b = Batch(systems)
    e2 = b.mp2()
    for s, o in enumerate(oracles):
        e_ref, ta, tb, tc, _ = o.mp2()
        assert e2[s] == pytest.approx(e_ref, rel=1e-12)
        ours = b.structure_factor(s)
        _check(ours, o.structure_factor(ta, tb, tc))
        assert 0.5 * float((ours["sum"] * ours["v"]).sum()) == pytest.approx(e2[s], rel=1e-12)


def _blocks(lines):
    out, cur = [], None
    for k, l in enumerate(lines):
        if l == " Starting a new structure factor":
            cur = []
            out.append(cur)
        elif cur is not None and l != " --------":
            cur.append(l)
    return out


def _block_energy(block, ncol):
    rows = [l.split() for l in block]
    assert rows and all(len(r) == ncol for r in rows)
    s = np.array([float(r[4]) for r in rows])
    v = np.array([float(r[5]) for r in rows])
    return 0.5 * float((s * v).sum())


def _cc_tables(out_lines):
    """(first, last) energies of every CCD iteration table in Output."""
    tabs, cur = [], None
    for l in out_lines:
        if "CCD summary follows" in l:
            cur = []
            tabs.append(cur)
        elif cur is not None and re.match(r"\s+\*\s+-?\d+\.\d+\s+\d+\s+\d+\.\d+\s+\*", l):
            cur.append(float(l.split()[1]))
    return [(t[0], t[-1]) for t in tabs]


def test_zcode_writes_structure_factor_files(goldens, tmp_path, monkeypatch):
    """The TA program of benchmarks/ZRun-v6-N14 on 4 twists with DoSFCalcMP2/CCD set:
    fort.81 has one block per DrvMBPT, fort.80 two per DrvCCD (start and converged
    amplitudes, twist by twist), fort.82 one per print_HF; every block's
    1/2 sum SfSum*SfV equals the energy Output prints for the same amplitudes."""
    g = goldens["G3"]
    text = g["input_text"].replace("TACalcN:          100", "TACalcN:          4")
    text = text.replace("EndInput:", "DoSFCalcMP2:      T\nDoSFCalcCCD:      T\nEndInput:")
    (tmp_path / "Input").write_text(text)
    with open(tmp_path / "Twists", "w") as f:
        for t in g["twists"][:4]:
            f.write("%.17g %.17g %.17g\n" % tuple(t))
    monkeypatch.chdir(tmp_path)
    zcode.run("Input", "Twists")
    out = (tmp_path / "Output").read_text().splitlines()
    e2 = [float(FLOAT.findall(l)[0]) for l in out if "* E(2) is" in l]
    b81 = _blocks((tmp_path / "fort.81").read_text().splitlines())
    b80 = _blocks((tmp_path / "fort.80").read_text().splitlines())
    assert len(e2) == len(b81) == 4 + 1
    for blk, e in zip(b81, e2):
        assert _block_energy(blk, 6) == pytest.approx(e, abs=2e-12)
    tabs = _cc_tables(out)
    assert len(tabs) == 4 + 1 and len(b80) == 2 * len(tabs)
    for k, (first, last) in enumerate(tabs):
        assert _block_energy(b80[2 * k], 8) == pytest.approx(first, abs=2e-10)
        assert _block_energy(b80[2 * k + 1], 8) == pytest.approx(last, abs=2e-10)
    # fort.81's MP2 block of twist 1 against the oracle's grid
    o = Oracle(parse_input_text(text))
    o.change_twist(g["twists"][0])
    _, ta, tb, tc, _ = o.mp2()
    ref = o.structure_factor(ta, tb, tc)
    S = ref["S"]
    rows = [l.split() for l in b81[0]]
    got = {tuple(int(x) for x in r[:3]): [float(x) for x in r[3:]] for r in rows}
    want = {(x, y, z): (ref["g"][z + S, y + S, x + S], ref["sum"][z + S, y + S, x + S], ref["v"][z + S, y + S, x + S])
            for x in range(-S, S + 1) for y in range(-S, S + 1) for z in range(-S, S + 1)
            if ref["g"][z + S, y + S, x + S] > 0}
    assert list(got) == list(want)   # same points in the reference's order (x outermost)
    scale = np.abs(ref["sum"]).max()
    for q, (gv, sv, vv) in want.items():
        assert got[q][0] == float(zcode.list_real(gv)) and got[q][2] == float(zcode.list_real(vv))
        assert abs(got[q][1] - sv) <= 1e-13 * scale
    f60 = (tmp_path / "fort.60").read_text()
    assert len(_blocks((tmp_path / "fort.82").read_text().splitlines())) == f60.count(" HF energy:")

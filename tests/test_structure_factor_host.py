"""Structure factors on the host side (no GPU): the oracle's restatement of
CCEnergyAndSF / DrvMBPT (CCD.f90:240-351, MP2.f90:86-117) and of print_ex_SF
(HEG.f90:617-674), and the library's exchange structure factor and fort.82 file.

The reference holds no fort.80/81/82 files, so the structure factors are pinned
through identities with numbers that are pinned to its files:
  * 1/2 sum_q SfSum(q) SfV(q) is the correlation energy of the amplitudes
    (the MP2 energy, pinned to source/Test/Output through the oracle);
  * sum_q ExSf(q) = O(O-1) and -sum_q ExSf(q) ExV(q) = XHF, whose
    'Exchange energy:' line in fort.60 equals the reference's file.
"""
import re

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import heg, zcode


def _g5_vals(goldens):
    v = parse_input_text("")
    v.update(goldens["G5"]["keys"])
    return v


def _g5_files(goldens, tmp_path):
    g = goldens["G5"]
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in g["keys"].items()))
    (tmp_path / "Twists").write_text("".join("%.17g %.17g %.17g\n" % tuple(t) for t in g["ta_twists"]))


def test_oracle_sf_sums_give_the_mp2_energy(goldens):
    o = Oracle(_g5_vals(goldens))
    e2, ta, tb, tc, _ = o.mp2()
    sf = o.structure_factor(ta, tb, tc)
    assert sf["oob"] == 0
    assert sf["ecorr"] == pytest.approx(e2, rel=1e-14)
    assert 0.5 * float((sf["sum"] * sf["v"]).sum()) == pytest.approx(e2, rel=1e-13)
    # SfSum = SfDSum + SfXSum term by term (T2aaaa+T2abab = (T2aaaa-T2abab) + 2 T2abab)
    np.testing.assert_allclose(sf["sum"], sf["dsum"] + sf["xsum"], rtol=0, atol=1e-15)
    # SfG = |q| 2 pi / L wherever an amplitude reaches q, and nowhere else
    S = sf["S"]
    z, y, x = np.meshgrid(*(np.arange(-S, S + 1),) * 3, indexing="ij")
    q = np.sqrt(x * x + y * y + z * z) * 2 * np.pi / o.scalars()["L"]
    seen = sf["g"] > 0
    assert seen.sum() > 0 and not seen[S, S, S]
    np.testing.assert_allclose(sf["g"][seen], q[seen], rtol=1e-15)
    assert np.all(sf["v"][~seen] == 0) and np.all(sf["sum"][~seen] == 0)


def test_oracle_sf_of_ccd_amplitudes():
    o = Oracle(parse_input_text(""))  # N=14, 19 plane waves, rs=1
    _, ta, tb, tc, _ = o.mp2()
    st, _, _ = o.ccd(ta, tb, tc, tol=1e-12)
    sf = o.structure_factor(ta, tb, tc)
    assert sf["ecorr"] == pytest.approx(st.ecorr, rel=1e-13)
    assert 0.5 * float((sf["sum"] * sf["v"]).sum()) == pytest.approx(st.ecorr, rel=1e-12)


def test_exchange_sf_matches_oracle(goldens, tmp_path):
    """Library print_ex_SF against the oracle, bit for bit, at the Input twist and another."""
    _g5_files(goldens, tmp_path)
    o = Oracle(_g5_vals(goldens))
    h = heg.Heg(heg.read_input(str(tmp_path / "Input"), require_all=False))
    for tw in (None, goldens["G5"]["ta_twists"][3]):
        if tw is not None:
            o.change_twist(tw)
            h.change_twist(tw)
        a, b = o.exchange_sf(), h.exchange_sf()
        assert a["maxq"] == b["maxq"]
        np.testing.assert_array_equal(a["n"], b["n"])
        np.testing.assert_array_equal(a["v"], b["v"])
        assert int(b["n"].sum()) == o.nocc * (o.nocc - 1)


def _blocks(lines):
    out, cur = [], None
    for k, l in enumerate(lines):
        if l == " Starting a new structure factor":
            assert lines[k - 1] == " --------" and lines[k + 1] == " --------"
            cur = []
            out.append(cur)
        elif cur is not None and l != " --------":
            cur.append(l)
    return out


def test_fort82_blocks(goldens, tmp_path, monkeypatch):
    """fort.82 of the set-up: one block per print_HF (each 'HF energy:' line of fort.60),
    the rSMin one equal to the oracle's grid in list-directed form, every block summing to
    the exchange energy that fort.60 prints beside it."""
    _g5_files(goldens, tmp_path)
    monkeypatch.chdir(tmp_path)
    zcode.host_logs("Input", "Twists", "fort.60", "fort.82")
    f60 = (tmp_path / "fort.60").read_text().splitlines()
    f82 = (tmp_path / "fort.82").read_text().splitlines()
    blocks = _blocks(f82)
    ex = [float(l.split()[-1]) for l in f60 if l.startswith(" Exchange energy:")]
    mad = [float(l.split()[-1]) for l in f60 if l.startswith(" Madelung:")]
    assert len(blocks) == len(ex) == len(mad) >= 10
    nel = int(goldens["G5"]["keys"]["# Electrons"])
    for blk, e, m in zip(blocks, ex, mad):
        rows = [l.split() for l in blk]
        assert all(len(r) == 5 for r in rows)
        n = np.array([int(r[3]) for r in rows])
        v = np.array([float(r[4]) for r in rows])
        assert n.sum() == (nel // 2) * (nel // 2 - 1)
        assert -(n * v).sum() / nel + m / 2 == pytest.approx(e, rel=1e-12)
    # the second block (change_rs to rSMin; the first is init_HEG's at rs = 1) from the
    # oracle's grids
    o = Oracle(_g5_vals(goldens))
    ref = o.exchange_sf()
    m = ref["maxq"]
    want = []
    for x in range(-m, m + 1):
        for y in range(-m, m + 1):
            for z in range(-m, m + 1):
                c = int(ref["n"][z + m, y + m, x + m])
                if c > 0:
                    want.append("".join(" %11d" % k for k in (x, y, z, c)) + zcode.list_real(ref["v"][z + m, y + m, x + m]))
    assert blocks[1] == want


def test_fort60_unchanged_by_fort82(goldens, tmp_path, monkeypatch):
    """Writing fort.82 leaves the fort.60 log as it was."""
    _g5_files(goldens, tmp_path)
    monkeypatch.chdir(tmp_path)
    zcode.host_logs("Input", "Twists", "a.60", "fort.82")
    zcode.host_logs("Input", "Twists", "b.60", None)
    assert (tmp_path / "a.60").read_text() == (tmp_path / "b.60").read_text()
    assert re.search(r"Starting a new structure factor", (tmp_path / "fort.82").read_text())

"""The product's host set-up (include/uegccd_host.h: ReadInput, init_HEG, change_rs,
ChangeTwist) reproduces the reference -- checked against the oracle and the goldens."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import _capi, heg


def _write(tmp_path, text, name="Input"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _g5_input_text(g):
    lines = [f"{k}: {v}" for k, v in g["G5"]["keys"].items()]
    return "\n".join(lines) + "\n"


def test_read_input_benchmark_key_set(goldens, tmp_path):
    inp = heg.read_input(_write(tmp_path, goldens["G1"]["input_text"]), require_all=False)
    assert (inp.nelectron, inp.maxkpoint, inp.do_drpa_sosex, inp.do_mosaic) == (14, 5, 1, 0)
    with pytest.raises(_capi.UegccdError, match="not set"):
        heg.read_input(_write(tmp_path, goldens["G1"]["input_text"]), require_all=True)


def test_read_input_errors(tmp_path):
    with pytest.raises(_capi.UegccdError, match="closed shell"):
        heg.read_input(_write(tmp_path, "# Electrons: 13\n"), require_all=False)
    with pytest.raises(_capi.UegccdError, match="not recognized"):
        heg.read_input(_write(tmp_path, "# Electrons: 14\nBogus Key: 3\n"), require_all=False)
    with pytest.raises(_capi.UegccdError, match="No Input file"):
        heg.read_input(str(tmp_path / "missing"), require_all=False)


@pytest.mark.parametrize("which", ["G1", "G3", "G5"])
def test_setup_matches_oracle_bitwise(goldens, which):
    if which == "G5":
        vals = parse_input_text("")
        vals.update(goldens["G5"]["keys"])
        inp = heg.default_input(nelectron=24, fcut2ecut=1, fcut=2.0, rsmin=5.0, rsmax=5.0,
                                ntwist=(0.1, 0.2, 0.45))
    else:
        vals = parse_input_text(goldens[which]["input_text"])
        inp = heg.default_input(nelectron=int(vals["# Electrons"]), maxkpoint=int(vals["Momentum Cutoff"]),
                                rsmin=float(vals["rSMin"]), rsmax=float(vals["rSMax"]),
                                ntwist=[float(x) for x in vals["NTwist"].split()])
    o = Oracle(vals)
    h = heg.Heg(inp)
    nocc, L, mad, eig, nv = h.system()
    sc = o.scalars()
    assert (nocc, len(eig)) == (o.nocc, o.nao)
    assert (L, mad, h.info()["ehf"]) == (sc["L"], sc["madelung"], sc["ehf"])
    np.testing.assert_array_equal(eig, o.eigen())
    np.testing.assert_array_equal(nv, o.nvec())
    if which == "G5":
        np.testing.assert_array_equal(eig, np.array(goldens["G5"]["eigen"]))
        for tw in goldens["G5"]["ta_twists"][:4]:
            h.change_twist(tw)
            o.change_twist(tw)
            np.testing.assert_array_equal(h.system()[3], o.eigen())
            assert h.info()["ehf"] == o.scalars()["ehf"]


def test_find_tol():
    assert heg.find_tol(1.0) == (1e-8, 100.0, 2.0)     # HEG.f90:1078-1079
    assert heg.find_tol(5.5) == (1e-6, 100.0, 5.0)
    assert heg.find_tol(0.5)[1] == 1e6


RANGE_KEYS = ["Rings Range", "XRings Range", "Ladders Range", "Mosaics Range", "DriverDir Range",
              "DriverEx Range", "Energy Range", "LinRings Range", "QuadRings Range", "DRings Range",
              "ExRings Range", "LinLadd Range", "QuadLadd Range", "DLadders Range", "ExLadders Range"]


@pytest.mark.parametrize("flags,total,uniform", [
    ({}, 0, 0),
    ({k: "2" for k in RANGE_KEYS}, 30, 2),
    ({"Rings Range": "1"}, 1, -1),
    ({**{k: "1" for k in RANGE_KEYS}, "Energy Range": "2"}, 16, -1),
])
def test_read_input_range_flags(tmp_path, flags, total, uniform):
    """ReadInput's "... Range" values: their |sum| (non-zero: CasedERI applies flags) and the
    one value they share, or -1 (the GPU path serves a shared flag only)."""
    from uegccd_b200 import heg

    (tmp_path / "Input").write_text("# Electrons: 14\n" + "".join(f"{k}: {v}\n" for k, v in flags.items()))
    p = heg.read_input(str(tmp_path / "Input"), require_all=False)
    assert p.range_flags == total
    assert p.range_uniform == uniform
    # the values themselves, in the order of UegccdRangeTerms (the Input's order)
    terms = [getattr(p.range_terms, name) for name in _capi.RANGE_TERMS]
    assert terms == [int(flags.get(k, 0)) for k in RANGE_KEYS]


@pytest.mark.parametrize("gap, ks", [(0.3, 0), (0.0, 1), (-0.2, 1)])
def test_setup_with_gap_and_kohn_sham_matches_oracle(gap, ks):
    """Gap (the occupied eigenvalues take + Madelung - Gap, HEG.f90:525) and DoKS (ExchangeFactor
    0 drops the exchange term, HEG.f90:298, 523; read at IO.f90:253-254) in the HF set-up, bitwise
    against the oracle, at the Gamma point and at a twist."""
    vals = parse_input_text("")
    vals.update({"Gap": str(gap), "DoKS": "T" if ks else "F"})
    o = Oracle(vals)
    h = heg.Heg(heg.default_input(gap=gap, do_ks=ks))
    for tw in (None, (0.1, -0.2, 0.35)):
        if tw is not None:
            h.change_twist(tw)
            o.change_twist(tw)
        nocc, L, mad, eig, nv = h.system()
        assert nocc == o.nocc
        np.testing.assert_array_equal(eig, o.eigen())
        np.testing.assert_array_equal(nv, o.nvec())
        assert h.info()["ehf"] == o.scalars()["ehf"]

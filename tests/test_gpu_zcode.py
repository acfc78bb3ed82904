"""The ZCode drop-in end to end on the GPU: Output and fort.59 against the
reference's own files (G5: source/Test; G3: benchmarks/ZRun-v6-N14) and the G1
dRPA benchmark.

Output is compared line by line: the text around the numbers (every label, width
and integer, iteration counts included) must be identical; each real number must
agree within 2e-10 (the last printed digit of the F15.10 iteration table).
"""
import os
import re
import subprocess

import numpy as np
import pytest

from uegccd_b200 import zcode

pytestmark = pytest.mark.gpu

FLOAT = re.compile(r"-?\d+\.\d+(?:E[+-]\d+)?")
TOL = 2e-10


def _skeleton(line):
    return FLOAT.sub(lambda m: "#" * len(m.group()), line)


def _compare_output(ours, ref):
    assert len(ours) == len(ref), (len(ours), len(ref))
    for k, (a, b) in enumerate(zip(ours, ref)):
        assert _skeleton(a) == _skeleton(b), (k, a, b)
        xa = [float(x) for x in FLOAT.findall(a)]
        xb = [float(x) for x in FLOAT.findall(b)]
        np.testing.assert_allclose(xa, xb, rtol=0, atol=TOL, err_msg=f"line {k}: {a!r} vs {b!r}")


def _write_twists(path, tws):
    with open(path, "w") as f:
        for t in tws:
            f.write("%.17g %.17g %.17g\n" % tuple(t))


def test_g5_output_and_fort59(goldens, tmp_path, monkeypatch):
    g = goldens["G5"]
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in g["keys"].items()))
    _write_twists(tmp_path / "Twists", g["ta_twists"])
    monkeypatch.chdir(tmp_path)
    zcode.run("Input", "Twists")
    _compare_output((tmp_path / "Output").read_text().splitlines(), g["output_lines"])
    ours = (tmp_path / "fort.59").read_text().splitlines()
    ref = g["fort59_lines"]
    assert len(ours) == len(ref)
    for a, b in zip(ours, ref):
        assert _skeleton(a) == _skeleton(b), (a, b)
        np.testing.assert_allclose([float(x) for x in FLOAT.findall(a)], [float(x) for x in FLOAT.findall(b)],
                                   rtol=1e-12, atol=1e-15)
    # the twist-independent host lines are bit-identical text
    for a, b in zip(ours, ref):
        if "conn" in b or "special" in b or "lowest" in b or re.fullmatch(r"\s+\d+\s+\S+\s*", b):
            assert a == b
    # fort.60: the set-up log, identical to the reference's up to its older 'om:' label
    # and its trailing change_rs block (tests/test_zcode_host.py)
    f60 = (tmp_path / "fort.60").read_text().splitlines()
    ref60 = [l.replace(" om:", " Omega:", 1) if l.startswith(" om:") else l for l in g["fort60_lines"]]
    assert len(f60) > 800 and f60 == ref60[: len(f60)]
    assert (tmp_path / "fort.61").read_text().splitlines() == g["fort61_lines"]


def test_g3_hundred_twists_ccd(goldens, tmp_path, monkeypatch):
    g = goldens["G3"]
    (tmp_path / "Input").write_text(g["input_text"])
    _write_twists(tmp_path / "Twists", g["twists"])
    monkeypatch.chdir(tmp_path)
    zcode.run("Input", "Twists")
    rows = [[float(x) for x in l.split()] for l in (tmp_path / "fort.59").read_text().splitlines()[:100]]
    rows = np.array(rows)
    np.testing.assert_array_equal(rows[:, :3], np.array(g["twists"]))
    np.testing.assert_allclose(rows[:, 3:6], np.array(g["hf_mp2_ccd"]), rtol=0, atol=1e-9)
    out = (tmp_path / "Output").read_text()
    ecs = [float(x) for x in re.findall(r"Ec\(CCD\) is\s+(-?\d+\.\d+)", out)]
    conv = [int(x) for x in re.findall(r"converged in\s+(\d+)", out)]
    assert len(ecs) == 101                       # 100 twists + the special twist
    assert conv[-1] == g["special_niter"]
    assert abs(ecs[-1] - g["special_ec_ccd"]) < 1e-9
    f59 = (tmp_path / "fort.59").read_text()
    special = [float(x) for x in FLOAT.findall([l for l in f59.splitlines() if "special" in l][0])]
    np.testing.assert_array_equal(special, g["special_twist"])


def test_g1_drpa_executable(goldens, tmp_path):
    """The uegccd_zcode executable on the G1 dRPA benchmark Input (no twist average)."""
    g = goldens["G1"]
    exe = os.path.join(os.path.dirname(zcode.__file__), "uegccd_zcode")
    (tmp_path / "Input").write_text(g["input_text"])
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = (tmp_path / "Output").read_text()
    ec = float(re.search(r"Ec\(dRPA\) is\s+(-?\d+\.\d+)", out).group(1))
    es = float(re.search(r"Ec\(SOSEX\) is\s+(-?\d+\.\d+)", out).group(1))
    niter = int(re.search(r"dRPA has converged in\s+(\d+)", out).group(1))
    assert niter == g["niter"]
    assert abs(ec - g["ec_drpa"]) < 2e-12 and abs(es - g["ec_sosex"]) < 2e-12
    e2 = float(re.search(r"E\(2\) is\s+(-?\d+\.\d+)", out).group(1))
    assert abs(e2 - g["e2"]) < 2e-12
    assert not (tmp_path / "fort.59").exists()   # TACalcN 0: no twist average


def test_ta_program_with_core_and_gap(goldens, tmp_path, monkeypatch):
    """The G5 program (source/Test) on 4 twists with CoreFactor 0.25 (CoreN = 3) and
    GapII 0.01 (NoCaseERI; the |q|^2 = 1 integrals are cut): every twist's E_HF and
    E_MP2 in fort.59 and the special-twist Ec(CCD) against the oracle's twist average."""
    from oracle.oracle import Oracle, parse_input_text

    g = goldens["G5"]
    keys = dict(g["keys"])
    keys.update({"CoreFactor": "0.25", "GapII": "0.01", "TACalcN": "4"})
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in keys.items()))
    _write_twists(tmp_path / "Twists", g["ta_twists"][:4])
    monkeypatch.chdir(tmp_path)
    zcode.run("Input", "Twists")
    rows = np.array([[float(x) for x in l.split()] for l in (tmp_path / "fort.59").read_text().splitlines()[:4]])
    vals = parse_input_text("")
    vals.update(keys)
    per, special, st, _ = Oracle(vals).twist_average(np.array(g["ta_twists"][:4]))
    np.testing.assert_allclose(rows[:, 3:6], per, rtol=0, atol=1e-12)
    out = (tmp_path / "Output").read_text()
    ecs = [float(x) for x in re.findall(r"Ec\(CCD\) is\s+(-?\d+\.\d+)", out)]
    assert abs(ecs[-1] - st.ecorr) < 1e-9
    assert (tmp_path / "fort.61").read_text().split() == ["6", "core", "electrons", "18", "active", "electrons"]


def test_range_flags_follow_setpointers(goldens, tmp_path, monkeypatch):
    """A "... Range" Input value acts only through CasedERI, which SetPointers (Main.f90:
    299-302) picks under Safe ERI (or with GapII and CoreN both set).  Without it the
    reference's ERI ignores the flags: the program runs as without them.  Under Safe ERI
    the flags act, and the program's answer changes."""
    g = goldens["G5"]
    base = dict(g["keys"])
    base.update({"Safe ERI": "F", "TACalcN": "2"})
    outs = []
    for extra in ({}, {"Rings Range": "1", "Energy Range": "2"}):
        d = tmp_path / ("r%d" % len(outs))
        d.mkdir()
        keys = dict(base)
        keys.update(extra)
        (d / "Input").write_text("".join(f"{k}: {v}\n" for k, v in keys.items()))
        _write_twists(d / "Twists", g["ta_twists"][:2])
        monkeypatch.chdir(d)
        zcode.run("Input", "Twists")
        outs.append(((d / "Output").read_text(), (d / "fort.59").read_text()))
    assert outs[0] == outs[1]
    d = tmp_path / "cased"
    d.mkdir()
    keys = dict(base)
    keys.update({"Safe ERI": "T", "Rings Range": "1", "Energy Range": "2"})
    (d / "Input").write_text("".join(f"{k}: {v}\n" for k, v in keys.items()))
    _write_twists(d / "Twists", g["ta_twists"][:2])
    monkeypatch.chdir(d)
    zcode.run("Input", "Twists")
    assert (d / "Output").read_text() != outs[0][0]


def test_ta_program_with_one_range_flag(goldens, tmp_path, monkeypatch):
    """The G5 program on 3 twists with all fifteen "... Range" values 1 under Safe ERI
    (CasedERI, short range for every CCD term): the per-twist MP2 (plain integrals) in
    fort.59 and the special-twist Ec(CCD) against the oracle."""
    from oracle.oracle import Oracle, parse_input_text

    g = goldens["G5"]
    keys = dict(g["keys"])
    keys.update({"TACalcN": "3", "Safe ERI": "T"})
    keys.update({k: "1" for k in ("Rings Range", "XRings Range", "Ladders Range", "Mosaics Range",
                                  "DriverDir Range", "DriverEx Range", "Energy Range", "LinRings Range",
                                  "QuadRings Range", "DRings Range", "ExRings Range", "LinLadd Range",
                                  "QuadLadd Range", "DLadders Range", "ExLadders Range")})
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in keys.items()))
    _write_twists(tmp_path / "Twists", g["ta_twists"][:3])
    monkeypatch.chdir(tmp_path)
    zcode.run("Input", "Twists")
    rows = np.array([[float(x) for x in l.split()] for l in (tmp_path / "fort.59").read_text().splitlines()[:3]])
    vals = parse_input_text("")
    vals.update(keys)
    per, special, st, _ = Oracle(vals).twist_average(np.array(g["ta_twists"][:3]))
    np.testing.assert_allclose(rows[:, 3:6], per, rtol=0, atol=1e-12)
    out = (tmp_path / "Output").read_text()
    ecs = [float(x) for x in re.findall(r"Ec\(CCD\) is\s+(-?\d+\.\d+)", out)]
    assert abs(ecs[-1] - st.ecorr) < 1e-9


@pytest.mark.parametrize("case", ["per-term flags", "rings without crossed rings"])
def test_ta_program_two_channel(goldens, tmp_path, monkeypatch, case):
    """The G5 program on 3 twists, with CCD at every twist (DoCalcTACCD), in the two-channel
    form: "... Range" values that differ between terms under Safe ERI (direct and exchange
    integrals of a term on different flags), or Do XRings F.  Every twist's CCD runs in its
    own context; fort.59 (E_HF, E_MP2, Ec(CCD) per twist) and the special-twist Ec(CCD)
    against the oracle's twist average."""
    from oracle.oracle import Oracle, parse_input_text

    g = goldens["G5"]
    keys = dict(g["keys"])
    keys.update({"TACalcN": "3", "DoCalcTACCD": "T"})
    if case == "per-term flags":
        # (many flag sets make the reference's own iteration diverge; this one converges)
        keys.update({"Safe ERI": "T", "Rings Range": "2", "XRings Range": "1", "Ladders Range": "2",
                     "DriverEx Range": "1", "Energy Range": "2"})
    else:
        keys.update({"Do XRings": "F"})
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in keys.items()))
    _write_twists(tmp_path / "Twists", g["ta_twists"][:3])
    monkeypatch.chdir(tmp_path)
    zcode.run("Input", "Twists")
    rows = np.array([[float(x) for x in l.split()] for l in (tmp_path / "fort.59").read_text().splitlines()[:3]])
    vals = parse_input_text("")
    vals.update(keys)
    per, special, st, _ = Oracle(vals).twist_average(np.array(g["ta_twists"][:3]))
    np.testing.assert_allclose(rows[:, 3:6], per, rtol=0, atol=1e-10)
    out = (tmp_path / "Output").read_text()
    ecs = [float(x) for x in re.findall(r"Ec\(CCD\) is\s+(-?\d+\.\d+)", out)]
    assert abs(ecs[-1] - st.ecorr) < 1e-9


def test_g1_drpa_program_with_range_flags(goldens, tmp_path, monkeypatch):
    """The G1 dRPA program under Safe ERI with per-term flags (Rings Range 2, DriverDir Range 1):
    the general-flag dRPA (the terms on their flags, the energy on flag 0, dRPA.f90:206-207,
    363-529) against the oracle's DrvdRPA on the same Input."""
    from oracle.oracle import Oracle, parse_input_text

    g = goldens["G1"]
    vals = parse_input_text(g["input_text"])
    vals.update({"Safe ERI": "T", "Rings Range": "2", "DriverDir Range": "1"})
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in vals.items()))
    monkeypatch.chdir(tmp_path)
    zcode.run("Input")
    out = (tmp_path / "Output").read_text()
    ec = float(re.search(r"Ec\(dRPA\) is\s+(-?\d+\.\d+)", out).group(1))
    es = float(re.search(r"Ec\(SOSEX\) is\s+(-?\d+\.\d+)", out).group(1))
    niter = int(re.search(r"dRPA has converged in\s+(\d+)", out).group(1))
    o = Oracle(vals)
    _, ta, _, _, _ = o.mp2()
    st, _, _ = o.drpa(ta.copy())
    assert niter == st.niter
    assert abs(ec - st.ecorr) < 5e-12 and abs(es - st.ecorr_sosex) < 5e-12
    assert abs(ec - g["ec_drpa"]) > 1e-3   # the flags act

"""Host side of the ZCode drop-in (Main.f90 twist average): the connectivity histogram,
the special-twist choice and the fort.59 number format, against the oracle and the
reference's own fort.59 (source/Test/fort.59, G5).  No GPU needed."""
import re

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import heg, zcode


def _g5_vals(goldens):
    v = parse_input_text("")
    v.update(goldens["G5"]["keys"])
    return v


def _heg(tmp_path, text, twist=None):
    p = tmp_path / "Input"
    p.write_text(text)
    inp = heg.read_input(str(p), require_all=False)
    if twist is not None:
        for d in range(3):
            inp.ntwist[d] = float(twist[d])
    return heg.Heg(inp)


def _g5_text(goldens):
    return "".join(f"{k}: {v}\n" for k, v in goldens["G5"]["keys"].items())


def _split_items(line):
    """Fortran list-directed record -> [(kind, text)] with kind 'r', 'i' or 's'."""
    out = []
    for tok in line.split():
        if re.fullmatch(r"-?\d+", tok):
            out.append(("i", tok))
        elif re.fullmatch(r"-?\d+\.\d+(E[+-]\d+)?", tok):
            out.append(("r", tok))
        elif out and out[-1][0] == "s":
            out[-1] = ("s", out[-1][1] + " " + tok)
        else:
            out.append(("s", tok))
    return out


def _rebuild(line):
    s = ""
    for kind, text in _split_items(line):
        if kind == "r":
            s += zcode.list_real(float(text))
        elif kind == "i":
            s += " %11d" % int(text)
        else:
            s += " " + text
    return s


def test_list_directed_format_matches_reference_fort59(goldens):
    """Every line of the reference's fort.59 re-written from its own numbers is identical."""
    lines = goldens["G5"]["fort59_lines"]
    assert len(lines) > 20
    for line in lines:
        assert _rebuild(line) == line, line


def test_list_real_forms():
    assert zcode.list_real(0.1766364574432373) == "  0.17663645744323730     "
    assert zcode.list_real(-1.3357699958295419) == "  -1.3357699958295419     "
    assert zcode.list_real(0.0) == "   0.0000000000000000     "
    assert zcode.list_real(5.438685417175293e-02) == "   5.4386854171752930E-002"
    assert zcode.list_real(-3.0e20) == "  -3.0000000000000000E+020"


def test_connectivity_matches_oracle(goldens, tmp_path):
    h = _heg(tmp_path, _g5_text(goldens))
    conn = zcode.connectivity(h.system())
    e, *_, oconn = Oracle(_g5_vals(goldens)).mp2()
    np.testing.assert_array_equal(conn, oconn)
    assert conn.sum() > 0


def test_special_twist_matches_reference_fort59(goldens, tmp_path):
    """G5: 10 twists -> the reference's special twist and its connectivity distances."""
    g = goldens["G5"]
    tws = np.array(g["ta_twists"])
    conns = np.stack([zcode.connectivity(_heg(tmp_path, _g5_text(goldens), tw).system()) for tw in tws])
    best, avg, d2 = zcode.special_twist(conns)
    np.testing.assert_array_equal(tws[best], np.array(g["special_twist"]))
    ref_d2 = [float(l.split()[1]) for l in g["fort59_lines"] if re.fullmatch(r"\s+\d+\s+\S+\s*", l)]
    np.testing.assert_allclose(d2, ref_d2, rtol=1e-14, atol=0)
    conn_line = [l for l in g["fort59_lines"] if l.rstrip().endswith("conn")][0]
    ref_avg = [float(x) for x in conn_line.split()[:-1]]
    np.testing.assert_array_equal(avg[: len(ref_avg)], ref_avg)


def test_special_twist_g3(goldens, tmp_path):
    g = goldens["G3"]
    tws = np.array(g["twists"])
    conns = np.stack([zcode.connectivity(_heg(tmp_path, g["input_text"], tw).system()) for tw in tws])
    best, _, _ = zcode.special_twist(conns)
    np.testing.assert_array_equal(tws[best], np.array(g["special_twist"]))


def test_special_twist_first_minimum_wins():
    c = np.zeros((3, zcode.CONN_LIMIT), dtype=np.int32)
    c[0, 0], c[1, 0], c[2, 0] = 4, 2, 2      # average 8/3: twists 1 and 2 tie at the minimum
    best, avg, d2 = zcode.special_twist(c)
    assert best == 1 and d2[1] == d2[2] < d2[0]


def test_zcode_without_gpu_reports_error(goldens, tmp_path, monkeypatch):
    """Without a GPU the program stops with an error before writing results."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    (tmp_path / "Input").write_text(goldens["G3"]["input_text"])
    monkeypatch.chdir(tmp_path)
    from uegccd_b200 import _capi

    with pytest.raises(_capi.UegccdError):
        zcode.run("Input")
    assert not (tmp_path / "fort.59").exists()


def test_fort60_log_matches_reference(goldens, tmp_path, monkeypatch):
    """The set-up log (fort.60) of the G5 program against the reference's own file.

    Every line is identical, with two differences. The reference's stored file is
    from a build that labelled Omega as 'om:'; the current source (HEG.f90:606)
    writes 'Omega:'. It also ends with one more change_rs block, which the current
    Main.f90 has commented out (Main.f90:236-242)."""
    import ctypes as C

    g = goldens["G5"]
    (tmp_path / "Input").write_text("".join(f"{k}: {v}\n" for k, v in g["keys"].items()))
    (tmp_path / "Twists").write_text("".join("%.17g %.17g %.17g\n" % tuple(t) for t in g["ta_twists"]))
    monkeypatch.chdir(tmp_path)
    L = heg._lib()
    L.uegccd_zcode_fort60.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
    assert L.uegccd_zcode_fort60(b"Input", b"Twists", b"fort.60") == 0
    ours = (tmp_path / "fort.60").read_text().splitlines()
    ref = [l.replace(" om:", " Omega:", 1) if l.startswith(" om:") else l for l in g["fort60_lines"]]
    assert len(ours) > 800
    assert ours == ref[: len(ours)]
    tail = ref[len(ours):]
    assert tail[2].strip() == "Calculating Madelung Constant - Fraser et al. PRB 53 4 1814"
    assert sum(1 for l in tail if l.startswith(" Omega:")) == 1


def test_fort61_matches_reference(goldens, tmp_path, monkeypatch):
    """fort.61, ReadInput's core and active electron counts (IO.f90:232-234), against the
    reference's source/Test/fort.61 (G5) and benchmarks/ZRun-v6-N14/fort.61 (G3), and for
    CoreFactor 0.3 at N=14 (CoreN = int(7*0.3) = 2)."""
    monkeypatch.chdir(tmp_path)
    g5 = goldens["G5"]
    cases = [("".join(f"{k}: {v}\n" for k, v in g5["keys"].items()), g5["fort61_lines"]),
             (goldens["G3"]["input_text"], goldens["G3"]["fort61_lines"]),
             (goldens["G3"]["input_text"].replace("CoreFactor:       0.0", "CoreFactor:       0.3")
              .replace("TACalcN:          100", "TACalcN:          2"),
              ["           4 core electrons", "          10 active electrons"])]
    for text, want in cases:
        (tmp_path / "Input").write_text(text)
        zcode.host_logs("Input", None, "fort.60", None, "fort.61")
        assert (tmp_path / "fort.61").read_text().splitlines() == want

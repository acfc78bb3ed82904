"""The plane-wave set-up of many twists on the GPU (uegccd_heg_twists) against the host
set-up (uegccd_heg_change_twist): basis order, HF eigenvalues and E_HF bit for bit.

The host set-up is itself pinned to the reference's fort.60 listings and fort.59 columns
(tests/test_host_setup.py, tests/test_gpu_zcode.py); the stable sort decides which orbitals
fcut keeps, so the order must match exactly.  Systems: G3's 100 listed twists (N=14,
'Momentum Cutoff: 2'), G5 (N=24, fcut2ecut with fcut 2, rs=5) and the batched-twist
benchmark workload (N=54, |n|^2 <= 30 pool cut to 485 orbitals, 100 twists of seed 2024).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compare(h, twists):
    systems, ehf = h.twist_systems(twists)
    for k, tw in enumerate(twists):
        h.change_twist(tw)
        nocc, L, mad, eig, nv = h.system()
        d = systems[k]
        assert d[0] == nocc and d[1] == L and d[2] == mad
        np.testing.assert_array_equal(d[4], nv)
        np.testing.assert_array_equal(d[3], eig)      # bit-equal eigenvalues
        assert ehf[k] == h.info()["ehf"], (k, ehf[k], h.info()["ehf"])


def test_g3_twists(goldens, tmp_path):
    from uegccd_b200 import heg

    p = tmp_path / "Input"
    p.write_text(goldens["G3"]["input_text"])
    h = heg.Heg(heg.read_input(str(p), require_all=False))
    _compare(h, np.array(goldens["G3"]["twists"]))


def test_g5_twists():
    from uegccd_b200 import heg

    h = heg.Heg(heg.default_input(nelectron=24, fcut2ecut=1, fcut=2.0, rsmin=5.0, rsmax=5.0,
                                  ntwist=(0.1, 0.2, 0.45)))
    tw = np.random.default_rng(11).random((10, 3)) - 0.5
    _compare(h, np.vstack([[0.1, 0.2, 0.45], tw]))


def test_benchmark_twists():
    import bench
    from uegccd_b200 import heg

    h = heg.Heg(heg.default_input(nelectron=bench.N_ELECTRONS, maxkpoint=bench.MAXK, rsmin=bench.RS,
                                  rsmax=bench.RS, fcut=bench.FCUT))
    _compare(h, bench.twists(100))


@pytest.mark.parametrize("gap, ks", [(0.3, 0), (-0.2, 1)])
def test_device_twists_with_gap_and_kohn_sham(gap, ks):
    """uegccd_heg_twists with Gap and DoKS set (HEG.f90:298, 523-525): bitwise against the host
    set-up of the same twists."""
    from uegccd_b200 import heg

    tws = np.random.default_rng(11).random((8, 3)) - 0.5
    inp = heg.default_input(gap=gap, do_ks=ks)
    dev_sys, dev_ehf = heg.Heg(inp).twist_systems(tws)
    h = heg.Heg(heg.default_input(gap=gap, do_ks=ks))
    for k, tw in enumerate(tws):
        h.change_twist(tw)
        nocc, L, mad, eig, nv = h.system()
        assert dev_sys[k][0] == nocc
        np.testing.assert_array_equal(dev_sys[k][3], eig)
        np.testing.assert_array_equal(dev_sys[k][4], nv)
        assert dev_ehf[k] == h.info()["ehf"]

"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is the C restatement in ``ueg_oracle.c`` of the reference Fortran
(shepherd-group/uegccd).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module, as the checker; the product
package never imports it.

Amplitude arrays use the reference's layout: ``T(NOcc, NOcc, NOcc+1:NAO)``
column-major, which is a numpy array of shape ``(V, O, O)`` in C order indexed
``[a-O-1, j-1, i-1]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libuegoracle.so")


class UoInput(C.Structure):
    _fields_ = [
        ("nelectron", C.c_int), ("maxkpoint", C.c_int),
        ("rsmin", C.c_double), ("rsmax", C.c_double), ("num_rs_points", C.c_int),
        ("safe_eri", C.c_int),
        ("do_ring", C.c_int), ("do_xring", C.c_int), ("do_ladder", C.c_int), ("do_mosaic", C.c_int),
        ("irange_ring", C.c_int), ("irange_xring", C.c_int), ("irange_ladder", C.c_int),
        ("irange_mosaic", C.c_int), ("irange_driver_direct", C.c_int),
        ("irange_driver_exchange", C.c_int), ("irange_energy", C.c_int),
        ("irange_lin_rings", C.c_int), ("irange_quad_rings", C.c_int),
        ("irange_direct_rings", C.c_int), ("irange_exchange_rings", C.c_int),
        ("irange_lin_ladders", C.c_int), ("irange_quad_ladders", C.c_int),
        ("irange_direct_ladders", C.c_int), ("irange_exchange_ladders", C.c_int),
        ("ntwist", C.c_double * 3), ("core_factor", C.c_double), ("tacalcn", C.c_int),
        ("do_calc_ta_ccd", C.c_int), ("do_drpa_sosex", C.c_int), ("do_ks", C.c_int),
        ("madelung_factor", C.c_double), ("do_single_calc", C.c_int), ("gap", C.c_double),
        ("fcut", C.c_double), ("corefcut", C.c_double), ("fcut2ecut", C.c_int),
        ("gapii", C.c_double), ("do_skip_ta", C.c_int),
    ]


class UoSolveStats(C.Structure):
    _fields_ = [
        ("ecorr", C.c_double), ("ecorr_sosex", C.c_double), ("max_res", C.c_double),
        ("last_dt", C.c_double), ("niter", C.c_int), ("fail", C.c_int), ("n_recorded", C.c_int),
    ]


def build() -> str:
    """Compile the oracle library with its Makefile (gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(
            os.path.getmtime(os.path.join(_HERE, f)) for f in ("ueg_oracle.c", "ueg_oracle.h")
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER
        dp = P(C.c_double)
        L.uo_create.restype = C.c_void_p
        L.uo_create.argtypes = [P(UoInput)]
        L.uo_destroy.argtypes = [C.c_void_p]
        L.uo_last_error.restype = C.c_char_p
        for f in ("uo_nocc", "uo_nao", "uo_cell", "uo_maxkpoint"):
            getattr(L, f).restype = C.c_int
            getattr(L, f).argtypes = [C.c_void_p]
        L.uo_scalars.argtypes = [C.c_void_p, dp]
        L.uo_get_eigen.argtypes = [C.c_void_p, dp]
        L.uo_set_eigen.argtypes = [C.c_void_p, dp]
        L.uo_get_nvec.argtypes = [C.c_void_p, P(C.c_int)]
        L.uo_get_kvec.argtypes = [C.c_void_p, dp]
        L.uo_change_twist.restype = C.c_int
        L.uo_change_twist.argtypes = [C.c_void_p, dp]
        L.uo_mp2.restype = C.c_double
        L.uo_mp2.argtypes = [C.c_void_p, dp, dp, dp, P(C.c_int)]
        L.uo_ccd.restype = C.c_int
        L.uo_ccd.argtypes = [C.c_void_p, dp, dp, dp, C.c_int, P(UoSolveStats), dp, dp, C.c_int]
        L.uo_drpa.restype = C.c_int
        L.uo_drpa.argtypes = [C.c_void_p, dp, C.c_int, P(UoSolveStats), dp, dp, C.c_int]
        L.uo_ccd_g2.argtypes = [C.c_void_p, dp, dp, C.c_int, dp, dp]
        L.uo_set_tol_override.argtypes = [C.c_double]
        L.uo_set_tol_override.restype = None
        L.uo_drpa_g2.argtypes = [C.c_void_p, dp, C.c_int, dp]
        L.uo_ccd_energy.restype = C.c_double
        L.uo_ccd_energy.argtypes = [C.c_void_p, dp, dp, dp]
        L.uo_drpa_energy.restype = C.c_double
        L.uo_drpa_energy.argtypes = [C.c_void_p, dp, C.c_double]
        L.uo_sf_length.restype = C.c_int
        L.uo_sf_length.argtypes = [C.c_void_p]
        L.uo_structure_factor.restype = C.c_double
        L.uo_structure_factor.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp, dp, dp, P(C.c_int)]
        L.uo_exchange_sf.restype = C.c_int
        L.uo_exchange_sf.argtypes = [C.c_void_p, P(C.c_int), dp]
        L.uo_twist_average.restype = C.c_int
        L.uo_twist_average.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, P(UoSolveStats), dp]
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ctype=C.c_double):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


# Defaults for keys that older Input files (the benchmarks' key set) do not set.  A key
# added after those files were written takes the behaviour of the code that predates it:
# DoSkipTA F (the twist average always ran; Main.f90:95 added the stop).
DEFAULTS = {
    "# Electrons": "14", "Momentum Cutoff": "2", "rSMin": "1.0", "rSMax": "1.0", "# rS Points": "1",
    "Safe ERI": "F", "Do Rings": "T", "Do XRings": "T", "Do Ladders": "T", "Do Mosaics": "T",
    "Rings Range": "0", "XRings Range": "0", "Ladders Range": "0", "Mosaics Range": "0",
    "DriverDir Range": "0", "DriverEx Range": "0", "Energy Range": "0", "LinRings Range": "0",
    "QuadRings Range": "0", "DRings Range": "0", "ExRings Range": "0", "LinLadd Range": "0",
    "QuadLadd Range": "0", "DLadders Range": "0", "ExLadders Range": "0", "NTwist": "0 0 0",
    "CoreFactor": "0.0", "TACalcN": "0", "DoCalcTACCD": "F", "DodRPASOSEX": "F",
    "DoTruncCoulombHF": "F", "DoTruncCoulombAll": "F", "DoKS": "F", "MadelungFactor": "1.0",
    "DoSingleCalc": "T", "Gap": "0.0", "fcut": "10.0", "corefcut": "1.0", "fcut2ecut": "F",
    "GapII": "-0.01", "DoSFCalcMP2": "F", "DoSFCalcCCD": "F", "DoSkipTA": "F", "DoOnlyMP2Grid": "F",
}


def parse_input_text(text: str) -> dict:
    """Key: Value lines, '!' comments (IO.f90:355-391); missing keys take DEFAULTS."""
    vals = dict(DEFAULTS)
    for line in text.splitlines():
        line = line.split("!", 1)[0]
        if not line.strip() or ":" not in line:
            continue
        k, v = line.split(":", 1)
        vals[k.strip()] = v.strip()
    return vals


def _b(v: str) -> int:
    v = v.strip().upper().lstrip(".")
    return 1 if v.startswith("T") else 0


def make_input(vals: dict) -> UoInput:
    g = lambda k: vals[k]
    p = UoInput()
    p.nelectron = int(g("# Electrons"))
    p.maxkpoint = int(g("Momentum Cutoff"))
    p.rsmin = float(g("rSMin")); p.rsmax = float(g("rSMax")); p.num_rs_points = int(g("# rS Points"))
    p.safe_eri = _b(g("Safe ERI"))
    p.do_ring = _b(g("Do Rings")); p.do_xring = _b(g("Do XRings"))
    p.do_ladder = _b(g("Do Ladders")); p.do_mosaic = _b(g("Do Mosaics"))
    for f, k in (("irange_ring", "Rings Range"), ("irange_xring", "XRings Range"),
                 ("irange_ladder", "Ladders Range"), ("irange_mosaic", "Mosaics Range"),
                 ("irange_driver_direct", "DriverDir Range"), ("irange_driver_exchange", "DriverEx Range"),
                 ("irange_energy", "Energy Range"), ("irange_lin_rings", "LinRings Range"),
                 ("irange_quad_rings", "QuadRings Range"), ("irange_direct_rings", "DRings Range"),
                 ("irange_exchange_rings", "ExRings Range"), ("irange_lin_ladders", "LinLadd Range"),
                 ("irange_quad_ladders", "QuadLadd Range"), ("irange_direct_ladders", "DLadders Range"),
                 ("irange_exchange_ladders", "ExLadders Range")):
        setattr(p, f, int(g(k)))
    tw = [float(x) for x in g("NTwist").split()[:3]]
    for d in range(3):
        p.ntwist[d] = tw[d]
    p.core_factor = float(g("CoreFactor")); p.tacalcn = int(g("TACalcN"))
    p.do_calc_ta_ccd = _b(g("DoCalcTACCD")); p.do_drpa_sosex = _b(g("DodRPASOSEX"))
    p.do_ks = _b(g("DoKS")); p.madelung_factor = float(g("MadelungFactor"))
    p.do_single_calc = _b(g("DoSingleCalc")); p.gap = float(g("Gap"))
    p.fcut = float(g("fcut")); p.corefcut = float(g("corefcut")); p.fcut2ecut = _b(g("fcut2ecut"))
    p.gapii = float(g("GapII")); p.do_skip_ta = _b(g("DoSkipTA"))
    return p


class Oracle:
    """One set-up uniform electron gas (init_HEG + change_rs) in the oracle."""

    def __init__(self, vals: dict | str):
        if isinstance(vals, str):
            vals = parse_input_text(vals)
        self.vals = vals
        self._inp = make_input(vals)
        self.L = lib()
        self.h = self.L.uo_create(C.byref(self._inp))
        if not self.h:
            raise RuntimeError(self.L.uo_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.uo_destroy(self.h)
            self.h = None

    @property
    def nocc(self) -> int:
        return self.L.uo_nocc(self.h)

    @property
    def nao(self) -> int:
        return self.L.uo_nao(self.h)

    @property
    def nvir(self) -> int:
        return self.nao - self.nocc

    @property
    def cell(self) -> int:
        return self.L.uo_cell(self.h)

    @property
    def maxkpoint(self) -> int:
        return self.L.uo_maxkpoint(self.h)

    def scalars(self) -> dict:
        out = np.zeros(7)
        self.L.uo_scalars(self.h, _ptr(out))
        return dict(L=out[0], omega=out[1], madelung=out[2], ehf=out[3], twist=out[4:7].copy())

    def eigen(self) -> np.ndarray:
        e = np.zeros(self.nao)
        self.L.uo_get_eigen(self.h, _ptr(e))
        return e

    def set_eigen(self, e: np.ndarray) -> None:
        e = np.ascontiguousarray(e, dtype=np.float64)
        self.L.uo_set_eigen(self.h, _ptr(e))

    def nvec(self) -> np.ndarray:
        n = np.zeros((self.nao, 3), dtype=np.int32)
        self.L.uo_get_nvec(self.h, _ptr(n, C.c_int))
        return n

    def kvec(self) -> np.ndarray:
        k = np.zeros((self.nao, 3))
        self.L.uo_get_kvec(self.h, _ptr(k))
        return k

    def change_twist(self, tw) -> None:
        t = np.ascontiguousarray(tw, dtype=np.float64)
        if self.L.uo_change_twist(self.h, _ptr(t)) != 0:
            raise RuntimeError(self.L.uo_last_error().decode())

    def zeros_t(self) -> np.ndarray:
        return np.zeros((self.nvir, self.nocc, self.nocc))

    def mp2(self):
        ta, tb, tc = self.zeros_t(), self.zeros_t(), self.zeros_t()
        conn = np.zeros(400, dtype=np.int32)
        e = self.L.uo_mp2(self.h, _ptr(ta), _ptr(tb), _ptr(tc), _ptr(conn, C.c_int))
        return e, ta, tb, tc, conn

    def ccd(self, t_aaaa, t_abab, t_abba, max_iter: int = 0, max_rec: int = 1100, tol: float = 0.0):
        """DrvCCD; tol > 0 replaces TolMax (tight-mode parity only)."""
        st = UoSolveStats()
        self.L.uo_set_tol_override(tol)
        en = np.zeros(max_rec)
        dts = np.zeros(max_rec)
        rc = self.L.uo_ccd(self.h, _ptr(t_aaaa), _ptr(t_abab), _ptr(t_abba), max_iter, C.byref(st),
                           _ptr(en), _ptr(dts), max_rec)
        self.L.uo_set_tol_override(0.0)
        if rc != 0:
            raise RuntimeError(self.L.uo_last_error().decode())
        return st, en[: st.n_recorded].copy(), dts[: st.n_recorded].copy()

    def drpa(self, t2, max_iter: int = 0, max_rec: int = 1100):
        st = UoSolveStats()
        en = np.zeros(max_rec)
        dts = np.zeros(max_rec)
        rc = self.L.uo_drpa(self.h, _ptr(t2), max_iter, C.byref(st), _ptr(en), _ptr(dts), max_rec)
        if rc != 0:
            raise RuntimeError(self.L.uo_last_error().decode())
        return st, en[: st.n_recorded].copy(), dts[: st.n_recorded].copy()

    def ccd_g2(self, t_abab, t_abba, mask: int = 31):
        ga, gb = self.zeros_t(), self.zeros_t()
        self.L.uo_ccd_g2(self.h, _ptr(np.ascontiguousarray(t_abab)), _ptr(np.ascontiguousarray(t_abba)),
                         mask, _ptr(ga), _ptr(gb))
        return ga, gb

    def drpa_g2(self, t2, mask: int = 11):
        g = self.zeros_t()
        self.L.uo_drpa_g2(self.h, _ptr(np.ascontiguousarray(t2)), mask, _ptr(g))
        return g

    def ccd_energy(self, t_aaaa, t_abab, t_abba) -> float:
        return self.L.uo_ccd_energy(self.h, _ptr(t_aaaa), _ptr(t_abab), _ptr(t_abba))

    def drpa_energy(self, t2, csosex: float) -> float:
        return self.L.uo_drpa_energy(self.h, _ptr(t2), csosex)

    def sf_length(self) -> int:
        return self.L.uo_sf_length(self.h)

    def structure_factor(self, t_aaaa, t_abab, t_abba) -> dict:
        """CCEnergyAndSF grids (W,W,W) indexed [z+S, y+S, x+S] (Fortran order), and ECorr."""
        S = self.sf_length()
        W = 2 * S + 1
        g = {k: np.zeros((W, W, W)) for k in ("sum", "g", "v", "dsum", "xsum")}
        oob = C.c_int()
        e = self.L.uo_structure_factor(self.h, _ptr(np.ascontiguousarray(t_aaaa)), _ptr(np.ascontiguousarray(t_abab)),
                                       _ptr(np.ascontiguousarray(t_abba)), _ptr(g["sum"]), _ptr(g["g"]), _ptr(g["v"]),
                                       _ptr(g["dsum"]), _ptr(g["xsum"]), C.byref(oob))
        g.update(S=S, ecorr=e, oob=oob.value)
        return g

    def exchange_sf(self) -> dict:
        """print_ex_SF grids (W,W,W) indexed [z+maxq, y+maxq, x+maxq]."""
        maxq = self.L.uo_exchange_sf(self.h, None, None)
        W = 2 * maxq + 1
        n = np.zeros((W, W, W), dtype=np.int32)
        v = np.zeros((W, W, W))
        self.L.uo_exchange_sf(self.h, _ptr(n, C.c_int), _ptr(v))
        return dict(maxq=maxq, n=n, v=v)

    def twist_average(self, twists: np.ndarray):
        tw = np.ascontiguousarray(twists, dtype=np.float64).reshape(-1, 3)
        per = np.zeros((tw.shape[0], 3))
        special = np.zeros(3)
        st = UoSolveStats()
        mp2 = C.c_double()
        rc = self.L.uo_twist_average(self.h, tw.shape[0], _ptr(tw), _ptr(per), _ptr(special), C.byref(st),
                                     C.byref(mp2))
        if rc != 0:
            raise RuntimeError(self.L.uo_last_error().decode())
        return per, special, st, mp2.value

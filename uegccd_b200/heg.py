"""Host-side set-up of the drop-in (ReadInput, init_HEG, change_rs, ChangeTwist).

Binds include/uegccd_host.h.  Produces the system (NOcc, NAO, L, Madelung,
Eigen, nVec) that the GPU hot path takes; mirrors the reference's HEG module
(HEG.f90:16-615) and IO module (IO.f90:14-391).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi


class Input(C.Structure):
    _fields_ = [
        ("nelectron", C.c_int32), ("maxkpoint", C.c_int32), ("rsmin", C.c_double), ("rsmax", C.c_double),
        ("num_rs_points", C.c_int32), ("safe_eri", C.c_int32), ("do_ring", C.c_int32), ("do_xring", C.c_int32),
        ("do_ladder", C.c_int32), ("do_mosaic", C.c_int32), ("range_flags", C.c_int32),
        ("ntwist", C.c_double * 3), ("core_factor", C.c_double), ("tacalcn", C.c_int32),
        ("do_calc_ta_ccd", C.c_int32), ("do_drpa_sosex", C.c_int32), ("do_ks", C.c_int32),
        ("madelung_factor", C.c_double), ("do_single_calc", C.c_int32), ("gap", C.c_double),
        ("fcut", C.c_double), ("corefcut", C.c_double), ("fcut2ecut", C.c_int32), ("gapii", C.c_double),
        ("do_skip_ta", C.c_int32), ("do_sf_calc_mp2", C.c_int32),
        ("do_sf_calc_ccd", C.c_int32), ("do_only_mp2_grid", C.c_int32), ("core_factor_set", C.c_int32),
        ("range_uniform", C.c_int32), ("range_terms", capi.RangeTerms),
    ]


class HegInfo(C.Structure):
    _fields_ = [
        ("nocc", C.c_int32), ("nao", C.c_int32), ("maxkpoint", C.c_int32), ("cell", C.c_int32),
        ("core_n", C.c_int32), ("L", C.c_double), ("omega", C.c_double), ("madelung", C.c_double),
        ("ehf", C.c_double), ("twist", C.c_double * 3),
    ]


_bound = False


def _lib():
    global _bound
    L = capi.lib()
    if not _bound:
        P, vp = C.POINTER, C.c_void_p
        L.uegccd_default_input.argtypes = [P(Input)]
        L.uegccd_default_input.restype = None
        L.uegccd_read_input.argtypes = [C.c_char_p, C.c_int32, P(Input)]
        L.uegccd_heg_create.argtypes = [P(Input), P(vp)]
        L.uegccd_heg_destroy.argtypes = [vp]
        L.uegccd_heg_destroy.restype = None
        L.uegccd_heg_change_twist.argtypes = [vp, P(C.c_double)]
        L.uegccd_heg_set_eigen.argtypes = [vp, P(C.c_double)]
        L.uegccd_heg_system.argtypes = [vp, P(capi.System)]
        L.uegccd_heg_info.argtypes = [vp, P(HegInfo)]
        L.uegccd_find_tol.argtypes = [C.c_double, P(C.c_double), P(C.c_double), P(C.c_double)]
        L.uegccd_find_tol.restype = None
        L.uegccd_host_last_error.restype = C.c_char_p
        L.uegccd_heg_exchange_sf.argtypes = [vp, P(C.c_int32), P(C.c_int32), P(C.c_double)]
        L.uegccd_heg_twists.argtypes = [vp, C.c_int32, P(C.c_double), P(C.c_int32), P(C.c_double), P(C.c_double)]
        _bound = True
    return L


def _check(rc):
    if rc != 0:
        raise capi.UegccdError(rc, _lib().uegccd_host_last_error().decode())


def default_input(**kw) -> Input:
    p = Input()
    _lib().uegccd_default_input(C.byref(p))
    for k, v in kw.items():
        if k == "ntwist":
            for d in range(3):
                p.ntwist[d] = float(v[d])
        else:
            setattr(p, k, v)
    return p


def read_input(path: str, require_all: bool = True) -> Input:
    """ReadInput (IO.f90:14-348)."""
    p = Input()
    _check(_lib().uegccd_read_input(path.encode(), 1 if require_all else 0, C.byref(p)))
    return p


def find_tol(rs: float):
    t, f, d = C.c_double(), C.c_double(), C.c_double(2.0)
    _lib().uegccd_find_tol(rs, C.byref(t), C.byref(f), C.byref(d))
    return t.value, f.value, d.value


class Heg:
    """init_HEG + change_rs of one Input; change_twist re-runs SetupBasis."""

    def __init__(self, inp: Input):
        self.input = inp
        h = C.c_void_p()
        _check(_lib().uegccd_heg_create(C.byref(inp), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib().uegccd_heg_destroy(self._h)
            self._h = None

    def info(self) -> dict:
        i = HegInfo()
        _check(_lib().uegccd_heg_info(self._h, C.byref(i)))
        d = {k: getattr(i, k) for k, _ in HegInfo._fields_}
        d["twist"] = np.array(i.twist[:])
        return d

    def change_twist(self, tw) -> None:
        t = np.ascontiguousarray(tw, dtype=np.float64)
        _check(_lib().uegccd_heg_change_twist(self._h, t.ctypes.data_as(C.POINTER(C.c_double))))

    def set_eigen(self, e) -> None:
        e = np.ascontiguousarray(e, dtype=np.float64)
        _check(_lib().uegccd_heg_set_eigen(self._h, e.ctypes.data_as(C.POINTER(C.c_double))))

    def exchange_sf(self) -> dict:
        """print_ex_SF (HEG.f90:617-674): pair counts n and ExV v on (W,W,W) grids indexed
        [z+maxq, y+maxq, x+maxq]."""
        m = C.c_int32()
        _check(_lib().uegccd_heg_exchange_sf(self._h, C.byref(m), None, None))
        W = 2 * m.value + 1
        n = np.zeros((W, W, W), dtype=np.int32)
        v = np.zeros((W, W, W))
        _check(_lib().uegccd_heg_exchange_sf(self._h, C.byref(m), n.ctypes.data_as(C.POINTER(C.c_int32)),
                                             v.ctypes.data_as(C.POINTER(C.c_double))))
        return dict(maxq=m.value, n=n, v=v)

    def system(self):
        """(nocc, L, madelung, eigen copy, nvec (NAO,3) copy)"""
        s = capi.System()
        _check(_lib().uegccd_heg_system(self._h, C.byref(s)))
        eig = np.ctypeslib.as_array(s.eigen, shape=(s.nao,)).copy()
        nv = np.ctypeslib.as_array(s.nvec, shape=(3, s.nao)).T.copy()
        return s.nocc, s.L, s.madelung, eig, nv

    def twist_systems(self, twists):
        """The systems (nocc, L, madelung, eigen, nvec) of many twists, set up on the GPU in
        one launch (uegccd_heg_twists), and their E_HF: bit-equal to change_twist then system()
        for each twist.  The set-up itself is left unchanged."""
        tw = np.ascontiguousarray(np.asarray(twists, dtype=np.float64).reshape(-1, 3))
        info = self.info()
        T, M = tw.shape[0], info["nao"]
        nv = np.zeros((T, 3, M), dtype=np.int32)
        eig = np.zeros((T, M))
        ehf = np.zeros(T)
        capi.check(_lib().uegccd_heg_twists(self._h, T, tw.ctypes.data_as(C.POINTER(C.c_double)),
                                            nv.ctypes.data_as(C.POINTER(C.c_int32)),
                                            eig.ctypes.data_as(C.POINTER(C.c_double)),
                                            ehf.ctypes.data_as(C.POINTER(C.c_double))))
        systems = [(info["nocc"], info["L"], info["madelung"], eig[k], nv[k].T.copy()) for k in range(T)]
        return systems, ehf

    def context(self):
        from .solver import Context

        return Context(*self.system())

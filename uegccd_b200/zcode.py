"""The reference's ZCode program (Main.f90) over the C ABI: the twist-average
helpers (connectivity histogram, special twist, fort.59 number format) and the
whole program, which runs its solves on the GPU.

    python -m uegccd_b200.zcode [Input [Twists]]
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _capi, heg

CONN_LIMIT = 400
_bound = False


def _lib():
    global _bound
    L = heg._lib()
    if not _bound:
        P = C.POINTER
        L.uegccd_connectivity.argtypes = [P(_capi.System), C.c_int32, P(C.c_int32)]
        L.uegccd_special_twist.argtypes = [C.c_int32, P(C.c_int32), P(C.c_double), P(C.c_double), P(C.c_int32)]
        L.uegccd_list_real.argtypes = [C.c_double, C.c_char_p, C.c_int32]
        L.uegccd_list_real.restype = C.c_int32
        L.uegccd_zcode.argtypes = [C.c_char_p, C.c_char_p, C.c_int32]
        L.uegccd_zcode_fort60.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
        L.uegccd_zcode_host_logs.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p]
        L.uegccd_zcode_last_error.restype = C.c_char_p
        _bound = True
    return L


def _check(rc):
    if rc < 0:
        raise _capi.UegccdError(rc, _lib().uegccd_zcode_last_error().decode())
    return rc


def connectivity(system_tuple, core_n: int = 0) -> np.ndarray:
    """MP2.f90:56-87 connectivity histogram of one basis (index q-1 counts |dn|^2 = q)."""
    s = _capi.make_system(*system_tuple)
    conn = np.zeros(CONN_LIMIT, dtype=np.int32)
    _check(_lib().uegccd_connectivity(C.byref(s), core_n, conn.ctypes.data_as(C.POINTER(C.c_int32))))
    return conn


def special_twist(conn: np.ndarray):
    """Main.f90:213-231: (index of the special twist, average histogram, diff2 per twist)."""
    conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, CONN_LIMIT)
    n = conn.shape[0]
    avg = np.zeros(CONN_LIMIT)
    d2 = np.zeros(n)
    best = C.c_int32()
    _check(_lib().uegccd_special_twist(n, conn.ctypes.data_as(C.POINTER(C.c_int32)),
                                       avg.ctypes.data_as(C.POINTER(C.c_double)),
                                       d2.ctypes.data_as(C.POINTER(C.c_double)), C.byref(best)))
    return best.value, avg, d2


def list_real(x: float) -> str:
    """One REAL(8) item as gfortran's list-directed write prints it."""
    buf = C.create_string_buffer(64)
    _check(_lib().uegccd_list_real(float(x), buf, 64))
    return buf.value.decode()


def host_logs(input_path: str = "Input", twists_path: str | None = None, fort60: str = "fort.60",
              fort82: str | None = "fort.82", fort61: str | None = "fort.61") -> None:
    """The program's host set-up alone (no GPU): its fort.60 log, fort.82 exchange
    structure factors and fort.61 core/active electron counts."""
    enc = lambda x: x.encode() if x else None
    _check(_lib().uegccd_zcode_host_logs(enc(input_path), enc(twists_path), enc(fort60), enc(fort82),
                                         enc(fort61)))


def run(input_path: str = "Input", twists_path: str | None = None, diis: bool = False) -> None:
    """The ZCode program in the working directory (writes Output, fort.58-61, fort.80-82)."""
    _check(_lib().uegccd_zcode(input_path.encode(), twists_path.encode() if twists_path else None,
                               _capi.UEGCCD_DIIS if diis else _capi.UEGCCD_REPLAY))


if __name__ == "__main__":
    run(sys.argv[1] if len(sys.argv) > 1 else "Input", sys.argv[2] if len(sys.argv) > 2 else None)

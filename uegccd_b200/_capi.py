"""ctypes binding of the C ABI declared in include/uegccd.h (libuegccd.so).

This is the same binding a Fortran host makes with iso_c_binding: plain
pointers to FP64 arrays in the reference's T(NOcc,NOcc,NOcc+1:NAO) layout.
The library is loaded from the package directory; if it is missing the import
fails loudly -- there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libuegccd.so")

UEGCCD_OK = 0
UEGCCD_NOT_CONVERGED = 1
UEGCCD_ERR_ALLOC = -3
UEGCCD_FP64, UEGCCD_MIXED = 0, 1
UEGCCD_REPLAY, UEGCCD_DIIS = 0, 1


class UegccdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"uegccd error {code}: {msg}")
        self.code = code


class System(C.Structure):
    _fields_ = [
        ("nocc", C.c_int32), ("nao", C.c_int32), ("L", C.c_double), ("madelung", C.c_double),
        ("eigen", C.POINTER(C.c_double)), ("nvec", C.POINTER(C.c_int32)),
    ]


class Options(C.Structure):
    _fields_ = [
        ("do_ring", C.c_int32), ("do_xring", C.c_int32), ("do_ladder", C.c_int32), ("do_mosaic", C.c_int32),
        ("core_n", C.c_int32), ("gapii", C.c_double), ("range_flags", C.c_int32), ("max_iter", C.c_int32),
        ("tol", C.c_double), ("denom_factor", C.c_double), ("fail_ratio", C.c_double), ("scheme", C.c_int32),
        ("ndiis", C.c_int32), ("precision", C.c_int32), ("refine_sweeps", C.c_int32),
        ("energies", C.POINTER(C.c_double)), ("dts", C.POINTER(C.c_double)), ("max_rec", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("ecorr", C.c_double), ("ecorr_sosex", C.c_double), ("max_res", C.c_double), ("last_dt", C.c_double),
        ("niter", C.c_int32), ("fail", C.c_int32), ("n_recorded", C.c_int32), ("kernel_launches", C.c_int32),
        ("gpu_ms", C.c_double), ("status", C.c_int32), ("ndiis", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


EXPORTS = [
    "uegccd_default_options", "uegccd_ctx_create", "uegccd_ctx_destroy", "uegccd_ctx_set_eigen",
    "uegccd_mp2", "uegccd_ccd", "uegccd_drpa", "uegccd_ccd_g2", "uegccd_batch_create",
    "uegccd_batch_destroy", "uegccd_batch_solve", "uegccd_batch_get_amplitudes", "uegccd_last_error",
    "uegccd_version", "uegccd_batch_set_profiling", "uegccd_batch_kernel_stats",
    "uegccd_batch_transfer_bytes", "uegccd_ccd_g2_ex", "uegccd_footprint",
]

_lib = None


class SfGrid(C.Structure):
    _fields_ = [(k, C.POINTER(C.c_double)) for k in ("sum", "dsum", "xsum", "g", "v")]


RANGE_TERMS = ("ring", "xring", "ladder", "mosaic", "driver_direct", "driver_exchange", "energy", "lin_rings",
               "quad_rings", "direct_rings", "exchange_rings", "lin_ladders", "quad_ladders", "direct_ladders",
               "exchange_ladders")


class RangeTerms(C.Structure):
    """UegccdRangeTerms: the fifteen "... Range" Input values, in the Input file's order."""
    _fields_ = [(k, C.c_int32) for k in RANGE_TERMS]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m uegccd_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, dp, vp = C.POINTER, C.POINTER(C.c_double), C.c_void_p
        L.uegccd_default_options.argtypes = [P(Options)]
        L.uegccd_default_options.restype = None
        L.uegccd_ctx_create.argtypes = [P(System), P(vp)]
        L.uegccd_ctx_destroy.argtypes = [vp]
        L.uegccd_ctx_set_eigen.argtypes = [vp, dp]
        L.uegccd_mp2.argtypes = [vp, dp, dp, dp, dp]
        L.uegccd_ccd.argtypes = [vp, P(Options), dp, dp, dp, P(Result)]
        L.uegccd_drpa.argtypes = [vp, P(Options), dp, P(Result)]
        L.uegccd_ccd_g2.argtypes = [vp, dp, C.c_int32, dp]
        L.uegccd_ccd_g2_ex.argtypes = [vp, dp, C.c_int32, C.c_int32, dp]
        L.uegccd_batch_create.argtypes = [P(System), C.c_int32, P(vp)]
        L.uegccd_batch_destroy.argtypes = [vp]
        L.uegccd_batch_solve.argtypes = [vp, P(Options), C.c_int32, dp, P(Result)]
        L.uegccd_batch_get_amplitudes.argtypes = [vp, C.c_int32, dp]
        L.uegccd_batch_get_all_amplitudes.argtypes = [vp, dp]
        L.uegccd_batch_mp2.argtypes = [vp, dp]
        L.uegccd_diis_create.argtypes = [C.c_int64, C.c_int32, C.c_int32, dp, P(vp)]
        L.uegccd_diis_push.argtypes = [vp, dp, dp]
        L.uegccd_diis_get_t.argtypes = [vp, C.c_int32, dp]
        L.uegccd_diis_destroy.argtypes = [vp]
        L.uegccd_ctx_set_integrals.argtypes = [vp, C.c_int32, C.c_double]
        L.uegccd_batch_set_integrals.argtypes = [vp, C.c_int32, C.c_double]
        L.uegccd_ctx_set_range.argtypes = [vp, C.c_int32, C.c_double]
        L.uegccd_ctx_set_eri.argtypes = [vp, P(RangeTerms), C.c_int32, C.c_double]
        L.uegccd_ccd_g2_2ch.argtypes = [vp, dp, dp, C.c_int32, dp, dp]
        L.uegccd_drpa_g2.argtypes = [vp, dp, C.c_int32, dp]
        L.uegccd_batch_set_range.argtypes = [vp, C.c_int32, C.c_double]
        L.uegccd_sf_length.argtypes = [P(System)]
        L.uegccd_sf_length.restype = C.c_int32
        L.uegccd_structure_factor.argtypes = [vp, dp, P(SfGrid)]
        L.uegccd_batch_structure_factor.argtypes = [vp, C.c_int32, P(SfGrid)]
        L.uegccd_batch_set_profiling.argtypes = [vp, C.c_int32]
        L.uegccd_batch_ring_threads.argtypes = [vp, P(C.c_int32), C.c_int32]
        L.uegccd_batch_ring_threads.restype = C.c_int32
        L.uegccd_batch_launch_shapes.argtypes = [vp, P(C.c_int32), C.c_int32]
        L.uegccd_batch_launch_shapes.restype = C.c_int32
        L.uegccd_batch_kernel_stats.argtypes = [vp, C.c_int32, P(C.c_char_p), dp, P(C.c_int64)]
        L.uegccd_batch_transfer_bytes.argtypes = [vp, P(C.c_int64), P(C.c_int64)]
        L.uegccd_footprint.argtypes = [P(System), C.c_int32, C.c_int32, P(C.c_int64), P(C.c_int64)]
        L.uegccd_batch_start.argtypes = [vp, P(Options), C.c_int32, dp]
        L.uegccd_batch_history.argtypes = [vp, C.c_int32, dp, dp, C.c_int32, P(C.c_int32)]
        L.uegccd_batch_advance.argtypes = [vp, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_int32), P(Result)]
        L.uegccd_set_memory_limit.argtypes = [C.c_int64]
        L.uegccd_memory_info.argtypes = [P(C.c_int64), P(C.c_int64)]
        L.uegccd_last_error.restype = C.c_char_p
        L.uegccd_version.restype = C.c_char_p
        _lib = L
    return _lib


def check(rc: int, allow_not_converged: bool = True) -> int:
    if rc < 0 or (rc > 0 and not allow_not_converged):
        raise UegccdError(rc, lib().uegccd_last_error().decode())
    return rc


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def default_options(**kw) -> Options:
    o = Options()
    lib().uegccd_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def make_system(nocc: int, L: float, madelung: float, eigen: np.ndarray, nvec: np.ndarray):
    """nvec: (NAO, 3) integer plane-wave vectors, row p = orbital p+1."""
    eigen = np.ascontiguousarray(eigen, dtype=np.float64)
    # Fortran HEGData%nVec(NAO,3) is column-major: store the transpose in C order
    nv = np.ascontiguousarray(np.asarray(nvec, dtype=np.int32).T)
    s = System(nocc, eigen.shape[0], L, madelung, eigen.ctypes.data_as(C.POINTER(C.c_double)),
               nv.ctypes.data_as(C.POINTER(C.c_int32)))
    s._keep = (eigen, nv)
    return s


def footprint(system_tuple, ndiis: int = 6, mixed: bool = False):
    """(device bytes, allowed amplitudes) of one system; no GPU needed."""
    s = make_system(*system_tuple)
    b, a = C.c_int64(), C.c_int64()
    check(lib().uegccd_footprint(C.byref(s), ndiis, 1 if mixed else 0, C.byref(b), C.byref(a)))
    return b.value, a.value


def set_memory_limit(nbytes: int) -> None:
    """Caps the device memory the library holds per device (0: no cap)."""
    check(lib().uegccd_set_memory_limit(int(nbytes)))


def memory_info():
    """(bytes held, of which cached) on the calling thread's current device."""
    h, c = C.c_int64(), C.c_int64()
    check(lib().uegccd_memory_info(C.byref(h), C.byref(c)))
    return h.value, c.value


def trim_cache() -> None:
    check(lib().uegccd_trim_cache())


_cudart = None


def set_device(device: int) -> None:
    """Makes `device` the calling thread's current CUDA device (the device a batch or
    context created next on this thread lives on)."""
    global _cudart
    lib()   # the library loads the CUDA runtime it uses
    if _cudart is None:
        _cudart = C.CDLL("libcudart.so.12")
    rc = _cudart.cudaSetDevice(C.c_int(int(device)))
    if rc != 0:
        raise UegccdError(-2, f"cudaSetDevice({device}) failed ({rc})")

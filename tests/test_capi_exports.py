"""The C ABI library loads on a machine without a GPU, exports every function that
include/*.h declares, and fails cleanly (status, message) when no device exists."""
import ctypes as C
import os
import re

import pytest

from uegccd_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in ("uegccd.h", "uegccd_host.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(uegccd_\w+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = _capi.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_defaults_are_the_reference_values():
    o = _capi.default_options()
    assert (o.max_iter, o.tol, o.denom_factor, o.fail_ratio) == (1000, 1e-8, 2.0, 100.0)  # CCD.f90:11,36; HEG.f90:1078-1079
    assert (o.do_ring, o.do_xring, o.do_ladder, o.do_mosaic) == (1, 1, 1, 1)
    assert o.scheme == _capi.UEGCCD_REPLAY and o.precision == _capi.UEGCCD_FP64


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU error path")
def test_no_gpu_is_an_error_not_a_fallback():
    import numpy as np

    from uegccd_b200 import Context

    with pytest.raises(_capi.UegccdError) as e:
        Context(7, 3.9, -0.73, np.zeros(19), np.zeros((19, 3), dtype=np.int32))
    assert e.value.code == -2
    assert _capi.lib().uegccd_version().startswith(b"uegccd_b200")


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU error path")
def test_diis_without_gpu_is_an_error():
    h = C.c_void_p()
    rc = _capi.lib().uegccd_diis_create(10, 3, _capi.UEGCCD_DIIS, None, C.byref(h))
    assert rc == -2 and not h.value


def test_argument_checks_without_device_work():
    """Bad arguments are refused before any device call (null handles, sizes, schemes)."""
    L = _capi.lib()
    h = C.c_void_p()
    assert L.uegccd_diis_create(0, 3, _capi.UEGCCD_DIIS, None, C.byref(h)) == -1
    assert L.uegccd_diis_create(10, 17, _capi.UEGCCD_DIIS, None, C.byref(h)) == -1
    assert L.uegccd_diis_create(10, 3, 7, None, C.byref(h)) == -1
    assert L.uegccd_batch_mp2(None, None) == -1
    assert L.uegccd_batch_structure_factor(None, 0, None) == -1
    assert L.uegccd_structure_factor(None, None, None) == -1
    assert L.uegccd_ctx_set_integrals(None, 0, 0.0) == -1
    assert L.uegccd_batch_set_integrals(None, 0, 0.0) == -1
    assert L.uegccd_diis_push(None, None, None) == -1
    assert L.uegccd_diis_get_t(None, 0, None) == -1
    assert L.uegccd_batch_ring_threads(None, None, 0) == -1


def test_sf_length_matches_oracle():
    """uegccd_sf_length (host-only) is the reference's SfLength = 2*maxval(nVec)+1."""
    import numpy as np

    from oracle.oracle import Oracle, parse_input_text

    for vals in ({}, {"# Electrons": "54", "Momentum Cutoff": "24"}):
        v = parse_input_text("")
        v.update(vals)
        o = Oracle(v)
        o.change_twist((0.3, -0.2, 0.45))
        sc = o.scalars()
        s = _capi.make_system(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())
        assert _capi.lib().uegccd_sf_length(C.byref(s)) == o.sf_length() == 2 * int(o.nvec().max()) + 1

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

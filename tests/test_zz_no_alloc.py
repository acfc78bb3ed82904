"""uegccd_mp2_energy_static -- E(2) with no device allocation (its storage is one
fixed array inside the library) -- against uegccd_mp2 through the C ABI.

Two calls in a row on each system must both agree with uegccd_mp2 within 1e-12 Ha
(the two paths sum the same terms in different orders), so the second call shows
that nothing left in the shared array by the first one leaks into its result.
This file is collected last on purpose: it must pass both alone in a fresh process
and after every other GPU test has run in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text

pytestmark = pytest.mark.gpu

TOL = 1e-12
ERR_ARG = -1   # UEGCCD_ERR_ARG, include/uegccd.h


def _systems(goldens):
    g5 = parse_input_text("")
    g5.update(goldens["G5"]["keys"])
    v54 = parse_input_text("")
    v54.update({"# Electrons": "54", "Momentum Cutoff": "24", "rSMin": "2.0", "rSMax": "2.0",
                "NTwist": "0.31 -0.12 0.07"})
    out = []
    for vals in (g5, goldens["G1"]["input_text"], v54):
        o = Oracle(vals)
        sc = o.scalars()
        out.append((o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec()))
    return out


def _static_e2(system_tuple):
    from uegccd_b200 import _capi

    L = _capi.lib()
    L.uegccd_mp2_energy_static.argtypes = [C.POINTER(_capi.System), C.c_void_p, C.POINTER(C.c_double)]
    L.uegccd_mp2_energy_static.restype = C.c_int
    s = _capi.make_system(*system_tuple)
    e = C.c_double(float("nan"))
    rc = L.uegccd_mp2_energy_static(C.byref(s), None, C.byref(e))
    return rc, e.value


def test_static_mp2_matches_mp2_two_calls_in_a_row(goldens):
    from uegccd_b200 import Context

    for sys_t in _systems(goldens):
        e_ref = Context(*sys_t).mp2()[0]
        rc1, e1 = _static_e2(sys_t)
        rc2, e2 = _static_e2(sys_t)
        assert rc1 == 0 and rc2 == 0
        assert abs(e1 - e_ref) < TOL, (e1, e_ref)
        assert abs(e2 - e_ref) < TOL, (e2, e_ref)


def test_static_mp2_alternating_sizes(goldens):
    """A small system after a large one: the lattice and partial sums are re-set per call."""
    from uegccd_b200 import Context

    small, _, large = _systems(goldens)
    refs = [Context(*t).mp2()[0] for t in (large, small)]
    for t, ref in zip((large, small), refs):
        rc, e = _static_e2(t)
        assert rc == 0 and abs(e - ref) < TOL


def test_static_mp2_refuses_oversize():
    from uegccd_b200 import _capi

    M = 2049
    nvec = np.zeros((M, 3), dtype=np.int32)
    nvec[:, 0] = np.arange(M) % 9 - 4
    rc, _ = _static_e2((7, 10.0, 1.0, np.linspace(-1, 1, M), nvec))
    assert rc == ERR_ARG
    assert "2048" in _capi.lib().uegccd_last_error().decode()
    nvec = np.zeros((20, 3), dtype=np.int32)
    nvec[:, 2] = np.arange(20) * 2 - 19     # |n_z| up to 19, and one |n_y| of 32
    nvec[19, 1] = 32
    rc, _ = _static_e2((7, 10.0, 1.0, np.linspace(-1, 1, 20), nvec))
    assert rc == ERR_ARG
    assert "31" in _capi.lib().uegccd_last_error().decode()


def test_static_mp2_leaves_device_memory_unchanged(goldens):
    """The entry point's contract is that it allocates nothing: after one warm-up call, the
    device's free memory (cudaMemGetInfo) stays the same over several more calls, and the
    library's own device-memory count does not move either."""
    from uegccd_b200 import _capi

    rt = C.CDLL("libcudart.so.12")
    free_b, total_b = C.c_size_t(), C.c_size_t()
    held = C.c_int64()
    sys_t = _systems(goldens)[2]
    assert _static_e2(sys_t)[0] == 0   # warm-up: the module and the array are loaded
    assert rt.cudaMemGetInfo(C.byref(free_b), C.byref(total_b)) == 0
    _capi.lib().uegccd_memory_info(C.byref(held), None)
    free0, held0 = free_b.value, held.value
    for _ in range(4):
        assert _static_e2(sys_t)[0] == 0
    assert rt.cudaMemGetInfo(C.byref(free_b), C.byref(total_b)) == 0
    _capi.lib().uegccd_memory_info(C.byref(held), None)
    assert free_b.value == free0
    assert held.value == held0

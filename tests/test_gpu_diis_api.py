"""The DIIS entry points (uegccd_diis_*, the reference's DIISCC module) on the GPU.

* REPLAY gives back the newest T bit for bit, as the reference's singular solve does
  (DIISCC.f90:110-125).
* DIIS: the Pulay combination over the pairs held, against a numpy solve of the same
  system (1e-12 relative), with the reference's NIter >= NDIIS + 5 wait and the
  oldest pair dropped when the history is full.
* A host-side CCD loop (G2 terms from uegccd_ccd_g2, Jacobi step, DIIS) converges to
  the amplitudes of the library's own solve.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Oracle, parse_input_text
from uegccd_b200 import Context
from uegccd_b200 import _capi as capi

pytestmark = pytest.mark.gpu


class Diis:
    def __init__(self, n, ndiis, scheme, t0=None):
        self.n = n
        h = C.c_void_p()
        t0 = None if t0 is None else np.ascontiguousarray(t0, dtype=np.float64)
        capi.check(capi.lib().uegccd_diis_create(n, ndiis, scheme, capi.dptr(t0), C.byref(h)))
        self.h = h

    def push(self, t, r):
        t = np.ascontiguousarray(t, dtype=np.float64)
        r = np.ascontiguousarray(r, dtype=np.float64)
        capi.check(capi.lib().uegccd_diis_push(self.h, capi.dptr(t), capi.dptr(r)))

    def get_t(self, niter):
        out = np.empty(self.n)
        capi.check(capi.lib().uegccd_diis_get_t(self.h, niter, capi.dptr(out)))
        return out

    def __del__(self):
        capi.lib().uegccd_diis_destroy(self.h)


def test_replay_returns_the_newest_t():
    rng = np.random.default_rng(5)
    n = 70001
    t0 = rng.standard_normal(n)
    d = Diis(n, 3, capi.UEGCCD_REPLAY, t0)
    np.testing.assert_array_equal(d.get_t(1), t0)
    for k in range(5):
        t = rng.standard_normal(n)
        d.push(t, rng.standard_normal(n))
        np.testing.assert_array_equal(d.get_t(20 + k), t)


def _pulay(ts, rs):
    m = len(ts)
    B = np.array([[a @ b for b in rs] for a in rs])
    B /= np.max(np.diag(B))
    M = np.zeros((m + 1, m + 1))
    M[:m, :m] = B
    M[:m, m] = M[m, :m] = 1.0
    v = np.zeros(m + 1)
    v[m] = 1.0
    c = np.linalg.solve(M, v)[:m]
    return sum(ci * ti for ci, ti in zip(c, ts))


def test_pulay_matches_numpy():
    rng = np.random.default_rng(6)
    n, ndiis = 123457, 4
    d = Diis(n, ndiis, capi.UEGCCD_DIIS)
    ts, rs = [], []
    for k in range(6):
        t = rng.standard_normal(n)
        r = rng.standard_normal(n) * 0.5 ** k
        d.push(t, r)
        ts.append(t)
        rs.append(r)
    np.testing.assert_array_equal(d.get_t(ndiis + 4), ts[-1])      # before the reference's wait
    got = d.get_t(ndiis + 5)
    want = _pulay(ts[-ndiis:], rs[-ndiis:])                         # the oldest two dropped
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def _valid_partner(o):
    O, M = o.nocc, o.nao
    nv = o.nvec()
    idx = {tuple(nv[p]): p for p in range(M)}
    mask = np.zeros((M - O, O, O), dtype=bool)
    for i in range(O):
        for j in range(O):
            for a in range(O, M):
                if idx.get(tuple(nv[i] + nv[j] - nv[a]), -1) >= O:
                    mask[a - O, j, i] = True
    return mask


def test_host_ccd_loop_with_diis():
    """N=14, rs=1: T <- G/D with the library's G2 and DIIS, to max|dT| < 1e-11."""
    o = Oracle(parse_input_text(""))
    sc = o.scalars()
    ctx = Context(o.nocc, sc["L"], sc["madelung"], o.eigen(), o.nvec())
    _, ta, tb, tc = ctx.mp2()
    mask = _valid_partner(o)
    e = o.eigen()
    O, M = o.nocc, o.nao
    # D(i,j,a) = e_i + e_j - e_a - e_b, b the partner of (i,j,a); 1 where no amplitude exists
    nv = o.nvec()
    idx = {tuple(nv[p]): p for p in range(M)}
    D = np.ones((M - O, O, O))
    for i in range(O):
        for j in range(O):
            for a in range(O, M):
                b = idx.get(tuple(nv[i] + nv[j] - nv[a]), -1)
                if b >= O:
                    D[a - O, j, i] = e[i] + e[j] - e[a] - e[b]
    t = tb.copy()
    d = Diis(t.size, 6, capi.UEGCCD_DIIS, t.ravel())
    for it in range(1, 200):
        g = ctx.ccd_g2(t, 31)
        r = np.where(mask, -g + D * t, 0.0)
        t_new = np.where(mask, g / D, 0.0)
        d.push(t_new.ravel(), r.ravel())
        t_next = d.get_t(it + 6).reshape(t.shape)
        dt = np.abs(t_next - t).max()
        t = t_next
        if dt < 1e-11:
            break
    assert dt < 1e-11 and it < 60
    # the library's own solve (Pulay DIIS on its device history) to the same point
    _, ta2, tb2, tc2 = ctx.mp2()
    rc, r2, _, _ = ctx.ccd(ta2, tb2, tc2, scheme=1, ndiis=6, denom_factor=1.0, tol=1e-12)
    assert rc == 0
    assert np.abs(t - tb2).max() < 1e-10

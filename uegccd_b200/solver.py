"""Python face of the C ABI: one system (context) or many (batch).

Mirrors the reference's driver entry points on the hot path:
    DrvMBPT  (MP2.f90:11)   -> Context.mp2
    DrvCCD   (CCD.f90:18)   -> Context.ccd
    DrvdRPA  (dRPA.f90:23)  -> Context.drpa
    CCEnergyAndSF (CCD.f90:240), the SF of DrvMBPT (MP2.f90:86) -> Context.structure_factor
Amplitude arrays use the reference layout T(NOcc,NOcc,NOcc+1:NAO) column-major,
which is a C-ordered numpy array of shape (V, O, O) indexed [a-O-1, j-1, i-1].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi


def _sf_call(system, call) -> dict:
    """Runs one structure-factor call into fresh (W,W,W) grids indexed [z+S, y+S, x+S]."""
    S = capi.lib().uegccd_sf_length(C.byref(system))
    if S < 0:
        capi.check(S)
    W = 2 * S + 1
    out = {k: np.zeros((W, W, W)) for k in ("sum", "dsum", "xsum", "g", "v")}
    grid = capi.SfGrid(*(capi.dptr(out[k]) for k in ("sum", "dsum", "xsum", "g", "v")))
    capi.check(call(C.byref(grid)))
    out["S"] = S
    return out


class Context:
    """uegccd_ctx_*: the momentum-block plan of one system, resident on the GPU."""

    def __init__(self, nocc: int, L: float, madelung: float, eigen, nvec):
        self.nocc = int(nocc)
        self.nao = int(len(eigen))
        self.nvir = self.nao - self.nocc
        self._sys = capi.make_system(nocc, L, madelung, eigen, nvec)
        h = C.c_void_p()
        capi.check(capi.lib().uegccd_ctx_create(C.byref(self._sys), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            capi.lib().uegccd_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def zeros_t(self) -> np.ndarray:
        return np.zeros((self.nvir, self.nocc, self.nocc))

    def set_eigen(self, eigen) -> None:
        e = np.ascontiguousarray(eigen, dtype=np.float64)
        capi.check(capi.lib().uegccd_ctx_set_eigen(self._h, capi.dptr(e)))

    def set_integrals(self, core_n: int = 0, gapii: float = 0.0) -> None:
        """CoreN and GapII of the integrals for the calls that follow (CoreERI/GapERI)."""
        capi.check(capi.lib().uegccd_ctx_set_integrals(self._h, int(core_n), float(gapii)))

    def set_range(self, flag: int, screening: float = 0.0) -> None:
        """One CasedERI range flag for every CCD term (1 short, 2 long range, 3 none; 0 clears),
        used by the CCD calls whose options carry range_flags != 0."""
        capi.check(capi.lib().uegccd_ctx_set_range(self._h, int(flag), float(screening)))

    def set_eri(self, flags=None, safe_eri: bool = False, screening: float = 0.0) -> None:
        """SetPointers in full for the two-channel form: flags maps the names of
        capi.RANGE_TERMS to the "... Range" Input values (missing: 0).  Every later ccd, drpa,
        ccd_g2_2ch and drpa_g2 takes per-term integral flags; None returns to the spin-adapted
        kernels."""
        if flags is None:
            capi.check(capi.lib().uegccd_ctx_set_eri(self._h, None, 0, 0.0))
            return
        unknown = set(flags) - set(capi.RANGE_TERMS)
        if unknown:
            raise ValueError(f"unknown range terms: {sorted(unknown)}")
        rt = capi.RangeTerms(*[int(flags.get(k, 0)) for k in capi.RANGE_TERMS])
        capi.check(capi.lib().uegccd_ctx_set_eri(self._h, C.byref(rt), 1 if safe_eri else 0, float(screening)))

    def ccd_g2_2ch(self, t_abab, t_abba, mask: int = 31):
        """TermsWrapper on both channels: (G2abab, G2abba) of the selected terms."""
        ga, gb = self.zeros_t(), self.zeros_t()
        ta = np.ascontiguousarray(t_abab, dtype=np.float64)
        tb = np.ascontiguousarray(t_abba, dtype=np.float64)
        capi.check(capi.lib().uegccd_ccd_g2_2ch(self._h, capi.dptr(ta), capi.dptr(tb), mask, capi.dptr(ga),
                                                 capi.dptr(gb)))
        return ga, gb

    def drpa_g2(self, t2, mask: int = 11) -> np.ndarray:
        """The dRPA residual G2 of one amplitude array (bit0 drivers, bit1 mosaics, bit3 rings)."""
        g = self.zeros_t()
        t = np.ascontiguousarray(t2, dtype=np.float64)
        capi.check(capi.lib().uegccd_drpa_g2(self._h, capi.dptr(t), mask, capi.dptr(g)))
        return g

    def mp2(self):
        """DrvMBPT: returns (E2, T2aaaa, T2abab, T2abba)."""
        ta, tb, tc = self.zeros_t(), self.zeros_t(), self.zeros_t()
        e2 = C.c_double()
        capi.check(capi.lib().uegccd_mp2(self._h, capi.dptr(ta), capi.dptr(tb), capi.dptr(tc), C.byref(e2)))
        return e2.value, ta, tb, tc

    def ccd(self, t_aaaa, t_abab, t_abba, max_rec: int = 1100, **opts):
        """DrvCCD: iterates in place; returns (status, result dict, energies, dts)."""
        en, dts = np.zeros(max_rec), np.zeros(max_rec)
        o = capi.default_options(**opts)
        o.energies, o.dts, o.max_rec = capi.dptr(en), capi.dptr(dts), max_rec
        r = capi.Result()
        rc = capi.check(capi.lib().uegccd_ccd(self._h, C.byref(o), capi.dptr(t_aaaa), capi.dptr(t_abab),
                                              capi.dptr(t_abba), C.byref(r)))
        return rc, r.as_dict(), en[: r.n_recorded].copy(), dts[: r.n_recorded].copy()

    def drpa(self, t2, max_rec: int = 1100, **opts):
        """DrvdRPA on one amplitude array (T2aaaa of the MP2 step)."""
        en, dts = np.zeros(max_rec), np.zeros(max_rec)
        o = capi.default_options(**opts)
        o.fail_ratio = opts.get("fail_ratio", 1.0e4)
        o.energies, o.dts, o.max_rec = capi.dptr(en), capi.dptr(dts), max_rec
        r = capi.Result()
        rc = capi.check(capi.lib().uegccd_drpa(self._h, C.byref(o), capi.dptr(t2), C.byref(r)))
        return rc, r.as_dict(), en[: r.n_recorded].copy(), dts[: r.n_recorded].copy()

    def ccd_g2(self, t_abab, mask: int = 31, precision: int = 0) -> np.ndarray:
        """One residual G2 of the selected terms (precision 1: tensor-core ladder)."""
        g = self.zeros_t()
        t = np.ascontiguousarray(t_abab, dtype=np.float64)
        capi.check(capi.lib().uegccd_ccd_g2_ex(self._h, capi.dptr(t), mask, precision, capi.dptr(g)))
        return g

    def structure_factor(self, t_abab) -> dict:
        """CCEnergyAndSF grids of spin-adapted amplitudes: sum, dsum, xsum, g, v and S."""
        t = np.ascontiguousarray(t_abab, dtype=np.float64)
        return _sf_call(self._sys, lambda g: capi.lib().uegccd_structure_factor(self._h, capi.dptr(t), g))


class SystemSet:
    """The UegccdSystem structs of many systems, built once.  A host that creates batch after
    batch of the same systems (a pipeline) passes this to Batch instead of the tuples: the
    conversion holds the interpreter lock, which the other pipeline threads then wait on."""

    def __init__(self, systems):
        self.systems = [capi.make_system(*s) for s in systems]
        self.arr = (capi.System * len(self.systems))(*self.systems)


class Batch:
    """uegccd_batch_*: many independent systems solved together."""

    def __init__(self, systems, device: int | None = None):
        """systems: iterable of (nocc, L, madelung, eigen, nvec), or a SystemSet.  device: the
        CUDA device to create the batch on (made current on this thread first); None: the
        current one.  Every later call on the batch runs on its device, from any thread."""
        if device is not None:
            capi.set_device(device)
        sset = systems if isinstance(systems, SystemSet) else SystemSet(systems)
        self._sset = sset
        self._systems = sset.systems
        arr = sset.arr
        self._arr = arr
        h = C.c_void_p()
        capi.check(capi.lib().uegccd_batch_create(arr, len(self._systems), C.byref(h)))
        self._h = h
        self.n = len(self._systems)
        self._shapes = [(s.nao - s.nocc, s.nocc, s.nocc) for s in self._systems]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            capi.lib().uegccd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, drpa: bool = False, raise_on_error: bool = True, **opts):
        """MP2 start + CCD (dRPA) of every system: (status, E(2) per system, result dicts).
        raise_on_error=False returns a negative status too, with each solve's own status in
        its result (e.g. UEGCCD_ERR_NUMERIC for the solves that met a NaN)."""
        o = capi.default_options(**opts)
        if drpa and "fail_ratio" not in opts:
            o.fail_ratio = 1.0e4
        e2 = np.zeros(self.n)
        res = (capi.Result * self.n)()
        rc = capi.lib().uegccd_batch_solve(self._h, C.byref(o), 1 if drpa else 0, capi.dptr(e2), res)
        if raise_on_error:
            capi.check(rc)
        return rc, e2, [r.as_dict() for r in res]

    def start(self, drpa: bool = False, **opts) -> np.ndarray:
        """Opens an incremental solve (uegccd_batch_start): the MP2 start of every system;
        returns E(2).  advance() then iterates and hands back the solves that stopped."""
        o = capi.default_options(**opts)
        if drpa and "fail_ratio" not in opts:
            o.fail_ratio = 1.0e4
        e2 = np.zeros(self.n)
        capi.check(capi.lib().uegccd_batch_start(self._h, C.byref(o), 1 if drpa else 0, capi.dptr(e2)))
        self._done_ids = (C.c_int32 * self.n)()
        self._done_res = (capi.Result * self.n)()
        return e2

    def advance(self, rounds: int = 1):
        """Up to `rounds` rounds of four iterations; returns (solves still iterating,
        [(solve index, result dict) of every solve that stopped since the last call])."""
        na, nd = C.c_int32(), C.c_int32()
        capi.check(capi.lib().uegccd_batch_advance(self._h, int(rounds), C.byref(na), C.byref(nd), self._done_ids,
                                                     self._done_res))
        return na.value, [(int(self._done_ids[k]), self._done_res[k].as_dict()) for k in range(nd.value)]

    def set_integrals(self, core_n: int = 0, gapii: float = 0.0) -> None:
        """CoreN and GapII of the integrals for the calls that follow (CoreERI/GapERI)."""
        capi.check(capi.lib().uegccd_batch_set_integrals(self._h, int(core_n), float(gapii)))

    def set_range(self, flag: int, screening: float = 0.0) -> None:
        """One CasedERI range flag for every CCD term of every solve (see Context.set_range)."""
        capi.check(capi.lib().uegccd_batch_set_range(self._h, int(flag), float(screening)))

    def mp2(self) -> np.ndarray:
        """DrvMBPT of every system; the MP2 amplitudes stay in the batch.  Returns E(2)."""
        e2 = np.zeros(self.n)
        capi.check(capi.lib().uegccd_batch_mp2(self._h, capi.dptr(e2)))
        return e2

    def structure_factor(self, s: int) -> dict:
        """Structure-factor grids of solve s from the amplitudes the batch holds."""
        return _sf_call(self._systems[s], lambda g: capi.lib().uegccd_batch_structure_factor(self._h, s, g))

    def ring_threads(self) -> list:
        """CTA size of each ring pair class (after the first CCD solve: the tuned ones)."""
        a = (C.c_int32 * 8)()
        n = capi.lib().uegccd_batch_ring_threads(self._h, a, 8)
        if n < 0:
            capi.check(n)
        return list(a[:n])

    def launch_shapes(self) -> dict:
        """The tuner's picks (after the first CCD solve): ring CTA sizes per class, the ring
        staging CTA size, the ladder tile order (0 block order, 1 longest first), the hole-hole
        intermediate's column chunk."""
        a = (C.c_int32 * 8)()
        n = capi.lib().uegccd_batch_launch_shapes(self._h, a, 8)
        if n < 0:
            capi.check(n)
        v = list(a[:n])
        return {"ring_threads": v[:4], "stage_threads": v[4], "ladder_order": "longest first" if v[5] else "block",
                "hh_chunk": v[6]}

    def set_profiling(self, on: bool) -> None:
        capi.check(capi.lib().uegccd_batch_set_profiling(self._h, 1 if on else 0))

    def kernel_stats(self) -> dict:
        n = 16
        names = (C.c_char_p * n)()
        ms = np.zeros(n)
        la = np.zeros(n, dtype=np.int64)
        k = capi.lib().uegccd_batch_kernel_stats(self._h, n, names, capi.dptr(ms),
                                                   la.ctypes.data_as(C.POINTER(C.c_int64)))
        return {names[i].decode(): (float(ms[i]), int(la[i])) for i in range(k)}

    def transfer_bytes(self):
        h, d = C.c_int64(), C.c_int64()
        capi.check(capi.lib().uegccd_batch_transfer_bytes(self._h, C.byref(h), C.byref(d)))
        return h.value, d.value

    def amplitudes(self, s: int) -> np.ndarray:
        t = np.zeros(self._shapes[s])
        capi.check(capi.lib().uegccd_batch_get_amplitudes(self._h, s, capi.dptr(t)))
        return t

    def history(self, s: int, max_rec: int = 1100):
        """Solve s's per-iteration energies and max|dT| from the last batch solve."""
        en, dt = np.zeros(max_rec), np.zeros(max_rec)
        n = C.c_int32()
        capi.check(capi.lib().uegccd_batch_history(self._h, int(s), capi.dptr(en), capi.dptr(dt), int(max_rec),
                                                    C.byref(n)))
        return en[: n.value].copy(), dt[: n.value].copy()

    def amplitude_count(self) -> int:
        """Doubles that all_amplitudes fills (every solve's NOcc^2 (NAO - NOcc))."""
        return sum(int(np.prod(sh)) for sh in self._shapes)

    def all_amplitudes(self, out: np.ndarray | None = None) -> list:
        """T2abab of every solve (views into one host buffer, one device-to-host copy);
        out: a float64 buffer of amplitude_count() entries to fill (page-locked memory
        takes the copy directly)."""
        sizes = [int(np.prod(sh)) for sh in self._shapes]
        buf = np.empty(sum(sizes)) if out is None else out
        assert buf.dtype == np.float64 and buf.flags["C_CONTIGUOUS"] and buf.size == sum(sizes)
        capi.check(capi.lib().uegccd_batch_get_all_amplitudes(self._h, capi.dptr(buf)))
        views, off = [], 0
        for sh, n in zip(self._shapes, sizes):
            views.append(buf[off:off + n].reshape(sh))
            off += n
        return views

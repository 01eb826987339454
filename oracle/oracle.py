"""oracle.py — TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

Two checkers live under oracle/:
  * liboracle.so — my C restatement of the reference tracking path (accel_oracle.c), built by
    oracle/Makefile; it takes the same accel_elem_desc descriptors as the engine.
  * _ref/libaccel_ref.so — the reference library itself (its own sources, compiled here by the
    same Makefile) behind a C shim (ref_shim.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs import this
module, and only to check or to time the CPU path; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libaccel_ref.so")

_port = None
_ref = None


def port_available() -> bool:
    return os.path.exists(PORT_PATH)


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def port():
    global _port
    if _port is None:
        L = C.CDLL(PORT_PATH)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        L.orc_pass_element.argtypes = [P, P, I, P]
        L.orc_pass_line.argtypes = [P, I, P, I, I, I, I, P]
        L.orc_track.argtypes = [P, I, P, I, I, P, I, C.c_uint64]
        L.orc_m66.argtypes = [P, I, I, I, D, D, P]
        L.orc_m66_at.argtypes = [P, I, I, I, P, D, P]
        L.orc_beam_stat.argtypes = [P, I, P, P, P]
        L.orc_set_flags.argtypes = [P, I, I, I, I]
        L.orc_longwake_voltage.argtypes = [I, D, P, D, D, D, D, P]
        for f in ("orc_pass_element", "orc_pass_line", "orc_track", "orc_beam_stat"):
            getattr(L, f).restype = I
        L.orc_m66.restype = None
        L.orc_m66_at.restype = None
        L.orc_set_flags.restype = None
        L.orc_longwake_voltage.restype = None
        _port = L
    return _port


def _arr(elems):
    """Contiguous ctypes array of descriptors (any ctypes Structure with the header's layout)."""
    if isinstance(elems, C.Array):
        return elems
    T = type(elems[0])
    return (T * len(elems))(*elems)


def port_track(elems, r: np.ndarray, nturn: int, loss: bool = True, nthreads: int = 1,
               seed: int = 1) -> np.ndarray | None:
    """Track AoS r (N x 6, float64, updated in place) nturn turns; returns loss turns or None."""
    arr = _arr(elems)
    r = np.ascontiguousarray(r)
    n = r.size // 6
    lt = np.empty(n, dtype=np.int32) if loss else None
    s = port().orc_track(arr, len(arr), r.ctypes.data, n, nturn,
                         lt.ctypes.data if loss else None, nthreads, seed)
    if s != 0:
        raise RuntimeError(f"orc_track status {s}")
    return lt


def port_pass_line(elems, r: np.ndarray, st: int, ed: int, nthreads: int = 1) -> None:
    arr = _arr(elems)
    s = port().orc_pass_line(arr, len(arr), r.ctypes.data, r.size // 6, st, ed, nthreads, None)
    if s != 0:
        raise RuntimeError(f"orc_pass_line status {s}")


def port_m66(elems, dpp=0.0, delta=1e-8, st=0, ed=None) -> np.ndarray:
    arr = _arr(elems)
    ed = len(arr) if ed is None else ed
    m = np.zeros(36)
    port().orc_m66(arr, len(arr), st, ed, dpp, delta, m.ctypes.data)
    return m.reshape(6, 6)


def port_m66_at(elems, r0, delta=1e-8, st=0, ed=None) -> np.ndarray:
    arr = _arr(elems)
    ed = len(arr) if ed is None else ed
    p = np.ascontiguousarray(r0, dtype=np.float64)
    m = np.zeros(36)
    port().orc_m66_at(arr, len(arr), st, ed, p.ctypes.data, delta, m.ctypes.data)
    return m.reshape(6, 6)


def port_set_flags(elems, rad=-1, cavity=-1, wake=-1):
    """ALine::set_rad_onoff / set_cavity_onoff / set_wake_onoff on a list of descriptors, in place."""
    arr = _arr(elems)
    port().orc_set_flags(arr, len(arr), rad, cavity, wake)
    if not isinstance(elems, C.Array):
        for i, d in enumerate(elems):
            C.memmove(C.byref(d), C.byref(arr[i]), C.sizeof(d))
    return elems


def port_beam_stat(r: np.ndarray):
    r = np.ascontiguousarray(r, dtype=np.float64)
    mean, sig, cross = np.zeros(6), np.zeros(6), np.zeros(6)
    nl = port().orc_beam_stat(r.ctypes.data, r.size // 6, mean.ctypes.data, sig.ctypes.data,
                              cross.ctypes.data)
    return mean, sig, cross, nl


# ---- the reference library --------------------------------------------------------------------
def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_PATH)
        P, I, D, S = C.c_void_p, C.c_int, C.c_double, C.c_char_p
        pd = C.POINTER(C.c_double)
        sig = {
            "ref_line_load": (P, [S]), "ref_line_free": (None, [P]), "ref_line_nelem": (I, [P]),
            "ref_set_threads": (None, [I]), "ref_max_threads": (I, []),
            "ref_set_crab": (None, [P, I]),
            "ref_pass": (None, [P, P, I, I]), "ref_pass_range": (None, [P, P, I, I, I]),
            "ref_track_loss": (None, [P, P, I, I, P]),
            "ref_track_loss_last": (None, [P, P, I, I, P, P]),
            "ref_m66": (None, [P, I, I, D, D, P]),
            "ref_calc_tune": (None, [P, pd, pd]), "ref_calc_chrom": (None, [P, pd, pd]),
            "ref_correct_chrom": (None, [P, S, S, S, pd, pd]),
            "ref_correct_tune": (None, [P, S, S, S, pd, pd]),
            "ref_setrfphase": (D, [P]), "ref_set_rad": (None, [P, I]),
            "ref_set_cavity": (None, [P, I]), "ref_set_wake": (None, [P, I]),
            "ref_set_energy": (None, [P, D]),
            "ref_set_poly": (I, [P, I, I, I, D]), "ref_get_poly": (I, [P, I, I, I, pd]),
            "ref_set_double_field": (I, [P, I, S, D]), "ref_get_double_field": (I, [P, I, S, pd]),
            "ref_set_nslice": (I, [P, I, I]), "ref_srand": (None, [C.c_uint]),
            "ref_grandn": (D, []),
            "ref_trackDA": (D, [P, D, D, D, I, I, I, P, P]),
            "ref_trackMA": (D, [P, D, D, I, I, P, P, I, P]),
            "ref_beam_stat": (I, [P, I, P, P, P]), "ref_getco4": (None, [P, D, P]),
            "ref_trackDiffusion": (D, [P, I, I, P, P, P, P, P, D, D, D, D]),
            "ref_tracktune": (None, [P, I, D, D, D, D, D, D, pd, pd]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ref = L
    return _ref


class RefLine:
    """The reference's ALine loaded from a lattice file (ALine::deserialize)."""

    def __init__(self, path: str):
        self.h = ref().ref_line_load(path.encode())
        if not self.h:
            raise RuntimeError(f"reference could not load {path}")

    def __del__(self):
        try:
            if self.h:
                ref().ref_line_free(self.h)
        except Exception:
            pass

    def __len__(self):
        return ref().ref_line_nelem(self.h)

    def track(self, r: np.ndarray, nturn: int, threads: int = 1) -> np.ndarray:
        ref().ref_set_threads(threads)
        ref().ref_pass(self.h, r.ctypes.data, r.size // 6, nturn)
        return r

    def pass_range(self, r: np.ndarray, st: int, ed: int, threads: int = 1) -> np.ndarray:
        ref().ref_set_threads(threads)
        ref().ref_pass_range(self.h, r.ctypes.data, r.size // 6, st, ed)
        return r

    def track_loss(self, r: np.ndarray, nturn: int, threads: int = 1, last=None) -> np.ndarray:
        """Loss turns (-1: survived) by a per-turn NaN scan; with `last` (N x 6), each particle's
        state at the end of the last turn it survived."""
        ref().ref_set_threads(threads)
        lt = np.empty(r.size // 6, dtype=np.int32)
        if last is None:
            ref().ref_track_loss(self.h, r.ctypes.data, r.size // 6, nturn, lt.ctypes.data)
        else:
            ref().ref_track_loss_last(self.h, r.ctypes.data, r.size // 6, nturn, lt.ctypes.data,
                                      last.ctypes.data)
        return lt

    def m66(self, dpp=0.0, delta=1e-8, st=0, ed=None) -> np.ndarray:
        ed = len(self) if ed is None else ed
        m = np.zeros(36)
        ref().ref_m66(self.h, st, ed, dpp, delta, m.ctypes.data)
        return m.reshape(6, 6)

    def tune(self):
        a, b = C.c_double(), C.c_double()
        ref().ref_calc_tune(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def chrom(self):
        a, b = C.c_double(), C.c_double()
        ref().ref_calc_chrom(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def correct_chrom(self, fam1: str, fam2: str, cx: float, cy: float, type_="StrMPole"):
        a, b = C.c_double(cx), C.c_double(cy)
        ref().ref_correct_chrom(self.h, type_.encode(), fam1.encode(), fam2.encode(),
                                C.byref(a), C.byref(b))
        return a.value, b.value

    def correct_tune(self, fam1: str, fam2: str, nux: float, nuy: float, type_="StrMPole"):
        a, b = C.c_double(nux), C.c_double(nuy)
        ref().ref_correct_tune(self.h, type_.encode(), fam1.encode(), fam2.encode(),
                               C.byref(a), C.byref(b))
        return a.value, b.value

    def setrfphase(self) -> float:
        return ref().ref_setrfphase(self.h)

    def set_crab(self, on):
        ref().ref_set_crab(self.h, int(bool(on)))

    def set_flags(self, rad=None, cavity=None, wake=None):
        if rad is not None:
            ref().ref_set_rad(self.h, rad)
        if cavity is not None:
            ref().ref_set_cavity(self.h, int(cavity))
        if wake is not None:
            ref().ref_set_wake(self.h, int(wake))

    def set_poly(self, idx, index, value, skew=False):
        if ref().ref_set_poly(self.h, idx, int(skew), index, value) != 0:
            raise RuntimeError("set_poly failed")

    def get_poly(self, idx, index, skew=False) -> float:
        v = C.c_double()
        if ref().ref_get_poly(self.h, idx, int(skew), index, C.byref(v)) != 0:
            raise RuntimeError("get_poly failed")
        return v.value

    def get_field(self, idx, name) -> float:
        v = C.c_double()
        ref().ref_get_double_field(self.h, idx, name.encode(), C.byref(v))
        return v.value

    def set_field(self, idx, name, value):
        ref().ref_set_double_field(self.h, idx, name.encode(), value)

    def trackDA(self, xmax, xmin, ymax, nturn, nray, nstep, threads=1):
        ref().ref_set_threads(threads)
        rx, ry = np.zeros(nray), np.zeros(nray)
        area = ref().ref_trackDA(self.h, xmax, xmin, ymax, nturn, nray, nstep, rx.ctypes.data,
                                 ry.ctypes.data)
        return area, rx, ry

    def trackDiffusion(self, nturn, x0, y0, xlow=0.0, xhi=0.5, ylow=0.0, yhi=0.5):
        """ALine::trackDiffusion: (nux, nuy, dif, total) of the points (x0[i], y0[i])."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        n = len(x0)
        nux, nuy, dif = np.zeros(n), np.zeros(n), np.zeros(n)
        tot = ref().ref_trackDiffusion(self.h, nturn, n, x0.ctypes.data, y0.ctypes.data, nux.ctypes.data,
                                       nuy.ctypes.data, dif.ctypes.data, xlow, xhi, ylow, yhi)
        return nux, nuy, dif, tot

    def tracktune(self, nturn, x0, y0, xlow=0.0, xhi=0.5, ylow=0.0, yhi=0.5):
        a, b = C.c_double(), C.c_double()
        ref().ref_tracktune(self.h, nturn, x0, y0, xlow, xhi, ylow, yhi, C.byref(a), C.byref(b))
        return a.value, b.value

    def trackMA(self, dppmax, dppmin, nturn, nstep, lfam, threads=1):
        ref().ref_set_threads(threads)
        lf = np.ascontiguousarray(lfam, dtype=np.int32)
        dp, dm = np.zeros(len(lf)), np.zeros(len(lf))
        avg = ref().ref_trackMA(self.h, dppmax, dppmin, nturn, nstep, dp.ctypes.data,
                                dm.ctypes.data, len(lf), lf.ctypes.data)
        return avg, dp, dm

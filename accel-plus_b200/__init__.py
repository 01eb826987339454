"""accel-plus_b200 — Python binding of the B200 tracking engine's C-ABI (include/accel_gpu.h).

The engine itself is libaccelgpu.so (CUDA for sm_100a plus its C++ host layer, built in-tree by
the Makefile beside this file).  This module is a thin ctypes layer over it, used by the test
suite and the benchmark; it never computes a tracking result itself, and every call fails
loudly (AccelError) when the library or a CUDA device is missing.

The directory name carries a hyphen, so import it with importlib:

    accel = importlib.import_module("accel-plus_b200")
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Iterable, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaccelgpu.so")

# ---- constants (mirror include/accel_gpu.h) -------------------------------------------------
OK, E_INVALID, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_IO, E_TIMEOUT, E_NODEVICE, E_TOO_LARGE = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)
DRIFT, QUAD, CORRECTOR, APERTURE, MONITOR, BEND, BENDMPOLE, STRMPOLE, CAVITY = range(1, 10)
WIGTABLE, IDEALWIG, CRABCAV, RFMULT, TRANSWAKE, MATRIX, SYNCRAD, LONGWAKE = range(10, 18)
TYPE_NAMES = {DRIFT: "Drift", QUAD: "Quad", CORRECTOR: "Corrector", APERTURE: "Aperture",
              MONITOR: "Monitor", BEND: "Bend", BENDMPOLE: "BendMPole", STRMPOLE: "StrMPole",
              CAVITY: "Cavity", WIGTABLE: "WigTable", IDEALWIG: "IdealWig", CRABCAV: "CrabCav",
              RFMULT: "RFMult", TRANSWAKE: "TransWake", MATRIX: "Matrix", SYNCRAD: "SyncRad",
              LONGWAKE: "LongWake"}
MAX_MPOLE = 10
RAD_OFF, RAD_RAD, RAD_RADQE, RAD_LUMP, RAD_LUMP_DAMP, RAD_LUMP_QE = range(6)
(F_LENGTH, F_K, F_POLYNOMB, F_POLYNOMA, F_NSLICE, F_MAXNPOLE, F_ANGLE, F_E1, F_E2, F_VOLTAGE,
 F_FREQUENCY, F_PHIS, F_ENERGY, F_KICKX, F_KICKY, F_XLIM, F_YLIM) = range(1, 18)
MODE_FUSED, MODE_PLAIN, MODE_EXACT = 0, 1, 2
LAYOUT_AOS, LAYOUT_SOA = 0, 1


class ElemDesc(C.Structure):
    """accel_elem_desc: one lattice element (field meanings per type in accel_gpu.h)."""
    _fields_ = [("type", C.c_int32), ("nslice", C.c_int32), ("max_npole", C.c_int32),
                ("flags", C.c_int32), ("len", C.c_double), ("f", C.c_double * 12),
                ("poly_a", C.c_double * MAX_MPOLE), ("poly_b", C.c_double * MAX_MPOLE),
                ("mat", C.c_double * 36), ("famname", C.c_char * 48)]

    @property
    def name(self) -> str:
        return self.famname.decode()

    @property
    def type_name(self) -> str:
        return TYPE_NAMES.get(self.type, "undefined")

    def copy(self) -> "ElemDesc":
        d = ElemDesc()
        C.memmove(C.byref(d), C.byref(self), C.sizeof(ElemDesc))
        return d


class AccelError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: status {status} ({detail})")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """Load libaccelgpu.so; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AccelError(E_UNSUPPORTED, "load", f"{LIB_PATH} is missing: run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    P, I, D = C.c_void_p, C.c_int, C.c_double
    pd = C.POINTER(ElemDesc)
    sig = {
        "accel_status_string": (C.c_char_p, [I]),
        "accel_last_error": (C.c_char_p, []),
        "accel_version": (I, []),
        "accel_device_count": (I, [C.POINTER(I)]),
        "accel_ctx_create": (I, [I, C.POINTER(P)]),
        "accel_ctx_destroy": (I, [P]),
        "accel_nccl_unique_id": (I, [C.c_char_p]),
        "accel_ctx_set_comm": (I, [P, C.c_char_p, I, I]),
        "accel_lattice_read": (I, [C.c_char_p, C.POINTER(pd), C.POINTER(I)]),
        "accel_lattice_parse": (I, [C.c_char_p, C.POINTER(pd), C.POINTER(I)]),
        "accel_lattice_write": (I, [C.c_char_p, pd, I, I]),
        "accel_lattice_free": (None, [pd]),
        "accel_state_write": (I, [C.c_char_p, P, C.c_int64, C.c_int64, P]),
        "accel_state_read": (I, [C.c_char_p, C.POINTER(C.POINTER(D)), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_int32))]),
        "accel_state_free": (None, [P]),
        "accel_wigtable_create": (I, [I, I, P, P, P, P, C.POINTER(C.c_int32)]),
        "accel_wigtable_info": (I, [C.c_int32, C.POINTER(I), C.POINTER(I)]),
        "accel_wigtable_get": (I, [C.c_int32, P, P, P, P]),
        "accel_wigtable_destroy": (I, [C.c_int32]),
        "accel_elem_default": (I, [I, pd]),
        "accel_line_create": (I, [P, pd, I, C.POINTER(P)]),
        "accel_line_destroy": (I, [P]),
        "accel_line_count": (I, [P, C.POINTER(I)]),
        "accel_line_get_desc": (I, [P, I, pd]),
        "accel_line_set_field": (I, [P, I, I, I, C.POINTER(D)]),
        "accel_line_get_field": (I, [P, I, I, I, C.POINTER(D)]),
        "accel_line_set_flags": (I, [P, I, I, I]),
        "accel_line_set_energy": (I, [P, D]),
        "accel_line_set_crab_onoff": (I, [P, I, C.POINTER(I)]),
        "accel_line_setrfphase": (I, [P, C.POINTER(D)]),
        "accel_line_set_seed": (I, [P, C.c_uint64]),
        "accel_track": (I, [P, P, I, I, I, I, I, P, I, P]),
        "accel_track_batched": (I, [P, I, P, P, C.c_int64, I, P, I, P]),
        "accel_autotune": (I, [P, I, P, P, C.c_int64, C.POINTER(I)]),
        "accel_set_tile": (I, [P, I, I, I]),
        "accel_get_tile": (I, [P, C.POINTER(I)]),
        "accel_set_stage_wait": (I, [P, I]),
        "accel_m66": (I, [P, I, I, D, D, I, C.POINTER(D)]),
        "accel_m66_at": (I, [P, I, I, C.POINTER(D), I, D, C.POINTER(D)]),
        "accel_m66_knob": (I, [P, I, I, C.POINTER(D), I, P, P, P, C.POINTER(D), C.POINTER(D)]),
        "accel_correct_tune": (I, [P, P, I, P, I, C.POINTER(D), C.POINTER(D), I, I, C.POINTER(I)]),
        "accel_correct_chrom": (I, [P, P, I, P, I, C.POINTER(D), C.POINTER(D), I, I, C.POINTER(I)]),
        "accel_adjoint_create": (I, [P, I, I, I, P, P, P, I, C.POINTER(P)]),
        "accel_adjoint_destroy": (I, [P]),
        "accel_adjoint_forward": (I, [P, P, P]),
        "accel_adjoint_backward": (I, [P, P, P, P]),
        "accel_beam_stat": (I, [P, P, I, I, C.POINTER(D), C.POINTER(D), C.POINTER(D), C.POINTER(I)]),
        "accel_beam_stat_noalloc": (I, [P, I, C.c_int64, P, P]),
        "accel_naff": (I, [P, I, D, D, C.POINTER(D)]),
        "accel_track_diffusion": (I, [P, I, I, P, P, P, P, P, D, D, D, D, I, C.POINTER(D)]),
        "accel_track_tune": (I, [P, I, D, D, D, D, D, D, I, C.POINTER(D), C.POINTER(D)]),
        "accel_fp64_peak": (I, [P, C.POINTER(D)]),
        "accel_fp64_peak_clocked": (I, [P, C.POINTER(D), C.POINTER(D)]),
        "accel_set_device_memory_limit": (I, [C.c_int64]),
        "accel_set_adjoint_tape_budget": (I, [C.c_int64]),
        "accel_device_memory_held": (I, [C.POINTER(C.c_int64)]),
        "accel_launch_count": (I, [P, C.POINTER(C.c_int64)]),
        "accel_transwake_pair_passes": (I, [P, C.POINTER(C.c_int64)]),
        "accel_profile_enable": (I, [P, I]),
        "accel_profile_read": (I, [P, C.POINTER(D), C.POINTER(C.c_int64), C.POINTER(D)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Every entry point include/accel_gpu.h declares, in declaration order."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "accel_gpu.h")
    with open(hdr) as f:
        text = f.read()
    return re.findall(r"^\s*(?:const char\*|int|void)\s+(accel_\w+)\s*\(", text, re.M)


def _check(status: int, where: str) -> None:
    if status != OK:
        L = lib()
        detail = (L.accel_last_error() or b"").decode() or L.accel_status_string(status).decode()
        raise AccelError(status, where, detail)


def status_string(s: int) -> str:
    return lib().accel_status_string(s).decode()


# ---- lattice files (host only) ------------------------------------------------------------------
def _take_desc(p, n) -> list[ElemDesc]:
    out = [p[i].copy() for i in range(n.value)]
    lib().accel_lattice_free(p)
    return out


def read_lattice(path: str) -> list[ElemDesc]:
    """Read an Accel+ lattice file (AccelElement::deserialize format)."""
    p, n = C.POINTER(ElemDesc)(), C.c_int()
    _check(lib().accel_lattice_read(path.encode(), C.byref(p), C.byref(n)), "accel_lattice_read")
    return _take_desc(p, n)


def parse_lattice(text: str) -> list[ElemDesc]:
    p, n = C.POINTER(ElemDesc)(), C.c_int()
    _check(lib().accel_lattice_parse(text.encode(), C.byref(p), C.byref(n)), "accel_lattice_parse")
    return _take_desc(p, n)


def write_lattice(path: str, elems: Sequence[ElemDesc], precision: int = 17) -> None:
    arr = (ElemDesc * len(elems))(*elems)
    _check(lib().accel_lattice_write(path.encode(), arr, len(elems), precision), "accel_lattice_write")


def elem(type_: int, famname: str = "undefined", length: float = 0.0, **kw) -> ElemDesc:
    """Build a descriptor with the reference constructor's defaults, then apply keywords:
    f=[...], poly_a=[...], poly_b=[...], mat=[...], nslice, max_npole, flags."""
    d = ElemDesc()
    _check(lib().accel_elem_default(type_, C.byref(d)), "accel_elem_default")
    d.famname = famname.encode()
    d.len = length
    for k, v in kw.items():
        if k in ("f", "poly_a", "poly_b", "mat"):
            arr = getattr(d, k)
            for i, x in enumerate(v):
                arr[i] = float(x)
        else:
            setattr(d, k, v)
    if type_ in (BEND, BENDMPOLE) and length != 0:
        d.f[4] = d.f[0] / length
    return d


def write_state(path: str, r, turn: int = 0, loss=None) -> None:
    """Lossless particle-state checkpoint (accel_state_write): r is (N, 6) float64 on the host."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    lt = None if loss is None else np.ascontiguousarray(loss, dtype=np.int32)
    _check(lib().accel_state_write(path.encode(), C.c_void_p(r.ctypes.data), r.size // 6, int(turn),
                                   None if lt is None else C.c_void_p(lt.ctypes.data)), "accel_state_write")


def read_state(path: str):
    """(r (N, 6), turn, loss turns or None) from a checkpoint written by write_state."""
    pr, pl = C.POINTER(C.c_double)(), C.POINTER(C.c_int32)()
    n, turn = C.c_int64(), C.c_int64()
    _check(lib().accel_state_read(path.encode(), C.byref(pr), C.byref(n), C.byref(turn), C.byref(pl)),
           "accel_state_read")
    r = np.ctypeslib.as_array(pr, shape=(max(1, n.value) * 6,))[: 6 * n.value].reshape(n.value, 6).copy()
    loss = None
    if pl:
        loss = np.ctypeslib.as_array(pl, shape=(max(1, n.value),))[: n.value].copy()
        lib().accel_state_free(C.cast(pl, C.c_void_p))
    lib().accel_state_free(C.cast(pr, C.c_void_p))
    return r, turn.value, loss


def set_device_memory_limit(nbytes: int | None) -> None:
    """Cap the device memory this process's library holds (None or a negative value: no cap);
    a request beyond it fails with E_NOMEM before any allocation (accel_set_device_memory_limit)."""
    _check(lib().accel_set_device_memory_limit(-1 if nbytes is None else int(nbytes)),
           "accel_set_device_memory_limit")


def set_adjoint_tape_budget(nbytes: int | None) -> None:
    """Device memory each tape of an adjoint created afterwards may take (None or <= 0: the
    default, 4e9 bytes); accel_set_adjoint_tape_budget."""
    _check(lib().accel_set_adjoint_tape_budget(0 if nbytes is None else int(nbytes)),
           "accel_set_adjoint_tape_budget")


def device_memory_held() -> int:
    """Bytes of device memory the library's buffers hold, all devices together."""
    v = C.c_int64()
    _check(lib().accel_device_memory_held(C.byref(v)), "accel_device_memory_held")
    return v.value


def wigtable(xl, yl, xkick, ykick) -> int:
    """Register a WigTable kick table (accel_wigtable_create) and return its id, the value of a
    WigTable descriptor's f[0].  xkick and ykick are [len(yl)][len(xl)]: kick[i][j] at
    (xl[j], yl[i])."""
    xl = np.ascontiguousarray(xl, dtype=np.float64)
    yl = np.ascontiguousarray(yl, dtype=np.float64)
    xk = np.ascontiguousarray(xkick, dtype=np.float64)
    yk = np.ascontiguousarray(ykick, dtype=np.float64)
    if xk.shape != (len(yl), len(xl)) or yk.shape != xk.shape:
        raise ValueError("kick tables must be [len(yl)][len(xl)]")
    tid = C.c_int32()
    _check(lib().accel_wigtable_create(len(xl), len(yl), C.c_void_p(xl.ctypes.data), C.c_void_p(yl.ctypes.data),
                                       C.c_void_p(xk.ctypes.data), C.c_void_p(yk.ctypes.data), C.byref(tid)),
           "accel_wigtable_create")
    return tid.value


def wigtable_get(tid: int):
    """(xl, yl, xkick, ykick) of a registered table (accel_wigtable_info / accel_wigtable_get)."""
    mx, my = C.c_int(), C.c_int()
    _check(lib().accel_wigtable_info(tid, C.byref(mx), C.byref(my)), "accel_wigtable_info")
    xl, yl = np.empty(mx.value), np.empty(my.value)
    xk, yk = np.empty((my.value, mx.value)), np.empty((my.value, mx.value))
    _check(lib().accel_wigtable_get(tid, C.c_void_p(xl.ctypes.data), C.c_void_p(yl.ctypes.data),
                                    C.c_void_p(xk.ctypes.data), C.c_void_p(yk.ctypes.data)), "accel_wigtable_get")
    return xl, yl, xk, yk


def wigtable_destroy(tid: int) -> None:
    _check(lib().accel_wigtable_destroy(tid), "accel_wigtable_destroy")


def desc_array(elems: Sequence[ElemDesc]):
    return (ElemDesc * len(elems))(*elems)


# ---- device objects ---------------------------------------------------------------------------
def device_count() -> int:
    n = C.c_int()
    _check(lib().accel_device_count(C.byref(n)), "accel_device_count")
    return n.value


def _process_nccl():
    """Load torch (when present) before the library loads NCCL: libtorch links its own
    libnccl.so.2, and a process can hold only one library of that name.  The library's dlopen then
    returns torch's copy instead of loading another one that torch could not use."""
    try:
        import torch  # noqa: F401
    except ImportError:
        pass


def naff(record, xlow: float = 0.0, xhi: float = 0.5) -> float:
    """Tune of a turn-by-turn record (accel_naff; host only)."""
    x = np.ascontiguousarray(record, dtype=np.float64)
    nu = C.c_double()
    _check(lib().accel_naff(C.c_void_p(x.ctypes.data), len(x), xlow, xhi, C.byref(nu)), "accel_naff")
    return nu.value


def nccl_unique_id() -> bytes:
    """A new NCCL communicator id (accel_nccl_unique_id), to be shared with the other ranks."""
    _process_nccl()
    buf = C.create_string_buffer(128)
    _check(lib().accel_nccl_unique_id(buf), "accel_nccl_unique_id")
    return buf.raw


class Context:
    """One CUDA device: streams, scratch buffers, tuned tiles (accel_ctx)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        _check(lib().accel_ctx_create(device, C.byref(self.h)), "accel_ctx_create")

    def close(self):
        """Release the context handle.  The library keeps it alive for lines still open on it, so
        handles may be closed (or garbage-collected) in any order."""
        if self.h:
            lib().accel_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_comm(self, uid: bytes, nranks: int, rank: int):
        """Join a bunch spread over nranks GPUs (accel_ctx_set_comm); uid from nccl_unique_id()
        on rank 0, the same bytes on every rank.  Blocks until every rank has joined."""
        if len(uid) != 128:
            raise ValueError("uid must be 128 bytes")
        _process_nccl()
        _check(lib().accel_ctx_set_comm(self.h, uid, nranks, rank), "accel_ctx_set_comm")

    def set_tile(self, block=0, seg_turns=0, variant=-1):
        _check(lib().accel_set_tile(self.h, block, seg_turns, variant), "accel_set_tile")

    def set_stage_wait(self, probes: int = 0):
        """accel_set_stage_wait: the staged schedule's first-wait probes (0 default, < 0 none)."""
        _check(lib().accel_set_stage_wait(self.h, int(probes)), "accel_set_stage_wait")

    def get_tile(self):
        t = (C.c_int * 3)()
        _check(lib().accel_get_tile(self.h, t), "accel_get_tile")
        return tuple(t)

    def fp64_peak(self) -> float:
        v = C.c_double()
        _check(lib().accel_fp64_peak(self.h, C.byref(v)), "accel_fp64_peak")
        return v.value

    def fp64_peak_clocked(self) -> tuple[float, float]:
        """(TFLOP/s, SM MHz during the fastest probe run): accel_fp64_peak_clocked."""
        v, m = C.c_double(), C.c_double()
        _check(lib().accel_fp64_peak_clocked(self.h, C.byref(v), C.byref(m)), "accel_fp64_peak_clocked")
        return v.value, m.value

    def launch_count(self) -> int:
        v = C.c_int64()
        _check(lib().accel_launch_count(self.h, C.byref(v)), "accel_launch_count")
        return v.value

    def transwake_pair_passes(self) -> int:
        """Fused-mode transverse wake passes that fell back to the O(N^2) pair sum."""
        v = C.c_int64()
        _check(lib().accel_transwake_pair_passes(self.h, C.byref(v)), "accel_transwake_pair_passes")
        return v.value

    def profile(self, on: bool):
        """Issue tracking launches directly with CUDA events around every tracking kernel."""
        _check(lib().accel_profile_enable(self.h, int(on)), "accel_profile_enable")

    def profile_read(self):
        """(summed tracking-kernel ms, their launch count, whole-call ms) of the last call."""
        f, t, n = C.c_double(), C.c_double(), C.c_int64()
        _check(lib().accel_profile_read(self.h, C.byref(f), C.byref(n), C.byref(t)), "accel_profile_read")
        return f.value, n.value, t.value

    def beam_stat(self, r, layout=LAYOUT_AOS, n=None):
        ptr, n = _ptr_and_n(r, n, layout)
        mean, sig, cross = (C.c_double * 6)(), (C.c_double * 6)(), (C.c_double * 6)()
        nl = C.c_int()
        _check(lib().accel_beam_stat(self.h, ptr, layout, n, mean, sig, cross, C.byref(nl)),
               "accel_beam_stat")
        return np.array(mean), np.array(sig), np.array(cross), nl.value


def beam_stat_noalloc(r, out, layout=LAYOUT_AOS, n=None, stream=None):
    """accel_beam_stat_noalloc: beam moments of a device tensor into the device tensor `out`
    (19 float64: mean[6], sigma[6], cross[6], live count), without any device allocation.
    Returns once the kernels are queued on `stream` (None = the legacy default stream)."""
    for name, t in (("r", r), ("out", out)):
        if not hasattr(t, "data_ptr") or not getattr(t, "is_cuda", False):
            raise ValueError(f"{name} must be a CUDA tensor")
        if str(t.dtype) != "torch.float64" or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float64 tensor")
    if out.device != r.device:
        raise ValueError("r and out must be on the same device")
    if out.numel() < 19:
        raise ValueError("out must hold 19 doubles")
    ptr, n = _ptr_and_n(r, n, layout)
    if n <= 0 or 6 * n > r.numel():
        raise ValueError(f"n = {n} particles needs {6 * n} doubles; r holds {r.numel()}")
    s = C.c_void_p(stream) if stream is not None else None
    _check(lib().accel_beam_stat_noalloc(ptr, layout, n, C.c_void_p(out.data_ptr()), s),
           "accel_beam_stat_noalloc")


def _ptr_and_n(r, n=None, layout=LAYOUT_AOS):
    """Pointer of a numpy array (host) or a torch tensor / object with data_ptr (device)."""
    if isinstance(r, np.ndarray):
        if r.dtype != np.float64 or not r.flags.c_contiguous:
            raise ValueError("state must be a C-contiguous float64 array")
        ptr = r.ctypes.data
        size = r.size
    elif hasattr(r, "data_ptr"):
        if not r.is_contiguous():
            raise ValueError("state tensor must be contiguous")
        ptr = r.data_ptr()
        size = r.numel()
    else:
        raise TypeError("state must be a numpy array or a tensor")
    if n is None:
        if size % 6:
            raise ValueError("state size is not a multiple of 6")
        n = size // 6
    return C.c_void_p(ptr), n


def _iptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype != np.int32 or not a.flags.c_contiguous:
            raise ValueError("loss array must be C-contiguous int32")
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())


class Line:
    """A lattice uploaded to a context (accel_line), with the reference ALine's pass API."""

    def __init__(self, ctx: Context, elems: Sequence[ElemDesc]):
        self.ctx = ctx
        self.h = C.c_void_p()
        arr = desc_array(elems)
        _check(lib().accel_line_create(ctx.h, arr, len(elems), C.byref(self.h)), "accel_line_create")

    def close(self):
        """Release the line handle (the library keeps it for adjoints still open on it)."""
        if self.h:
            lib().accel_line_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        n = C.c_int()
        _check(lib().accel_line_count(self.h, C.byref(n)), "accel_line_count")
        return n.value

    def desc(self, i: int) -> ElemDesc:
        d = ElemDesc()
        _check(lib().accel_line_get_desc(self.h, i, C.byref(d)), "accel_line_get_desc")
        return d

    def descs(self) -> list[ElemDesc]:
        return [self.desc(i) for i in range(len(self))]

    def set_field(self, idx: int, field: int, value, index: int = 0):
        v = (C.c_double * 2)(*np.atleast_1d(np.asarray(value, dtype=np.float64))[:2])
        _check(lib().accel_line_set_field(self.h, idx, field, index, v), "accel_line_set_field")

    def get_field(self, idx: int, field: int, index: int = 0):
        v = (C.c_double * 2)()
        _check(lib().accel_line_get_field(self.h, idx, field, index, v), "accel_line_get_field")
        return v[0] if field not in (F_XLIM, F_YLIM) else (v[0], v[1])

    def set_flags(self, rad=-1, cavity=-1, wake=-1):
        _check(lib().accel_line_set_flags(self.h, rad, cavity, wake), "accel_line_set_flags")

    def set_crab(self, on: bool) -> int:
        """ALine::set_crab_onoff: every CrabCav on or off; returns their number."""
        n = C.c_int()
        _check(lib().accel_line_set_crab_onoff(self.h, int(bool(on)), C.byref(n)), "accel_line_set_crab_onoff")
        return n.value

    def set_energy(self, en: float):
        _check(lib().accel_line_set_energy(self.h, en), "accel_line_set_energy")

    def setrfphase(self) -> float:
        v = C.c_double()
        _check(lib().accel_line_setrfphase(self.h, C.byref(v)), "accel_line_setrfphase")
        return v.value

    def set_seed(self, seed: int):
        _check(lib().accel_line_set_seed(self.h, C.c_uint64(seed)), "accel_line_set_seed")

    def track(self, r, nturn: int = 1, st: int = 0, ed: int | None = None, loss=None,
              mode: int = MODE_FUSED, layout: int = LAYOUT_AOS, stream=None, n=None):
        """ALine::pass(r, N, nturn) / pass(r, N, st, ed): r is updated in place."""
        ptr, n = _ptr_and_n(r, n, layout)
        ed = len(self) if ed is None else ed
        s = C.c_void_p(stream) if stream is not None else None
        _check(lib().accel_track(self.h, ptr, layout, n, st, ed, nturn, _iptr(loss), mode, s),
               "accel_track")
        return r

    def track_diffusion(self, nturn, x0, y0, xlow=0.0, xhi=0.5, ylow=0.0, yhi=0.5, mode=MODE_FUSED):
        """ALine::trackDiffusion (accel_track_diffusion): (nux, nuy, dif, total) of the points."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        n = len(x0)
        nux, nuy, dif = np.zeros(n), np.zeros(n), np.zeros(n)
        tot = C.c_double()
        _check(lib().accel_track_diffusion(self.h, nturn, n, C.c_void_p(x0.ctypes.data), C.c_void_p(y0.ctypes.data),
                                           C.c_void_p(nux.ctypes.data), C.c_void_p(nuy.ctypes.data),
                                           C.c_void_p(dif.ctypes.data), xlow, xhi, ylow, yhi, mode,
                                           C.byref(tot)), "accel_track_diffusion")
        return nux, nuy, dif, tot.value

    def track_tune(self, nturn, x0, y0, xlow=0.0, xhi=0.5, ylow=0.0, yhi=0.5, mode=MODE_FUSED):
        """ALine::tracktune (accel_track_tune): (tunex, tuney) of one starting point."""
        a, b = C.c_double(), C.c_double()
        _check(lib().accel_track_tune(self.h, nturn, x0, y0, xlow, xhi, ylow, yhi, mode, C.byref(a), C.byref(b)),
               "accel_track_tune")
        return a.value, b.value

    def m66(self, dpp=0.0, delta=1e-8, method=0, st=0, ed=None) -> np.ndarray:
        m = (C.c_double * 36)()
        ed = len(self) if ed is None else ed
        _check(lib().accel_m66(self.h, st, ed, dpp, delta, method, m), "accel_m66")
        return np.array(m).reshape(6, 6)

    def m66_knob(self, knob, r0=(0, 0, 0, 0, 0, 0), st=0, ed=None):
        """(m66, dm66/dknob) for a knob moving the (element, field, index) coefficients in `knob`
        together (accel_m66_knob): exact, from hyper-dual numbers."""
        knob = list(knob)
        e = np.array([k[0] for k in knob], dtype=np.int32)
        f = np.array([k[1] for k in knob], dtype=np.int32)
        i = np.array([k[2] for k in knob], dtype=np.int32)
        m, dm = (C.c_double * 36)(), (C.c_double * 36)()
        p = (C.c_double * 6)(*[float(x) for x in r0])
        ed = len(self) if ed is None else ed
        _check(lib().accel_m66_knob(self.h, st, ed, p, len(knob), C.c_void_p(e.ctypes.data), C.c_void_p(f.ctypes.data),
                                    C.c_void_p(i.ctypes.data), m, dm), "accel_m66_knob")
        return np.array(m).reshape(6, 6), np.array(dm).reshape(6, 6)

    def _correct(self, fn, fam1, fam2, a, b, method, maxit):
        f1 = np.ascontiguousarray(fam1, dtype=np.int32)
        f2 = np.ascontiguousarray(fam2, dtype=np.int32)
        x, y, it = C.c_double(a), C.c_double(b), C.c_int(0)
        _check(fn(self.h, C.c_void_p(f1.ctypes.data), len(f1), C.c_void_p(f2.ctypes.data), len(f2),
                  C.byref(x), C.byref(y), method, maxit, C.byref(it)), fn.__name__)
        return x.value, y.value, it.value

    def correct_tune(self, fam1, fam2, tunex, tuney, method=0, maxit=8):
        """accel_correct_tune: (achieved x, y, iterations); method 0 exact Newton, 1 the reference's fit."""
        return self._correct(lib().accel_correct_tune, fam1, fam2, tunex, tuney, method, maxit)

    def correct_chrom(self, fam1, fam2, chromx, chromy, method=0, maxit=8):
        """accel_correct_chrom: (achieved x, y, iterations); method 0 exact Newton, 1 the reference's fit."""
        return self._correct(lib().accel_correct_chrom, fam1, fam2, chromx, chromy, method, maxit)

    def m66_at(self, r0, method=0, delta=1e-8, st=0, ed=None) -> np.ndarray:
        m = (C.c_double * 36)()
        p = (C.c_double * 6)(*[float(x) for x in r0])
        ed = len(self) if ed is None else ed
        _check(lib().accel_m66_at(self.h, st, ed, p, method, delta, m), "accel_m66_at")
        return np.array(m).reshape(6, 6)


def _line_array(lines: Sequence[Line]):
    return (C.c_void_p * len(lines))(*[l.h.value for l in lines])


def track_batched(lines: Sequence[Line], part_off: np.ndarray, r_soa, nturn: int, loss=None,
                  mode: int = MODE_FUSED, stream=None):
    """Track many lattice instances in one launch; r_soa is 6 x Ntot (SoA), a device tensor or a
    host array (numpy, or a pinned CPU tensor), updated in place; loss likewise host or device."""
    off = np.ascontiguousarray(part_off, dtype=np.int64)
    ntot = int(off[-1])
    if isinstance(r_soa, np.ndarray):
        if r_soa.dtype != np.float64 or not r_soa.flags.c_contiguous or r_soa.size != 6 * ntot:
            raise ValueError("r_soa must be a C-contiguous float64 array of 6 x Ntot")
        ptr = r_soa.ctypes.data
    else:
        if not r_soa.is_contiguous() or r_soa.numel() != 6 * ntot or str(r_soa.dtype) != "torch.float64":
            raise ValueError("r_soa must be a contiguous float64 tensor of 6 x Ntot")
        ptr = r_soa.data_ptr()
    s = C.c_void_p(stream) if stream is not None else None
    _check(lib().accel_track_batched(_line_array(lines), len(lines), C.c_void_p(off.ctypes.data),
                                     C.c_void_p(ptr), ntot, nturn, _iptr(loss), mode, s),
           "accel_track_batched")


def autotune(lines: Sequence[Line], part_off: np.ndarray, r_soa) -> tuple:
    off = np.ascontiguousarray(part_off, dtype=np.int64)
    t = (C.c_int * 3)()
    _check(lib().accel_autotune(_line_array(lines), len(lines), C.c_void_p(off.ctypes.data),
                                C.c_void_p(r_soa.data_ptr()), int(off[-1]), t), "accel_autotune")
    return tuple(t)


class Adjoint:
    """accel_adjoint_forward / accel_adjoint_backward pair for one line."""

    def __init__(self, line: Line, n: int, nturn: int, ckpt_every: int,
                 params: Iterable[tuple[int, int, int]]):
        params = list(params)
        pe = np.array([p[0] for p in params], dtype=np.int32)
        pf = np.array([p[1] for p in params], dtype=np.int32)
        pi = np.array([p[2] for p in params], dtype=np.int32)
        self._keep = (pe, pf, pi)
        self.nparam = len(params)
        self.n = n
        self.line = line
        self.h = C.c_void_p()
        _check(lib().accel_adjoint_create(line.h, n, nturn, ckpt_every,
                                          C.c_void_p(pe.ctypes.data), C.c_void_p(pf.ctypes.data),
                                          C.c_void_p(pi.ctypes.data), self.nparam, C.byref(self.h)),
               "accel_adjoint_create")

    def close(self):
        if self.h:
            lib().accel_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, r0: np.ndarray) -> np.ndarray:
        r0 = np.ascontiguousarray(r0, dtype=np.float64)
        out = np.empty_like(r0)
        _check(lib().accel_adjoint_forward(self.h, C.c_void_p(r0.ctypes.data),
                                           C.c_void_p(out.ctypes.data)), "accel_adjoint_forward")
        return out

    def backward(self, g: np.ndarray):
        g = np.ascontiguousarray(g, dtype=np.float64)
        dr0 = np.empty_like(g)
        dp = np.zeros(max(1, self.nparam))
        _check(lib().accel_adjoint_backward(self.h, C.c_void_p(g.ctypes.data),
                                            C.c_void_p(dr0.ctypes.data), C.c_void_p(dp.ctypes.data)),
               "accel_adjoint_backward")
        return dr0, dp[: self.nparam]

"""ctypes binding of librgf's C ABI (include/rgf.h).

This is the Python counterpart of the MEX gateway: plain structs and
pointers, no torch types.  Loading fails loudly when the shared library is
missing -- there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes
import os
import threading
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_void_p
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "librgf.so"

RGF_OK, RGF_ERR_ARG, RGF_ERR_NONFINITE, RGF_ERR_SINGULAR, RGF_ERR_TIMEOUT, RGF_ERR_CUDA, RGF_ERR_OOM, \
    RGF_ERR_NODEVICE, RGF_ERR_ILLCOND = range(9)
STATUS_NAMES = {0: "RGF_OK", 1: "RGF_ERR_ARG", 2: "RGF_ERR_NONFINITE", 3: "RGF_ERR_SINGULAR",
                4: "RGF_ERR_TIMEOUT", 5: "RGF_ERR_CUDA", 6: "RGF_ERR_OOM", 7: "RGF_ERR_NODEVICE",
                8: "RGF_ERR_ILLCOND"}

BC_PERIODIC, BC_DIRICHLET, BC_NEUMANN, BC_DIRICHLET_NEUMANN, BC_NEUMANN_DIRICHLET, BC_BLOCH = range(6)
RGF_ALL = -1
RGF_FP64 = 0
RGF_TF32X3 = 1  # split-precision form (3xTF32 factorization + FP64 refinement)
RGF_NOALLOC_SCRATCH_BYTES = 32 << 20  # include/rgf.h
RGF_NOALLOC_SCRATCH_BYTES = 32 << 20  # include/rgf.h


class Cplx(ctypes.Structure):
    _fields_ = [("re", c_double), ("im", c_double)]


def cplx(z) -> Cplx:
    z = complex(z)
    return Cplx(z.real, z.imag)


class Syst2D(ctypes.Structure):
    _fields_ = [("ny", c_int64), ("nx", c_int64), ("epsilon", c_void_p), ("eps_on_device", c_int32),
                ("epsilon_L", Cplx), ("epsilon_R", Cplx), ("k0dx", Cplx), ("yBC", c_int32), ("ka", c_double)]


class Syst3D(ctypes.Structure):
    _fields_ = [("nx", c_int64), ("ny", c_int64), ("nz", c_int64), ("epsilon", c_void_p),
                ("eps_on_device", c_int32), ("epsilon_L", Cplx), ("epsilon_R", Cplx), ("k0dx", Cplx),
                ("xyBC", c_int32), ("kxa", c_double), ("kya", c_double)]


class Request(ctypes.Structure):
    _fields_ = [("ind_out_L", c_void_p), ("n_out_L", c_int64), ("ind_out_R", c_void_p), ("n_out_R", c_int64),
                ("ind_in_L", c_void_p), ("n_in_L", c_int64), ("ind_in_R", c_void_p), ("n_in_R", c_int64)]


class Options(ctypes.Structure):
    _fields_ = [("precision", c_int32), ("engine", c_int32), ("S_on_device", c_int32), ("profile", c_int32)]


class Channels(ctypes.Structure):
    _fields_ = [("kydx", c_void_p), ("kxdx_t", c_void_p), ("kxdx_L", c_void_p), ("kxdx_R", c_void_p),
                ("sqrt_mu_L", c_void_p), ("sqrt_mu_R", c_void_p), ("ind_prop_L", c_void_p),
                ("ind_prop_R", c_void_p), ("ind_prop_conj_L", c_void_p), ("ind_prop_conj_R", c_void_p),
                ("N_prop_L", c_int64), ("N_prop_R", c_int64), ("has_prop_conj", c_int32), ("reserved", c_int32)]


# every symbol include/rgf.h declares, with its ctypes signature
SIGNATURES = {
    "rgf_create": (c_int, [c_int, POINTER(c_void_p)]),
    "rgf_destroy": (c_int, [c_void_p]),
    "rgf_smatrix_2d": (c_int, [c_void_p, POINTER(Syst2D), POINTER(Request), POINTER(Options), c_void_p, c_int64,
                               POINTER(Channels)]),
    "rgf_smatrix_3d": (c_int, [c_void_p, POINTER(Syst3D), POINTER(Request), POINTER(Options), c_void_p, c_int64,
                               POINTER(Channels)]),
    "rgf_smatrix_batch_2d": (c_int, [c_void_p, c_int64, POINTER(Syst2D), POINTER(Request), POINTER(Options),
                                     POINTER(c_void_p), POINTER(c_int64), POINTER(c_int), c_int32]),
    "rgf_smatrix_grad_2d": (c_int, [c_void_p, POINTER(Syst2D), POINTER(Request), POINTER(Options), c_void_p,
                                    c_int64, c_void_p, c_int64, c_void_p, c_int64]),
    "rgf_smatrix_grad_3d": (c_int, [c_void_p, POINTER(Syst3D), POINTER(Request), POINTER(Options), c_void_p,
                                    c_int64, c_void_p, c_int64, c_void_p, c_int64]),
    "rgf_fields_2d": (c_int, [c_void_p, POINTER(Syst2D), POINTER(Request), POINTER(Options), c_void_p, c_int64,
                              c_void_p, c_int64]),
    "rgf_fields_3d": (c_int, [c_void_p, POINTER(Syst3D), POINTER(Request), POINTER(Options), c_void_p, c_int64,
                              c_void_p, c_int64]),
    "rgf_segment_sweep_2d": (c_int, [c_void_p, POINTER(Syst2D), POINTER(Request), POINTER(Options), c_int32,
                                     c_int64, c_void_p]),
    "rgf_segment_sweep_3d": (c_int, [c_void_p, POINTER(Syst3D), POINTER(Request), POINTER(Options), c_int32,
                                     c_int64, c_void_p]),
    "rgf_segment_merge_2d": (c_int, [c_void_p, POINTER(Syst2D), POINTER(Request), POINTER(Options), c_void_p,
                                     c_void_p, c_void_p, c_int64]),
    "rgf_segment_merge_3d": (c_int, [c_void_p, POINTER(Syst3D), POINTER(Request), POINTER(Options), c_void_p,
                                     c_void_p, c_void_p, c_int64]),
    "rgf_smatrix_size_2d": (c_int, [c_void_p, POINTER(Syst2D), POINTER(Request), POINTER(c_int64),
                                    POINTER(c_int64)]),
    "rgf_smatrix_size_3d": (c_int, [c_void_p, POINTER(Syst3D), POINTER(Request), POINTER(c_int64),
                                    POINTER(c_int64)]),
    "rgf_setup_channels_2d": (c_int, [c_void_p, c_int64, c_int32, c_double, Cplx, Cplx, Cplx, c_int32,
                                      POINTER(Channels)]),
    "rgf_setup_channels_3d": (c_int, [c_void_p, c_int64, c_int64, c_int32, c_double, c_double, Cplx, Cplx, Cplx,
                                      c_int32, POINTER(Channels)]),
    "rgf_build_laplacian_1d": (c_int, [c_void_p, c_int64, c_int32, c_double, c_void_p]),
    "rgf_last_error": (c_char_p, []),
    "rgf_version": (c_char_p, []),
    "rgf_last_stats": (c_int, [c_void_p, POINTER(c_int64), POINTER(c_double)]),
    "rgf_last_engine": (c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_double)]),
    "rgf_last_refinement": (c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_double),
                                    POINTER(c_double), POINTER(c_double)]),
    "rgf_last_profile": (c_int, [c_void_p, POINTER(c_int64), POINTER(c_double), POINTER(c_double), c_char_p,
                                 ctypes.c_size_t]),
    "rgf_set_stream": (c_int, [c_void_p, c_void_p]),
    "rgf_set_tile_table": (c_int, [c_void_p, c_int32, c_void_p, c_void_p]),
    "rgf_smatrix_2d_noalloc": (c_int, [POINTER(Syst2D), POINTER(Request), POINTER(Options), c_void_p, c_int64,
                                       POINTER(Channels), c_void_p]),
}

_lib = None
_lock = threading.Lock()


class RGFError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load() -> ctypes.CDLL:
    """Load librgf.so (built in-tree by ``python -m rgf_b200.build``)."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(f"librgf.so not found at {LIB_PATH}; build it with `python -m rgf_b200.build`")
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


class IllConditionedWarning(UserWarning):
    """A slice inverse failed its a-posteriori check even under partial
    pivoting over the whole column (RGF_ERR_ILLCOND): the result is returned
    but may be inaccurate -- where MATLAB's inv warns that the matrix is close
    to singular or badly scaled."""


def check(status: int) -> None:
    if status == RGF_ERR_ILLCOND:
        import warnings
        msg = load().rgf_last_error()
        warnings.warn(msg.decode() if msg else "ill-conditioned slice matrix", IllConditionedWarning, stacklevel=3)
        return
    if status != RGF_OK:
        msg = load().rgf_last_error()
        raise RGFError(status, msg.decode() if msg else "")


class Handle:
    """Owns one rgf_handle (device workspace + stream)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = c_void_p()
        check(self.lib.rgf_create(int(device), ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.rgf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr) -> None:
        check(self.lib.rgf_set_stream(self.h, c_void_p(stream_ptr) if stream_ptr else None))

    def profile(self):
        n = c_int64()
        ms = c_double()
        fl = c_double()
        name = ctypes.create_string_buffer(128)
        check(self.lib.rgf_last_profile(self.h, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(fl), name, 128))
        return int(n.value), float(ms.value), float(fl.value), name.value.decode()

    def engine(self):
        """(engine, fallback, rejected probe residual) of the last S-matrix call."""
        e, f, r = c_int32(), c_int32(), c_double()
        check(self.lib.rgf_last_engine(self.h, ctypes.byref(e), ctypes.byref(f), ctypes.byref(r)))
        return int(e.value), int(f.value), float(r.value)

    def refinement(self):
        """Split-precision form of the last S-matrix call: dict with form
        (RGF_TF32X3 when its S stands, -RGF_TF32X3 after a fallback to FP64,
        RGF_FP64 when not asked for), iterations, last_change, factor_ms,
        solve_ms."""
        f, it = c_int32(), c_int32()
        ch, fm, sm = c_double(), c_double(), c_double()
        check(self.lib.rgf_last_refinement(self.h, ctypes.byref(f), ctypes.byref(it), ctypes.byref(ch),
                                           ctypes.byref(fm), ctypes.byref(sm)))
        return {"form": int(f.value), "iterations": int(it.value), "last_change": float(ch.value),
                "factor_ms": float(fm.value), "solve_ms": float(sm.value)}

    def stats(self):
        n = c_int64()
        r = c_double()
        check(self.lib.rgf_last_stats(self.h, ctypes.byref(n), ctypes.byref(r)))
        return int(n.value), float(r.value)


_tls = threading.local()


def default_handle(device: int = 0, mode: str = "latency") -> Handle:
    """This thread's handle on `device`, with the tuned tile table of this GPU
    model (rgf_b200/tuned, written by rgf_b200.autotune) installed when there
    is one: the fastest tiles for single S-matrices (mode "latency") or the
    fewest SM-microseconds for batches (mode "throughput")."""
    hs = getattr(_tls, "handles", None)
    if hs is None:
        hs = _tls.handles = {}
    key = (device, mode)
    if key not in hs:
        h = Handle(device)
        _install_tuned(h, mode)
        hs[key] = h
    return hs[key]


def _install_tuned(h: Handle, mode: str) -> None:
    from . import autotune
    # the table is keyed by the GPU model and SM count, read here from torch
    # when it is importable
    try:
        import torch
        p = torch.cuda.get_device_properties(h.device)
        name, sms = p.name, p.multi_processor_count
    except Exception:
        return
    table = autotune.load(name, sms)
    if table:
        autotune.install(h, table, mode)


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size else None


def index_array(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.int64).reshape(-1))

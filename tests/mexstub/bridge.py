"""Python side of the MEX stand-in (test infrastructure): converts Python
values to the stub's mxArrays, calls the gateway's mexFunction, converts the
results back.  MATLAB semantics: column-major arrays, 1-based channel
indices, cell arrays as lists, 1x1 structs as dicts."""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_size_t, c_void_p

import numpy as np

LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmexstub.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        L.stub_double.restype = c_void_p
        L.stub_double.argtypes = [c_size_t, POINTER(c_size_t), c_void_p, c_void_p]
        L.stub_char.restype = c_void_p
        L.stub_char.argtypes = [c_char_p]
        L.stub_cell.restype = c_void_p
        L.stub_cell.argtypes = [c_size_t, POINTER(c_void_p)]
        L.stub_struct.restype = c_void_p
        L.stub_struct.argtypes = [c_int, POINTER(c_char_p), POINTER(c_void_p)]
        L.stub_info.restype = c_int
        L.stub_info.argtypes = [c_void_p, POINTER(c_size_t), POINTER(c_int), POINTER(c_int)]
        L.stub_read.argtypes = [c_void_p, c_void_p, c_void_p]
        L.stub_field.restype = c_void_p
        L.stub_field.argtypes = [c_void_p, c_char_p]
        L.stub_destroy.argtypes = [c_void_p]
        L.stub_err_id.restype = c_char_p
        L.stub_err_msg.restype = c_char_p
        L.stub_warning.restype = c_char_p
        L.stub_warning.argtypes = [c_int]
        L.stub_call.restype = c_int
        L.stub_call.argtypes = [c_int, POINTER(c_void_p), c_int, POINTER(c_void_p)]
        _lib = L
    return _lib


class MexError(Exception):
    def __init__(self, ident, msg):
        super().__init__(f"{ident}: {msg}")
        self.ident = ident
        self.msg = msg


def to_mx(v):
    L = lib()
    if isinstance(v, str):
        return L.stub_char(v.encode())
    if isinstance(v, dict):
        names = (c_char_p * len(v))(*[k.encode() for k in v])
        vals = (c_void_p * len(v))(*[to_mx(x) for x in v.values()])
        return L.stub_struct(len(v), names, vals)
    if isinstance(v, (list, tuple)):
        el = (c_void_p * len(v))(*[to_mx(x) for x in v])
        return L.stub_cell(len(v), el)
    a = np.asarray(v)
    if a.ndim < 2:
        a = a.reshape(1, -1) if a.ndim == 1 else a.reshape(1, 1)
    dims = (c_size_t * a.ndim)(*a.shape)
    re = np.asfortranarray(a.real, dtype=float)
    im = np.asfortranarray(a.imag, dtype=float) if np.iscomplexobj(a) else None
    return L.stub_double(a.ndim, dims, re.ctypes.data, im.ctypes.data if im is not None else None)


def from_mx(p):
    L = lib()
    dims = (c_size_t * 8)()
    kind, cplx = c_int(), c_int()
    nd = L.stub_info(p, dims, ctypes.byref(kind), ctypes.byref(cplx))
    shape = tuple(dims[i] for i in range(nd))
    if kind.value == 0:
        n = int(np.prod(shape))
        re = np.zeros(max(n, 1))
        im = np.zeros(max(n, 1))
        L.stub_read(p, re.ctypes.data, im.ctypes.data)
        out = (re[:n] + 1j * im[:n]) if cplx.value else re[:n]
        return out.reshape(shape, order="F")
    raise TypeError("only numeric results are read back directly; use field()")


def field(p, name):
    f = lib().stub_field(p, name.encode())
    if not f:
        raise KeyError(name)
    return f


def call(nlhs, *args):
    """[out1, ..., out_nlhs] = rgf_mex(args...) -> (list of mxArray pointers, warnings)."""
    L = lib()
    prhs = (c_void_p * len(args))(*[to_mx(a) for a in args])
    plhs = (c_void_p * max(nlhs, 1))()
    rc = L.stub_call(nlhs, plhs, len(args), prhs)
    warns = [L.stub_warning(i).decode() for i in range(L.stub_nwarnings())]
    for i in range(len(args)):
        L.stub_destroy(prhs[i])
    if rc:
        raise MexError(L.stub_err_id().decode(), L.stub_err_msg().decode())
    return [plhs[i] for i in range(nlhs)], warns


def destroy(p):
    lib().stub_destroy(p)

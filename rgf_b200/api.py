"""Python mirror of the reference's MATLAB interface, on top of the C ABI.

    cal_smatrix_RGF(syst, out, in_)      <- src/cal_smatrix_RGF.m:1
    cal_smatrix_RGF_3D(syst, out, in_)   <- src/cal_smatrix_RGF_3D.m:1
    setup_channels(ny, BC, k0dx, eL, eR) <- src/setup_channels.m:1
    setup_channels_3D(nx, ny, BC, ...)   <- src/setup_channels_3D.m:1
    build_laplacian_1d(n, BC)            <- src/build_laplacian_1d.m:1

Argument meaning, channel ordering, 1-based channel indices and error
behaviour follow the MATLAB functions (``syst`` is a dict or any object with
the same fields, ``out``/``in_`` a dict (MATLAB struct) or a list (MATLAB
cell)).  Deviation: a numeric ``yBC`` (Bloch phase ka) is accepted by
cal_smatrix_RGF although cal_smatrix_RGF.m:89 rejects it; its help text
(:32-34) and setup_channels.m:105-111 support it.

All arithmetic runs on the GPU through librgf; errors surface as
``ValueError`` (invalid input, the MATLAB ``error`` cases) or
``rgf_b200._abi.RGFError`` (device-side failures).
"""
from __future__ import annotations

import ctypes
import warnings
from typing import Any, Dict

import numpy as np

from . import _abi
from ._abi import RGF_ALL, Channels, Options, Request, Syst2D, Syst3D, check, cplx, ptr

__all__ = ["cal_smatrix_RGF", "cal_smatrix_RGF_3D", "setup_channels", "setup_channels_3D",
           "build_laplacian_1d"]


# ---------------------------------------------------------------------------
# argument helpers
# ---------------------------------------------------------------------------
def _get(s, k):
    return s[k] if isinstance(s, dict) else getattr(s, k)


def _has(s, k):
    return (k in s) if isinstance(s, dict) else hasattr(s, k)


def _is_num_scalar(x) -> bool:
    return np.isscalar(x) and isinstance(x, (int, float, complex, np.number)) and not isinstance(x, bool)


def _bc_2d(BC):
    """BC argument -> (rgf_bc, ka) (setup_channels.m:98-159)."""
    if isinstance(BC, str):
        b = BC.lower()
        if b == "bloch":
            raise ValueError("To use Bloch periodic boundary condition, set BC to k*a where k is the Bloch wave "
                             "number and a is the periodicity")
        table = {"periodic": _abi.BC_PERIODIC, "dirichlet": _abi.BC_DIRICHLET, "pec": _abi.BC_DIRICHLET,
                 "neumann": _abi.BC_NEUMANN, "pmc": _abi.BC_NEUMANN,
                 "dirichletneumann": _abi.BC_DIRICHLET_NEUMANN, "pecpmc": _abi.BC_DIRICHLET_NEUMANN,
                 "neumanndirichlet": _abi.BC_NEUMANN_DIRICHLET, "pmcpec": _abi.BC_NEUMANN_DIRICHLET}
        if b not in table:
            raise ValueError(f"Boundary condition BC = {BC} is not an eligible option")
        return table[b], 0.0
    if _is_num_scalar(BC):
        if np.imag(BC) != 0:
            raise ValueError(f"k*a = {np.real(BC):g} + 1i*{np.imag(BC):g} is a complex number; has to be real for a "
                             "complete orthonormal transverse basis.")
        return _abi.BC_BLOCH, float(np.real(BC))
    raise ValueError("Boundary condition BC has to be a character vector or string, or numeric scalar "
                     "(for Bloch periodic BC)")


def _bc_3d(BC):
    """xyBC -> (rgf_bc, kxa, kya) (setup_channels_3D.m:66-126)."""
    if isinstance(BC, str):
        b = BC.lower()
        if b == "bloch":
            raise ValueError("To use Bloch periodic boundary condition, set BC to [kx*ax, ky*ay] where (kx,ky) is "
                             "the Bloch wave vector and (ax,ay) is the periodicity")
        if b == "periodic":
            return _abi.BC_PERIODIC, 0.0, 0.0
        if b in ("dirichlet", "pec"):
            return _abi.BC_DIRICHLET, 0.0, 0.0
        raise ValueError(f"Boundary condition BC = {BC} is not an eligible option")
    arr = np.asarray(BC)
    if arr.size == 2 and np.issubdtype(arr.dtype, np.number):
        kxa, kya = arr.ravel()
        if np.imag(kxa) != 0 or np.imag(kya) != 0:
            raise ValueError("kx*a and ky*a have to be real for a complete orthonormal transverse basis.")
        return _abi.BC_BLOCH, float(np.real(kxa)), float(np.real(kya))
    raise ValueError("Boundary condition BC has to be a character vector or string, or numeric vector with 2 "
                     "elements (for Bloch periodic BC)")


def _check_syst(syst, bc_key):
    """cal_smatrix_RGF.m:79-88."""
    if not (isinstance(syst, dict) or hasattr(syst, "__dict__")):
        raise ValueError("syst must be a structure")
    for key in ("epsilon", "epsilon_L", "epsilon_R", "k0dx", bc_key):
        if not _has(syst, key):
            raise ValueError(f"syst.{key} must be provided")
    for key in ("epsilon_L", "epsilon_R", "k0dx"):
        if not _is_num_scalar(_get(syst, key)):
            raise ValueError(f"syst.{key} must be a numeric scalar")


def _parse_request(req, kind: str):
    """out/in -> [(array or None, n)] for sides L, R (cal_smatrix_RGF.m:103-178).

    Returns 0-based index arrays; n == RGF_ALL for the cell form."""
    sides = [(None, 0), (None, 0)]
    if isinstance(req, dict):
        for s, side in enumerate(("L", "R")):
            key = f"ind_{kind}_{side}"
            if key in req:
                v = np.asarray(req[key]).reshape(-1)
                if v.size:
                    ok = np.issubdtype(v.dtype, np.number) and not np.iscomplexobj(v)
                    ok = ok and bool(np.all(np.round(v) == v)) and v.min() > 0
                    if not ok:
                        raise ValueError(f"{kind}.{key}, when specified, must be an array of positive integers "
                                         f"not exceeding N_prop_{side}")
                a = _abi.index_array(v.astype(np.int64) - 1)
                sides[s] = (a, int(a.size))
    elif isinstance(req, (list, tuple)):
        for k, el in enumerate(req, start=1):
            if not isinstance(el, str):
                warnings.warn(f"element {kind}{{{k}}} has wrong format and is ignored; should be one of "
                              "{'left', 'right', 'L', 'R'}")
                continue
            if el in ("left", "L"):
                sides[0] = (None, RGF_ALL)
            elif el in ("right", "R"):
                sides[1] = (None, RGF_ALL)
            else:
                warnings.warn(f"element {kind}{{{k}}} = {el} ignored; should be one of {{'left', 'right', 'L', 'R'}}")
    else:
        raise ValueError(f"input argument '{kind}' must be a structure or a cell array")
    return sides


def _request(out, in_):
    o = _parse_request(out, "out")
    i = _parse_request(in_, "in")
    keep = [o[0][0], o[1][0], i[0][0], i[1][0]]
    r = Request(ptr(o[0][0]), o[0][1], ptr(o[1][0]), o[1][1], ptr(i[0][0]), i[0][1], ptr(i[1][0]), i[1][1])
    return r, keep


class _ChanBuf:
    def __init__(self, N: int, dim: int):
        self.N = N
        self.kydx = np.zeros(N)
        self.kxdx_t = np.zeros(N) if dim == 3 else None
        self.kx = [np.zeros(N, complex), np.zeros(N, complex)]
        self.mu = [np.zeros(N, complex), np.zeros(N, complex)]
        self.ip = [np.zeros(N, np.int64), np.zeros(N, np.int64)]
        self.ic = [np.zeros(N, np.int64), np.zeros(N, np.int64)]
        self.c = Channels(ptr(self.kydx), ptr(self.kxdx_t), ptr(self.kx[0]), ptr(self.kx[1]), ptr(self.mu[0]),
                          ptr(self.mu[1]), ptr(self.ip[0]), ptr(self.ip[1]), ptr(self.ic[0]), ptr(self.ic[1]),
                          0, 0, 0, 0)

    def side(self, s: int, dim: int, shape=None) -> Dict[str, Any]:
        n = self.c.N_prop_L if s == 0 else self.c.N_prop_R
        if n < 0:
            return {"N_prop": np.nan}
        d = {"N_prop": int(n), "ind_prop": self.ip[s][:n] + 1, "sqrt_mu": self.mu[s][:n].copy()}
        if dim == 3:
            d["kzdx"] = self.kx[s].reshape(shape, order="F").copy()  # nx-by-ny, setup_channels_3D.m:47-59
        else:
            d["kxdx"] = self.kx[s].copy()
        if self.c.has_prop_conj:
            d["ind_prop_conj"] = self.ic[s][:n] + 1
        return d


def _fun_phi_2d(ny: int, bc: int):
    """channels.fun_phi of setup_channels.m:133-156."""
    m = np.arange(1, ny + 1, dtype=float)
    mh = np.arange(0.5, ny, 1.0)

    def f(k):
        k = np.atleast_1d(np.asarray(k, dtype=float))
        if bc in (_abi.BC_PERIODIC, _abi.BC_BLOCH):
            return np.exp(1j * np.outer(m, k)) / np.sqrt(ny)
        if bc == _abi.BC_DIRICHLET:
            return np.sin(np.outer(m, k)) * np.sqrt(2 / (ny + 1))
        if bc == _abi.BC_NEUMANN:
            return (np.cos(np.outer(mh, k)) - ((k == 0) * (1 - np.sqrt(0.5)))[None, :]) * np.sqrt(2 / ny)
        if bc == _abi.BC_DIRICHLET_NEUMANN:
            return np.sin(np.outer(m, k)) * np.sqrt(2 / (ny + 0.5))
        return np.cos(np.outer(mh, k)) * np.sqrt(2 / (ny + 0.5))
    return f


def _fun_phi_3d(nx: int, ny: int, bc: int):
    """channels.fun_phi of setup_channels_3D.m:118-123 (nx-by-ny profile)."""
    mx = np.arange(1, nx + 1, dtype=float)
    my = np.arange(1, ny + 1, dtype=float)

    def f(kx, ky):
        if bc == _abi.BC_DIRICHLET:
            return np.outer(np.sin(mx * kx), np.sin(my * ky) * np.sqrt(4 / ((nx + 1) * (ny + 1))))
        return np.outer(np.exp(1j * mx * kx), np.exp(1j * my * ky) / np.sqrt(nx * ny))
    return f


def _channels_dict_2d(cb: _ChanBuf, ny: int, bc: int) -> Dict[str, Any]:
    return {"kydx": cb.kydx.copy(), "fun_phi": _fun_phi_2d(ny, bc), "L": cb.side(0, 2), "R": cb.side(1, 2)}


def _channels_dict_3d(cb: _ChanBuf, nx: int, ny: int, bc: int) -> Dict[str, Any]:
    return {"kxdx": cb.kxdx_t.reshape((nx, ny), order="F").copy(), "kydx": cb.kydx.reshape((nx, ny), order="F").copy(),
            "fun_phi": _fun_phi_3d(nx, ny, bc), "L": cb.side(0, 3, (nx, ny)), "R": cb.side(1, 3, (nx, ny))}


def _options(options) -> Options:
    if options is None:
        return Options(_abi.RGF_FP64, 0, 0, 0)
    if isinstance(options, Options):
        return options
    return Options(int(options.get("precision", 0)), int(options.get("engine", 0)),
                   int(options.get("S_on_device", 0)), 0)


# ---------------------------------------------------------------------------
# public API
# ---------------------------------------------------------------------------
def cal_smatrix_RGF(syst, out, in_, *, device: int = 0, options=None, handle=None):
    """[smatrix, channels] = cal_smatrix_RGF(syst, out, in) on the GPU."""
    _check_syst(syst, "yBC")
    eps = np.asarray(_get(syst, "epsilon"))
    if eps.ndim != 2 or not np.issubdtype(eps.dtype, np.number):
        raise ValueError("syst.epsilon must be a numeric matrix")
    ny, nx = eps.shape
    if ny == 0:
        raise ValueError("need at least one site along the transverse (y) direction")
    bc, ka = _bc_2d(_get(syst, "yBC"))
    req, keep = _request(out, in_)
    h = handle or _abi.default_handle(device)
    epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
    sy = Syst2D(ny, nx, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                cplx(_get(syst, "k0dx")), bc, ka)
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    check(h.lib.rgf_smatrix_size_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no), ctypes.byref(ni)))
    S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
    cb = _ChanBuf(ny, 2)
    opt = _options(options)
    check(h.lib.rgf_smatrix_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), S.ctypes.data,
                               S.shape[0], ctypes.byref(cb.c)))
    del keep
    S = S[:no.value, :ni.value] if (no.value and ni.value) else np.zeros((no.value, ni.value))
    return S, _channels_dict_2d(cb, ny, bc)


def cal_smatrix_RGF_3D(syst, out, in_, *, device: int = 0, options=None, handle=None):
    """[smatrix, channels] = cal_smatrix_RGF_3D(syst, out, in) on the GPU."""
    _check_syst(syst, "xyBC")
    eps = np.asarray(_get(syst, "epsilon"))
    if eps.ndim not in (2, 3) or not np.issubdtype(eps.dtype, np.number):
        raise ValueError("syst.epsilon must be a 3D array")
    if eps.ndim == 2:
        eps = eps[:, :, None]
    nx, ny, nz = eps.shape
    if nx * ny == 0:
        raise ValueError("need at least one site along the transverse directions (x,y)")
    bc, kxa, kya = _bc_3d(_get(syst, "xyBC"))
    req, keep = _request(out, in_)
    h = handle or _abi.default_handle(device)
    epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
    sy = Syst3D(nx, ny, nz, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                cplx(_get(syst, "k0dx")), bc, kxa, kya)
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    check(h.lib.rgf_smatrix_size_3d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no), ctypes.byref(ni)))
    S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
    cb = _ChanBuf(nx * ny, 3)
    opt = _options(options)
    check(h.lib.rgf_smatrix_3d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), S.ctypes.data,
                               S.shape[0], ctypes.byref(cb.c)))
    del keep
    S = S[:no.value, :ni.value] if (no.value and ni.value) else np.zeros((no.value, ni.value))
    return S, _channels_dict_3d(cb, nx, ny, bc)


def cal_smatrix_RGF_batch(systs, outs, ins, *, workers: int = 0, device: int = 0, options=None, handle=None):
    """[S_1, ..., S_n] for n independent 2D structures (cal_smatrix_RGF on
    each); outs / ins are lists (one request per structure) or a single
    request used for all.  workers = 0: all slice sweeps in one persistent
    launch (gangs of CTAs sized to each structure from a device work queue);
    workers > 0: that many concurrent pipelines."""
    n = len(systs)
    if not isinstance(outs, (list, tuple)) or (outs and isinstance(outs[0], str)):
        outs = [outs] * n
    if not isinstance(ins, (list, tuple)) or (ins and isinstance(ins[0], str)):
        ins = [ins] * n
    h = handle or _abi.default_handle(device, "throughput")
    keep, sy_list, rq_list, S_list = [], [], [], []
    for syst, out, in_ in zip(systs, outs, ins):
        _check_syst(syst, "yBC")
        eps = np.asarray(_get(syst, "epsilon"))
        ny, nx = eps.shape
        bc, ka = _bc_2d(_get(syst, "yBC"))
        req, k = _request(out, in_)
        epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
        sy = Syst2D(ny, nx, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                    cplx(_get(syst, "k0dx")), bc, ka)
        no, ni = ctypes.c_int64(), ctypes.c_int64()
        check(h.lib.rgf_smatrix_size_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no),
                                        ctypes.byref(ni)))
        S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
        keep += [k, epsf]
        sy_list.append(sy)
        rq_list.append(req)
        S_list.append((S, no.value, ni.value))
    systs_c = (Syst2D * n)(*sy_list)
    reqs_c = (Request * n)(*rq_list)
    Sp = (ctypes.c_void_p * n)(*[S.ctypes.data for S, _, _ in S_list])
    ld = (ctypes.c_int64 * n)(*[S.shape[0] for S, _, _ in S_list])
    stat = (ctypes.c_int * n)()
    opt = _options(options)
    check(h.lib.rgf_smatrix_batch_2d(h.h, n, systs_c, reqs_c, ctypes.byref(opt), Sp, ld, stat, int(workers)))
    del keep
    return [S[:no, :ni] if (no and ni) else np.zeros((no, ni)) for S, no, ni in S_list]


def smatrix_grad_RGF(syst, out, in_, D, *, checkpoint: int = 0, device: int = 0, options=None, handle=None):
    """(S, g) for a 2D syst: S as cal_smatrix_RGF, and
    g[m, n] = sum_ab D[a, b] dS_ab / d epsilon[m, n] (complex, shape [ny, nx]).

    For a real objective F(S) with dF = 2 Re sum D dS (D = conj(S) for
    F = sum |S|^2), dF/d Re(epsilon) = 2 Re g.  An addition of this library:
    the reference computes S only."""
    _check_syst(syst, "yBC")
    eps = np.asarray(_get(syst, "epsilon"))
    if eps.ndim != 2 or not np.issubdtype(eps.dtype, np.number):
        raise ValueError("syst.epsilon must be a numeric matrix")
    ny, nx = eps.shape
    bc, ka = _bc_2d(_get(syst, "yBC"))
    req, keep = _request(out, in_)
    h = handle or _abi.default_handle(device)
    epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
    sy = Syst2D(ny, nx, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                cplx(_get(syst, "k0dx")), bc, ka)
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    check(h.lib.rgf_smatrix_size_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no), ctypes.byref(ni)))
    Dm = np.asfortranarray(np.asarray(D, dtype=complex).reshape(no.value, ni.value))
    S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
    g = np.zeros((ny, nx), dtype=complex, order="F")
    Dp = Dm if Dm.size else np.zeros((1, 1), dtype=complex, order="F")
    opt = _options(options)
    check(h.lib.rgf_smatrix_grad_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), Dp.ctypes.data,
                                    max(no.value, 1), S.ctypes.data, S.shape[0], g.ctypes.data, int(checkpoint)))
    del keep
    S = S[:no.value, :ni.value] if (no.value and ni.value) else np.zeros((no.value, ni.value))
    return S, g


def smatrix_grad_RGF_3D(syst, out, in_, D, *, checkpoint: int = 0, device: int = 0, options=None, handle=None):
    """(S, g) for a 3D syst; g has the shape of syst.epsilon ([nx, ny, nz])."""
    _check_syst(syst, "xyBC")
    eps = np.asarray(_get(syst, "epsilon"))
    if eps.ndim == 2:
        eps = eps[:, :, None]
    nx, ny, nz = eps.shape
    bc, kxa, kya = _bc_3d(_get(syst, "xyBC"))
    req, keep = _request(out, in_)
    h = handle or _abi.default_handle(device)
    epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
    sy = Syst3D(nx, ny, nz, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                cplx(_get(syst, "k0dx")), bc, kxa, kya)
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    check(h.lib.rgf_smatrix_size_3d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no), ctypes.byref(ni)))
    Dm = np.asfortranarray(np.asarray(D, dtype=complex).reshape(no.value, ni.value))
    S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
    g = np.zeros((nx, ny, nz), dtype=complex, order="F")
    Dp = Dm if Dm.size else np.zeros((1, 1), dtype=complex, order="F")
    opt = _options(options)
    check(h.lib.rgf_smatrix_grad_3d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), Dp.ctypes.data,
                                    max(no.value, 1), S.ctypes.data, S.shape[0], g.ctypes.data, int(checkpoint)))
    del keep
    S = S[:no.value, :ni.value] if (no.value and ni.value) else np.zeros((no.value, ni.value))
    return S, g


def fields_RGF(syst, out, in_, *, checkpoint: int = 0, device: int = 0, options=None, handle=None):
    """(S, psi) for a 2D syst: S as cal_smatrix_RGF, and the fields inside the
    structure psi[m, n, b] = (G_{n, s(b)} B_b)_m -- the response at site m of
    slice n to input channel b (the columns of S) -- of shape [ny, nx, n_in].
    An addition of this library (the reference points to MESTI for fields)."""
    _check_syst(syst, "yBC")
    eps = np.asarray(_get(syst, "epsilon"))
    if eps.ndim != 2 or not np.issubdtype(eps.dtype, np.number):
        raise ValueError("syst.epsilon must be a numeric matrix")
    ny, nx = eps.shape
    bc, ka = _bc_2d(_get(syst, "yBC"))
    req, keep = _request(out, in_)
    h = handle or _abi.default_handle(device)
    epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
    sy = Syst2D(ny, nx, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                cplx(_get(syst, "k0dx")), bc, ka)
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    check(h.lib.rgf_smatrix_size_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no), ctypes.byref(ni)))
    S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
    psi = np.zeros((ny, nx, ni.value), dtype=complex, order="F")
    pp = psi if psi.size else np.zeros(1, dtype=complex)
    opt = _options(options)
    check(h.lib.rgf_fields_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), S.ctypes.data,
                              S.shape[0], pp.ctypes.data, int(checkpoint)))
    del keep
    S = S[:no.value, :ni.value] if (no.value and ni.value) else np.zeros((no.value, ni.value))
    return S, psi


def fields_RGF_3D(syst, out, in_, *, checkpoint: int = 0, device: int = 0, options=None, handle=None):
    """(S, psi) for a 3D syst; psi has shape [nx, ny, nz, n_in]."""
    _check_syst(syst, "xyBC")
    eps = np.asarray(_get(syst, "epsilon"))
    if eps.ndim == 2:
        eps = eps[:, :, None]
    nx, ny, nz = eps.shape
    bc, kxa, kya = _bc_3d(_get(syst, "xyBC"))
    req, keep = _request(out, in_)
    h = handle or _abi.default_handle(device)
    epsf = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
    sy = Syst3D(nx, ny, nz, ptr(epsf), 0, cplx(_get(syst, "epsilon_L")), cplx(_get(syst, "epsilon_R")),
                cplx(_get(syst, "k0dx")), bc, kxa, kya)
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    check(h.lib.rgf_smatrix_size_3d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no), ctypes.byref(ni)))
    S = np.zeros((max(no.value, 1), max(ni.value, 1)), dtype=complex, order="F")
    psi = np.zeros((nx, ny, nz, ni.value), dtype=complex, order="F")
    pp = psi if psi.size else np.zeros(1, dtype=complex)
    opt = _options(options)
    check(h.lib.rgf_fields_3d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), S.ctypes.data,
                              S.shape[0], pp.ctypes.data, int(checkpoint)))
    del keep
    S = S[:no.value, :ni.value] if (no.value and ni.value) else np.zeros((no.value, ni.value))
    return S, psi


def _one_sided(epsilon_R) -> bool:
    return epsilon_R is None or (np.isscalar(epsilon_R) and np.isnan(epsilon_R))


def setup_channels(ny, BC, k0dx, epsilon_L, epsilon_R=None, *, device: int = 0, handle=None):
    """channels = setup_channels(ny, BC, k0dx, epsilon_L, epsilon_R) on the GPU."""
    if not (isinstance(ny, (int, np.integer)) and ny > 0):
        raise ValueError("ny must be a positive integer scalar")
    if not _is_num_scalar(k0dx):
        raise ValueError("k0dx must be a numeric scalar")
    if not _is_num_scalar(epsilon_L):
        raise ValueError("epsilon_L must be a numeric scalar")
    two = not _one_sided(epsilon_R)
    if two and not _is_num_scalar(epsilon_R):
        raise ValueError("epsilon_R must be a numeric scalar")
    bc, ka = _bc_2d(BC)
    h = handle or _abi.default_handle(device)
    cb = _ChanBuf(int(ny), 2)
    check(h.lib.rgf_setup_channels_2d(h.h, int(ny), bc, ka, cplx(k0dx), cplx(epsilon_L),
                                      cplx(epsilon_R if two else 0), int(two), ctypes.byref(cb.c)))
    return _channels_dict_2d(cb, int(ny), bc)


def setup_channels_3D(nx, ny, BC, k0dx, epsilon_L, epsilon_R=None, *, device: int = 0, handle=None):
    """channels = setup_channels_3D(nx, ny, BC, k0dx, epsilon_L, epsilon_R) on the GPU."""
    for name, v in (("nx", nx), ("ny", ny)):
        if not (isinstance(v, (int, np.integer)) and v > 0):
            raise ValueError(f"{name} must be a positive integer scalar")
    two = not _one_sided(epsilon_R)
    bc, kxa, kya = _bc_3d(BC)
    h = handle or _abi.default_handle(device)
    cb = _ChanBuf(int(nx) * int(ny), 3)
    check(h.lib.rgf_setup_channels_3d(h.h, int(nx), int(ny), bc, kxa, kya, cplx(k0dx), cplx(epsilon_L),
                                      cplx(epsilon_R if two else 0), int(two), ctypes.byref(cb.c)))
    return _channels_dict_3d(cb, int(nx), int(ny), bc)


def build_laplacian_1d(n, BC, *, device: int = 0, handle=None) -> np.ndarray:
    """A = build_laplacian_1d(n, BC) (dense) on the GPU."""
    if not (isinstance(n, (int, np.integer)) and n >= 0):
        raise ValueError("The number of sites n must be a non-negative integer scalar")
    bc, ka = _bc_2d(BC)
    h = handle or _abi.default_handle(device)
    A = np.zeros((n, n), dtype=complex, order="F")
    check(h.lib.rgf_build_laplacian_1d(h.h, int(n), bc, ka, A.ctypes.data if n else None))
    return A

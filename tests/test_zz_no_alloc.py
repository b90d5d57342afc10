"""rgf_smatrix_2d_noalloc (static device scratch, no cudaMalloc) against
rgf_smatrix_2d on the same inputs, called through the C ABI.

The two share every kernel; only where the device workspace lives differs.
Two calls in a row check that what the previous call left in the shared
static scratch does not leak into the next result.  Tolerance: the relative
Frobenius error bound of the FP64 plain form, 1e-11."""
import ctypes

import numpy as np
import pytest

from rgf_b200 import _abi
from rgf_b200.api import _request

pytestmark = pytest.mark.gpu
TOL_S = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def problem(ny, nx, bc, seed):
    rng = np.random.default_rng(seed)
    eps = np.ascontiguousarray((1.0 + 2.0 * rng.random((ny, nx))).astype(complex).ravel(order="F"))
    sy = _abi.Syst2D(ny, nx, eps.ctypes.data, 0, _abi.Cplx(1.0, 0.0), _abi.Cplx(1.0, 0.0),
                     _abi.Cplx(2 * np.pi / 15, 0.0), bc, 0.0)
    return sy, eps


def s_size(h, sy, req):
    no, ni = ctypes.c_int64(), ctypes.c_int64()
    _abi.check(h.lib.rgf_smatrix_size_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no),
                                         ctypes.byref(ni)))
    return no.value, ni.value


@pytest.mark.parametrize("ny,nx,bc,out,inp", [
    (64, 200, _abi.BC_PERIODIC, ["left", "right"], ["left", "right"]),
    (100, 9, _abi.BC_DIRICHLET, ["left", "right"], ["left"]),
])
def test_noalloc_matches_allocating_entry(ny, nx, bc, out, inp):
    lib = _abi.load()
    h = _abi.Handle(0)
    sy, eps = problem(ny, nx, bc, seed=ny + nx)
    req, keep = _request(out, inp)
    opt = _abi.Options(_abi.RGF_FP64, 0, 0, 0)
    no, ni = s_size(h, sy, req)
    ref = np.zeros((no, ni), dtype=complex, order="F")
    _abi.check(lib.rgf_smatrix_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), ref.ctypes.data,
                                  no, None))
    for _ in range(2):
        S = np.full((no, ni), np.nan, dtype=complex, order="F")
        _abi.check(lib.rgf_smatrix_2d_noalloc(ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt),
                                              S.ctypes.data, no, None, None))
        assert rel(S, ref) <= TOL_S
    del keep, eps


def test_noalloc_rejects_oversized_problem():
    lib = _abi.load()
    sy, eps = problem(1024, 4096, _abi.BC_PERIODIC, seed=0)  # 64 MiB of epsilon alone
    req, keep = _request(["left"], ["left"])
    S = np.zeros((1024, 1024), dtype=complex, order="F")
    st = lib.rgf_smatrix_2d_noalloc(ctypes.byref(sy), ctypes.byref(req), None, S.ctypes.data, 1024, None, None)
    assert st == _abi.RGF_ERR_ARG
    assert b"static device scratch" in lib.rgf_last_error()
    del keep, eps


def noalloc_footprint_bytes(N, n_out, n_in, nx, eps_on_host=True, two_leads=False):
    """The workspace of rgf_smatrix_2d_noalloc as include/rgf.h states it."""
    R, C = N + n_out, N + n_in + 2
    b = 16 * (3 * N * N + R * (C + 1) + 64 * R + 288 * C + 110 * N)
    if two_leads:
        b += 16 * N * N
    if eps_on_host:
        b += 16 * N * nx
    return b


def test_noalloc_size_limit_is_the_documented_one():
    """The largest ny accepted for a full two-sided periodic S (epsilon on the
    host, 2 slices), found by bisection, is the one the header's footprint
    formula predicts (to 1%); ny + 1 is rejected and ny matches the
    allocating entry."""
    lib = _abi.load()
    h = _abi.Handle(0)
    req, keep = _request(["left", "right"], ["left", "right"])
    opt = _abi.Options(_abi.RGF_FP64, 0, 0, 0)

    def attempt(ny):
        sy, eps = problem(ny, 2, _abi.BC_PERIODIC, seed=ny)
        no, ni = s_size(h, sy, req)
        S = np.zeros((no, ni), dtype=complex, order="F")
        st = lib.rgf_smatrix_2d_noalloc(ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), S.ctypes.data, no,
                                        None, None)
        assert st in (_abi.RGF_OK, _abi.RGF_ERR_ARG), _abi.STATUS_NAMES.get(st, st)
        return st == _abi.RGF_OK, (sy, eps, no, ni, S)

    lo, hi = 300, 1200  # lo fits, hi does not
    assert attempt(lo)[0] and not attempt(hi)[0]
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if attempt(mid)[0]:
            lo = mid
        else:
            hi = mid
    ok, (sy, eps, no, ni, S) = attempt(lo)
    assert ok and not attempt(lo + 1)[0]
    ref = np.zeros((no, ni), dtype=complex, order="F")
    _abi.check(lib.rgf_smatrix_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), ref.ctypes.data, no,
                                  None))
    assert rel(S, ref) <= TOL_S
    # the documented formula's largest ny for this problem
    pred = max(n for n in range(300, 1200)
               if noalloc_footprint_bytes(n, *_sizes_for(h, n, req), nx=2) <= _abi.RGF_NOALLOC_SCRATCH_BYTES)
    assert abs(pred - lo) <= 0.01 * lo, (pred, lo)
    del keep


def _sizes_for(h, ny, req):
    sy, eps = problem(ny, 2, _abi.BC_PERIODIC, seed=ny)
    return s_size(h, sy, req)


def noalloc_footprint_bytes(N, n_out, n_in, nx, eps_on_host=True, two_leads=False):
    """The workspace of rgf_smatrix_2d_noalloc as include/rgf.h states it."""
    R, C = N + n_out, N + n_in + 2
    b = 16 * (3 * N * N + R * (C + 1) + 64 * R + 288 * C + 110 * N)
    if two_leads:
        b += 16 * N * N
    if eps_on_host:
        b += 16 * N * nx
    return b


def test_noalloc_size_limit_is_the_documented_one():
    """The largest ny accepted for a full two-sided periodic S (epsilon on the
    host, 2 slices), found by bisection, is the one the header's footprint
    formula predicts (to 1%); ny + 1 is rejected, and ny matches the
    allocating entry."""
    lib = _abi.load()
    h = _abi.Handle(0)
    req, keep = _request(["left", "right"], ["left", "right"])
    opt = _abi.Options(_abi.RGF_FP64, 0, 0, 0)

    def attempt(ny):
        sy, eps = problem(ny, 2, _abi.BC_PERIODIC, seed=ny)
        no, ni = s_size(h, sy, req)
        S = np.zeros((no, ni), dtype=complex, order="F")
        st = lib.rgf_smatrix_2d_noalloc(ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), S.ctypes.data, no,
                                        None, None)
        assert st in (_abi.RGF_OK, _abi.RGF_ERR_ARG), _abi.STATUS_NAMES.get(st, st)
        return st == _abi.RGF_OK, (sy, eps, no, ni, S)

    lo, hi = 300, 1200  # lo fits, hi does not
    assert attempt(lo)[0] and not attempt(hi)[0]
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if attempt(mid)[0]:
            lo = mid
        else:
            hi = mid
    ok, (sy, eps, no, ni, S) = attempt(lo)
    assert ok and not attempt(lo + 1)[0]
    ref = np.zeros((no, ni), dtype=complex, order="F")
    _abi.check(lib.rgf_smatrix_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt), ref.ctypes.data, no,
                                  None))
    assert rel(S, ref) <= TOL_S
    sizes = {}
    for n in range(lo - 30, lo + 31):
        sy_n, eps_n = problem(n, 2, _abi.BC_PERIODIC, seed=n)
        sizes[n] = s_size(h, sy_n, req)
    pred = max(n for n, (no_n, ni_n) in sizes.items()
               if noalloc_footprint_bytes(n, no_n, ni_n, nx=2) <= _abi.RGF_NOALLOC_SCRATCH_BYTES)
    assert abs(pred - lo) <= 0.01 * lo, (pred, lo)
    del keep

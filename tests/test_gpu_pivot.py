"""Pivoting and the a-posteriori slice-inverse check, on the GPU.

The reference inverts every slice matrix with MATLAB's inv
(cal_smatrix_RGF.m:265), i.e. LU with partial pivoting over the whole
column.  The persistent engine pivots inside each 32 x 32 pivot block only;
a probe vector carried through every slice checks each inverse, and a call
whose check fails is recomputed by the per-step engine, which pivots over
the whole remaining column like LAPACK zgetrf.  These cases leave diagonal
dominance behind (k0dx^2 eps_L >= 3.5, index contrast 12, gain) on N >= 96
(several pivot blocks), and one has a singular leading pivot block while the
slice matrix itself is well conditioned.

Tolerance: relative Frobenius error of S <= 1e-11 against the FP64 oracle
(itself within 4e-14 of a dense solve of the same operator on every case
here)."""
import ctypes
import glob
import os
import warnings

import numpy as np
import pytest

import rgf_b200
from rgf_b200 import _abi
from tests.golden_io import load_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
PIVOT = sorted(glob.glob(os.path.join(GOLDEN, "2d_pivot_*.npz")))
TOL_S = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("path", PIVOT, ids=lambda p: os.path.basename(p)[:-4])
def test_pivot_regime_matches_oracle(path, engine):
    case = load_case(path)
    h = _abi.Handle(0)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        S, _ = rgf_b200.cal_smatrix_RGF(case["syst"], case["out"], case["in"], handle=h,
                                        options={"engine": engine})
    assert rel(S, case["S"]) <= TOL_S
    used, fallback, _ = h.engine()
    _, probe = h.stats()
    # the residual scales with |G_n| |M_n|: at index contrast 12 it reaches
    # ~2e-10 under whole-column pivoting while S still matches to 1e-11
    assert probe < 1e-9
    if engine == 1:
        assert used == 1 and fallback == 0


def test_singular_leading_block_falls_back():
    """In-block pivoting cannot invert this slice matrix (its leading 32 x 32
    block is singular); the check must reject the persistent engine's result
    and the whole-column pivoting recompute must match the oracle."""
    case = load_case(os.path.join(GOLDEN, "2d_pivot_singular_block.npz"))
    h = _abi.Handle(0)
    S, _ = rgf_b200.cal_smatrix_RGF(case["syst"], case["out"], case["in"], handle=h)
    used, fallback, rejected = h.engine()
    assert fallback == 1 and used == 1
    assert not (rejected <= 1e-10)
    assert rel(S, case["S"]) <= TOL_S


def test_singular_leading_block_noalloc():
    """The same recompute inside the allocation-free entry point."""
    from rgf_b200.api import _request
    case = load_case(os.path.join(GOLDEN, "2d_pivot_singular_block.npz"))
    sy_ = case["syst"]
    eps = np.ascontiguousarray(np.asarray(sy_["epsilon"], dtype=complex).ravel(order="F"))
    ny, nx = sy_["epsilon"].shape
    sy = _abi.Syst2D(ny, nx, eps.ctypes.data, 0, _abi.cplx(1.0), _abi.cplx(1.0), _abi.cplx(sy_["k0dx"]),
                     _abi.BC_DIRICHLET, 0.0)
    req, keep = _request(case["out"], case["in"])
    no, ni = case["S"].shape
    S = np.full((no, ni), np.nan, dtype=complex, order="F")
    lib = _abi.load()
    _abi.check(lib.rgf_smatrix_2d_noalloc(ctypes.byref(sy), ctypes.byref(req), None, S.ctypes.data, no, None, None))
    assert rel(S, case["S"]) <= TOL_S
    del keep


def singular_slice_eps(ny, nx, k0dx):
    """eps whose first slice matrix A0 - k0dx^2 diag(eps_1) - G0_L is singular
    (eps_1 constant = lambda / k0dx^2, lambda an eigenvalue of A0 - G0_L)."""
    from oracle.rgf_ref import build_laplacian_1d, setup_channels
    ch = setup_channels(ny, "Dirichlet", k0dx, 1.0, 1.0)
    phi = ch["fun_phi"](ch["kydx"])
    G0 = (phi * np.exp(1j * ch["L"]["kxdx"])[None, :]) @ phi.conj().T
    A0 = -build_laplacian_1d(ny, "Dirichlet") + 2 * np.eye(ny)
    lam = np.linalg.eigvals(A0 - G0)
    eps = np.full((ny, nx), 2.0, dtype=complex)
    eps[:, 0] = lam[np.argmin(np.abs(lam - 2 * k0dx ** 2))] / k0dx ** 2
    return eps


@pytest.mark.parametrize("engine", [0, 1])
def test_singular_slice_is_reported(engine):
    """A slice matrix that is singular to working precision: no engine may
    return RGF_OK (MATLAB's inv would warn); the call reports
    RGF_ERR_ILLCOND (or RGF_ERR_SINGULAR on an exactly zero pivot)."""
    k0dx = 2 * np.pi / 15
    eps = singular_slice_eps(64, 5, k0dx)
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=k0dx, yBC="Dirichlet")
    h = _abi.Handle(0)
    caught = None
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        try:
            rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], handle=h,
                                     options={"engine": engine})
        except _abi.RGFError as e:
            caught = e.status
    if caught is None:
        assert any(issubclass(x.category, _abi.IllConditionedWarning) for x in w)
    else:
        assert caught == _abi.RGF_ERR_SINGULAR


def test_crecip_newton_reciprocal_ulp():
    """The persistent engine's pivot reciprocal (rcp.approx.ftz.f64 + two
    Newton steps) against IEEE division conj(z) / |z|^2 over |z| in
    [1e-150, 1e150]: within 2 ulp of the larger component; |z|^2 beyond
    ~2^1022 flushes to 0, which the engine flags as singular."""
    lib = ctypes.CDLL(os.path.join(os.path.dirname(__file__), "cuda", "libselftest.so"))
    lib.rgf_selftest_crecip.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    rng = np.random.default_rng(31)
    n = 200000
    mag = 10.0 ** rng.uniform(-150, 150, n)
    ang = rng.uniform(0, 2 * np.pi, n)
    z = np.ascontiguousarray(mag * np.exp(1j * ang))
    z[:4] = [1.0, 1j, -3.0 + 4.0j, 1e-150]
    out = np.zeros((n, 4))
    assert lib.rgf_selftest_crecip(z.ctypes.data, out.ctypes.data, n) == 0
    ours = out[:, 0] + 1j * out[:, 1]
    ieee = out[:, 2] + 1j * out[:, 3]
    scale = np.maximum(np.abs(ieee.real), np.abs(ieee.imag))
    ulp = np.spacing(scale)
    err = np.maximum(np.abs(ours.real - ieee.real), np.abs(ours.imag - ieee.imag)) / ulp
    assert np.all(np.isfinite(ours))
    assert err.max() <= 2.0, err.max()
    # |z|^2 = 2^1023: the reciprocal 2^-1023 is subnormal and flushed to 0;
    # |z|^2 = inf (|z| ~ 2^520): non-finite
    big = np.array([2.0 ** 511 * (1 + 1j), 2.0 ** 520 * (1 + 1j)])
    out1 = np.zeros((2, 4))
    assert lib.rgf_selftest_crecip(big.ctypes.data, out1.ctypes.data, 2) == 0
    assert out1[0, 0] == 0.0 and out1[0, 1] == 0.0
    assert not np.all(np.isfinite(out1[1, :2]))

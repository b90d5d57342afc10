"""The 3xTF32 tcgen05 GEMM (rgf_b200/csrc/tc32.cuh) against an FP64 product.

The operands are split into tf32 hi/lo parts on the host (round to nearest,
ties away, as cvt.rna.tf32.f32); the kernel's result must carry about 21 bits
(relative error ~1e-6), far below the ~1e-3 of a single TF32 product.
Complex products use the realified layout the precision form feeds it.
"""
import ctypes
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
K_STORE, K_PARTIAL, K_GJ = 0, 1, 2


def _lib():
    lib = ctypes.CDLL(os.path.join(HERE, "cuda", "libselftest.so"))
    f = lib.rgf_selftest_tc32
    f.argtypes = [ctypes.c_int] * 8 + [ctypes.c_void_p] * 5
    f.restype = ctypes.c_int
    return f


def tf32_split(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32)
    hi = ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)
    lo = (x - hi).astype(np.float32)
    return hi, lo


def realify_left(P):
    """complex rows x K -> real rows x 2K (interleaved re, im): the A operand."""
    return np.ascontiguousarray(P.astype(np.complex64)).view(np.float32)


def realify_right(Q):
    """complex K x cols -> real K-major B operand [2 cols x 2K]."""
    K, n = Q.shape
    Bt = np.empty((2 * n, 2 * K), np.float32)
    Bt[0::2, 0::2] = Q.real.T
    Bt[0::2, 1::2] = -Q.imag.T
    Bt[1::2, 0::2] = Q.imag.T
    Bt[1::2, 1::2] = Q.real.T
    return Bt


def run(A, Bt, bn, ksplit=1, mode=K_STORE, out=None, gj=(0, 0)):
    f = _lib()
    M, K = A.shape
    Nr = Bt.shape[0]
    ah, al = tf32_split(A)
    bh, bl = tf32_split(Bt)
    if out is None:
        out = np.zeros(((ksplit if mode == K_PARTIAL else 1), M, Nr), np.float32)
    out = np.ascontiguousarray(out, np.float32)
    rc = f(M, Nr, K, ksplit, bn, mode, gj[0], gj[1], ah.ctypes.data, al.ctypes.data, bh.ctypes.data,
           bl.ctypes.data, out.ctypes.data)
    assert rc == 0, rc
    return out


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("M,Kc,Nc,bn", [(128, 16, 32, 64), (256, 64, 96, 64), (200, 48, 68, 128),
                                         (384, 32, 128, 256), (130, 80, 200, 128), (256, 64, 204, 144),
                                         (130, 48, 100, 208)])
def test_complex_product(M, Kc, Nc, bn):
    rng = np.random.default_rng(M + Kc + Nc)
    P = (rng.standard_normal((M, Kc)) + 1j * rng.standard_normal((M, Kc))).astype(np.complex64)
    Q = (rng.standard_normal((Kc, Nc)) + 1j * rng.standard_normal((Kc, Nc))).astype(np.complex64)
    A, Bt = realify_left(P), realify_right(Q)
    D = run(A, Bt, bn)[0]
    ref = P.astype(np.complex128) @ Q.astype(np.complex128)
    got = D[:, 0::2].astype(np.float64) + 1j * D[:, 1::2]
    err = rel(got, ref)
    assert err < 3e-6, err
    # a single TF32 product would sit near 1e-3: the split must recover FP32-level accuracy
    tf = (tf32_split(A)[0].astype(np.float64) @ tf32_split(Bt)[0].astype(np.float64).T)
    assert rel(tf[:, 0::2] + 1j * tf[:, 1::2], ref) > 30 * err


@pytest.mark.gpu
def test_ksplit_partials():
    rng = np.random.default_rng(7)
    M, K, Nr = 256, 512, 192
    A = rng.standard_normal((M, K)).astype(np.float32)
    Bt = rng.standard_normal((Nr, K)).astype(np.float32)
    out = run(A, Bt, 64, ksplit=4, mode=K_PARTIAL)
    ref = A.astype(np.float64) @ Bt.astype(np.float64).T
    assert rel(out.sum(axis=0, dtype=np.float64), ref) < 3e-6
    for z in range(4):  # each split is its own quarter of K
        refz = A[:, z * 128:(z + 1) * 128].astype(np.float64) @ Bt[:, z * 128:(z + 1) * 128].astype(np.float64).T
        assert rel(out[z], refz) < 3e-6


@pytest.mark.gpu
def test_ragged_ksplit_partials():
    """A K-split that does not divide the chunk count (16 chunks in 3 splits:
    5, 5, 6 chunks of 32) on 144-wide tiles, as the refinement's solve uses."""
    rng = np.random.default_rng(8)
    M, K, Nr = 256, 512, 408
    A = rng.standard_normal((M, K)).astype(np.float32)
    Bt = rng.standard_normal((Nr, K)).astype(np.float32)
    out = run(A, Bt, 144, ksplit=3, mode=K_PARTIAL)
    ref = A.astype(np.float64) @ Bt.astype(np.float64).T
    assert rel(out.sum(axis=0, dtype=np.float64), ref) < 3e-6
    for z in range(3):
        lo, hi = 32 * (z * 16 // 3), 32 * ((z + 1) * 16 // 3)
        refz = A[:, lo:hi].astype(np.float64) @ Bt[:, lo:hi].astype(np.float64).T
        assert rel(out[z], refz) < 3e-6


@pytest.mark.gpu
def test_gauss_jordan_epilogue():
    rng = np.random.default_rng(11)
    N, nb, c0 = 192, 64, 64  # complex W is N x N, pivot block columns [c0, c0+nb)
    W = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    V = (rng.standard_normal((N, nb)) + 1j * rng.standard_normal((N, nb))).astype(np.complex64)
    U = (rng.standard_normal((nb, N)) + 1j * rng.standard_normal((nb, N))).astype(np.complex64)
    A, Bt = realify_left(V), realify_right(U)
    out = realify_left(W).reshape(1, N, 2 * N).copy()
    got = run(A, Bt, 128, mode=K_GJ, out=out, gj=(c0, nb))[0]
    Wp = W.astype(np.complex128)
    Wp[:, c0:c0 + nb] = 0
    Wp[np.arange(c0, c0 + nb), np.arange(c0, c0 + nb)] = 1
    ref = Wp - V.astype(np.complex128) @ U.astype(np.complex128)
    g = got[:, 0::2].astype(np.float64) + 1j * got[:, 1::2]
    assert rel(g, ref) < 3e-6

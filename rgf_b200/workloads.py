"""Seeded synthetic structures (the reference ships no benchmark inputs).

Each function returns a ``syst`` dict in the reference's MATLAB layout
(``epsilon`` is [ny, nx] in 2D and [nx, ny, nz] in 3D) plus the ``out``/``in``
request, reproducible from numpy's PCG64 ``default_rng(seed)``.

  config1  2D periodic, N=64,   L=200,  eps U[1,4),            full S
  config2  2D Dirichlet, N=1024, L=4096, 2.25 + 30% disks of 1 (r in [4,12]) + 1j*U[0,0.01), full S
  config3  3D Bloch (0.3, 0.7), 24x24, L=300, eps in {1, 2.25} (p=0.4), full S
  config4  256 periodic structures, N in [64,512], L in [100,2000], complex k0dx
  config5  2D periodic, N=256, L=512, eps U[1,4), t block out R 1:8 / in L 1:8
"""
from __future__ import annotations

import numpy as np


def config1(seed: int = 1, ny: int = 64, nx: int = 200):
    rng = np.random.default_rng(seed)
    eps = 1.0 + 3.0 * rng.random((ny, nx))
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15, yBC="periodic")
    return syst, ["left", "right"], ["left", "right"]


def disks_permittivity(ny: int, nx: int, seed: int, fill: float = 0.30, background: float = 2.25,
                       rmin: float = 4.0, rmax: float = 12.0, absorption: float = 0.01) -> np.ndarray:
    """Background permittivity with random disks of eps = 1 until a fraction
    ``fill`` of the pixels is 1, then + 1j*U[0, absorption) on every pixel.

    Disk k draws (cy, cx, r) = (U[0,ny), U[0,nx), U[rmin,rmax)); pixel (m, n)
    (0-based) is inside when (m-cy)^2 + (n-cx)^2 <= r^2.
    """
    rng = np.random.default_rng(seed)
    inside = np.zeros((ny, nx), dtype=bool)
    count = 0
    target = fill * ny * nx
    while count < target:
        cy, cx, r = rng.uniform(0, ny), rng.uniform(0, nx), rng.uniform(rmin, rmax)
        m0, m1 = max(int(np.floor(cy - r)), 0), min(int(np.ceil(cy + r)) + 1, ny)
        n0, n1 = max(int(np.floor(cx - r)), 0), min(int(np.ceil(cx + r)) + 1, nx)
        if m0 >= m1 or n0 >= n1:
            continue
        m = np.arange(m0, m1)[:, None]
        n = np.arange(n0, n1)[None, :]
        blk = (m - cy) ** 2 + (n - cx) ** 2 <= r * r
        sub = inside[m0:m1, n0:n1]
        count += int(np.count_nonzero(blk & ~sub))
        sub |= blk
    eps = np.where(inside, 1.0, background).astype(complex)
    eps += 1j * rng.uniform(0.0, absorption, size=(ny, nx))
    return eps


def config2(seed: int = 2, ny: int = 1024, nx: int = 4096):
    eps = disks_permittivity(ny, nx, seed)
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 20, yBC="Dirichlet")
    return syst, ["left", "right"], ["left", "right"]


def config3(seed: int = 3, nx: int = 24, ny: int = 24, nz: int = 300):
    rng = np.random.default_rng(seed)
    eps = np.where(rng.random((nx, ny, nz)) < 0.4, 2.25, 1.0)
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 12, xyBC=[0.3, 0.7])
    return syst, ["left", "right"], ["left", "right"]


def config4_params(seed: int = 4, count: int = 256):
    """(N, L, eta) of every structure of the batched workload."""
    rng = np.random.default_rng(seed)
    Ns = rng.integers(64, 513, size=count)
    Ls = rng.integers(100, 2001, size=count)
    etas = rng.uniform(0.0, 1e-3, size=count)
    return Ns, Ls, etas


# the 16-structure subsample of the batched workload that has oracle
# fixtures: the first twelve, then the largest N (k=70, N=511), the largest L
# (k=101, L=1997), the largest L*N^3 (k=142, N=503, L=1917) and the largest
# eta (k=218)
CONFIG4_SUBSAMPLE = tuple(range(12)) + (70, 101, 142, 218)


def config4_structure(k: int, seed: int = 4, count: int = 256):
    """Structure k of the batched workload: periodic, eps U[1,3) drawn from
    default_rng([seed, k]), k0dx = 2pi/15 (1 + 1j eta)."""
    Ns, Ls, etas = config4_params(seed, count)
    rng = np.random.default_rng([seed, k])
    eps = 1.0 + 2.0 * rng.random((int(Ns[k]), int(Ls[k])))
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15 * (1 + 1j * float(etas[k])),
                yBC="periodic")
    return syst, ["left", "right"], ["left", "right"]


def config5(seed: int = 5, ny: int = 256, nx: int = 512):
    rng = np.random.default_rng(seed)
    eps = 1.0 + 3.0 * rng.random((ny, nx))
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15, yBC="periodic")
    return syst, {"ind_out_R": np.arange(1, 9)}, {"ind_in_L": np.arange(1, 9)}


def canonical_slice_flops(N: int, pin: int, pout: int) -> float:
    """Channel-projected algorithmic flops of one slice of the recursion:
    inverse 8N^3, carriers X = G B_L and Z = C_L G (8N^2 each per channel),
    Y += Z X (8N P_out P_in); pin / pout are the left-side channel counts."""
    return 8.0 * N ** 3 + 8.0 * N * N * (pin + pout) + 8.0 * N * pout * pin


def canonical_flops(N: int, L: int, pin: int, pout: int, distinct_leads: bool = False) -> float:
    """Channel-projected algorithmic flop count of one S-matrix (real flops,
    complex multiply-add = 8): per slice 8N^3 (inverse) + 8N^2 (P_in + P_out)
    + 8N P_out P_in, plus the lead G0 GEMM(s), the attach inverse and the
    Fisher-Lee projection."""
    per_slice = 8.0 * N ** 3 + 8.0 * N * N * (pin + pout) + 8.0 * N * pout * pin
    setup = 8.0 * N ** 3 * (2 if distinct_leads else 1)
    attach = 8.0 * N ** 3 + 8.0 * N * N * (pin + pout) + 8.0 * N * pout * pin
    return L * per_slice + setup + attach

"""Permittivity gradient of an objective on S -- TEST INFRASTRUCTURE ONLY.

The reference computes S only; the gradient is an addition of this build.
Two independent CPU statements of it, both in FP64:

* ``grad_dense_2d``: from the dense inverse of the whole block-tridiagonal
  operator (sites 0 .. L+1, as ``oracle.dense_fdfd``).  With
  ``S = -2i C G B - delta`` and ``dH/d eps[m, n] = -k0dx^2 e_m e_m^T`` at site
  n+1, ``dG = -G dH G`` gives

      dS_ab / d eps[m, n] = -2i k0dx^2 (C_a G_{side(a), n+1})[m] (G_{n+1, side(b)} B_b)[m].

* ``grad_rgf_2d``: the slice recursion of ``cal_smatrix_RGF.m:257-280`` run
  forward in the sweep direction (start side s, end side e), keeping the
  start-connected blocks g_k and the carriers X_k = g_k ... g_0 B_s,
  Z_k = C_s g_0 ... g_k, followed by the backward recursions

      Psi_k = [X_k, 0] + g_k Psi_{k+1}      (columns in_s, in_e)
      Phi_k = [Z_k; 0] + Phi_{k+1} g_k      (rows out_s, out_e)

  from Psi_{L+1} = [X_{L+1}, g_{L+1} B_e], Phi_{L+1} = [Z_{L+1}; C_e g_{L+1}]
  (columns and rows of the inverse of the block LU factors of the operator),
  so that Psi_k = G_{k, ends} B and Phi_k = C G_{ends, k}.

Both return (S, g) where g[m, n] = sum_ab D[a, b] dS_ab/d eps[m, n] for the
weights D (complex); for a real objective F with dF = 2 Re sum D dS, the
gradient with respect to a real permittivity is 2 Re g.
"""
from __future__ import annotations

import numpy as np

from .rgf_ref import (build_laplacian_1d, cal_smatrix_RGF, parse_channel_request,
                      setup_channels)


def _setup(syst, out, in_):
    eps = np.asarray(syst["epsilon"], dtype=complex)
    ny, nx = eps.shape
    k0dx = syst["k0dx"]
    ch = setup_channels(int(ny), syst["yBC"], k0dx, syst["epsilon_L"], syst["epsilon_R"])
    chL, chR = ch["L"], ch["R"]
    iiL, iiR = parse_channel_request(in_, "in", chL["N_prop"], chR["N_prop"])
    ioL, ioR = parse_channel_request(out, "out", chL["N_prop"], chR["N_prop"])
    phi = ch["fun_phi"](ch["kydx"])
    G0 = {s: (phi * np.exp(1j * c["kxdx"])[None, :]) @ phi.conj().T for s, c in (("L", chL), ("R", chR))}
    B = {"L": phi[:, chL["ind_prop"][iiL - 1] - 1] * chL["sqrt_mu"][iiL - 1][None, :],
         "R": phi[:, chR["ind_prop"][iiR - 1] - 1] * chR["sqrt_mu"][iiR - 1][None, :]}
    C = {"L": chL["sqrt_mu"][ioL - 1][:, None] * phi[:, chL["ind_prop"][ioL - 1] - 1].conj().T,
         "R": chR["sqrt_mu"][ioR - 1][:, None] * phi[:, chR["ind_prop"][ioR - 1] - 1].conj().T}
    A0 = -build_laplacian_1d(int(ny), syst["yBC"]) + 2 * np.eye(ny)
    return eps, k0dx, G0, B, C, A0, (len(ioL), len(ioR), len(iiL), len(iiR))


def grad_dense_2d(syst, out, in_, D):
    """(S, g) from the dense inverse; small problems only."""
    eps, k0dx, G0, B, C, A0, _ = _setup(syst, out, in_)
    ny, nx = eps.shape
    N = ny
    nsite = nx + 2
    H = np.zeros((nsite * N, nsite * N), dtype=complex)

    def blk(i, j):
        return slice(i * N, (i + 1) * N), slice(j * N, (j + 1) * N)

    H[blk(0, 0)] = np.linalg.inv(G0["L"])
    H[blk(nsite - 1, nsite - 1)] = np.linalg.inv(G0["R"])
    for n in range(nx):
        H[blk(n + 1, n + 1)] = A0 - np.diag(k0dx ** 2 * eps[:, n])
    for s in range(nsite - 1):
        H[blk(s, s + 1)] = -np.eye(N)
        H[blk(s + 1, s)] = -np.eye(N)
    G = np.linalg.inv(H)
    site = {"L": 0, "R": nsite - 1}
    S, _ = cal_smatrix_RGF(syst, out, in_)
    D = np.asarray(D, dtype=complex)
    g = np.zeros((ny, nx), dtype=complex)
    for n in range(nx):
        k = n + 1
        Phi = np.vstack([C["L"] @ G[blk(site["L"], k)], C["R"] @ G[blk(site["R"], k)]])   # n_out x N
        Psi = np.hstack([G[blk(k, site["L"])] @ B["L"], G[blk(k, site["R"])] @ B["R"]])   # N x n_in
        g[:, n] = -2j * k0dx ** 2 * np.einsum("am,ab,mb->m", Phi, D, Psi)
    return S, g


def grad_rgf_2d(syst, out, in_, D):
    """(S, g) by the forward sweep + backward recursions (any request form).

    The sweep runs right-to-left when nothing enters from the right (the
    direction rule of the CUDA implementation); rows/columns of D are given
    in the reference's order [out_L; out_R] x [in_L; in_R]."""
    eps, k0dx, G0, B, C, A0, (noL, noR, niL, niR) = _setup(syst, out, in_)
    ny, nx = eps.shape
    mirror = niR == 0
    s, e = ("R", "L") if mirror else ("L", "R")
    no_e = noL if mirror else noR
    ni_e = niL if mirror else niR
    k2 = k0dx ** 2
    N = ny
    # forward sweep over sites 0 .. L+1 in sweep order
    g = [G0[s]]
    X = [G0[s] @ B[s]]
    Z = [C[s] @ G0[s]]
    for k in range(1, nx + 1):
        n = (nx - k) if mirror else (k - 1)
        gk = np.linalg.inv(A0 - np.diag(k2 * eps[:, n]) - g[-1])
        g.append(gk)
        X.append(gk @ X[-1])
        Z.append(Z[-1] @ gk)
    gL1 = np.linalg.inv(np.linalg.inv(G0[e]) - g[-1])
    Psi = np.hstack([gL1 @ X[-1], gL1 @ B[e]])
    Phi = np.vstack([Z[-1] @ gL1, C[e] @ gL1])
    # D in sweep order: rows [out_s; out_e], columns [in_s; in_e]
    D = np.asarray(D, dtype=complex)
    rows = (list(range(noL, noL + noR)) + list(range(noL))) if mirror else list(range(noL + noR))
    cols = (list(range(niL, niL + niR)) + list(range(niL))) if mirror else list(range(niL + niR))
    Ds = D[np.ix_(rows, cols)]
    grad = np.zeros((ny, nx), dtype=complex)
    for k in range(nx, 0, -1):
        Psi = np.hstack([X[k], np.zeros((N, ni_e), dtype=complex)]) + g[k] @ Psi
        Phi = np.vstack([Z[k], np.zeros((no_e, N), dtype=complex)]) + Phi @ g[k]
        n = (nx - k) if mirror else (k - 1)
        grad[:, n] = -2j * k2 * np.einsum("am,ab,mb->m", Phi, Ds, Psi)
    S, _ = cal_smatrix_RGF(syst, out, in_)
    return S, grad


def grad_fd_2d(syst, out, in_, D, pixels, h=1e-6):
    """Central finite differences of F = 2 Re sum(D * S) at real-eps pixels
    [(m, n), ...]; returns dF/d eps there (compare with 2 Re g)."""
    res = []
    for m, n in pixels:
        vals = []
        for sgn in (1, -1):
            eps = np.array(syst["epsilon"], dtype=complex)
            eps[m, n] += sgn * h
            S, _ = cal_smatrix_RGF(dict(syst, epsilon=eps), out, in_)
            vals.append(2 * np.real(np.sum(np.asarray(D) * S)))
        res.append((vals[0] - vals[1]) / (2 * h))
    return np.array(res)

"""Independent dense check of the slice recursion -- TEST INFRASTRUCTURE ONLY.

Builds the whole block-tridiagonal operator for sites n = 0 .. L+1 (the two
reference planes of cal_smatrix_RGF.m:66-68 included) with the exact lead
self-energies folded into the end blocks, solves it densely, and applies the
Fisher-Lee relation of cal_smatrix_RGF.m:277-289.  It shares only the
channel set-up (B, C, G0) with ``oracle.rgf_ref``, so agreement pins the
recursion algebra (all five branches of cal_smatrix_RGF.m:217-280) against a
plain linear solve.

Block structure (slice operator A_n = A0 - k0dx^2 diag(eps_n), hopping -I):
    site 0     : G0_L^{-1}       (left lead surface, exact retarded BC)
    site n=1..L: A_n
    site L+1   : G0_R^{-1}
"""
from __future__ import annotations

import numpy as np

from .rgf_ref import (_delta_matrix, build_laplacian_1d, parse_channel_request,
                      setup_channels, setup_channels_3D)


def smatrix_dense_2d(syst, out, in_):
    """S of cal_smatrix_RGF from a dense solve of the whole operator."""
    return _dense_2d(syst, out, in_, fields=False)


def fields_dense_2d(syst, out, in_):
    """(S, psi): psi[:, n, b] = G_{n+1, side(b)} B_b, the response at slice n
    (site n+1) to input channel b (columns in S's order [in_L; in_R]), from
    the same dense inverse."""
    return _dense_2d(syst, out, in_, fields=True)


def _dense_2d(syst, out, in_, fields):
    eps = np.asarray(syst["epsilon"], dtype=complex)
    ny, nx = eps.shape
    k0dx = syst["k0dx"]
    ch = setup_channels(int(ny), syst["yBC"], k0dx, syst["epsilon_L"], syst["epsilon_R"])
    phi = ch["fun_phi"](ch["kydx"])
    A0 = -build_laplacian_1d(int(ny), syst["yBC"]) + 2 * np.eye(ny)
    return _dense(phi, ch["L"], ch["R"], ch["L"]["kxdx"], ch["R"]["kxdx"], A0, k0dx, eps, out, in_, fields)


def fields_dense_3d(syst, out, in_):
    """(S, psi) of cal_smatrix_RGF_3D from a dense solve: psi[:, n, b] at the
    nx*ny sites (x fastest) of slice n, as fields_dense_2d."""
    eps = np.asarray(syst["epsilon"], dtype=complex)
    if eps.ndim == 2:
        eps = eps[:, :, None]
    nx, ny, nz = eps.shape
    k0dx = syst["k0dx"]
    xyBC = syst["xyBC"]
    ch = setup_channels_3D(int(nx), int(ny), xyBC, k0dx, syst["epsilon_L"], syst["epsilon_R"])
    kxf, kyf = ch["kxdx"].ravel(order="F"), ch["kydx"].ravel(order="F")
    phi = np.stack([ch["fun_phi"](kxf[a], kyf[a]).ravel(order="F") for a in range(nx * ny)], axis=1)
    if isinstance(xyBC, str):
        xBC = yBC = xyBC
    else:
        xBC, yBC = (float(np.real(v)) for v in np.asarray(xyBC).ravel()[:2])
    A0 = (-np.kron(np.eye(ny), build_laplacian_1d(int(nx), xBC)) - np.kron(build_laplacian_1d(int(ny), yBC), np.eye(nx))
          + 2 * np.eye(nx * ny))
    return _dense(phi, ch["L"], ch["R"], ch["L"]["kzdx"].ravel(order="F"), ch["R"]["kzdx"].ravel(order="F"), A0, k0dx,
                  eps.reshape((nx * ny, nz), order="F"), out, in_, True)


def _dense(phi, chL, chR, kxL, kxR, A0, k0dx, eps, out, in_, fields):
    N, nx = eps.shape
    iiL, iiR = parse_channel_request(in_, "in", chL["N_prop"], chR["N_prop"])
    ioL, ioR = parse_channel_request(out, "out", chL["N_prop"], chR["N_prop"])
    G0L = (phi * np.exp(1j * kxL)[None, :]) @ phi.conj().T
    G0R = (phi * np.exp(1j * kxR)[None, :]) @ phi.conj().T
    nsite = nx + 2
    H = np.zeros((nsite * N, nsite * N), dtype=complex)

    def blk(i, j):
        return slice(i * N, (i + 1) * N), slice(j * N, (j + 1) * N)

    H[blk(0, 0)] = np.linalg.inv(G0L)
    H[blk(nsite - 1, nsite - 1)] = np.linalg.inv(G0R)
    for n in range(nx):
        H[blk(n + 1, n + 1)] = A0 - np.diag(k0dx ** 2 * eps[:, n])
    for s in range(nsite - 1):
        H[blk(s, s + 1)] = -np.eye(N)
        H[blk(s + 1, s)] = -np.eye(N)
    Ginv = np.linalg.inv(H)
    G_LL = Ginv[blk(0, 0)]
    G_LR = Ginv[blk(0, nsite - 1)]
    G_RL = Ginv[blk(nsite - 1, 0)]
    G_RR = Ginv[blk(nsite - 1, nsite - 1)]
    B_L = phi[:, chL["ind_prop"][iiL - 1] - 1] * chL["sqrt_mu"][iiL - 1][None, :]
    B_R = phi[:, chR["ind_prop"][iiR - 1] - 1] * chR["sqrt_mu"][iiR - 1][None, :]
    C_L = chL["sqrt_mu"][ioL - 1][:, None] * phi[:, chL["ind_prop"][ioL - 1] - 1].conj().T
    C_R = chR["sqrt_mu"][ioR - 1][:, None] * phi[:, chR["ind_prop"][ioR - 1] - 1].conj().T
    S = (-2j) * np.block([[C_L @ G_LL @ B_L, C_L @ G_LR @ B_R],
                          [C_R @ G_RL @ B_L, C_R @ G_RR @ B_R]])
    S = S - _delta_matrix(ioL, ioR, iiL, iiR)
    if not fields:
        return S
    psi = np.zeros((N, nx, B_L.shape[1] + B_R.shape[1]), dtype=complex)
    for n in range(nx):
        r = slice((n + 1) * N, (n + 2) * N)
        psi[:, n, :B_L.shape[1]] = Ginv[r, 0:N] @ B_L
        psi[:, n, B_L.shape[1]:] = Ginv[r, (nsite - 1) * N:] @ B_R
    return S, psi

"""L-split S-matrix on the CPU -- TEST INFRASTRUCTURE ONLY.

The reference's general-branch loop (cal_smatrix_RGF.m:257-269) run over a
part of the slices only: the left part [0, cut) from the left lead, the
right part [cut, L) from the right lead (the mirror loop of :217-236 /
:226-236), each ending in a segment state [[g, X], [Z, Y]] (g the
lead-connected Green's function of the part's last slice, X = G_{b,0} B,
Z = C G_{0,b}, Y = C G_{00} B on that part's lead), then the two joined
across the cut by the Dyson equation of two Green's functions coupled by the
hopping -I:

    C_L G_00 B_L = Y_L + Z_L (I - g_R g_L)^{-1} g_R X_L
    C_L G_0e B_R = Z_L (I - g_R g_L)^{-1} X_R
    C_R G_e0 B_L = Z_R (I - g_L g_R)^{-1} X_L
    C_R G_ee B_R = Y_R + Z_R (I - g_L g_R)^{-1} g_L X_R

and S = -2i C G B - delta (:279-289).  The states use the layout of
rgf_segment_sweep_2d: row-major (N + n_out_side) x (N + n_in_side).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from .rgf_ref import _delta_matrix, build_laplacian_1d, parse_channel_request, setup_channels


def _setup(syst, out, in_):
    eps = np.asarray(syst["epsilon"], dtype=complex)
    ny, nx = eps.shape
    k0dx = syst["k0dx"]
    ch = setup_channels(int(ny), syst["yBC"], k0dx, syst["epsilon_L"], syst["epsilon_R"])
    iiL, iiR = parse_channel_request(in_, "in", ch["L"]["N_prop"], ch["R"]["N_prop"])
    ioL, ioR = parse_channel_request(out, "out", ch["L"]["N_prop"], ch["R"]["N_prop"])
    phi = ch["fun_phi"](ch["kydx"])
    A0 = -build_laplacian_1d(int(ny), syst["yBC"]) + 2 * np.eye(ny)
    return eps, k0dx, ch, phi, A0, (iiL, iiR), (ioL, ioR)


def segment_state_2d(syst, out, in_, side: int, cut: int) -> np.ndarray:
    eps, k0dx, ch, phi, A0, ii, io = _setup(syst, out, in_)
    L = eps.shape[1]
    c = ch["L"] if side == 0 else ch["R"]
    i_in, i_out = ii[side], io[side]
    B = phi[:, c["ind_prop"][i_in - 1] - 1] * c["sqrt_mu"][i_in - 1][None, :]
    C = c["sqrt_mu"][i_out - 1][:, None] * phi[:, c["ind_prop"][i_out - 1] - 1].conj().T
    G0 = (phi * np.exp(1j * c["kxdx"])[None, :]) @ phi.conj().T
    g, Gn0, G0n, G00 = G0, G0, G0, G0
    slices = range(cut) if side == 0 else range(L - 1, cut - 1, -1)
    for n in slices:
        g = sla.inv(A0 - np.diag(k0dx ** 2 * eps[:, n]) - g)
        Gn0 = g @ Gn0
        G00 = G00 + G0n @ Gn0
        G0n = G0n @ g
    return np.block([[g, Gn0 @ B], [C @ G0n, C @ G00 @ B]])


def segment_merge_2d(syst, out, in_, state_L: np.ndarray, state_R: np.ndarray) -> np.ndarray:
    eps, k0dx, ch, phi, A0, ii, io = _setup(syst, out, in_)
    N = eps.shape[0]
    nL, nR = len(ii[0]), len(ii[1])
    gL, XL, ZL, YL = state_L[:N, :N], state_L[:N, N:N + nL], state_L[N:, :N], state_L[N:, N:N + nL]
    gR, XR, ZR, YR = state_R[:N, :N], state_R[:N, N:N + nR], state_R[N:, :N], state_R[N:, N:N + nR]
    I = np.eye(N)
    Dp = sla.inv(I - gR @ gL)
    D = sla.inv(I - gL @ gR)
    blocks = [[YL + ZL @ Dp @ gR @ XL, ZL @ Dp @ XR], [ZR @ D @ XL, YR + ZR @ D @ gL @ XR]]
    S = (-2j) * np.block(blocks)
    return S - _delta_matrix(io[0], io[1], ii[0], ii[1])

"""Generate the golden S-matrix fixtures from the CPU oracle.

    python tests/golden/make_golden.py            # small cases + configs 1, 3, 5, 4-subset
    python tests/golden/make_golden.py --config2  # also config 2 (N=1024, L=4096; ~15 min on 8 cores)

Small cases store their inputs explicitly; the configs store a checksum of
the seeded input from ``rgf_b200.workloads`` (regenerated by the tests) and
the oracle's S.  The oracle itself is pinned by tests/test_oracle.py.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.rgf_ref import cal_smatrix_RGF, cal_smatrix_RGF_3D  # noqa: E402
from rgf_b200 import workloads  # noqa: E402

FULL = (["left", "right"], ["left", "right"])
REQUESTS = {
    "full": FULL,
    "LL": (["left"], ["left"]),                        # branch 1
    "inL": (["left", "right"], ["left"]),              # branch 2
    "RR": (["right"], ["right"]),                      # branch 3
    "inR": (["left", "right"], ["right"]),             # branch 4
    "lists": ({"ind_out_L": [2, 1, 2], "ind_out_R": [1]}, {"ind_in_L": [1, 2], "ind_in_R": [2, 1]}),
}


def eps_checksum(eps: np.ndarray) -> np.ndarray:
    e = np.asarray(eps, dtype=complex).ravel(order="F")
    w = np.cos(np.arange(e.size) * 0.618)
    return np.array([np.sum(e.real * w), np.sum(e.imag * w), np.sum(np.abs(e))])


def small_cases():
    rng = np.random.default_rng(12345)
    cases = {}
    for bc in ["periodic", "Dirichlet", "Neumann", "DirichletNeumann", "NeumannDirichlet", 0.7]:
        ny, nx = 11, 6
        eps = 1 + 2 * rng.random((ny, nx)) + 0.05j * rng.random((ny, nx))
        tag = bc if isinstance(bc, str) else "Bloch"
        for rname, (out, in_) in REQUESTS.items():
            syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.7, k0dx=2 * np.pi / 6, yBC=bc)
            cases[f"2d_{tag}_{rname}"] = ("2d", syst, out, in_)
    # edge cases
    cases["2d_interface_nx0"] = ("2d", dict(epsilon=np.zeros((16, 0)), epsilon_L=1.0, epsilon_R=2.5,
                                            k0dx=2 * np.pi / 8, yBC="Dirichlet"), *FULL)
    cases["2d_ny1"] = ("2d", dict(epsilon=1 + rng.random((1, 7)), epsilon_L=1.0, epsilon_R=1.0,
                                  k0dx=0.9, yBC="periodic"), *FULL)
    cases["2d_ny2_bloch"] = ("2d", dict(epsilon=1 + rng.random((2, 5)), epsilon_L=1.0, epsilon_R=1.3,
                                        k0dx=1.1, yBC=0.4), *FULL)
    cases["2d_complexk"] = ("2d", dict(epsilon=1 + 2 * rng.random((40, 30)), epsilon_L=1.0, epsilon_R=1.0,
                                       k0dx=2 * np.pi / 12 * (1 + 3e-3j), yBC="periodic"), *FULL)
    cases["2d_highk_k2e_gt4"] = ("2d", dict(epsilon=1 + 3 * rng.random((20, 12)), epsilon_L=2.5, epsilon_R=3.0,
                                            k0dx=1.6, yBC="Dirichlet"), *FULL)
    cases["2d_complex_epsLR"] = ("2d", dict(epsilon=1 + 2 * rng.random((24, 10)), epsilon_L=1.2 + 0.01j,
                                            epsilon_R=2.0 - 0.02j, k0dx=2 * np.pi / 7, yBC="Neumann"), *FULL)
    cases["2d_large_N_gt_block"] = ("2d", dict(epsilon=1 + 3 * rng.random((100, 9)), epsilon_L=1.0, epsilon_R=1.0,
                                               k0dx=2 * np.pi / 15, yBC="periodic"), *FULL)
    cases["3d_periodic"] = ("3d", dict(epsilon=1 + rng.random((5, 4, 6)), epsilon_L=1.0, epsilon_R=1.5,
                                       k0dx=2 * np.pi / 5, xyBC="periodic"), *FULL)
    cases["3d_dirichlet"] = ("3d", dict(epsilon=1 + rng.random((6, 5, 4)), epsilon_L=1.0, epsilon_R=1.0,
                                        k0dx=2 * np.pi / 4, xyBC="Dirichlet"), *FULL)
    cases["3d_bloch_inR"] = ("3d", dict(epsilon=1 + rng.random((4, 6, 5)), epsilon_L=1.2, epsilon_R=1.0,
                                        k0dx=2 * np.pi / 5, xyBC=[0.3, -0.8]), ["left", "right"], ["right"])
    cases["3d_nx1"] = ("3d", dict(epsilon=1 + rng.random((1, 9, 5)), epsilon_L=1.0, epsilon_R=1.0,
                                  k0dx=2 * np.pi / 6, xyBC="periodic"), *FULL)
    return cases


def singular_leading_block_eps(ny: int, nx: int, k0dx: float, seed: int) -> np.ndarray:
    """Permittivity whose first slice matrix M_1 = A0 - k0dx^2 diag(eps_1) -
    G0_L has an exactly singular leading 32 x 32 block (up to rounding) while
    M_1 itself is well conditioned: eps_1 on sites 0..31 is the constant
    lambda / k0dx^2, lambda an eigenvalue of (A0 - G0_L)[0:32, 0:32]
    (Dirichlet BC, epsilon_L = 1; cal_smatrix_RGF.m:209, 260, 265).  Pivoting
    inside that block alone cannot invert M_1 accurately; pivoting over the
    whole column (MATLAB's inv) can."""
    from oracle.rgf_ref import build_laplacian_1d, setup_channels
    rng = np.random.default_rng(seed)
    eps = (1.0 + 2.0 * rng.random((ny, nx))).astype(complex)
    ch = setup_channels(ny, "Dirichlet", k0dx, 1.0, 1.0)
    phi = ch["fun_phi"](ch["kydx"])
    G0 = (phi * np.exp(1j * ch["L"]["kxdx"])[None, :]) @ phi.conj().T
    A0 = -build_laplacian_1d(ny, "Dirichlet") + 2 * np.eye(ny)
    lam = np.linalg.eigvals((A0 - G0)[:32, :32])
    target = k0dx ** 2 * 2.0  # the eigenvalue closest to a plausible k0dx^2 eps
    eps[:32, 0] = lam[np.argmin(np.abs(lam - target))] / k0dx ** 2
    return eps


def pivot_cases():
    """Slice matrices far from diagonal dominance, several 32-wide pivot
    blocks each (N >= 100): k0dx^2 eps_L at and beyond 4 (setup_channels.m:
    211-215), high index contrast, gain (Im eps < 0), and a leading pivot
    block that is singular although the slice matrix is not."""
    rng = np.random.default_rng(777)
    cases = {}
    for tag, k2e in (("3p5", 3.5), ("3p95", 3.95), ("4p5", 4.5), ("6", 6.0)):
        k0dx = float(np.sqrt(k2e / 1.0))
        eps = 1.0 + 3.0 * rng.random((128, 14)) + 0.01j * rng.random((128, 14))
        cases[f"2d_pivot_k2e_{tag}"] = ("2d", dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.5, k0dx=k0dx,
                                                   yBC="Dirichlet"), *FULL)
    eps = np.where(rng.random((128, 20)) < 0.5, 12.0, 1.0) + 0.0j
    cases["2d_pivot_contrast12"] = ("2d", dict(epsilon=eps, epsilon_L=1.0, epsilon_R=12.0, k0dx=2 * np.pi / 10,
                                               yBC="periodic"), *FULL)
    eps = 2.0 + 2.0 * rng.random((100, 15)) - 0.3j * rng.random((100, 15))
    cases["2d_pivot_gain"] = ("2d", dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 9,
                                         yBC="Neumann"), *FULL)
    k0dx = 2 * np.pi / 15
    cases["2d_pivot_singular_block"] = ("2d", dict(epsilon=singular_leading_block_eps(96, 6, k0dx, 778),
                                                   epsilon_L=1.0, epsilon_R=1.0, k0dx=k0dx, yBC="Dirichlet"),
                                        *FULL)
    return cases


def config_cases(with_cfg2: bool):
    out = {}
    s, o, i = workloads.config1()
    out["cfg1"] = ("2d", s, o, i)
    s, o, i = workloads.config3()
    out["cfg3"] = ("3d", s, o, i)
    s, o, i = workloads.config5()
    out["cfg5"] = ("2d", s, o, i)
    for k in workloads.CONFIG4_SUBSAMPLE:
        s, o, i = workloads.config4_structure(k)
        out[f"cfg4_{k}"] = ("2d", s, o, i)
    if with_cfg2:
        s, o, i = workloads.config2()
        out["cfg2"] = ("2d", s, o, i)
    return out


def save_case(name, dim, syst, out, in_, store_inputs: bool):
    t = time.time()
    fn = cal_smatrix_RGF if dim == "2d" else cal_smatrix_RGF_3D
    S, ch = fn(syst, out, in_)
    dt = time.time() - t
    rec = {"S": S, "dim": dim, "oracle_seconds": dt, "eps_checksum": eps_checksum(syst["epsilon"])}
    bc = syst["yBC"] if dim == "2d" else syst["xyBC"]
    rec["bc"] = np.array(bc, dtype=object) if isinstance(bc, str) else np.asarray(bc, dtype=float)
    for k in ("epsilon_L", "epsilon_R", "k0dx"):
        rec[k] = np.complex128(syst[k])
    if store_inputs:
        rec["epsilon"] = np.asarray(syst["epsilon"])
    rec["request"] = np.array(repr((out, in_)), dtype=object)
    for side in ("L", "R"):
        rec[f"N_prop_{side}"] = ch[side]["N_prop"]
        rec[f"ind_prop_{side}"] = ch[side]["ind_prop"]
        rec[f"sqrt_mu_{side}"] = ch[side]["sqrt_mu"]
        rec[f"kx_{side}"] = ch[side]["kxdx" if dim == "2d" else "kzdx"]
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **rec)
    print(f"{name:28s} S{S.shape} oracle {dt:7.2f}s -> {os.path.relpath(path, ROOT)}")


def main():
    with_cfg2 = "--config2" in sys.argv
    only_cfg2 = "--only-config2" in sys.argv
    only = [a.split("=", 1)[1] for a in sys.argv if a.startswith("--only=")]
    if not only_cfg2:
        cases = dict(small_cases())
        cases.update(pivot_cases())
        for name, (dim, syst, out, in_) in cases.items():
            if only and name not in only:
                continue
            save_case(name, dim, syst, out, in_, store_inputs=True)
    for name, (dim, syst, out, in_) in config_cases(with_cfg2 or only_cfg2).items():
        if only_cfg2 and name != "cfg2":
            continue
        if only and name not in only:
            continue
        save_case(name, dim, syst, out, in_, store_inputs=False)


if __name__ == "__main__":
    main()

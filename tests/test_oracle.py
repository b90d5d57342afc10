"""Pins of the CPU oracle (no GPU): the reference ships no golden vectors,
so the oracle is checked against an independent dense solve, analytic known
answers and the invariants the reference's examples print
(examples/example_script.m:26-35)."""
import glob
import os

import numpy as np
import pytest

from oracle.dense_fdfd import smatrix_dense_2d
from oracle.rgf_ref import (build_laplacian_1d, cal_smatrix_RGF, cal_smatrix_RGF_3D, setup_channels,
                            setup_channels_3D)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
BCS = ["periodic", "Dirichlet", "Neumann", "DirichletNeumann", "NeumannDirichlet", 0.7]
REQS = {
    "full": (["left", "right"], ["left", "right"]),
    "LL": (["left"], ["left"]),
    "inL": (["left", "right"], ["left"]),
    "RR": (["right"], ["right"]),
    "inR": (["left", "right"], ["right"]),
    "lists": ({"ind_out_L": [2, 1, 2], "ind_out_R": [1]}, {"ind_in_L": [1, 2], "ind_in_R": [2, 1]}),
}


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _syst(bc, rng, ny=10, nx=5, eL=1.0, eR=1.6, k0dx=2 * np.pi / 6, absorb=0.0):
    eps = 1 + 2 * rng.random((ny, nx)) + 1j * absorb * rng.random((ny, nx))
    return dict(epsilon=eps, epsilon_L=eL, epsilon_R=eR, k0dx=k0dx, yBC=bc)


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("req", list(REQS))
def test_oracle_matches_dense_solve(bc, req):
    """All five branches of cal_smatrix_RGF.m:217-280 against a dense
    block-tridiagonal solve with exact lead self-energies."""
    rng = np.random.default_rng(7)
    syst = _syst(bc, rng, absorb=0.05)
    out, in_ = REQS[req]
    S, _ = cal_smatrix_RGF(syst, out, in_)
    Sd = smatrix_dense_2d(syst, out, in_)
    assert S.shape == Sd.shape
    assert rel(S, Sd) < 1e-12


@pytest.mark.parametrize("bc", ["periodic", "Dirichlet", "Neumann", 0.4])
@pytest.mark.parametrize("k0dx", [2 * np.pi / 5, 1.7])  # 1.7: k0dx^2 eps > 4 (branch flip active)
def test_homogeneous_slab_known_answer(bc, k0dx):
    """eps == eps_L == eps_R: r = 0 and t = diag(exp(1i kx (nx+1)))."""
    ny, nx = 8, 5
    syst = dict(epsilon=np.full((ny, nx), 1.3), epsilon_L=1.3, epsilon_R=1.3, k0dx=k0dx, yBC=bc)
    S, ch = cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"])
    P = ch["L"]["N_prop"]
    kx = ch["L"]["kxdx"][ch["L"]["ind_prop"] - 1]
    assert np.abs(S[:P, :P]).max() < 1e-13
    assert np.abs(S[P:, :P] - np.diag(np.exp(1j * kx * (nx + 1)))).max() < 1e-13


@pytest.mark.parametrize("bc", BCS)
def test_interface_nx0_unitary(bc):
    """L = 0 (cal_smatrix_RGF.m:15-16): the bare eps_L | eps_R interface."""
    syst = dict(epsilon=np.zeros((12, 0)), epsilon_L=1.0, epsilon_R=2.4, k0dx=2 * np.pi / 7, yBC=bc)
    S, _ = cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"])
    assert np.abs(S.conj().T @ S - np.eye(S.shape[0])).max() < 1e-13


@pytest.mark.parametrize("bc", BCS)
def test_unitarity_and_reciprocity(bc):
    """examples/example_script.m:26-35 on a random real structure."""
    rng = np.random.default_rng(3)
    syst = _syst(bc, rng, ny=14, nx=9, eL=1.0, eR=1.0)
    S, ch = cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"])
    assert np.abs(S.conj().T @ S - np.eye(S.shape[0])).max() < 1e-12
    if "ind_prop_conj" in ch["L"]:
        p = np.concatenate([ch["L"]["ind_prop_conj"], ch["L"]["N_prop"] + ch["R"]["ind_prop_conj"]]) - 1
        St = S[p, :]
        assert np.abs(St.T - St).max() < 1e-12
    else:
        assert bc == 0.7  # Bloch ka != 0 has no conj permutation (setup_channels.m:80-82)


def test_cross_branch_consistency():
    rng = np.random.default_rng(11)
    syst = _syst("Dirichlet", rng, ny=12, nx=7, absorb=0.02)
    S, ch = cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"])
    PL, PR = ch["L"]["N_prop"], ch["R"]["N_prop"]
    blocks = {"LL": S[:PL, :PL], "inL": S[:, :PL], "RR": S[PL:, PL:], "inR": S[:, PL:]}
    for name, ref in blocks.items():
        Sb, _ = cal_smatrix_RGF(syst, *REQS[name])
        assert rel(Sb, ref) < 1e-12, name


def test_2d_equals_3d_with_unit_axis():
    """Periodic 2D == 3D with nx = 1 (Lap_x = 0 there)."""
    rng = np.random.default_rng(5)
    ny, nx = 9, 6
    eps = 1 + 2 * rng.random((ny, nx))
    s2 = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.4, k0dx=2 * np.pi / 5, yBC="periodic")
    s3 = dict(epsilon=eps[None, :, :], epsilon_L=1.0, epsilon_R=1.4, k0dx=2 * np.pi / 5, xyBC="periodic")
    S2, c2 = cal_smatrix_RGF(s2, ["left", "right"], ["left", "right"])
    S3, c3 = cal_smatrix_RGF_3D(s3, ["left", "right"], ["left", "right"])
    assert S2.shape == S3.shape
    assert rel(S3, S2) < 1e-12


def test_complex_frequency_continuity():
    rng = np.random.default_rng(8)
    syst = _syst("periodic", rng, ny=16, nx=6, eL=1.0, eR=1.0, k0dx=2 * np.pi / 9)
    S0, _ = cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"])
    errs = []
    for eta in (1e-4, 1e-6, 1e-8):
        s = dict(syst, k0dx=syst["k0dx"] * (1 + 1j * eta))
        S, _ = cal_smatrix_RGF(s, ["left", "right"], ["left", "right"])
        errs.append(rel(S, S0))
    assert errs[2] < errs[1] < errs[0] and errs[2] < 1e-6


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("n", [1, 2, 7, 8])
def test_laplacian_eigenbasis(bc, n):
    """phi diagonalises -Lap with eigenvalues 4 sin^2(ky/2); phi is unitary."""
    ch = setup_channels(n, bc, 0.5, 1.0, 1.0)
    phi = ch["fun_phi"](ch["kydx"])
    A = -build_laplacian_1d(n, bc)
    assert np.abs(phi.conj().T @ phi - np.eye(n)).max() < 1e-13
    lam = 4 * np.sin(ch["kydx"] / 2) ** 2
    assert np.abs(A @ phi - phi * lam[None, :]).max() < 1e-12


def test_laplacian_1_site_bloch_is_physical():
    """Quirk Q9: n = 1 Bloch gives 2cos(ka) - 2."""
    ka = 0.9
    assert abs(build_laplacian_1d(1, ka)[0, 0] - (2 * np.cos(ka) - 2)) < 1e-15


@pytest.mark.parametrize("k0dx", [0.5, 1.7, 2.2, 1.7 * (1 + 1e-3j), 0.9 * (1 - 2e-3j)])
def test_kx_branch(k0dx):
    """setup_channels.m:201-215: real k0dx -> 0<kx<pi propagating, Im kx >= 0
    evanescent; the lead G0 is the fixed point G0 = (A_lead - G0)^{-1}."""
    ny = 9
    ch = setup_channels(ny, "Dirichlet", k0dx, 1.1)
    kx = ch["L"]["kxdx"]
    if np.imag(k0dx) == 0:
        prop = ch["L"]["ind_prop"] - 1
        assert np.all(np.abs(kx[prop].imag) == 0) and np.all((kx[prop].real > 0) & (kx[prop].real < np.pi))
        ev = np.setdiff1d(np.arange(ny), prop)
        assert np.all(kx[ev].imag >= 0)
    phi = ch["fun_phi"](ch["kydx"])
    G0 = (phi * np.exp(1j * kx)) @ phi.conj().T
    A = -build_laplacian_1d(ny, "Dirichlet") + 2 * np.eye(ny) - k0dx ** 2 * 1.1 * np.eye(ny)
    assert np.abs(G0 - np.linalg.inv(A - G0)).max() < 1e-12


def test_matlab_asin_convention_above_one():
    """For real z > 1 MATLAB's asin(sqrt(z)) is pi/2 - 1i*acosh(sqrt(z));
    after the flip kxdx = -pi + 2i*acosh(sqrt(z))."""
    ch = setup_channels(4, "Dirichlet", 2.5, 1.0)
    z = 0.25 * 2.5 ** 2 - np.sin(ch["kydx"] / 2) ** 2
    big = z > 1
    assert big.any()
    expect = -np.pi + 2j * np.arccosh(np.sqrt(z[big]))
    assert np.abs(ch["L"]["kxdx"][big] - expect).max() < 1e-14


def test_3d_channels_layout():
    ch = setup_channels_3D(3, 4, [0.2, -0.5], 2.0, 1.0, 1.0)
    assert ch["kxdx"].shape == (3, 4) and ch["kydx"].shape == (3, 4)
    assert np.all(ch["kxdx"][:, 0] == ch["kxdx"][:, 1]) and np.all(ch["kydx"][0] == ch["kydx"][1])


def test_request_parsing_errors():
    rng = np.random.default_rng(0)
    syst = _syst("periodic", rng)
    with pytest.raises(ValueError):
        cal_smatrix_RGF(syst, "left", ["left"])
    with pytest.raises(ValueError):
        cal_smatrix_RGF(syst, {"ind_out_L": [0]}, ["left"])
    with pytest.raises(ValueError):
        cal_smatrix_RGF(syst, {"ind_out_L": [1.5]}, ["left"])
    with pytest.warns(UserWarning):
        S, _ = cal_smatrix_RGF(syst, ["left", "up"], ["left"])
    S, _ = cal_smatrix_RGF(syst, ["left"], {})
    assert S.shape[1] == 0


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "2d_*.npz")) +
                                        glob.glob(os.path.join(GOLDEN, "3d_*.npz"))))
def test_golden_small_fixtures_reproduce(path):
    """The committed small fixtures are reproduced by the oracle."""
    from tests.golden_io import load_case
    case = load_case(path)
    fn = cal_smatrix_RGF if case["dim"] == "2d" else cal_smatrix_RGF_3D
    S, _ = fn(case["syst"], case["out"], case["in"])
    assert rel(S, case["S"]) < 1e-13


# ---------------------------------------------------------------------------
# permittivity gradient (an addition of this build; the reference has none)
# ---------------------------------------------------------------------------
GRAD_CASES = [
    ("periodic", ["left", "right"], ["left", "right"]),
    ("Dirichlet", {"ind_out_R": [1, 2]}, {"ind_in_L": [2, 1]}),
    ("Neumann", ["left"], ["left"]),
    (0.4, ["right"], ["left", "right"]),
    ("DirichletNeumann", ["left", "right"], ["right"]),
    ("periodic", {"ind_out_L": [1], "ind_out_R": [2, 1]}, {"ind_in_R": [1]}),
]


@pytest.mark.parametrize("bc,out,inp", GRAD_CASES)
def test_adjoint_recursion_matches_dense_gradient(bc, out, inp):
    """The backward recursions over the start-connected blocks give the same
    dS/d eps as the dense inverse, for every request form and direction."""
    from oracle.adjoint import grad_dense_2d, grad_rgf_2d
    rng = np.random.default_rng(11)
    syst = dict(epsilon=1 + 2 * rng.random((7, 5)) + 0.01j * rng.random((7, 5)), epsilon_L=1.0,
                epsilon_R=1.3, k0dx=1.1, yBC=bc)
    S0, _ = cal_smatrix_RGF(syst, out, inp)
    D = rng.standard_normal(S0.shape) + 1j * rng.standard_normal(S0.shape)
    _, g1 = grad_dense_2d(syst, out, inp, D)
    _, g2 = grad_rgf_2d(syst, out, inp, D)
    assert np.abs(g1 - g2).max() <= 1e-12 * np.abs(g1).max()


@pytest.mark.parametrize("bc,out,inp", GRAD_CASES[:3])
def test_adjoint_matches_finite_differences(bc, out, inp):
    from oracle.adjoint import grad_fd_2d, grad_rgf_2d
    rng = np.random.default_rng(12)
    syst = dict(epsilon=1 + 2 * rng.random((7, 5)), epsilon_L=1.0, epsilon_R=1.0, k0dx=1.1, yBC=bc)
    S0, _ = cal_smatrix_RGF(syst, out, inp)
    D = rng.standard_normal(S0.shape) + 1j * rng.standard_normal(S0.shape)
    _, g = grad_rgf_2d(syst, out, inp, D)
    pix = [(1, 2), (6, 0), (3, 4)]
    fd = grad_fd_2d(syst, out, inp, D, pix)
    an = 2 * np.real(np.array([g[m, n] for m, n in pix]))
    assert np.abs(an - fd).max() <= 1e-7 * np.abs(fd).max()

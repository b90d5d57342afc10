"""GPU parity of the permittivity gradient (rgf_smatrix_grad_2d/3d through the
C ABI) against the oracle's recursion form (oracle/adjoint.py, itself pinned
to the dense inverse and to finite differences), for every request form,
both engines and several checkpoint intervals.

Tolerance: max |g - g_oracle| <= 1e-10 max |g_oracle| (FP64 throughout)."""
import numpy as np
import pytest
import torch

import rgf_b200
from oracle.adjoint import grad_rgf_2d
from oracle.rgf_ref import cal_smatrix_RGF as ref_smatrix
from rgf_b200 import workloads

pytestmark = pytest.mark.gpu
TOL_G = 1e-10

CASES = [
    ("periodic", ["left", "right"], ["left", "right"]),
    ("Dirichlet", {"ind_out_R": [1, 2]}, {"ind_in_L": [2, 1]}),
    ("Neumann", ["left"], ["left"]),
    (0.4, ["right"], ["left", "right"]),
    ("DirichletNeumann", ["left", "right"], ["right"]),
    ("periodic", {"ind_out_L": [1], "ind_out_R": [2, 1]}, {"ind_in_R": [1]}),
]


def relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("ckpt", [0, 2])
@pytest.mark.parametrize("bc,out,inp", CASES)
def test_gradient_matches_oracle_small(bc, out, inp, engine, ckpt):
    rng = np.random.default_rng(21)
    syst = dict(epsilon=1 + 2 * rng.random((7, 5)) + 0.01j * rng.random((7, 5)), epsilon_L=1.0,
                epsilon_R=1.3, k0dx=1.1, yBC=bc)
    S0, _ = ref_smatrix(syst, out, inp)
    D = rng.standard_normal(S0.shape) + 1j * rng.standard_normal(S0.shape)
    S, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, D, checkpoint=ckpt, options={"engine": engine})
    _, g0 = grad_rgf_2d(syst, out, inp, D)
    assert np.linalg.norm(S - S0) <= 1e-11 * np.linalg.norm(S0)
    assert relmax(g, g0) <= TOL_G


@pytest.mark.parametrize("ny,nx,bc,out,inp", [
    (100, 9, "Dirichlet", ["left", "right"], ["left", "right"]),
    (70, 13, "periodic", {"ind_out_R": [1, 2, 3]}, {"ind_in_L": [1, 2]}),
])
def test_gradient_matches_oracle_multiblock(ny, nx, bc, out, inp):
    """N > 32: several pivot blocks per slice in the persistent kernel."""
    rng = np.random.default_rng(ny)
    syst = dict(epsilon=1 + 3 * rng.random((ny, nx)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15, yBC=bc)
    S0, _ = ref_smatrix(syst, out, inp)
    D = np.conj(S0)
    for ckpt in (0, 4):
        _, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, D, checkpoint=ckpt)
        _, g0 = grad_rgf_2d(syst, out, inp, D)
        assert relmax(g, g0) <= TOL_G


def test_gradient_config5_reduced():
    """The config-5 request (branch 2: 8 left inputs -> 8 right outputs,
    F = sum |t|^2) on its first 64 slices."""
    syst, out, inp = workloads.config5()
    syst = dict(syst, epsilon=np.ascontiguousarray(syst["epsilon"][:, :64]))
    S0, _ = ref_smatrix(syst, out, inp)
    _, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, np.conj(S0), checkpoint=23)
    _, g0 = grad_rgf_2d(syst, out, inp, np.conj(S0))
    assert relmax(g, g0) <= TOL_G


def test_gradient_config5_full():
    """The whole config-5 gradient (N=256, L=512: 256 x 512 pixels, 8 left
    inputs -> 8 right outputs, F = sum |t_ab|^2, checkpoint every 23 slices)
    against the oracle's recursion form."""
    syst, out, inp = workloads.config5()
    S0, _ = ref_smatrix(syst, out, inp)
    S, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, np.conj(S0), checkpoint=23)
    _, g0 = grad_rgf_2d(syst, out, inp, np.conj(S0))
    assert g.shape == (256, 512)
    assert np.linalg.norm(S - S0) <= 1e-11 * np.linalg.norm(S0)
    assert relmax(g, g0) <= TOL_G


def test_gradient_config5_finite_differences():
    """dF/d eps = 2 Re g of F = sum |t_ab|^2 at config 5 against central
    differences of the GPU's own S (h = 1e-6, FP64) on 32 pixels drawn with
    seed 55.  The difference quotient carries up to ~1e-13 |F| / h ~ 1e-6 of
    round-off (S is computed to ~1e-13 relative), hence the absolute floor."""
    syst, out, inp = workloads.config5()
    S, _ = rgf_b200.cal_smatrix_RGF(syst, out, inp)
    _, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, np.conj(S), checkpoint=23)
    F = lambda Sx: float(np.sum(np.abs(Sx) ** 2))  # noqa: E731
    rng = np.random.default_rng(55)
    ms, ns = rng.integers(0, 256, 32), rng.integers(0, 512, 32)
    h = 1e-6
    fds, gs = [], []
    for m, n in zip(ms, ns):
        vals = []
        for sgn in (1, -1):
            eps = syst["epsilon"].copy()
            eps[m, n] += sgn * h
            Sp, _ = rgf_b200.cal_smatrix_RGF(dict(syst, epsilon=eps), out, inp)
            vals.append(F(Sp))
        fds.append((vals[0] - vals[1]) / (2 * h))
        gs.append(2 * np.real(g[m, n]))
    fds, gs = np.array(fds), np.array(gs)
    floor = 1e-13 * F(S) / h  # round-off of the difference quotient
    assert np.all(np.abs(gs - fds) <= 1e-6 * np.abs(fds) + floor), np.abs(gs - fds).max()


def test_gradient_finite_differences_on_device():
    """2 Re g against central differences of the GPU's own S (h = 1e-6; the
    difference quotient carries ~eps_mach |F| / h ~ 1e-9 of round-off, hence
    the absolute floor of the tolerance)."""
    rng = np.random.default_rng(5)
    syst = dict(epsilon=1 + 3 * rng.random((40, 30)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15,
                yBC="periodic")
    out, inp = {"ind_out_R": [1, 2, 3]}, {"ind_in_L": [1, 2]}
    S, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, np.zeros((3, 2)))
    D = np.conj(S)
    _, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, D)
    pix = [(int(m), int(n)) for m, n in zip(rng.integers(0, 40, 8), rng.integers(0, 30, 8))]
    h = 1e-6
    for m, n in pix:
        vals = []
        for sgn in (1, -1):
            eps = syst["epsilon"].copy()
            eps[m, n] += sgn * h
            Sp, _ = rgf_b200.cal_smatrix_RGF(dict(syst, epsilon=eps), out, inp)
            vals.append(2 * np.real(np.sum(D * Sp)))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(2 * np.real(g[m, n]) - fd) <= 1e-6 * abs(fd) + 1e-8


def test_gradient_3d_finite_differences():
    rng = np.random.default_rng(6)
    syst = dict(epsilon=np.where(rng.random((5, 6, 7)) < 0.4, 2.25, 1.0), epsilon_L=1.0, epsilon_R=1.0,
                k0dx=2 * np.pi / 6, xyBC=[0.3, 0.7])
    out, inp = ["right"], ["left"]
    S, _ = rgf_b200.cal_smatrix_RGF_3D(syst, out, inp)
    D = np.conj(S)
    _, g = rgf_b200.smatrix_grad_RGF_3D(syst, out, inp, D, checkpoint=3)
    assert g.shape == (5, 6, 7)
    h = 1e-6
    for (x, y, z) in [(0, 0, 0), (4, 5, 6), (2, 3, 3), (1, 4, 5)]:
        vals = []
        for sgn in (1, -1):
            eps = syst["epsilon"].copy()
            eps[x, y, z] += sgn * h
            Sp, _ = rgf_b200.cal_smatrix_RGF_3D(dict(syst, epsilon=eps), out, inp)
            vals.append(2 * np.real(np.sum(D * Sp)))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(2 * np.real(g[x, y, z]) - fd) <= 1e-6 * abs(fd) + 1e-8


def test_torch_autograd_harness():
    from rgf_b200.autograd import SMatrix
    rng = np.random.default_rng(7)
    syst = dict(epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15, yBC="periodic")
    eps = torch.tensor(1 + 3 * rng.random((32, 20)), dtype=torch.float64, requires_grad=True)
    out, inp = {"ind_out_R": [1, 2]}, {"ind_in_L": [1, 2]}
    S = SMatrix.apply(eps, syst, out, inp)
    loss = (S.abs() ** 2).sum()
    loss.backward()
    S_np = S.detach().numpy()
    _, g = rgf_b200.smatrix_grad_RGF(dict(syst, epsilon=eps.detach().numpy()), out, inp, np.conj(S_np))
    assert np.abs(eps.grad.numpy() - 2 * np.real(g)).max() <= 1e-12 * np.abs(2 * np.real(g)).max()


def test_gradient_many_channels():
    """More than 32 channels on a side: the backward pass takes its GEMM path
    (the one-launch step serves up to 32 x 32)."""
    rng = np.random.default_rng(30)
    syst = dict(epsilon=1 + 2 * rng.random((260, 4)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15,
                yBC="periodic")
    out, inp = ["left", "right"], ["left", "right"]
    S0, _ = ref_smatrix(syst, out, inp)
    assert min(S0.shape) > 64
    D = np.conj(S0)
    _, g = rgf_b200.smatrix_grad_RGF(syst, out, inp, D, checkpoint=2)
    _, g0 = grad_rgf_2d(syst, out, inp, D)
    assert relmax(g, g0) <= TOL_G

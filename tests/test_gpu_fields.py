"""Fields inside the structure (rgf_fields_2d/3d through the C ABI) against a
dense solve of the whole block-tridiagonal operator (oracle/dense_fdfd.py):
psi[:, n, b] = G_{n, s(b)} B_b for every slice n and requested input b, for
every request form, both engines and several checkpoint intervals.

Tolerance: max |psi - psi_dense| <= 1e-11 max |psi_dense| (FP64 throughout)."""
import numpy as np
import pytest

import rgf_b200
from oracle.dense_fdfd import fields_dense_2d

pytestmark = pytest.mark.gpu
TOL = 1e-11


def relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


CASES = [
    ("periodic", ["left", "right"], ["left", "right"]),
    ("Dirichlet", {"ind_out_R": [1, 2]}, {"ind_in_L": [2, 1]}),
    ("Neumann", ["left"], ["left"]),
    (0.4, ["right"], ["right"]),
    ("DirichletNeumann", ["left", "right"], ["right"]),
]


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("ckpt", [0, 3])
@pytest.mark.parametrize("bc,out,inp", CASES)
def test_fields_match_dense_solve(bc, out, inp, engine, ckpt):
    rng = np.random.default_rng(12)
    syst = dict(epsilon=1 + 2 * rng.random((9, 7)) + 0.02j * rng.random((9, 7)), epsilon_L=1.0, epsilon_R=1.4,
                k0dx=1.1, yBC=bc)
    S, psi = rgf_b200.fields_RGF(syst, out, inp, checkpoint=ckpt, options={"engine": engine})
    S0, psi0 = fields_dense_2d(syst, out, inp)
    assert np.linalg.norm(S - S0) <= 1e-11 * np.linalg.norm(S0)
    assert psi.shape == psi0.shape
    assert relmax(psi, psi0) <= TOL


def test_fields_multiblock():
    """N > 32 (several pivot blocks) and the persistent engine."""
    rng = np.random.default_rng(13)
    syst = dict(epsilon=1 + 3 * rng.random((70, 11)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15,
                yBC="periodic")
    S, psi = rgf_b200.fields_RGF(syst, ["left", "right"], {"ind_in_L": [1, 3], "ind_in_R": [2]})
    S0, psi0 = fields_dense_2d(syst, ["left", "right"], {"ind_in_L": [1, 3], "ind_in_R": [2]})
    assert relmax(psi, psi0) <= TOL


def test_fields_energy_flux_real_eps():
    """A homogeneous slab (eps = eps_L = 1): the field of channel b is the
    lead's own propagating mode, psi[:, n, b] = G0-propagated profile with
    |psi| constant along the slab (no reflection)."""
    syst = dict(epsilon=np.ones((16, 10)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 8, yBC="periodic")
    _, psi = rgf_b200.fields_RGF(syst, ["right"], {"ind_in_L": [1]})
    amp = np.linalg.norm(psi[:, :, 0], axis=0)
    assert np.abs(amp - amp[0]).max() <= 1e-12 * amp[0]


@pytest.mark.parametrize("bc,out,inp", [
    ("periodic", ["left", "right"], ["left", "right"]),
    ("Dirichlet", ["right"], ["left"]),
    ([0.3, -0.2], {"ind_out_L": [1]}, {"ind_in_R": [2, 1]}),
])
def test_fields_3d_match_dense_solve(bc, out, inp):
    """3D: psi[x, y, n, b] against the dense solve of the whole operator."""
    from oracle.dense_fdfd import fields_dense_3d
    rng = np.random.default_rng(15)
    syst = dict(epsilon=1 + rng.random((4, 3, 5)), epsilon_L=1.0, epsilon_R=1.3, k0dx=2 * np.pi / 5, xyBC=bc)
    S, psi = rgf_b200.fields_RGF_3D(syst, out, inp, checkpoint=2)
    S0, psi0 = fields_dense_3d(syst, out, inp)
    assert np.linalg.norm(S - S0) <= 1e-11 * np.linalg.norm(S0)
    assert psi.shape == (4, 3, 5, psi0.shape[2])
    assert relmax(psi.reshape((12, 5, -1), order="F"), psi0) <= TOL

"""GPU parity of the split-precision form (options precision = RGF_TF32X3):
slice inverses factored in FP32 with 3xTF32 tcgen05 updates, S won back by
FP64 iterative refinement.  Against the FP64 oracle's golden S-matrices:

* relative Frobenius error of S <= 1e-10 (the tolerance this form is held
  to), for every fixture, whether the refinement's result stands or the call
  fell back to the FP64 form;
* on the configurations it is built for (config 1, 2 and 3 and the small
  cases) the refinement must converge: its own result stands;
* reciprocity S = S^T for Dirichlet structures at <= 1e-12.
"""
import glob
import os

import numpy as np
import pytest

import rgf_b200
from rgf_b200 import _abi
from tests.golden_io import config_case, load_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SMALL = sorted(glob.glob(os.path.join(GOLDEN, "2d_*.npz")) + glob.glob(os.path.join(GOLDEN, "3d_*.npz")))
TOL_S = 1e-10
OPT = {"precision": _abi.RGF_TF32X3}


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run(case, h):
    fn = rgf_b200.cal_smatrix_RGF if case["dim"] == "2d" else rgf_b200.cal_smatrix_RGF_3D
    return fn(case["syst"], case["out"], case["in"], options=OPT, handle=h)


@pytest.fixture(scope="module")
def handle():
    return _abi.Handle(0)


@pytest.mark.parametrize("path", SMALL, ids=lambda p: os.path.basename(p)[:-4])
def test_small_golden(path, handle):
    case = load_case(path)
    S, ch = run(case, handle)
    info = handle.refinement()
    assert S.shape == case["S"].shape
    err = rel(S, case["S"])
    assert err <= TOL_S, (err, info)
    nx = np.asarray(case["syst"]["epsilon"]).shape[-1] if "epsilon" in case["syst"] else 0
    if nx > 0 and "pivot" not in case["name"]:
        assert info["form"] == _abi.RGF_TF32X3, info  # the refinement's own result
    for side in ("L", "R"):
        assert ch[side]["N_prop"] == case[f"N_prop_{side}"]


@pytest.mark.parametrize("name", ["cfg1", "cfg3", "cfg5", "cfg4_0", "cfg4_7"])
def test_config_golden(name, handle):
    case = config_case(name)
    if case is None:
        pytest.skip(f"no fixture {name}")
    S, _ = run(case, handle)
    info = handle.refinement()
    print(name, info)
    assert rel(S, case["S"]) <= TOL_S, info
    assert info["form"] == _abi.RGF_TF32X3, info


def test_config2_golden(handle):
    """The headline workload (N=1024, L=4096): the refinement's S against the oracle."""
    case = config_case("cfg2")
    if case is None:
        pytest.skip("config-2 fixture not generated")
    S, _ = run(case, handle)
    info = handle.refinement()
    err = rel(S, case["S"])
    print(f"config 2 split precision: rel. error {err:.3g}, {info}")
    assert info["form"] == _abi.RGF_TF32X3, info
    assert err <= TOL_S
    assert np.abs(S - S.T).max() <= 1e-12  # Dirichlet: S = S^T (setup_channels.m:75-79)


def test_pivot_regime_never_wrong(handle):
    """Past diagonal dominance the FP32 factor may be too poor a preconditioner;
    then the call must fall back to FP64, never return an inaccurate S."""
    for path in sorted(glob.glob(os.path.join(GOLDEN, "2d_pivot_*.npz"))):
        case = load_case(path)
        if "singular" in case["name"]:
            continue
        S, _ = run(case, handle)
        info = handle.refinement()
        assert rel(S, case["S"]) <= TOL_S, (case["name"], info)
        assert info["form"] in (_abi.RGF_TF32X3, -_abi.RGF_TF32X3)


def test_unsupported_combinations(handle):
    case = load_case(os.path.join(GOLDEN, "2d_periodic_full.npz"))
    T0, _ = rgf_b200.cal_smatrix_RGF(case["syst"], ["right"], ["left"], handle=handle)
    with pytest.raises(_abi.RGFError):
        rgf_b200.smatrix_grad_RGF(case["syst"], ["right"], ["left"], np.conj(T0), options=OPT, handle=handle)


@pytest.mark.parametrize("ny,nx,bc", [(40, 7, "periodic"), (40, 8, "Dirichlet"), (70, 9, "Neumann"),
                                      (96, 16, 0.4), (33, 17, "DirichletNeumann"), (130, 64, "periodic")])
def test_two_sided_edges(ny, nx, bc, handle):
    """One chain below 8 slices, the two-sided factorization from 8 on (odd and
    even L: sides of equal or unequal length), N not a multiple of the 32-wide
    pivot block; against the FP64 form of the same call."""
    rng = np.random.default_rng(ny * 100 + nx)
    syst = dict(epsilon=1 + 2 * rng.random((ny, nx)) + 0.01j * rng.random((ny, nx)), epsilon_L=1.0,
                epsilon_R=1.5, k0dx=2 * np.pi / 12, yBC=bc)
    S64, _ = rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], handle=handle)
    S, _ = rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], options=OPT, handle=handle)
    info = handle.refinement()
    assert info["form"] == _abi.RGF_TF32X3, info
    assert rel(S, S64) <= TOL_S, (rel(S, S64), info)


def test_two_sided_3d(handle):
    rng = np.random.default_rng(9)
    eps = np.where(rng.random((8, 6, 21)) < 0.4, 2.25, 1.0)
    syst = dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 10, xyBC="periodic")
    S64, _ = rgf_b200.cal_smatrix_RGF_3D(syst, ["left", "right"], ["left", "right"], handle=handle)
    S, _ = rgf_b200.cal_smatrix_RGF_3D(syst, ["left", "right"], ["left", "right"], options=OPT, handle=handle)
    assert handle.refinement()["form"] == _abi.RGF_TF32X3
    assert rel(S, S64) <= TOL_S

"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle's
golden S-matrices, channel data and the reference's invariants.

Tolerances (FP64 plain form): relative Frobenius error of S <= 1e-11
against the FP64 oracle; reciprocity |S - S^T| <= 1e-12; unitarity for real
eps <= 1e-12."""
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
TOL_S = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run(case):
    fn = rgf_b200.cal_smatrix_RGF if case["dim"] == "2d" else rgf_b200.cal_smatrix_RGF_3D
    return fn(case["syst"], case["out"], case["in"])


@pytest.mark.parametrize("path", SMALL, ids=lambda p: os.path.basename(p)[:-4])
def test_small_golden(path):
    case = load_case(path)
    S, ch = run(case)
    assert S.shape == case["S"].shape
    assert rel(S, case["S"]) <= TOL_S
    for side in ("L", "R"):
        assert ch[side]["N_prop"] == case[f"N_prop_{side}"]
        assert np.array_equal(ch[side]["ind_prop"], case[f"ind_prop_{side}"])
        assert np.abs(ch[side]["sqrt_mu"] - case[f"sqrt_mu_{side}"]).max(initial=0) < 1e-13
        kx = ch[side]["kxdx" if case["dim"] == "2d" else "kzdx"]
        assert np.abs(np.ravel(kx, order="F") - np.ravel(case[f"kx_{side}"], order="F")).max() < 1e-12


@pytest.mark.parametrize("name", ["cfg1", "cfg3", "cfg5", "cfg4_0", "cfg4_1", "cfg4_2"])
def test_config_golden(name):
    case = config_case(name)
    if case is None:
        pytest.skip(f"no fixture {name}")
    S, ch = run(case)
    assert S.shape == case["S"].shape
    assert rel(S, case["S"]) <= TOL_S


def test_config2_golden():
    """Full-size headline workload (N=1024, L=4096) against the oracle."""
    case = config_case("cfg2")
    if case is None:
        pytest.skip("config-2 fixture not generated")
    h = _abi.Handle(0)
    S, _ = rgf_b200.cal_smatrix_RGF(case["syst"], case["out"], case["in"], handle=h)
    used, fallback, _ = h.engine()
    _, probe = h.stats()
    print(f"config 2: engine {used}, fallback {fallback}, probe residual {probe:.3g}")
    assert fallback == 0 and probe < 1e-12  # the persistent engine's result stands
    assert rel(S, case["S"]) <= TOL_S
    # Dirichlet: literal reciprocity S = S^T (setup_channels.m:75-79)
    assert np.abs(S - S.T).max() <= 1e-12


def test_config1_invariants():
    """examples/example_script.m:26-35: unitarity (real eps) and reciprocity
    under ind_prop_conj."""
    case = config_case("cfg1")
    S, ch = run(case)
    assert np.abs(S.conj().T @ S - np.eye(S.shape[0])).max() <= 1e-12
    p = np.concatenate([ch["L"]["ind_prop_conj"], ch["L"]["N_prop"] + ch["R"]["ind_prop_conj"]]) - 1
    St = S[p, :]
    assert np.abs(St.T - St).max() <= 1e-12


@pytest.mark.parametrize("bc", ["periodic", "Dirichlet", "Neumann", "DirichletNeumann", "NeumannDirichlet", 0.3])
@pytest.mark.parametrize("k0dx", [2 * np.pi / 7, 1.8, 1.1 * (1 + 2e-3j), 0.7 * (1 - 1e-3j)])
def test_setup_channels_parity(bc, k0dx):
    from oracle.rgf_ref import setup_channels as ref
    for eR in (1.0, 2.3, None):
        got = rgf_b200.setup_channels(13, bc, k0dx, 1.4, eR)
        exp = ref(13, bc, k0dx, 1.4, eR)
        assert np.abs(got["kydx"] - exp["kydx"]).max() < 1e-14
        for side in ("L", "R"):
            if eR is None and side == "R":
                assert np.isnan(got["R"]["N_prop"])
                continue
            g, e = got[side], exp[side]
            assert g["N_prop"] == e["N_prop"]
            assert np.array_equal(g["ind_prop"], e["ind_prop"])
            assert np.abs(g["kxdx"] - e["kxdx"]).max() < 1e-12
            assert np.abs(g["sqrt_mu"] - e["sqrt_mu"]).max(initial=0) < 1e-13
            if "ind_prop_conj" in e:
                assert np.array_equal(g["ind_prop_conj"], e["ind_prop_conj"])
            else:
                assert "ind_prop_conj" not in g
        phi_g = got["fun_phi"](got["kydx"])
        phi_e = exp["fun_phi"](exp["kydx"])
        assert np.abs(phi_g - phi_e).max() < 1e-14


@pytest.mark.parametrize("bc", ["periodic", "Dirichlet", [0.2, -1.1]])
def test_setup_channels_3d_parity(bc):
    from oracle.rgf_ref import setup_channels_3D as ref
    got = rgf_b200.setup_channels_3D(5, 7, bc, 1.3, 1.0, 2.0)
    exp = ref(5, 7, bc, 1.3, 1.0, 2.0)
    assert np.abs(got["kxdx"] - exp["kxdx"]).max() < 1e-14
    assert np.abs(got["kydx"] - exp["kydx"]).max() < 1e-14
    for side in ("L", "R"):
        assert got[side]["N_prop"] == exp[side]["N_prop"]
        assert np.array_equal(got[side]["ind_prop"], exp[side]["ind_prop"])
        assert np.abs(got[side]["kzdx"] - exp[side]["kzdx"]).max() < 1e-12


@pytest.mark.parametrize("bc", ["periodic", "Dirichlet", [0.2, -1.1]])
@pytest.mark.parametrize("k0dx", [1.3, 0.9 * (1 + 1e-3j)])
def test_setup_channels_3d_one_sided(bc, k0dx):
    """setup_channels_3D with epsilon_R omitted (setup_channels_3D.m:74,
    138-141): the left side only, channels.R.N_prop = NaN."""
    from oracle.rgf_ref import setup_channels_3D as ref
    got = rgf_b200.setup_channels_3D(6, 5, bc, k0dx, 1.7)
    exp = ref(6, 5, bc, k0dx, 1.7)
    assert np.abs(got["kxdx"] - exp["kxdx"]).max() < 1e-14
    assert np.abs(got["kydx"] - exp["kydx"]).max() < 1e-14
    assert got["L"]["N_prop"] == exp["L"]["N_prop"]
    assert np.array_equal(got["L"]["ind_prop"], exp["L"]["ind_prop"])
    assert np.abs(got["L"]["kzdx"] - exp["L"]["kzdx"]).max() < 1e-12
    assert np.abs(got["L"]["sqrt_mu"] - exp["L"]["sqrt_mu"]).max(initial=0) < 1e-13
    assert np.isnan(got["R"]["N_prop"])


@pytest.mark.parametrize("bc", ["periodic", "Dirichlet", "Neumann", "DirichletNeumann", "NeumannDirichlet", 1.3])
@pytest.mark.parametrize("n", [1, 2, 3, 10])
def test_build_laplacian_parity(bc, n):
    from oracle.rgf_ref import build_laplacian_1d as ref
    assert np.abs(rgf_b200.build_laplacian_1d(n, bc) - ref(n, bc)).max(initial=0) < 1e-15


def test_nonfinite_epsilon_rejected():
    s = dict(epsilon=np.ones((8, 4)), epsilon_L=1.0, epsilon_R=1.0, k0dx=1.0, yBC="periodic")
    s["epsilon"][3, 2] = np.nan
    with pytest.raises(_abi.RGFError) as ei:
        rgf_b200.cal_smatrix_RGF(s, ["left"], ["left"])
    assert ei.value.status == _abi.RGF_ERR_NONFINITE


def test_channel_index_out_of_range():
    s = dict(epsilon=np.ones((8, 4)), epsilon_L=1.0, epsilon_R=1.0, k0dx=1.0, yBC="periodic")
    with pytest.raises(_abi.RGFError, match="N_prop"):
        rgf_b200.cal_smatrix_RGF(s, {"ind_out_L": [99]}, ["left"])


def test_empty_request_returns_empty():
    s = dict(epsilon=np.ones((8, 4)), epsilon_L=1.0, epsilon_R=1.0, k0dx=1.0, yBC="periodic")
    S, ch = rgf_b200.cal_smatrix_RGF(s, ["left"], {})
    assert S.shape == (ch["L"]["N_prop"], 0)


def test_repeated_calls_reuse_workspace():
    """A handle serves differently sized problems back to back."""
    a = load_case(os.path.join(GOLDEN, "2d_large_N_gt_block.npz"))
    b = load_case(os.path.join(GOLDEN, "2d_periodic_full.npz"))
    for case in (a, b, a):
        S, _ = run(case)
        assert rel(S, case["S"]) <= TOL_S


@pytest.mark.parametrize("name", ["cfg1", "cfg5", "2d_large_N_gt_block", "3d_bloch_inR", "2d_Bloch_inL"])
def test_engines_agree_and_probe(name):
    """The persistent register-resident engine (default) and the per-step
    engine give the same S; the per-slice probe residual max|G_n M_n v - v|
    stays at round-off level."""
    case = config_case(name) if name.startswith("cfg") else load_case(os.path.join(GOLDEN, name + ".npz"))
    h = _abi.Handle(0)
    fn = rgf_b200.cal_smatrix_RGF if case["dim"] == "2d" else rgf_b200.cal_smatrix_RGF_3D
    S0, _ = fn(case["syst"], case["out"], case["in"], handle=h, options={"engine": 0})
    launches0, probe = h.stats()
    S1, _ = fn(case["syst"], case["out"], case["in"], handle=h, options={"engine": 1})
    launches1, _ = h.stats()
    assert rel(S0, case["S"]) <= TOL_S and rel(S1, case["S"]) <= TOL_S
    assert rel(S0, S1) <= 1e-12
    assert probe < 1e-10
    assert launches0 < launches1

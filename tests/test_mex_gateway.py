"""The MEX gateway (matlab/rgf_mex.c) driven through the test harness's
stand-in for MATLAB's MEX API (tests/mexstub): MATLAB values in (1-based
channel indices, cell/struct requests, real epsilon promoted to complex),
mexFunction, MATLAB values out, errors as rgf:<status> identifiers.

The CPU tests need no GPU (argument errors; rgf:nodevice without a device);
the GPU tests compare the gateway's S, channels, Laplacian and gradient with
the oracle's golden fixtures (relative Frobenius error of S <= 1e-11)."""
import os

import numpy as np
import pytest

from tests.conftest import gpu_available
from tests.golden_io import load_case
from tests.mexstub import bridge

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def mx_request(r):
    """Python request (list of sides or dict of 1-based lists) as MATLAB values."""
    if isinstance(r, dict):
        return {k: np.asarray(v, dtype=float).reshape(1, -1) for k, v in r.items()}
    return list(r)


def syst_mx(syst, bc_key="yBC"):
    return {"epsilon": np.asarray(syst["epsilon"]), "epsilon_L": syst["epsilon_L"], "epsilon_R": syst["epsilon_R"],
            "k0dx": syst["k0dx"], bc_key: syst[bc_key] if isinstance(syst[bc_key], str)
            else np.asarray(syst[bc_key], dtype=float)}


def test_gateway_requires_a_command():
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1)
    assert ei.value.ident == "rgf:arg"
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1, 3.0)
    assert ei.value.ident == "rgf:arg"


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_gateway_reports_missing_device():
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1, "laplacian", 4.0, "periodic")
    assert ei.value.ident == "rgf:nodevice"


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["2d_periodic_full", "2d_Dirichlet_lists", "2d_Bloch_inL", "2d_Neumann_RR",
                                  "2d_pivot_k2e_4p5", "2d_interface_nx0"])
def test_smatrix2d_through_gateway(name):
    case = load_case(os.path.join(GOLDEN, name + ".npz"))
    (S, ch), warns = bridge.call(2, "smatrix2d", syst_mx(case["syst"]), mx_request(case["out"]),
                                 mx_request(case["in"]))
    try:
        Sg = bridge.from_mx(S)
        assert Sg.shape == case["S"].shape
        assert rel(Sg, case["S"]) <= 1e-11
        for side in ("L", "R"):
            t = bridge.field(ch, side)
            assert int(bridge.from_mx(bridge.field(t, "N_prop"))[0, 0]) == case[f"N_prop_{side}"]
            ip = bridge.from_mx(bridge.field(t, "ind_prop")).ravel()
            assert np.array_equal(ip.astype(int), case[f"ind_prop_{side}"])  # 1-based, as MATLAB's
    finally:
        bridge.destroy(S)
        bridge.destroy(ch)
    assert not warns


@pytest.mark.gpu
def test_smatrix3d_through_gateway():
    case = load_case(os.path.join(GOLDEN, "3d_bloch_inR.npz"))
    (S,), _ = bridge.call(1, "smatrix3d", syst_mx(case["syst"], "xyBC"), mx_request(case["out"]),
                          mx_request(case["in"]))
    try:
        assert rel(bridge.from_mx(S), case["S"]) <= 1e-11
    finally:
        bridge.destroy(S)


@pytest.mark.gpu
def test_cell_forms_and_ignored_elements():
    """{'L','R'} equals {'left','right'}; a non-side element is ignored with
    the reference's warning (cal_smatrix_RGF.m:120-135)."""
    case = load_case(os.path.join(GOLDEN, "2d_periodic_full.npz"))
    (S,), warns = bridge.call(1, "smatrix2d", syst_mx(case["syst"]), ["L", "R", "up"], ["left", "R", 3.0])
    try:
        assert rel(bridge.from_mx(S), case["S"]) <= 1e-11
    finally:
        bridge.destroy(S)
    assert len(warns) == 2 and all(w.startswith("rgf:ignored") for w in warns)
    assert "out{3} = up ignored" in warns[0] and "in{3} has wrong format" in warns[1]


@pytest.mark.gpu
def test_gateway_errors():
    case = load_case(os.path.join(GOLDEN, "2d_periodic_full.npz"))
    s = syst_mx(case["syst"])
    n = case["N_prop_L"]
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1, "smatrix2d", s, {"ind_out_L": np.array([[n + 1.0]])}, ["left"])
    assert ei.value.ident == "rgf:arg" and f"not exceeding N_prop_L={n}" in ei.value.msg
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1, "smatrix2d", s, {"ind_out_L": np.array([[1.5]])}, ["left"])
    assert ei.value.ident == "rgf:arg" and "out.ind_out_L" in ei.value.msg
    bad = dict(s, epsilon=np.array(s["epsilon"], dtype=float))
    bad["epsilon"][0, 0] = np.nan
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1, "smatrix2d", bad, ["left"], ["left"])
    assert ei.value.ident == "rgf:nonfinite"
    with pytest.raises(bridge.MexError) as ei:
        bridge.call(1, "smatrix2d", s, 5.0, ["left"])
    assert ei.value.ident == "rgf:arg"


@pytest.mark.gpu
def test_channels_and_laplacian_through_gateway():
    from oracle.rgf_ref import build_laplacian_1d, setup_channels, setup_channels_3D
    (ch,), _ = bridge.call(1, "channels2d", 13.0, "Neumann", 1.1 * (1 + 2e-3j), 1.4, 2.3)
    try:
        exp = setup_channels(13, "Neumann", 1.1 * (1 + 2e-3j), 1.4, 2.3)
        assert np.abs(bridge.from_mx(bridge.field(ch, "kydx")).ravel() - exp["kydx"]).max() < 1e-14
        for side in ("L", "R"):
            t = bridge.field(ch, side)
            assert np.array_equal(bridge.from_mx(bridge.field(t, "ind_prop")).ravel().astype(int),
                                  exp[side]["ind_prop"])
            assert np.abs(bridge.from_mx(bridge.field(t, "kxdx")).ravel() - exp[side]["kxdx"]).max() < 1e-12
            assert np.array_equal(bridge.from_mx(bridge.field(t, "ind_prop_conj")).ravel().astype(int),
                                  exp[side]["ind_prop_conj"])
    finally:
        bridge.destroy(ch)
    (ch3,), _ = bridge.call(1, "channels3d", 4.0, 5.0, np.array([[0.3, -0.2]]), 1.2, 1.0)  # one-sided
    try:
        exp = setup_channels_3D(4, 5, [0.3, -0.2], 1.2, 1.0)
        t = bridge.field(ch3, "L")
        assert int(bridge.from_mx(bridge.field(t, "N_prop"))[0, 0]) == exp["L"]["N_prop"]
        assert np.isnan(bridge.from_mx(bridge.field(bridge.field(ch3, "R"), "N_prop"))[0, 0])
    finally:
        bridge.destroy(ch3)
    for bc in ("periodic", "Dirichlet", "NeumannDirichlet", 0.7):
        (A,), _ = bridge.call(1, "laplacian", 6.0, bc)
        try:
            assert np.abs(bridge.from_mx(A) - build_laplacian_1d(6, bc)).max() < 1e-15
        finally:
            bridge.destroy(A)


@pytest.mark.gpu
def test_gradient_through_gateway():
    from oracle.adjoint import grad_rgf_2d
    from oracle.rgf_ref import cal_smatrix_RGF as ref
    rng = np.random.default_rng(8)
    syst = dict(epsilon=1 + 2 * rng.random((12, 7)), epsilon_L=1.0, epsilon_R=1.2, k0dx=1.0, yBC="periodic")
    out, inp = {"ind_out_R": [1, 2]}, {"ind_in_L": [2]}
    S0, _ = ref(syst, out, inp)
    D = np.conj(S0)
    (S, g), _ = bridge.call(2, "grad2d", syst_mx(syst), mx_request(out), mx_request(inp), D)
    try:
        _, g0 = grad_rgf_2d(syst, out, inp, D)
        assert rel(bridge.from_mx(S), S0) <= 1e-11
        gg = bridge.from_mx(g)
        assert gg.shape == (12, 7)
        assert np.abs(gg - g0).max() <= 1e-10 * np.abs(g0).max()
    finally:
        bridge.destroy(S)
        bridge.destroy(g)


@pytest.mark.gpu
def test_fields_through_gateway():
    from oracle.dense_fdfd import fields_dense_2d
    rng = np.random.default_rng(9)
    syst = dict(epsilon=1 + 2 * rng.random((10, 6)), epsilon_L=1.0, epsilon_R=1.2, k0dx=1.0, yBC="Neumann")
    out, inp = ["left", "right"], {"ind_in_R": [1, 2]}
    (S, psi), _ = bridge.call(2, "fields2d", syst_mx(syst), mx_request(out), mx_request(inp))
    try:
        S0, psi0 = fields_dense_2d(syst, out, inp)
        assert rel(bridge.from_mx(S), S0) <= 1e-11
        p = bridge.from_mx(psi)
        assert p.shape == (10, 6, 2)
        assert np.abs(p - psi0).max() <= 1e-11 * np.abs(psi0).max()
    finally:
        bridge.destroy(S)
        bridge.destroy(psi)

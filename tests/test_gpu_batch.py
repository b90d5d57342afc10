"""Batched form (rgf_smatrix_batch_2d through the C ABI): independent 2D
structures of uneven N and L, complex frequency, run as concurrent
pipelines, against the oracle's golden S (config 4 structures) and against
one-at-a-time calls.  Tolerance: relative Frobenius error of S <= 1e-11."""
import numpy as np
import pytest

import rgf_b200
from rgf_b200 import _abi, workloads
from tests.golden_io import config_case

pytestmark = pytest.mark.gpu
TOL_S = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def mixed_batch(n=12, seed=40):
    rng = np.random.default_rng(seed)
    systs, outs, ins = [], [], []
    bcs = ["periodic", "Dirichlet", "Neumann", 0.37]
    for k in range(n):
        ny, nx = int(rng.integers(8, 140)), int(rng.integers(0, 40))
        eps = 1 + 2 * rng.random((ny, nx))
        systs.append(dict(epsilon=eps, epsilon_L=1.0, epsilon_R=1.0 + 0.5 * (k % 2),
                          k0dx=2 * np.pi / 15 * (1 + 1j * 1e-3 * rng.random()), yBC=bcs[k % 4]))
        outs.append(["left", "right"] if k % 3 else {"ind_out_R": [1]})
        ins.append(["left", "right"] if k % 3 != 1 else ["left"])
    return systs, outs, ins


@pytest.mark.parametrize("workers", [0, 1, 4, 8])
def test_batch_matches_single_calls(workers):
    systs, outs, ins = mixed_batch()
    Sb = rgf_b200.cal_smatrix_RGF_batch(systs, outs, ins, workers=workers)
    for s, o, i, S in zip(systs, outs, ins, Sb):
        S1, _ = rgf_b200.cal_smatrix_RGF(s, o, i)
        assert S.shape == S1.shape
        assert rel(S, S1) <= 1e-12


def test_batch_config4_golden():
    """The 16-structure subsample of config 4 (the first twelve structures,
    the largest N, the largest L, the largest L N^3 and the largest eta)
    through the batched entry, against the oracle's S."""
    cases = [config_case(f"cfg4_{k}") for k in workloads.CONFIG4_SUBSAMPLE]
    cases = [c for c in cases if c is not None]
    if not cases:
        pytest.skip("no config-4 fixtures")
    for workers in (0, 3):  # one launch for all; three pipelines
        Sb = rgf_b200.cal_smatrix_RGF_batch([c["syst"] for c in cases], [c["out"] for c in cases],
                                            [c["in"] for c in cases], workers=workers)
        for c, S in zip(cases, Sb):
            assert rel(S, c["S"]) <= TOL_S


def test_batch_reports_failing_item():
    systs, outs, ins = mixed_batch(5)
    bad = dict(systs[2])
    bad["epsilon"] = bad["epsilon"].copy()
    if bad["epsilon"].size == 0:
        bad["epsilon"] = np.ones((9, 3))
    bad["epsilon"][0, 0] = np.nan
    systs[2] = bad
    for workers in (0, 3):
        with pytest.raises(_abi.RGFError) as ei:
            rgf_b200.cal_smatrix_RGF_batch(systs, outs, ins, workers=workers)
        assert ei.value.status == _abi.RGF_ERR_NONFINITE
        assert "batch item 2" in str(ei.value)


def test_one_launch_batch_runs_one_gang_launch():
    """workers = 0: every sweep of the batch in one persistent launch (gangs
    from the device work queue), with structures of very different size."""
    systs, outs, ins = mixed_batch(20, seed=41)
    h = _abi.Handle(0)
    Sb = rgf_b200.cal_smatrix_RGF_batch(systs, outs, ins, workers=0, handle=h)
    launches, _ = h.stats()
    assert launches == 1
    for s, o, i, S in zip(systs, outs, ins, Sb):
        S1, _ = rgf_b200.cal_smatrix_RGF(s, o, i)
        assert rel(S, S1) <= 1e-12


@pytest.mark.parametrize("workers", [0, 3])
def test_batch_split_precision(workers):
    """The batched entry with the split-precision form: config-4 structures
    against the oracle fixtures at the form's 1e-10, and the mixed batch
    against single FP64 calls."""
    names = ["cfg4_0", "cfg4_7", "cfg4_9"]
    cases = [config_case(n) for n in names]
    cases = [c for c in cases if c is not None]
    opt = {"precision": _abi.RGF_TF32X3}
    Sb = rgf_b200.cal_smatrix_RGF_batch([c["syst"] for c in cases], [c["out"] for c in cases],
                                        [c["in"] for c in cases], workers=workers, options=opt)
    for c, S in zip(cases, Sb):
        assert rel(S, c["S"]) <= 1e-10, c["name"]
    systs, outs, ins = mixed_batch(n=6, seed=41)
    Sb = rgf_b200.cal_smatrix_RGF_batch(systs, outs, ins, workers=workers, options=opt)
    for s, o, i, S in zip(systs, outs, ins, Sb):
        S1, _ = rgf_b200.cal_smatrix_RGF(s, o, i)
        assert S.shape == S1.shape
        if S1.size:
            assert rel(S, S1) <= 1e-10

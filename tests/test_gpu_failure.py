"""Failure detection on the GPU without a fault: the T-server withholds the
first pivot-block inverse (a flag that nothing sets), every dependent wait
runs out after RGF_WAIT_TIMEOUT_MS, the kernel returns on its own, the host
reports RGF_ERR_TIMEOUT, and the same handle then computes a correct S."""
import os

import numpy as np
import pytest

import rgf_b200
from rgf_b200 import _abi
from oracle.rgf_ref import cal_smatrix_RGF as ref

pytestmark = pytest.mark.gpu


def test_withheld_flag_times_out_and_handle_recovers(monkeypatch):
    rng = np.random.default_rng(3)
    syst = dict(epsilon=1 + 3 * rng.random((70, 12)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15,
                yBC="periodic")
    h = _abi.Handle(0)
    monkeypatch.setenv("RGF_WAIT_TIMEOUT_MS", "200")
    monkeypatch.setenv("RGF_TEST_WITHHOLD_T", "1")
    with pytest.raises(_abi.RGFError) as ei:
        rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], handle=h)
    assert ei.value.status == _abi.RGF_ERR_TIMEOUT
    monkeypatch.delenv("RGF_TEST_WITHHOLD_T")
    S, _ = rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], handle=h)
    S0, _ = ref(syst, ["left", "right"], ["left", "right"])
    assert np.linalg.norm(S - S0) <= 1e-11 * np.linalg.norm(S0)

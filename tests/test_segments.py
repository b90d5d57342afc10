"""L-split S-matrix (rgf_b200.segments): two parts of the slices swept from
their own leads and joined across the cut.

CPU: the split's algebra (oracle/segments.py, checked against the oracle's
unsplit S) and its two-rank plumbing over gloo with the CPU statement of the
two operations standing in for the GPU.  GPU: the C ABI's segment sweeps
and merge against the oracle's golden S, on one GPU.  Tolerance: relative
Frobenius error of S <= 1e-11."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle.rgf_ref import cal_smatrix_RGF as ref
from oracle.segments import segment_merge_2d, segment_state_2d

CASES = [
    ("periodic", ["left", "right"], ["left", "right"]),
    ("Dirichlet", {"ind_out_R": [1, 2]}, {"ind_in_L": [2, 1]}),
    ("Neumann", ["left"], ["left", "right"]),
    (0.3, ["right"], ["right"]),
    ("NeumannDirichlet", {"ind_out_L": [1, 1, 2], "ind_out_R": [3]}, {"ind_in_L": [1], "ind_in_R": [2, 1]}),
]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def syst_of(bc, seed=3):
    rng = np.random.default_rng(seed)
    return dict(epsilon=1 + 2 * rng.random((15, 11)) + 0.01j * rng.random((15, 11)), epsilon_L=1.0,
                epsilon_R=1.6, k0dx=1.0, yBC=bc)


class CpuSegments:
    """The two operations of the split, from the CPU oracle (test stand-in
    for the GPU)."""

    def __init__(self, syst, out, in_):
        self.args = (syst, out, in_)

    def state(self, side, cut):
        return segment_state_2d(*self.args, side, cut)

    def merge(self, a, b):
        return segment_merge_2d(*self.args, a, b)


@pytest.mark.parametrize("cut", [1, 5, 10])
@pytest.mark.parametrize("bc,out,inp", CASES)
def test_split_algebra_matches_unsplit(bc, out, inp, cut):
    s = syst_of(bc)
    S0, _ = ref(s, out, inp)
    S = segment_merge_2d(s, out, inp, segment_state_2d(s, out, inp, 0, cut), segment_state_2d(s, out, inp, 1, cut))
    assert rel(S, S0) <= 1e-13


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, res):
    import datetime

    import torch.distributed as dist

    from rgf_b200.segments import cal_smatrix_RGF_split
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        for k, (bc, out, inp) in enumerate(CASES):
            s = syst_of(bc)
            S = cal_smatrix_RGF_split(s, out, inp, cut=4, group=dist.group.WORLD, segments=CpuSegments(s, out, inp))
            if rank == 0:
                res[k] = S
            else:
                res[100 + k] = S is None
    finally:
        dist.destroy_process_group()


def test_split_over_two_gloo_ranks():
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    res = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, res), nprocs=world, start_method="spawn", join=True)
    for k, (bc, out, inp) in enumerate(CASES):
        S0, _ = ref(syst_of(bc), out, inp)
        assert rel(res[k], S0) <= 1e-13
        assert res[100 + k]


@pytest.mark.gpu
@pytest.mark.parametrize("bc,out,inp", CASES)
@pytest.mark.parametrize("engine", [0, 1])
def test_split_on_one_gpu(bc, out, inp, engine):
    from rgf_b200.segments import DeviceSegments, cal_smatrix_RGF_split
    s = syst_of(bc)
    S0, _ = ref(s, out, inp)
    for cut in (1, 6, 10):
        seg = DeviceSegments(s, out, inp, options={"engine": engine})
        S = cal_smatrix_RGF_split(s, out, inp, cut=cut, segments=seg)
        assert rel(S, S0) <= 1e-11
        # the GPU's segment states equal the CPU statement's
        for side in (0, 1):
            assert rel(seg.state(side, cut), segment_state_2d(s, out, inp, side, cut)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cfg1", "cfg5"])
def test_split_config_golden(name):
    """Configs 1 and 5 split at L/2 and at L/3 (multi-block N for config 5)."""
    from rgf_b200.segments import cal_smatrix_RGF_split
    from tests.golden_io import config_case
    case = config_case(name)
    L = case["syst"]["epsilon"].shape[1]
    for cut in (L // 2, L // 3):
        S = cal_smatrix_RGF_split(case["syst"], case["out"], case["in"], cut=cut)
        assert rel(S, case["S"]) <= 1e-11

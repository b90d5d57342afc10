"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol include/rgf.h declares, and the host-side argument handling mirrors
the reference's error behaviour (cal_smatrix_RGF.m:79-93, 103-178)."""
import ctypes
import os
import re

import numpy as np
import pytest

from rgf_b200 import _abi
from rgf_b200 import api
from tests.conftest import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rgf.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^RGF_API\s+[\w\s\*]+?\b(rgf_\w+)\s*\(", src, flags=re.M)))


def test_header_parsed():
    names = header_functions()
    assert "rgf_smatrix_2d" in names and "rgf_smatrix_3d" in names and len(names) >= 12


def test_library_exports_every_header_symbol():
    lib = _abi.load()
    for name in header_functions():
        assert hasattr(lib, name), name


def test_ctypes_signatures_cover_header():
    assert sorted(_abi.SIGNATURES) == header_functions()


def test_struct_layouts():
    # rgf_cplx is two doubles; the syst structs follow C alignment rules
    assert ctypes.sizeof(_abi.Cplx) == 16
    assert _abi.Syst2D.epsilon_L.offset % 8 == 0 and _abi.Syst3D.kya.offset % 8 == 0
    assert ctypes.sizeof(_abi.Request) == 64


def test_version_string():
    assert b"sm_100a" in _abi.load().rgf_version()


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_without_device_fails_loudly():
    lib = _abi.load()
    h = ctypes.c_void_p()
    st = lib.rgf_create(0, ctypes.byref(h))
    assert st == _abi.RGF_ERR_NODEVICE
    assert b"no CUDA device" in lib.rgf_last_error()
    with pytest.raises(_abi.RGFError):
        _abi.Handle(0)


def test_null_handle_rejected():
    lib = _abi.load()
    st = lib.rgf_smatrix_2d(None, None, None, None, None, 0, None)
    assert st == _abi.RGF_ERR_ARG


def _syst():
    return dict(epsilon=np.ones((4, 3)), epsilon_L=1.0, epsilon_R=1.0, k0dx=0.5, yBC="periodic")


@pytest.mark.parametrize("bad,msg", [
    ("missing", "must be provided"),
    ("eps3d", "numeric matrix"),
    ("k0dx_vec", "numeric scalar"),
    ("bloch_str", "Bloch"),
    ("bad_bc", "not an eligible"),
    ("ny0", "at least one site"),
    ("bad_out", "structure or a cell"),
    ("bad_index", "positive integers"),
])
def test_python_validation_before_device(bad, msg):
    s = _syst()
    out, in_ = ["left"], ["left"]
    if bad == "missing":
        del s["k0dx"]
    elif bad == "eps3d":
        s["epsilon"] = np.ones((2, 2, 2))
    elif bad == "k0dx_vec":
        s["k0dx"] = np.array([1.0, 2.0])
    elif bad == "bloch_str":
        s["yBC"] = "Bloch"
    elif bad == "bad_bc":
        s["yBC"] = "absorbing"
    elif bad == "ny0":
        s["epsilon"] = np.ones((0, 3))
    elif bad == "bad_out":
        out = "left"
    elif bad == "bad_index":
        out = {"ind_out_L": [0]}
    with pytest.raises(ValueError, match=msg):
        api.cal_smatrix_RGF(s, out, in_)


def test_request_parsing():
    reqs = api._parse_request({"ind_in_L": [3, 1], "ind_in_R": []}, "in")
    assert list(reqs[0][0]) == [2, 0] and reqs[1][1] == 0
    with pytest.warns(UserWarning):
        reqs = api._parse_request(["left", 5, "up"], "in")
    assert reqs[0][1] == _abi.RGF_ALL and reqs[1][1] == 0


def test_workload_inputs_match_fixtures():
    """Seeded inputs regenerate bit-for-bit (the fixtures store a checksum)."""
    from tests.golden.make_golden import eps_checksum
    from tests.golden_io import config_case
    for name in ("cfg1", "cfg3", "cfg5"):
        case = config_case(name)
        assert case is not None
        assert np.allclose(eps_checksum(case["syst"]["epsilon"]), case["eps_checksum"], rtol=0, atol=1e-9)


def test_constants_match_header():
    src = open(HEADER).read()
    m = re.search(r"#define RGF_NOALLOC_SCRATCH_BYTES \(\(size_t\)(\d+) << (\d+)\)", src)
    assert m and int(m.group(1)) << int(m.group(2)) == _abi.RGF_NOALLOC_SCRATCH_BYTES
    enum = dict(re.findall(r"^\s*(RGF_ERR_\w+|RGF_OK) = (\d+)", src, flags=re.M))
    for name, val in enum.items():
        assert _abi.STATUS_NAMES[int(val)] == name


def test_cpu_stand_ins_of_segments_and_fields_exist():
    """The test-only CPU statements the GPU tests of the split and of the
    fields check against (oracle/segments.py, oracle/dense_fdfd.py)."""
    from oracle.dense_fdfd import fields_dense_2d
    from oracle.segments import segment_merge_2d, segment_state_2d
    s = _syst()
    S, psi = fields_dense_2d(s, ["left", "right"], ["left"])
    assert psi.shape == (4, 3, S.shape[1])
    st = segment_state_2d(s, ["left"], ["left"], 0, 1)
    assert st.shape[0] == 4 + S.shape[0] // 2 or st.shape[0] >= 4
    assert callable(segment_merge_2d)


def test_constants_match_header():
    src = open(HEADER).read()
    m = re.search(r"#define RGF_NOALLOC_SCRATCH_BYTES \(\(size_t\)(\d+) << (\d+)\)", src)
    assert m and int(m.group(1)) << int(m.group(2)) == _abi.RGF_NOALLOC_SCRATCH_BYTES
    enum = dict(re.findall(r"^\s*(RGF_ERR_\w+|RGF_OK) = (\d+)", src, flags=re.M))
    assert len(enum) == 9
    for name, val in enum.items():
        assert _abi.STATUS_NAMES[int(val)] == name

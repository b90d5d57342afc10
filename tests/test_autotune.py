"""Tile-shape autotuner (rgf_b200.autotune): the table it builds from
measurements, its JSON cache, and on the GPU a short tuning run and an
installed table that changes the tile the persistent engine uses but not S."""
import json

import numpy as np
import pytest

from rgf_b200 import autotune


def test_table_covers_sizes_to_the_midpoint():
    rows = [{"rows": 300, "best": 64}, {"rows": 100, "best": 32}, {"rows": 1100, "best": 96}]
    rmax, tile = autotune.table_from_measurements(rows)
    assert rmax == [200, 700, 1 << 40] and tile == [32, 64, 96]


def test_cache_path_names_the_gpu():
    assert autotune.cache_path("NVIDIA B200", 148).name == "tiles_nvidia_b200_148sm.json"


def test_load_rejects_other_sm_count(tmp_path):
    f = tmp_path / "t.json"
    f.write_text(json.dumps({"gpu": "x", "sms": 132, "entries": []}))
    assert autotune.load("x", 148, str(f)) is None
    assert autotune.load("x", 132, str(f))["sms"] == 132


@pytest.mark.gpu
def test_tuning_run_and_installed_table():
    import rgf_b200
    from rgf_b200 import _abi
    t = autotune.tune(sizes=(64, 160), slices=6, reps=1)
    assert t["sms"] > 0 and len(t["entries"]) == 2
    for e in t["entries"]:
        assert e["best"] in e["us_per_slice"] and all(v > 0 for v in e["us_per_slice"].values())
    rng = np.random.default_rng(9)
    syst = dict(epsilon=1 + 2 * rng.random((160, 12)), epsilon_L=1.0, epsilon_R=1.0, k0dx=2 * np.pi / 15,
                yBC="periodic")
    h = _abi.Handle(0)
    S0, _ = rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], handle=h)
    for tile in (32, 64):
        autotune.install(h, {"entries": [{"rows": 10 ** 6, "best": tile}]})
        S, _ = rgf_b200.cal_smatrix_RGF(syst, ["left", "right"], ["left", "right"], handle=h,
                                        options=_abi.Options(_abi.RGF_FP64, 0, 0, 1))
        assert h.profile()[3].startswith(f"k_persist<{tile},")
        assert np.linalg.norm(S - S0) <= 1e-12 * np.linalg.norm(S0)


def test_annotate_picks_fewest_sm_microseconds():
    t = autotune.annotate({"entries": [{"N": 256, "rows": 291, "us_per_slice": {"96": 193.0, "64": 147.0, "32": 129.0},
                                        "best": 32}]})
    e = t["entries"][0]
    assert e["best_throughput"] == 96  # 18 SMs x 193 us beats 27 x 147 and 102 x 129
    assert autotune.grid_sms(291, 96) == 18 and autotune.grid_sms(291, 32) == 102


def test_committed_b200_table():
    """The table measured on this pool's B200s (148 SMs) is in the package."""
    t = autotune.load("NVIDIA B200", 148)
    assert t is not None and t["sms"] == 148 and len(t["entries"]) >= 8
    for e in t["entries"]:
        assert e["best"] in (32, 64, 96) and e["best_throughput"] in (32, 64, 96)

"""Tile-shape autotuner of the persistent sweep (tile tables for
rgf_set_tile_table).

For a set of transverse sizes N it times the persistent engine on a short
synthetic 2D structure (periodic, eps 1 + 2U, k0dx = 2 pi / 15, full S, a
fixed number of slices) with each square tile that fits the GPU (96, 64,
32), keeps the fastest per size, and writes a table keyed by the matrix's
active rows Rp (N plus the carried output channels): an entry covers sizes up
to the midpoint towards the next measured one.  The table is cached as JSON
(one file per GPU model and SM count) and installed on a handle with
``install``.

    python -m rgf_b200.autotune [--out FILE] [--slices K] [--sizes 64,128,...]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time
from pathlib import Path

import numpy as np

from . import _abi
from .api import _request

TILES = (96, 64, 32)
DEFAULT_SIZES = (64, 96, 128, 192, 256, 320, 384, 448, 512, 640, 768, 1024)
CACHE_DIR = Path(__file__).resolve().parent / "tuned"


def cache_path(gpu_name: str, sms: int) -> Path:
    slug = "".join(c if c.isalnum() else "_" for c in gpu_name).strip("_").lower()
    return CACHE_DIR / f"tiles_{slug}_{sms}sm.json"


def table_from_measurements(rows: list) -> tuple:
    """rows: [{"rows": Rp, "best": tile}, ...] -> (rows_max, tile), each entry
    reaching to the midpoint towards the next measured size."""
    rows = sorted(rows, key=lambda r: r["rows"])
    rmax, tile = [], []
    for k, r in enumerate(rows):
        upper = (r["rows"] + rows[k + 1]["rows"]) // 2 if k + 1 < len(rows) else 1 << 40
        rmax.append(int(upper))
        tile.append(int(r["best"]))
    return rmax, tile


def grid_sms(rows: int, tile: int) -> int:
    """SMs one persistent sweep of a full request holds: its tiles (Rp rows,
    Rp + 2 columns rounded up to even) plus the T-server and prep CTAs."""
    cols = ((rows + 1) & ~1) + 2
    return -(-rows // tile) * -(-cols // tile) + 2


def annotate(table: dict) -> dict:
    """Adds to every entry the tile that needs the fewest SM-microseconds per
    slice ("best_throughput": the choice when many structures share the GPU,
    as in a batch) beside the fastest one ("best")."""
    for e in table["entries"]:
        cost = {int(t): us * grid_sms(e["rows"], int(t)) for t, us in e["us_per_slice"].items()}
        e["sm_us_per_slice"] = {str(t): round(c, 1) for t, c in cost.items()}
        e["best_throughput"] = min(cost, key=cost.get)
    return table


def install(handle, table: dict, mode: str = "latency") -> None:
    """Install a tuned table (as written by ``tune``) on an _abi.Handle: the
    fastest tile per size (mode "latency", single S-matrices) or the one with
    the fewest SM-microseconds (mode "throughput", batches)."""
    key = "best" if mode == "latency" else "best_throughput"
    rmax, tile = table_from_measurements([{"rows": e["rows"], "best": e[key]} for e in table["entries"]])
    a = (ctypes.c_int64 * max(len(rmax), 1))(*rmax)
    b = (ctypes.c_int32 * max(len(tile), 1))(*tile)
    _abi.check(handle.lib.rgf_set_tile_table(handle.h, len(rmax), a, b))


def load(gpu_name: str, sms: int, path: str | None = None) -> dict | None:
    """The cached table of this GPU model and SM count, or None."""
    p = Path(path) if path else cache_path(gpu_name, sms)
    if not p.exists():
        return None
    t = json.loads(p.read_text())
    if t.get("sms") != sms:
        return None
    return t


def _force(handle, tile: int) -> None:
    a = (ctypes.c_int64 * 1)(1 << 40)
    b = (ctypes.c_int32 * 1)(tile)
    _abi.check(handle.lib.rgf_set_tile_table(handle.h, 1, a, b))


def tune(device: int = 0, sizes=DEFAULT_SIZES, slices: int = 24, reps: int = 3) -> dict:
    import torch
    h = _abi.Handle(device)
    props = torch.cuda.get_device_properties(device)
    lib = h.lib
    req, keep = _request(["left", "right"], ["left", "right"])
    entries = []
    for N in sizes:
        rng = np.random.default_rng(N)
        epsn = np.ascontiguousarray((1 + 2 * rng.random((N, slices))).astype(complex).ravel(order="F"))
        eps = torch.from_numpy(epsn).to(f"cuda:{device}")
        sy = _abi.Syst2D(N, slices, eps.data_ptr(), 1, _abi.cplx(1.0), _abi.cplx(1.0), _abi.cplx(2 * np.pi / 15),
                         _abi.BC_PERIODIC, 0.0)
        no, ni = ctypes.c_int64(), ctypes.c_int64()
        _abi.check(lib.rgf_smatrix_size_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(no),
                                           ctypes.byref(ni)))
        S = torch.zeros((ni.value, no.value), dtype=torch.complex128, device=f"cuda:{device}")
        opt = _abi.Options(_abi.RGF_FP64, 0, 1, 1)  # the persistent launch is timed with CUDA events
        times = {}
        for t in TILES:
            _force(h, t)
            best = None
            try:
                for r in range(reps + 1):
                    _abi.check(lib.rgf_smatrix_2d(h.h, ctypes.byref(sy), ctypes.byref(req), ctypes.byref(opt),
                                                  S.data_ptr(), no.value, None))
                    n, ms, _, name = h.profile()
                    if not name.startswith(f"k_persist<{t},"):
                        best = None  # this tile did not fit: the engine chose another
                        break
                    if r and n:
                        best = ms / slices if best is None else min(best, ms / slices)
            except _abi.RGFError:
                best = None
            if best is not None:
                times[t] = best * 1e3  # us per slice
        if times:
            entries.append({"N": N, "rows": N + no.value // 2, "us_per_slice": times,
                            "best": min(times, key=times.get)})
    _abi.check(lib.rgf_set_tile_table(h.h, 0, None, None))
    del keep
    h.close()
    return annotate({"gpu": props.name, "sms": props.multi_processor_count, "slices": slices,
                     "workload": "2D periodic, eps 1+2U, k0dx 2pi/15, full S",
                     "time": time.strftime("%Y-%m-%d %H:%M:%S"), "entries": entries})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--slices", type=int, default=24)
    ap.add_argument("--sizes", default=",".join(map(str, DEFAULT_SIZES)))
    args = ap.parse_args()
    t = tune(sizes=[int(x) for x in args.sizes.split(",")], slices=args.slices)
    out = Path(args.out) if args.out else cache_path(t["gpu"], t["sms"])
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text(json.dumps(t, indent=1))
    print(json.dumps(t, indent=1))
    print(f"-> {out}")


if __name__ == "__main__":
    main()

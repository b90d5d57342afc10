"""L-split S-matrix of a 2D structure: the slices are cut in two parts, each
swept from its own lead (on its own GPU, or one after the other on one), and
the two segment states are joined across the cut (rgf_segment_sweep_2d /
rgf_segment_merge_2d of the C ABI).

The reference's slice loop (cal_smatrix_RGF.m:263-269) is strictly
sequential; this split lets two GPUs share one S-matrix with a single
message between them: rank 1 sends its segment state, (N + n_out_R) x
(N + n_in_R) complex, to rank 0, which merges.  Each part is the ordinary
channel-projected sweep, so the split costs one merge (about three slices of
work) on top of the two half sweeps.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from .api import _bc_2d, _check_syst, _get, _options, _request
from ._abi import Syst2D, check, cplx, ptr


class DeviceSegments:
    """The two operations of the split on this process's GPU (C ABI)."""

    def __init__(self, syst, out, in_, device: int = 0, handle=None, options=None):
        _check_syst(syst, "yBC")
        eps = np.asarray(_get(syst, "epsilon"))
        self.ny, self.nx = eps.shape
        bc, ka = _bc_2d(_get(syst, "yBC"))
        self.req, self._keep = _request(out, in_)
        self.h = handle or _abi.default_handle(device)
        self._eps = np.ascontiguousarray(eps.astype(complex).ravel(order="F"))
        self.sy = Syst2D(self.ny, self.nx, ptr(self._eps), 0, cplx(_get(syst, "epsilon_L")),
                         cplx(_get(syst, "epsilon_R")), cplx(_get(syst, "k0dx")), bc, ka)
        self.opt = _options(options)
        no, ni = ctypes.c_int64(), ctypes.c_int64()
        check(self.h.lib.rgf_smatrix_size_2d(self.h.h, ctypes.byref(self.sy), ctypes.byref(self.req),
                                             ctypes.byref(no), ctypes.byref(ni)))
        self.n_out, self.n_in = no.value, ni.value
        self._sides = self._side_counts(out, in_)

    def _side_counts(self, out, in_):
        """(n_out, n_in) per side: the S block sizes of one-sided requests."""
        counts = []
        for side in ("left", "right"):
            o = _one_side(out, side, "out")
            i = _one_side(in_, side, "in")
            r, keep = _request(o, i)
            no, ni = ctypes.c_int64(), ctypes.c_int64()
            check(self.h.lib.rgf_smatrix_size_2d(self.h.h, ctypes.byref(self.sy), ctypes.byref(r), ctypes.byref(no),
                                                 ctypes.byref(ni)))
            counts.append((no.value, ni.value))
            del keep
        return counts

    def state(self, side: int, cut: int) -> np.ndarray:
        no, ni = self._sides[side]
        st = np.zeros((self.ny + no, self.ny + ni), dtype=complex)  # row-major, as the ABI writes it
        check(self.h.lib.rgf_segment_sweep_2d(self.h.h, ctypes.byref(self.sy), ctypes.byref(self.req),
                                              ctypes.byref(self.opt), int(side), int(cut), st.ctypes.data))
        return st

    def merge(self, state_L: np.ndarray, state_R: np.ndarray) -> np.ndarray:
        S = np.zeros((max(self.n_out, 1), max(self.n_in, 1)), dtype=complex, order="F")
        sL = np.ascontiguousarray(state_L, dtype=complex)
        sR = np.ascontiguousarray(state_R, dtype=complex)
        check(self.h.lib.rgf_segment_merge_2d(self.h.h, ctypes.byref(self.sy), ctypes.byref(self.req),
                                              ctypes.byref(self.opt), sL.ctypes.data, sR.ctypes.data, S.ctypes.data,
                                              S.shape[0]))
        return S[:self.n_out, :self.n_in]


def _one_side(req, side: str, kind: str):
    """The part of a request on one side (struct or cell form)."""
    if isinstance(req, dict):
        key = f"ind_{kind}_{'L' if side == 'left' else 'R'}"
        return {key: req[key]} if key in req else {}
    names = ("left", "L") if side == "left" else ("right", "R")
    return [side] if any(isinstance(el, str) and el in names for el in req) else []


def cal_smatrix_RGF_split(syst, out, in_, *, cut: int | None = None, group=None, segments=None, device: int = 0):
    """S of a 2D structure with its slices split at `cut` (default L // 2).

    With a torch.distributed group of two ranks, rank 0 sweeps [0, cut) from
    the left lead and rank 1 [cut, L) from the right lead; rank 1 sends its
    state to rank 0, which merges and returns S (rank 1 returns None).
    Without a group (or with one rank) both parts run here.  `segments`
    supplies the two operations (default: this process's GPU through the C
    ABI)."""
    L = np.asarray(_get(syst, "epsilon")).shape[1]
    cut = L // 2 if cut is None else int(cut)
    seg = segments or DeviceSegments(syst, out, in_, device=device)
    dist = None
    if group is not None:
        import torch.distributed as dist
    world = 1 if dist is None else dist.get_world_size(group)
    if world == 1:
        return seg.merge(seg.state(0, cut), seg.state(1, cut))
    if world != 2:
        raise ValueError("the split runs on one or two ranks")
    import torch
    rank = dist.get_rank(group)
    dev = "cpu" if dist.get_backend(group) == "gloo" else f"cuda:{torch.cuda.current_device()}"
    if rank == 1:
        st = seg.state(1, cut)
        dist.send(torch.tensor(st.shape, dtype=torch.int64, device=dev), dst=0, group=group)
        dist.send(torch.from_numpy(np.ascontiguousarray(st).view(np.float64)).to(dev), dst=0, group=group)
        return None
    st_L = seg.state(0, cut)
    shape = torch.zeros(2, dtype=torch.int64, device=dev)
    dist.recv(shape, src=1, group=group)
    buf = torch.zeros((int(shape[0]), 2 * int(shape[1])), dtype=torch.float64, device=dev)
    dist.recv(buf, src=1, group=group)
    st_R = buf.cpu().numpy().view(np.complex128)
    return seg.merge(st_L, st_R)

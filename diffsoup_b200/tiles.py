"""Screen-tile bins of a batch of views (host side of csrc/tiled.cu).

`bin_views` runs ds_tiles_bin once per (clip positions, triangles,
resolutions) and returns a `Bins` object that the tiled rasterizer and the
tiled opacity-aux pass share, so the training step bins each batch once.

List capacity: the number of (triangle, tile) entries is data dependent.  The
bins are sized from a per-device estimate that doubles whenever a kernel
reports DS_STATUS_LIST_OVERFLOW; tiles whose list did not fit fall back to
testing every triangle of their view, so results are exact either way and no
host synchronisation is needed.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _core

DS_TILE = 16
DS_STATUS_LIST_OVERFLOW = 1
DS_STATUS_RECORD_FALLBACK = 2

_capacity: Dict[int, int] = {}
_pending_status: Dict[int, Tuple[torch.Tensor, torch.cuda.Event, int]] = {}
_view_tables: Dict[Tuple, Tuple[torch.Tensor, int, int, List[int]]] = {}


def view_table(hw: Sequence[Tuple[int, int]], device: torch.device):
    """(device table of ds_view_desc, num_tiles, num_pixels, pixel offsets)."""
    key = (tuple(hw), device.index if device.index is not None else torch.cuda.current_device())
    hit = _view_tables.get(key)
    if hit is not None:
        return hit
    B = len(hw)
    Hs = (C.c_int * max(B, 1))(*[h for h, _ in hw])
    Ws = (C.c_int * max(B, 1))(*[w for _, w in hw])
    desc = (_core.ViewDesc * max(B, 1))()
    npix = C.c_int64(0)
    nt = _core.lib.ds_make_view_table(B, Hs, Ws, desc, C.byref(npix))
    if nt < 0 or (nt == 0 and B > 0):
        _core.check(nt if nt > 0 else 1)
    raw = torch.frombuffer(bytearray(C.string_at(C.addressof(desc), C.sizeof(_core.ViewDesc) * max(B, 1))),
                           dtype=torch.uint8)
    table = raw.to(device)
    offs = [int(desc[b].pix_offset) for b in range(B)]
    out = (table, int(nt), int(npix.value), offs)
    _view_tables[key] = out
    return out


def _device_index(device: torch.device) -> int:
    return device.index if device.index is not None else torch.cuda.current_device()


def _capacity_for(device: torch.device, B: int, T: int) -> int:
    di = _device_index(device)
    pend = _pending_status.get(di)
    if pend is not None:
        status, ev, cap = pend
        if ev.query():
            if int(status.item()) & DS_STATUS_LIST_OVERFLOW:
                _capacity[di] = max(_capacity.get(di, 0), 2 * cap)
            del _pending_status[di]
    want = max(1 << 16, 8 * B * T)
    cap = max(_capacity.get(di, 0), want)
    _capacity[di] = cap
    return min(cap, 0x7FFFFFFF)


@dataclass
class Bins:
    B: int
    T: int
    V: int
    hw: Tuple[Tuple[int, int], ...]
    views: torch.Tensor
    num_tiles: int
    num_pixels: int
    pix_offsets: List[int]
    capacity: int
    workspace: torch.Tensor
    status: torch.Tensor
    pos: torch.Tensor
    tri: torch.Tensor
    key: Tuple


_last: Optional[Bins] = None


def _key(pos: torch.Tensor, tri: torch.Tensor, hw) -> Tuple:
    return (pos.data_ptr(), pos._version, tuple(pos.shape), tri.data_ptr(), tri._version, tuple(tri.shape),
            tuple(hw), torch.cuda.current_stream(pos.device).cuda_stream)


def bin_views(pos: torch.Tensor, tri: torch.Tensor, hw: Sequence[Tuple[int, int]], reuse: bool = True) -> Bins:
    """Bin every (view, triangle) of pos [B,V,4] into 16x16 screen tiles."""
    global _last
    hw = tuple((int(h), int(w)) for h, w in hw)
    key = _key(pos, tri, hw)
    if reuse and _last is not None and _last.key == key:
        return _last
    B, V, _ = pos.shape
    T = tri.shape[0]
    dev = pos.device
    table, nt, npix, offs = view_table(hw, dev)
    cap = _capacity_for(dev, B, T)
    ws = _core.workspace(_core.lib.ds_tiles_workspace_size(B, T, nt, cap), dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    _core.check(_core.lib.ds_tiles_bin(B, _core.ptr(table), nt, V, _core.ptr(pos), T, _core.ptr(tri), _core.ptr(ws),
                                       ws.numel(), cap, _core.ptr(status), _core.stream()))
    host = torch.empty(1, dtype=torch.int32, pin_memory=True)
    host.copy_(status, non_blocking=True)
    ev = torch.cuda.Event()
    ev.record()
    _pending_status[_device_index(dev)] = (host, ev, cap)
    bins = Bins(B, T, V, hw, table, nt, npix, offs, cap, ws, status, pos, tri, key)
    _last = bins
    return bins


def rasterize(bins: Bins, level: int, alpha_src_2d: torch.Tensor, rast: torch.Tensor, thr_mode: int,
              thr_const: float = 0.5, rng: Optional[torch.Tensor] = None) -> None:
    """ds_tiles_rasterize into rast (packed pixels x 4)."""
    _core.check(_core.lib.ds_tiles_rasterize(bins.B, _core.ptr(bins.views), bins.num_tiles, bins.V,
                                             _core.ptr(bins.pos), bins.T, _core.ptr(bins.tri), level,
                                             alpha_src_2d.shape[1], _core.ptr(alpha_src_2d), thr_mode, thr_const,
                                             _core.ptr(rng), _core.ptr(rast), _core.ptr(bins.workspace),
                                             bins.workspace.numel(), bins.capacity, _core.stream()))


def opacity_aux(bins: Bins, level: int, alpha_src_2d: torch.Tensor, color: torch.Tensor, target: torch.Tensor,
                rast: torch.Tensor, grad_alpha_src: torch.Tensor, scale: float = 1.0) -> None:
    """ds_tiles_opacity_aux: grad_alpha_src += scale * dL_aux/dalpha_src."""
    Cd = color.shape[-1]
    _core.check(_core.lib.ds_tiles_opacity_aux(bins.B, _core.ptr(bins.views), bins.num_tiles, bins.V,
                                               _core.ptr(bins.pos), bins.T, _core.ptr(bins.tri), level,
                                               alpha_src_2d.shape[1], _core.ptr(alpha_src_2d), Cd, _core.ptr(color),
                                               _core.ptr(target), _core.ptr(rast), float(scale),
                                               _core.ptr(grad_alpha_src), _core.ptr(bins.workspace),
                                               bins.workspace.numel(), bins.capacity, _core.stream()))

"""Adaptive triangle-soup subdivision on the GPU (csrc/remesh.cu), with the
signatures of the reference's python/diffsoup/remesh.py.

The reference splits on the CPU with a global priority queue of edges
(src/remesh.cpp, src/remesh_clip.cpp).  In a soup every face is split
independently, so here each input face walks its own split tree on the GPU:
the same triangles as the reference, bit for bit, with the new vertices and
faces numbered per input face (depth first) instead of in the queue's global
order.  Training uses the threshold mode (`*_until`, num_splits = -1).  A
split budget (num_splits > 0) keeps the queue's global choice: the
num_splits longest splits, found by a search over counting passes; splits of
exactly equal length at the cut-off are taken in face order.
"""

from __future__ import annotations

import ctypes as C
from typing import Tuple

import torch

from . import _core

Quad = Tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]
DS_STATUS_SPLIT_LIMIT = 4


def _split(mode: int, verts: torch.Tensor, faces: torch.Tensor, num_splits: int, tau: float,
           mvp: torch.Tensor = None, valid: torch.Tensor = None, aspect_wh: float = 1.0) -> Quad:
    out_dev = verts.device
    dev = out_dev if out_dev.type == "cuda" else torch.device("cuda", torch.cuda.current_device())
    v = verts.detach().to(dev, torch.float32).contiguous()
    f = faces.detach().to(dev, torch.int32).contiguous()
    N, M = v.shape[0], f.shape[0]
    vm = None
    if mode == 1:
        vm = valid.detach().to(dev, torch.int32).contiguous()
    m_host = None
    if mvp is not None:
        m_host = (C.c_float * 16)(*mvp.detach().to("cpu", torch.float32).reshape(-1).tolist())
    with torch.cuda.device(dev):
        offsets = torch.empty(M + 1, dtype=torch.int64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        ws = _core.workspace(_core.lib.ds_split_soup_workspace_size(M), dev)
        total = C.c_int64(0)
        _core.check(_core.lib.ds_split_soup_count(mode, m_host, float(aspect_wh), float(tau), int(num_splits), N,
                                                  _core.ptr(v), M, _core.ptr(f), _core.ptr(vm), _core.ptr(offsets),
                                                  C.byref(total), _core.ptr(ws), ws.numel(), _core.ptr(status),
                                                  _core.stream()))
        if int(status.item()) & DS_STATUS_SPLIT_LIMIT:
            raise RuntimeError("split_triangle_soup: a face's split tree exceeds the limits (2^20 splits per face, "
                               "depth 40, 2^27 per call); the threshold is too small for this soup")
        S = int(total.value)
        out_v = torch.empty(N + 3 * S, 3, dtype=torch.float32, device=dev)
        out_f = torch.empty(M + S, 3, dtype=torch.int32, device=dev)
        out_map = torch.empty(M + S, dtype=torch.int32, device=dev)
        out_flag = torch.empty(M + S, dtype=torch.int32, device=dev)
        _core.check(_core.lib.ds_split_soup_emit(mode, m_host, float(aspect_wh), N, _core.ptr(v), M, _core.ptr(f),
                                                 _core.ptr(offsets), S, _core.ptr(ws), _core.ptr(out_v),
                                                 _core.ptr(out_f), _core.ptr(out_map), _core.ptr(out_flag),
                                                 _core.ptr(status), _core.stream()))
    return (out_v.to(out_dev), out_f.to(out_dev), out_map.to(out_dev), out_flag.to(out_dev))


def split_triangle_soup(verts: torch.Tensor, faces: torch.Tensor, num_splits: int, tau: float = 0.0) -> Quad:
    """Bisects longest world-space edges (python/diffsoup/remesh.py:9-47).
    Returns (verts [N',3] f32, faces [M',3] i32, face_mapping [M'] i32,
    face_flags [M'] i32 = 1 for faces never split)."""
    assert verts.ndim == 2 and verts.shape[1] == 3, "verts must be (N, 3)"
    assert faces.ndim == 2 and faces.shape[1] == 3, "faces must be (M, 3)"
    return _split(0, verts, faces, int(num_splits), float(tau))


def split_triangle_soup_until(verts: torch.Tensor, faces: torch.Tensor, tau: float, hard_cap: int = None) -> Quad:
    """Splits until every world-space edge is below tau (remesh.py:50-70)."""
    ns = -1 if hard_cap is None else int(hard_cap)
    return split_triangle_soup(verts, faces, ns, tau=float(tau))


def split_triangle_soup_clip(resolution: Tuple[int, int], mvp: torch.Tensor, verts: torch.Tensor,
                             faces: torch.Tensor, valid_faces: torch.Tensor, num_splits: int,
                             tau_ratio: float = 0.0) -> Quad:
    """Bisects longest screen-space edges under one MVP (remesh.py:73-129):
    lengths in NDC with x scaled by W/H (image-height units), edges with an end
    outside the NDC cube ignored, only faces with valid_faces > 0 split."""
    H, W = resolution
    assert mvp.shape == (4, 4)
    assert verts.ndim == 2 and verts.shape[1] == 3
    assert faces.ndim == 2 and faces.shape[1] == 3
    assert valid_faces.shape == (faces.shape[0],)
    return _split(1, verts, faces, int(num_splits), float(tau_ratio), mvp=mvp, valid=valid_faces,
                  aspect_wh=float(W) / float(H))


def split_triangle_soup_clip_until(resolution: Tuple[int, int], mvp: torch.Tensor, verts: torch.Tensor,
                                   faces: torch.Tensor, valid_faces: torch.Tensor, tau_ratio: float,
                                   hard_cap: int = None) -> Quad:
    """Splits until every screen-space edge is below tau_ratio image heights
    (remesh.py:132-158)."""
    ns = -1 if hard_cap is None else int(hard_cap)
    return split_triangle_soup_clip(resolution, mvp, verts, faces, valid_faces, ns, tau_ratio)


def expand_by_index(source: torch.Tensor, index_map: torch.Tensor) -> torch.Tensor:
    """result[j] = source[index_map[j]] (remesh.py:161-190): per-face data of
    the parents carried to their children."""
    if not (torch.is_tensor(source) and torch.is_tensor(index_map)):
        raise TypeError("expand_by_index: `source` and `index_map` must be torch tensors")
    idx = index_map.to(device=source.device, dtype=torch.long)
    if idx.numel() > 0 and (int(idx.min()) < 0 or int(idx.max()) >= source.shape[0]):
        raise ValueError("expand_by_index: `index_map` holds indices outside [0, len(source))")
    return source[idx]


def split_edges_from_training_views(resolution: Tuple[int, int], MVPs: torch.Tensor, V: torch.Tensor,
                                    F: torch.Tensor, Rmax: int, alpha_acc: torch.Tensor, tau_ratio: float,
                                    num_views_cap: int) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """The resampling step of training (examples/utils.py:493-545): for up to
    num_views_cap random views, the faces visible in that view (binned
    rasterizer, deterministic opacity threshold) are split until their
    screen-space edges are below tau_ratio image heights.  Returns (V, F,
    face_map into the input F)."""
    from . import visibility
    from . import tiles as _tiles

    H, W = int(resolution[0]), int(resolution[1])
    dev = V.device
    M0 = F.shape[0]
    perm = torch.randperm(MVPs.shape[0], device=dev, dtype=torch.long)
    mvps = MVPs[perm[:min(MVPs.shape[0], int(num_views_cap))]]
    S = _core.feats_at_level(int(Rmax))
    a2 = alpha_acc.reshape(alpha_acc.shape[0], -1).float().contiguous()
    assert a2.shape[1] == S, "Invalid feature size."
    pos = visibility.project_vertices(V.float(), mvps.float())
    Fi = F.int().contiguous()
    bins = _tiles.bin_views(pos, Fi, [(H, W)] * pos.shape[0], reuse=False)
    rast = torch.empty(bins.num_pixels, 4, device=dev)
    _tiles.rasterize(bins, int(Rmax), a2, rast, thr_mode=0, thr_const=0.5)
    fmap = torch.arange(M0, device=dev, dtype=torch.long)
    for i in range(mvps.shape[0]):
        ids = rast[i * H * W:(i + 1) * H * W, 3]
        seen = torch.zeros(M0, dtype=torch.int32, device=dev)
        seen[(ids[ids > 0].long() - 1).unique()] = 1
        valid = seen[fmap].contiguous()
        V, F, fmap_next, _ = split_triangle_soup_clip_until((H, W), mvps[i], V, F, valid, tau_ratio=tau_ratio)
        fmap = fmap[fmap_next.long()].contiguous()
    return V, F, fmap

"""Per-triangle visibility over a set of views, the statistic that drives the
resampling of the soup (examples/utils.py:445-482, count_visible_triangles).

Same signature and result as the reference's helper; all views of a batch
go through one binned rasterizer launch with the deterministic opacity
threshold (0.5, stochastic=False) and the ID buffer is counted by one kernel
(ds_count_triangle_ids) into the running total.
"""

from __future__ import annotations

from typing import Tuple

import torch

from . import _core
from . import tiles as _tiles


def project_vertices(V: torch.Tensor, MVPs: torch.Tensor) -> torch.Tensor:
    """Clip-space positions [B, Nv, 4] = MVPs[b] . (V, 1) (examples/utils.py:
    412-426), by the projection kernel of the training step."""
    V = V.float().contiguous()
    M = MVPs.float().contiguous()
    out = torch.empty(M.shape[0], V.shape[0], 4, dtype=torch.float32, device=V.device)
    _core.check(_core.lib.ds_project_vertices(M.shape[0], V.shape[0], _core.ptr(V), _core.ptr(M), _core.ptr(out),
                                              _core.stream()))
    return out


def count_visible_triangles(resolution: Tuple[int, int], MVPs: torch.Tensor, V: torch.Tensor, F: torch.Tensor,
                            level: int, alpha_src: torch.Tensor, batch_size: int = 16) -> torch.Tensor:
    """(Nf,) int64 pixel counts per triangle summed over the views MVPs [N,4,4]."""
    H, W = int(resolution[0]), int(resolution[1])
    S = _core.feats_at_level(level)
    a2 = alpha_src.reshape(alpha_src.shape[0], -1)
    assert a2.shape[1] == S, "Invalid feature size."
    a2 = a2.float().contiguous()
    F = F.int().contiguous()
    count = torch.zeros(F.shape[0], dtype=torch.int64, device=V.device)
    status = torch.zeros(1, dtype=torch.int32, device=V.device)
    for start in range(0, MVPs.shape[0], max(1, int(batch_size))):
        mvp = MVPs[start:start + batch_size]
        pos = project_vertices(V.float(), mvp.float())
        bins = _tiles.bin_views(pos, F, [(H, W)] * pos.shape[0], reuse=False)
        rast = torch.empty(bins.num_pixels, 4, device=V.device)
        _tiles.rasterize(bins, level, a2, rast, thr_mode=0, thr_const=0.5)
        _core.check(_core.lib.ds_count_triangle_ids(bins.num_pixels, _core.ptr(rast), F.shape[0], _core.ptr(count),
                                                    _core.ptr(status), _core.stream()))
    return count

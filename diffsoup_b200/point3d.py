"""Point-cloud helpers of the training scripts (python/diffsoup/point3d.py):
the soup's initial spacing and triangles, and vertex compaction after faces
are pruned.  Torch operations on whatever device the input lives on (the
spacing search runs on the GPU when one is present); none of them is on the
per-view path.
"""

from __future__ import annotations

import math

import numpy as np
import torch


def nn_spacing(points, reduction: str = "median") -> float:
    """Median (or mean) distance from each point to its nearest other point
    (point3d.py:11-39).  points: (N, 3).  Exact nearest neighbours by a
    blocked all-pairs search in FP32 on the GPU (on the CPU without one)."""
    P = torch.as_tensor(np.asarray(points, dtype=np.float32) if not torch.is_tensor(points) else points,
                        dtype=torch.float32)
    if P.dim() != 2 or P.shape[1] != 3:
        raise ValueError("`points` must be shaped (N, 3).")
    red = reduction.lower()
    if red not in ("median", "med", "mean", "avg", "average"):
        raise ValueError("`reduction` must be one of {'median', 'mean'}.")
    n = P.shape[0]
    if n < 2:
        return 0.0
    dev = torch.device("cuda") if torch.cuda.is_available() else P.device
    P = P.to(dev).contiguous()
    best = torch.empty(n, dtype=torch.float32, device=dev)
    rows = max(1, min(n, (1 << 25) // n))  # about 400 MB of coordinate differences per block
    for s in range(0, n, rows):
        q = P[s:s + rows]
        d2 = ((q[:, None, :] - P[None, :, :]) ** 2).sum(-1)  # exact differences, no Gram-matrix cancellation
        idx = torch.arange(s, s + q.shape[0], device=dev)
        d2[torch.arange(q.shape[0], device=dev), idx] = float("inf")  # not the point itself
        best[s:s + q.shape[0]] = d2.min(dim=1).values
    nn = best.sqrt()
    vals = nn[torch.isfinite(nn)].double().cpu().numpy()
    if vals.size == 0:
        return 0.0
    return float(np.mean(vals)) if red in ("mean", "avg", "average") else float(np.median(vals))


def triangle_soup_from_points(xyz: torch.Tensor, scale: float):
    """One equilateral triangle of circumradius `scale` per point, centred on
    it and turned by a uniformly random rotation (point3d.py:42-112; the
    rotation is a unit quaternion from three uniforms, Shoemake's method).
    Returns V (3N, 3) and F (N, 3) int32 on xyz's device."""
    if xyz.dim() != 2 or xyz.shape[-1] != 3:
        raise ValueError("`xyz` must be shaped (N, 3).")
    n = xyz.shape[0]
    dt, dev = xyz.dtype, xyz.device
    if n == 0:
        return xyz.new_zeros((0, 3)), torch.empty((0, 3), dtype=torch.int32, device=dev)
    h = math.sqrt(3.0) / 2.0
    corners = torch.tensor([[1.0, 0.0, 0.0], [-0.5, h, 0.0], [-0.5, -h, 0.0]], dtype=dt, device=dev) * scale
    u = torch.rand(3, n, device=dev, dtype=dt)
    a, b = torch.sqrt(1.0 - u[0]), torch.sqrt(u[0])
    t1, t2 = 2.0 * math.pi * u[1], 2.0 * math.pi * u[2]
    x, y, z, w = a * torch.sin(t1), a * torch.cos(t1), b * torch.sin(t2), b * torch.cos(t2)
    R = torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        torch.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)  # (N, 3, 3)
    V = (corners[None, :, None, :] * R[:, None, :, :]).sum(-1) + xyz[:, None, :]  # R @ corner, per triangle
    F = torch.arange(3 * n, device=dev, dtype=torch.int32).reshape(n, 3)
    return V.reshape(-1, 3).contiguous(), F


def remove_unreferenced_vertices_from_soup(verts: torch.Tensor, faces: torch.Tensor):
    """Drops the vertices no face uses and renumbers the faces, keeping the
    vertices' order (point3d.py:115-143).  Returns (verts', faces' int32)."""
    assert verts.dim() == 2 and verts.shape[1] == 3
    assert faces.dim() == 2 and faces.shape[1] == 3
    used = torch.zeros(verts.shape[0], dtype=torch.bool, device=faces.device)
    used[faces.reshape(-1).long()] = True
    new_index = torch.cumsum(used.long(), 0) - 1
    return verts[used.to(verts.device)].contiguous(), new_index[faces.long()].int().contiguous()

"""Rasterisation, edge gradients and view-direction encodings.

Drop-in for kenji-tojo/diffsoup python/diffsoup/rasterize.py: same public
functions, signatures, tensor layouts and assertions.  The fragment pipeline
of the reference (_compute_fragments + _depth_test, rasterize.py:14-126) is
still available for callers of the `_core` layer, but the public entry points
run the tiled B200 kernels (csrc/tiled.cu), which never materialise a fragment
list and never synchronise with the host.
"""

from __future__ import annotations

from typing import Tuple

import torch

from . import _core
from . import tiles as _tiles


# ---------------------------------------------------------------------------
#  Fragment computation (reference layer, rasterize.py:14-76)
# ---------------------------------------------------------------------------

def _filter_valid_fragments(frag_pix: torch.Tensor, frag_attrs: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """Compact fragment buffers, dropping rejected (-1) entries (rasterize.py:14-37)."""
    frag_pix_out = torch.empty_like(frag_pix)
    frag_attrs_out = torch.empty_like(frag_attrs)
    n = _core.filter_valid_fragments(frag_pix, frag_attrs, frag_pix_out, frag_attrs_out)
    return frag_pix_out[:n].contiguous(), frag_attrs_out[:n].contiguous()


def _compute_fragments(resolution: Tuple[int, int], pos: torch.Tensor, tri: torch.Tensor):
    """Per-pixel fragments of every view (rasterize.py:40-76)."""
    H, W = resolution
    B, V, _ = pos.shape
    T, _ = tri.shape
    device = pos.device
    assert pos.shape == (B, V, 4) and pos.dtype == torch.float32 and pos.is_contiguous()
    assert tri.shape == (T, 3) and tri.dtype == torch.int32 and tri.is_contiguous()
    assert pos.is_cuda and tri.device == device
    rects = torch.empty((B * T, 4), dtype=torch.int32, device=device)
    prefix = torch.empty(B * T, dtype=torch.int32, device=device)
    n = _core.compute_triangle_rects(H, W, pos, tri, rects, prefix)
    frag_pix = torch.full((n, 3), -1, dtype=torch.int32, device=device)
    frag_attrs = torch.empty((n, 4), dtype=torch.float32, device=device)
    _core.compute_fragments(H, W, pos, tri, prefix, rects, frag_pix, frag_attrs)
    return _filter_valid_fragments(frag_pix, frag_attrs)


def _depth_test(resolution, pos, frag_pix, frag_attrs, frag_alpha, alpha_thresh) -> torch.Tensor:
    """Depth test of a fragment list (rasterize.py:83-126)."""
    H, W = resolution
    B, V, _ = pos.shape
    n, _ = frag_pix.shape
    assert pos.shape == (B, V, 4) and pos.dtype == torch.float32 and pos.is_contiguous()
    assert frag_pix.shape == (n, 3) and frag_pix.dtype == torch.int32 and frag_pix.is_contiguous()
    assert frag_attrs.shape == (n, 4) and frag_attrs.dtype == torch.float32 and frag_attrs.is_contiguous()
    assert frag_alpha.shape == (n,) and frag_alpha.dtype == torch.float32 and frag_alpha.is_contiguous()
    assert alpha_thresh.shape == (n,) and alpha_thresh.dtype == torch.float32 and alpha_thresh.is_contiguous()
    assert pos.is_cuda
    rast = torch.zeros(B, H, W, 4, dtype=torch.float32, device=pos.device)
    _core.depth_test(frag_pix, frag_attrs, frag_alpha, alpha_thresh, rast)
    return rast


# ---------------------------------------------------------------------------
#  Stochastic opacity masking (rasterize.py:139-252)
# ---------------------------------------------------------------------------

class _OpacityAuxLossFn(torch.autograd.Function):
    """Zero-valued loss whose backward delivers dL_aux/dalpha_src.

    The forward re-enumerates every fragment tile by tile (ds_tiles_opacity_aux)
    instead of materialising the fragment list; the gradient is scaled by
    1/numel(color) in backward as in the reference (rasterize.py:183-196).
    """

    @staticmethod
    def forward(ctx, color, target, rast, pos, tri, level, alpha_src):
        B, H, W, _ = rast.shape
        assert alpha_src.ndim == 2
        bins = _tiles.bin_views(pos, tri, [(H, W)] * B)
        grad_alpha_src = torch.zeros_like(alpha_src)
        _tiles.opacity_aux(bins, level, alpha_src, color, target, rast, grad_alpha_src)
        ctx.save_for_backward(grad_alpha_src)
        ctx.weight = 1.0 / color.numel()
        return torch.zeros(1, dtype=torch.float32, device=rast.device)

    @staticmethod
    def backward(ctx, grad_loss):
        (grad_alpha_src,) = ctx.saved_tensors
        return None, None, None, None, None, None, ctx.weight * grad_loss * grad_alpha_src


def opacity_aux_loss(color, target, rast, pos, tri, level: int, alpha_src) -> torch.Tensor:
    """Stochastic opacity masking auxiliary loss (identically zero; its backward
    populates alpha_src.grad).  Same contract as rasterize.py:199-252."""
    B, H, W, C = color.shape
    dev = color.device
    _, V, _ = pos.shape
    T, _ = tri.shape
    _, S, _ = alpha_src.shape
    assert color.is_contiguous() and color.dtype == torch.float32
    assert target.shape == (B, H, W, C) and target.is_contiguous() and target.dtype == torch.float32
    assert rast.shape == (B, H, W, 4) and rast.is_contiguous() and rast.dtype == torch.float32
    assert pos.shape == (B, V, 4) and pos.is_contiguous() and pos.dtype == torch.float32
    assert tri.shape == (T, 3) and tri.is_contiguous() and tri.dtype == torch.int32
    assert alpha_src.shape == (T, S, 1) and alpha_src.dtype == torch.float32 and alpha_src.is_contiguous()
    assert color.is_cuda
    assert target.device == dev and rast.device == dev
    assert pos.device == dev and tri.device == dev
    return _OpacityAuxLossFn.apply(color, target, rast, pos, tri, level, alpha_src.squeeze(-1))


# ---------------------------------------------------------------------------
#  Edge gradients (rasterize.py:259-312)
# ---------------------------------------------------------------------------

class _EdgeGradFn(torch.autograd.Function):
    """Identity on colour; backward adds silhouette/edge gradients to pos."""

    @staticmethod
    def forward(ctx, color, rast, pos, tri):
        ctx.save_for_backward(color, rast, pos, tri)
        return color

    @staticmethod
    def backward(ctx, grad_color):
        color, rast, pos, tri = ctx.saved_tensors
        grad_color = grad_color.contiguous()
        grad_pos = torch.zeros_like(pos)
        _core.backward_edge_grad(color, grad_color, rast, pos, grad_pos, tri)
        return grad_color, None, grad_pos, None


def edge_grad(color, rast, pos, tri) -> torch.Tensor:
    """Attach silhouette edge gradients to vertex positions (rasterize.py:277-312)."""
    B, H, W, C = color.shape
    _, V, _ = pos.shape
    T, _ = tri.shape
    assert color.is_contiguous() and color.dtype == torch.float32
    assert rast.shape == (B, H, W, 4) and rast.is_contiguous() and rast.dtype == torch.float32
    assert pos.shape == (B, V, 4) and pos.is_contiguous() and pos.dtype == torch.float32
    assert tri.shape == (T, 3) and tri.is_contiguous() and tri.dtype == torch.int32
    assert color.is_cuda
    assert rast.device == color.device and pos.device == color.device and tri.device == color.device
    return _EdgeGradFn.apply(color, rast, pos, tri)


# ---------------------------------------------------------------------------
#  View-direction encodings (rasterize.py:319-341)
# ---------------------------------------------------------------------------

def encode_view_dir_sh2(rast, inv_mvp) -> torch.Tensor:
    """Degree-2 spherical-harmonic basis of the per-pixel view direction: (B,H,W,9)."""
    B, H, W, _ = rast.shape
    dev = rast.device
    assert rast.shape == (B, H, W, 4) and rast.is_contiguous() and rast.dtype == torch.float32
    assert inv_mvp.shape == (B, 4, 4) and inv_mvp.is_contiguous() and inv_mvp.dtype == torch.float32
    assert rast.is_cuda and inv_mvp.device == dev
    enc = torch.zeros(B, H, W, 9, dtype=torch.float32, device=dev)
    _core.encode_view_dir_sh2(rast, inv_mvp, enc)
    return enc


def encode_view_dir(rast, inv_mvp) -> torch.Tensor:
    """Unit view direction per covered pixel, (B,H,W,3): the vector the
    reference's SH2 encoder evaluates (encoding.cu:28-53), for shaders that take
    the raw direction."""
    B, H, W, _ = rast.shape
    dev = rast.device
    assert rast.shape == (B, H, W, 4) and rast.is_contiguous() and rast.dtype == torch.float32
    assert inv_mvp.shape == (B, 4, 4) and inv_mvp.is_contiguous() and inv_mvp.dtype == torch.float32
    assert rast.is_cuda and inv_mvp.device == dev
    enc = torch.zeros(B, H, W, 3, dtype=torch.float32, device=dev)
    _core.encode_view_dir(rast, inv_mvp, enc)
    return enc


# ---------------------------------------------------------------------------
#  Utilities (rasterize.py:348-366)
# ---------------------------------------------------------------------------

def count_triangle_ids(rast: torch.Tensor, num_tris: int) -> torch.Tensor:
    """Pixels covered per triangle in a rasterisation buffer: (num_tris,) int64
    (rasterize.py:348-366; one kernel, ds_count_triangle_ids).  Like the
    reference's bincount, an ID beyond num_tris fails the assertion; checking
    it synchronises with the device."""
    assert rast.is_cuda and rast.dtype == torch.float32 and rast.shape[-1] == 4
    r = rast.contiguous()
    count = torch.zeros(num_tris, dtype=torch.int64, device=rast.device)
    status = torch.zeros(1, dtype=torch.int32, device=rast.device)
    _core.check(_core.lib.ds_count_triangle_ids(r.numel() // 4, _core.ptr(r), int(num_tris), _core.ptr(count),
                                                _core.ptr(status), _core.stream()))
    assert int(status.item()) == 0, "triangle id beyond num_tris"
    return count

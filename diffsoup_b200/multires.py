"""Multi-resolution triangle features: opacity, colour, level accumulation and
the shading MLP.

Drop-in for kenji-tojo/diffsoup python/diffsoup/multires.py (same public
functions, signatures, layouts and assertions).  rasterize_multires_triangle_alpha
runs the tiled rasterizer of csrc/tiled.cu with a counter-based stochastic
threshold instead of the fragment list plus torch.rand of the reference.
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch
from torch import nn

from . import _core
from . import tiles as _tiles


def feats_at_level(level: int) -> int:
    """Lattice samples per triangle at one level (multires.py:16-23)."""
    assert level >= 0
    return 3 if level == 0 else ((1 << (level - 1)) + 1) * ((1 << level) + 1)


def build_multires_triangle_color(T: int, min_level: int, max_level: int, feat_dim: int) -> torch.Tensor:
    """Zero (T, S, feat_dim) float32 buffer for levels [min_level, max_level] (multires.py:26-45)."""
    S = sum(feats_at_level(l) for l in range(min_level, max_level + 1))
    return torch.zeros(T, S, feat_dim, dtype=torch.float32)


# ---------------------------------------------------------------------------
#  Stochastic-opacity rasterisation (multires.py:52-102)
# ---------------------------------------------------------------------------

_iteration = 0


def _rng_state(device: torch.device) -> torch.Tensor:
    """Device (seed, iteration) for the Philox threshold.  The seed is drawn
    from torch's default CPU generator, so torch.manual_seed makes the masks
    reproducible."""
    global _iteration
    seed = int(torch.randint(0, 2 ** 62, (1,)).item())
    _iteration += 1
    return torch.tensor([seed, _iteration], dtype=torch.int64, device=device)


def rasterize_multires_triangle_alpha(resolution: Tuple[int, int], pos: torch.Tensor, tri: torch.Tensor, level: int,
                                      alpha_src: torch.Tensor, stochastic: bool = True) -> torch.Tensor:
    """Rasterise with per-fragment multires opacity and depth testing.

    Returns rast (B, H, W, 4) float32 = (b0, b1, z_ndc, tri_id + 1), 0 where
    nothing passes.  A fragment is kept when its opacity is >= its threshold:
    0.5 when stochastic is False (bit-identical IDs to the reference), else a
    uniform draw keyed by (seed, iteration, view, pixel, triangle).
    """
    H, W = resolution
    B, V, _ = pos.shape
    T, _ = tri.shape
    _, S, _ = alpha_src.shape
    dev = pos.device
    assert pos.shape == (B, V, 4) and pos.dtype == torch.float32 and pos.is_contiguous()
    assert tri.shape == (T, 3) and tri.dtype == torch.int32 and tri.is_contiguous()
    assert alpha_src.shape == (T, S, 1) and alpha_src.dtype == torch.float32 and alpha_src.is_contiguous()
    assert S == feats_at_level(level)
    assert pos.is_cuda and tri.device == dev and alpha_src.device == dev
    rast = torch.empty(B, H, W, 4, dtype=torch.float32, device=dev)
    if B == 0:
        return rast
    bins = _tiles.bin_views(pos, tri, [(H, W)] * B)
    a2 = alpha_src.view(T, S)
    if stochastic:
        _tiles.rasterize(bins, level, a2, rast, thr_mode=1, rng=_rng_state(dev))
    else:
        _tiles.rasterize(bins, level, a2, rast, thr_mode=0, thr_const=0.5)
    return rast


# ---------------------------------------------------------------------------
#  Colour MLP (multires.py:109-207)
# ---------------------------------------------------------------------------

class ColorMLP(nn.Module):
    """Per-pixel shading MLP with a residual blend.

    output = (1 - x[..., 3]) * x[..., :3] + x[..., 3] * sigmoid(MLP(x)), where
    MLP = n_layers hidden Linear+ReLU layers of width hidden_dim and a final
    Linear.  Module layout (``mlp`` = Sequential of Linear/ReLU/.../Sigmoid) and
    initialisation (Kaiming-uniform hidden layers, Xavier-uniform or zero output
    layer, zero biases) follow multires.py:128-167 so checkpoints interchange.
    """

    def __init__(self, input_dim: int, output_dim: int, hidden_dim: int = 16, n_layers: int = 2,
                 zero_last: bool = False):
        super().__init__()
        dims = [input_dim] + [hidden_dim] * n_layers
        mods = []
        for a, b in zip(dims[:-1], dims[1:]):
            mods += [nn.Linear(a, b), nn.ReLU()]
        mods += [nn.Linear(dims[-1], output_dim), nn.Sigmoid()]
        self.input_dim = input_dim
        self.output_dim = output_dim
        self.mlp = nn.Sequential(*mods)
        self._init_weights(zero_last)

    def _init_weights(self, zero_last: bool = False) -> None:
        lins = [m for m in self.mlp if isinstance(m, nn.Linear)]
        for lin in lins[:-1]:
            nn.init.kaiming_uniform_(lin.weight, a=0.0, mode="fan_in", nonlinearity="relu")
            nn.init.zeros_(lin.bias)
        last = lins[-1]
        if zero_last:
            nn.init.zeros_(last.weight)
        else:
            nn.init.xavier_uniform_(last.weight, gain=1.0)
        nn.init.zeros_(last.bias)

    def forward(self, x: torch.Tensor, mask: Optional[torch.Tensor] = None) -> torch.Tensor:
        B, H, W, _ = x.shape
        assert x.shape == (B, H, W, self.input_dim)
        assert mask is None or mask.shape == (B, H, W)
        rgb, res = x[..., :3], x[..., 3:4]
        if mask is None:
            y = self.mlp(x.reshape(-1, self.input_dim)).view(B, H, W, self.output_dim)
            return (1.0 - res) * rgb + res * y
        flat = x.reshape(-1, self.input_dim)
        m = mask.reshape(-1)
        out = torch.zeros(B * H * W, self.output_dim, device=x.device, dtype=x.dtype)
        if m.any():
            sel = flat[m]
            y = self.mlp(sel)
            r = sel[:, 3:4]
            out[m] = (1.0 - r) * sel[:, :3] + r * y
        return out.view(B, H, W, self.output_dim)


# ---------------------------------------------------------------------------
#  Per-pixel feature interpolation (multires.py:214-272)
# ---------------------------------------------------------------------------

class _MultiresTriangleColorFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rast, min_level, max_level, feat):
        B, H, W, _ = rast.shape
        out = torch.zeros((B, H, W, feat.shape[2]), dtype=torch.float32, device=rast.device)
        _core.multires_triangle_color(rast, min_level, max_level, feat, out)
        ctx.save_for_backward(rast)
        ctx.levels = (min_level, max_level)
        ctx.feat_shape = tuple(feat.shape)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (rast,) = ctx.saved_tensors
        lo, hi = ctx.levels
        grad_feat = torch.zeros(ctx.feat_shape, dtype=torch.float32, device=rast.device)
        _core.backward_multires_triangle_color(rast, lo, hi, grad_feat, grad_out.contiguous())
        return None, None, None, grad_feat


def multires_triangle_color(rast: torch.Tensor, level: int, feat: torch.Tensor) -> torch.Tensor:
    """Interpolate (T, S, C) features at one level per pixel: (B, H, W, C)."""
    B, H, W, _ = rast.shape
    _, S, _ = feat.shape
    dev = rast.device
    assert rast.shape == (B, H, W, 4) and rast.dtype == torch.float32 and rast.is_contiguous()
    assert feat.dim() == 3 and feat.dtype == torch.float32 and feat.is_contiguous()
    assert S == feats_at_level(level)
    assert rast.is_cuda and feat.device == dev
    return _MultiresTriangleColorFn.apply(rast, level, level, feat)


# ---------------------------------------------------------------------------
#  Cross-level accumulation (multires.py:279-339)
# ---------------------------------------------------------------------------

class _AccumulateToLevelFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, min_level, max_level, target_level, feat):
        T, _, Cd = feat.shape
        out = torch.empty(T, feats_at_level(target_level), Cd, dtype=torch.float32, device=feat.device)
        _core.accumulate_to_level_forward(min_level, max_level, target_level, feat, out)
        ctx.levels = (min_level, max_level, target_level)
        ctx.feat_shape = tuple(feat.shape)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        lo, hi, tl = ctx.levels
        grad_feat = torch.zeros(ctx.feat_shape, dtype=torch.float32, device=grad_out.device)
        _core.accumulate_to_level_backward(lo, hi, tl, grad_feat, grad_out.contiguous())
        return None, None, None, grad_feat


def accumulate_to_level(min_level: int, max_level: int, feat: torch.Tensor,
                        target_level: Optional[int] = None) -> torch.Tensor:
    """Evaluate levels [min_level, max_level] on the lattice of target_level
    (default max_level): (T, S_target, C)."""
    assert min_level >= 0
    assert feat.ndim == 3 and feat.dtype == torch.float32
    assert feat.is_contiguous() and feat.is_cuda
    if target_level is None:
        target_level = max_level
    return _AccumulateToLevelFn.apply(min_level, max_level, target_level, feat)

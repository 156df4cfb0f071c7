"""The training step of oracle/pipeline.py run with the reference's own CUDA
kernels (oracle/_ref, through oracle/ref.py) and torch on the GPU.

TEST INFRASTRUCTURE ONLY.  It composes, view after view, what the
reference's Python layer runs for one training view (examples/02_synthetic.py
:340-380 over python/diffsoup/rasterize.py and multires.py): the level
accumulation and its sigmoid (multires.cu:314-450), the fragment rasterizer
with the lattice opacity and a deterministic 0.5 threshold
(rasterize.cu:43-487, multires.cu:130-222), the feature lattice
(multires.cu:224-266), the SH2 view encoding (encoding.cu:56-118), the torch
ColorMLP with the residual blend and the MSE loss, and the adjoints (feature
lattice, edge gradients rasterize.cu:489-921, the opacity auxiliary gradient
:923-992 scaled by 1/(pixels*3), the accumulation adjoint), in the order and
with the arithmetic of oracle/pipeline.py's FP32 path.  Tests compare the
batched step with it at full size and time both.
"""

from __future__ import annotations

from typing import List, Tuple

import torch

from . import ref as oref


def _mlp_forward(x: torch.Tensor, mlp: List[Tuple[torch.Tensor, torch.Tensor]]) -> torch.Tensor:
    h = x
    for i, (W, b) in enumerate(mlp):
        h = h @ W.T + b
        h = torch.relu(h) if i < len(mlp) - 1 else torch.sigmoid(h)
    return h


def ref_train_step(R: oref.Ref, verts, tri, mvps, inv_mvps, hw, feat_src, alpha_src, mlp, targets, lo, hi,
                   feats_at_level, pos=None, alpha_rast=None):
    """One step over the views of `hw` (cuda tensors; view encoding SH2).
    pos [B,V,4] and alpha_rast [T,ST] replace the clip positions and the
    opacities the rasterizer tests (by default computed here) with a caller's,
    so that a comparison isolates the kernels from their inputs' last bits.
    Returns (loss, colours per view, grad_verts, grad_feat_src, grad_alpha_src,
    [(gW, gb)] per layer, ID buffers per view)."""
    dev = verts.device
    T = tri.shape[0]
    ST = feats_at_level(hi)
    N = float(sum(h * w for h, w in hw) * 3)
    a_acc = torch.sigmoid(R.accumulate_forward(lo, hi, hi, alpha_src[..., None].contiguous(), ST))[..., 0].contiguous()
    f_acc = torch.sigmoid(R.accumulate_forward(lo, hi, hi, feat_src, ST)).contiguous()
    if pos is None:
        vh = torch.cat([verts, torch.ones(verts.shape[0], 1, device=dev)], dim=1)
        pos = torch.einsum("bij,nj->bni", mvps, vh).contiguous()
    a_rast = a_acc if alpha_rast is None else alpha_rast
    mlp_t = [(W.detach().clone().requires_grad_(True), b.detach().clone().requires_grad_(True)) for W, b in mlp]
    grad_f_acc = torch.zeros_like(f_acc)
    grad_a_acc = torch.zeros_like(a_acc)
    grad_pos = torch.zeros_like(pos)
    loss = torch.zeros((), device=dev)
    colors, rasts = [], []
    for b, (H, W) in enumerate(hw):
        pb = pos[b:b + 1].contiguous()
        rast, _, _, _ = R.rasterize_alpha(H, W, pb, tri, hi, a_rast)
        rasts.append(rast[0])
        vdir = R.encode_sh2(rast, inv_mvps[b:b + 1].contiguous())
        feat = R.multires_color(rast, hi, hi, f_acc)
        xf = feat.detach().requires_grad_(True)
        x = torch.cat([xf, vdir], dim=-1)
        mask = rast[..., 3] > 0
        y = _mlp_forward(x, mlp_t)
        shaded = (1.0 - x[..., 3:4]) * x[..., :3] + x[..., 3:4] * y
        color = torch.where(mask[..., None], shaded, torch.ones_like(shaded))
        tgt = targets[b][None]
        lv = ((color - tgt) ** 2).sum() / N
        lv.backward()
        loss = loss + lv.detach()
        col = color.detach().contiguous()
        colors.append(col[0])
        gcol = (2.0 * (col - tgt) / N).contiguous()
        grad_f_acc += R.multires_color_backward(rast, hi, hi, f_acc.shape, xf.grad.contiguous())
        grad_pos[b:b + 1] += R.edge_grad(col, gcol, rast, pb, tri)
        gas, _, _, _, _ = R.opacity_aux(col, tgt.contiguous(), rast, pb, tri, hi, a_acc)
        grad_a_acc += gas / N
    gf_src = R.accumulate_backward(lo, hi, hi, feat_src.shape, (grad_f_acc * f_acc * (1.0 - f_acc)).contiguous())
    ga_src = R.accumulate_backward(lo, hi, hi, alpha_src[..., None].shape,
                                   (grad_a_acc * a_acc * (1.0 - a_acc))[..., None].contiguous())[..., 0]
    g_verts = torch.einsum("bri,bvr->vi", mvps[:, :, :3], grad_pos[..., :4])
    grad_mlp = [(W.grad, b.grad) for W, b in mlp_t]
    return loss, colors, g_verts, gf_src, ga_src, grad_mlp, rasts

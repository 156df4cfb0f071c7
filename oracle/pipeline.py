"""CPU oracle of one DiffSoup training step (examples/02_synthetic.py:354-385
with an MSE photometric loss), the checker of diffsoup_b200.step.TrainStep.

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU
baseline of bench.py.

The step is restated view by view from the oracle's kernel restatements
(oracle/oracle.cpp) and torch on the CPU for the shading MLP, whose reference
implementation is torch itself (python/diffsoup/multires.py:109-207):

  precision="f64": every continuous quantity in float64 (the FP64 oracle the
                   precision reports are measured against).  The discrete
                   decisions (which triangle covers which pixel) come from
                   the FP32 rasterization, exactly as in the reference.
  precision="f32": the reference's own FP32 arithmetic, multi-threaded (the
                   CPU baseline).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import cpu


@dataclass
class StepInputs:
    verts: np.ndarray            # [V,3] f32
    tri: np.ndarray              # [T,3] i32
    mvps: np.ndarray             # [B,4,4] f32
    inv_mvps: np.ndarray         # [B,4,4] f32
    hw: Sequence[Tuple[int, int]]
    feat_src: np.ndarray         # [T,S,C] f32 (pre-sigmoid)
    alpha_src: np.ndarray        # [T,S] f32 (pre-sigmoid)
    mlp: List[Tuple[np.ndarray, np.ndarray]]  # [(W[out,in], b[out])]
    targets: List[np.ndarray]    # per view [H,W,3] f32
    min_level: int
    max_level: int
    stochastic: bool = True
    seed: int = 0
    iteration: int = 0


@dataclass
class StepResult:
    loss: float
    rast: List[np.ndarray]
    color: List[np.ndarray]
    grad_verts: np.ndarray
    grad_feat_src: np.ndarray
    grad_alpha_src: np.ndarray
    grad_mlp: List[Tuple[np.ndarray, np.ndarray]]
    covered_fragments: int


def _mlp_forward(x: torch.Tensor, mlp: List[Tuple[torch.Tensor, torch.Tensor]]) -> torch.Tensor:
    h = x
    for i, (W, b) in enumerate(mlp):
        h = h @ W.T + b
        h = torch.relu(h) if i < len(mlp) - 1 else torch.sigmoid(h)
    return h


def train_step(inp: StepInputs, precision: str = "f64", rast_in: Optional[List[np.ndarray]] = None,
               pos32: Optional[np.ndarray] = None, alpha32: Optional[np.ndarray] = None) -> StepResult:
    """One forward+backward.  rast_in / pos32 / alpha32 let a caller supply the
    FP32 rasterization inputs of the device under test (they are recomputed
    here otherwise)."""
    f64 = precision == "f64"
    npdt = np.float64 if f64 else np.float32
    tdt = torch.float64 if f64 else torch.float32
    lo, hi = inp.min_level, inp.max_level
    T = inp.tri.shape[0]
    B = len(inp.hw)
    npix = sum(h * w for h, w in inp.hw)
    N = float(npix * 3)

    # opacity / features: sigmoid(accumulate_to_level(...)) (02_synthetic.py:355-356)
    if f64:
        a_acc = 1.0 / (1.0 + np.exp(-cpu.accumulate_forward(lo, hi, hi, inp.alpha_src[..., None], "f64")[..., 0]))
        f_acc = 1.0 / (1.0 + np.exp(-cpu.accumulate_forward(lo, hi, hi, inp.feat_src, "f64")))
    else:
        a_acc = cpu.accumulate_sigmoid_f32(lo, hi, hi, inp.alpha_src[..., None])[..., 0]
        f_acc = cpu.accumulate_sigmoid_f32(lo, hi, hi, inp.feat_src)
    if alpha32 is None:
        alpha32 = cpu.accumulate_sigmoid_f32(lo, hi, hi, inp.alpha_src[..., None])[..., 0]
    if pos32 is None:
        pos32 = cpu.project(inp.verts, inp.mvps)
    vh = np.concatenate([inp.verts.astype(np.float64), np.ones((inp.verts.shape[0], 1))], axis=1)
    pos = np.einsum("bij,nj->bni", inp.mvps.astype(np.float64), vh) if f64 else pos32

    mlp_t = [(torch.tensor(W, dtype=tdt, requires_grad=True), torch.tensor(b, dtype=tdt, requires_grad=True))
             for W, b in inp.mlp]
    grad_f_acc = np.zeros(f_acc.shape, np.float64)
    grad_a_acc = np.zeros(a_acc.shape, np.float64)
    grad_pos = np.zeros((B,) + pos.shape[1:], np.float64)
    loss = 0.0
    rasts, colors = [], []
    nfrag = 0
    for b, (H, W) in enumerate(inp.hw):
        if rast_in is not None:
            rast = rast_in[b]
        else:
            rast, nf = cpu.rasterize_alpha(H, W, pos32[b:b + 1], inp.tri, hi, alpha32, inp.stochastic, inp.seed,
                                           inp.iteration, view0=b)
            nfrag += nf
        rasts.append(rast)
        feat = cpu.multires_color(rast, hi, hi, f_acc, "f64" if f64 else "f32")
        vdir = cpu.encode_view(rast, inp.inv_mvps[b:b + 1], sh=False, precision="f64" if f64 else "f32")
        xf = torch.tensor(feat, dtype=tdt, requires_grad=True)
        x = torch.cat([xf, torch.tensor(vdir, dtype=tdt)], dim=-1)
        mask = torch.tensor(rast[..., 3] > 0)
        y = _mlp_forward(x, mlp_t)
        shaded = (1.0 - x[..., 3:4]) * x[..., :3] + x[..., 3:4] * y
        color = torch.where(mask[..., None], shaded, torch.ones_like(shaded))
        tgt = torch.tensor(inp.targets[b][None], dtype=tdt)
        lv = ((color - tgt) ** 2).sum() / N
        lv.backward()
        loss += float(lv.detach())
        col = color.detach()
        colors.append(col.numpy()[0].astype(np.float32) if not f64 else col.numpy()[0])
        gcol = (2.0 * (col - tgt) / N).numpy()
        grad_f_acc += cpu.multires_color_backward(rast, hi, hi, T, xf.grad.numpy())
        grad_pos[b:b + 1] += cpu.edge_grad(col.numpy(), gcol, rast, pos[b:b + 1], inp.tri,
                                           precision="f64" if f64 else "f32")
        grad_a_acc += cpu.opacity_aux(col.numpy(), tgt.numpy(), rast, pos32[b:b + 1], inp.tri, hi,
                                      a_acc, precision="f64" if f64 else "f32") / N
    gf_src = cpu.accumulate_backward(lo, hi, hi, T, grad_f_acc * f_acc * (1.0 - f_acc))
    ga_src = cpu.accumulate_backward(lo, hi, hi, T, (grad_a_acc * a_acc * (1.0 - a_acc))[..., None])[..., 0]
    g_verts = np.einsum("bri,bvr->vi", inp.mvps.astype(np.float64)[:, :, :3], grad_pos)
    grad_mlp = [(W.grad.numpy().astype(npdt), b.grad.numpy().astype(npdt)) for W, b in mlp_t]
    return StepResult(loss=loss, rast=rasts, color=colors, grad_verts=g_verts.astype(npdt),
                      grad_feat_src=gf_src.astype(npdt), grad_alpha_src=ga_src.astype(npdt), grad_mlp=grad_mlp,
                      covered_fragments=nfrag)

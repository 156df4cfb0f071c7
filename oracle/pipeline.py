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

  mlp_rounding="bf16" (with "f64"): the shading MLP with the BF16 operand
                   rounding of the fused step's BF16 mode and FP64 arithmetic
                   otherwise -- features gathered from the BF16-rounded
                   feature table, MLP inputs, weights, hidden activations and
                   the back-propagated pre-activation gradients rounded to
                   BF16 where the kernel feeds them to the tensor cores, biases
                   and their gradients unrounded (csrc/shade_reg.cuh,
                   csrc/shade.cuh).  It separates the kernel's own arithmetic
                   from the rounding of its BF16 operands.
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
    view_enc: str = "dir3"       # "dir3": 3-D view direction; "sh2": encode_view_dir_sh2 (9)


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


def bf16(a) -> np.ndarray:
    """Round to BF16 (nearest even, through FP32) and widen to float64."""
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float64)))
    return t.float().bfloat16().double().numpy()


def _mlp_bf16(feat: np.ndarray, enc: np.ndarray, mlp, tgt: np.ndarray, N: float):
    """Forward and backward of the blended ColorMLP over the covered pixels
    (rows of feat [n,C] and enc [n,E]) with the BF16 operand rounding of the
    fused step.  Returns colour [n,3], dL/dfeat [n,C], [(dW, db)] and the
    summed squared error."""
    C = feat.shape[1]
    xm = bf16(np.concatenate([feat, enc], axis=1))
    Wr = [bf16(W) for W, _ in mlp]
    acts = [xm]
    a = xm
    for (W, b), Wq in zip(mlp[:-1], Wr[:-1]):
        a = bf16(np.maximum(a @ Wq.T + b.astype(np.float64), 0.0))
        acts.append(a)
    logit = a @ Wr[-1].T + mlp[-1][1].astype(np.float64)
    s = 1.0 / (1.0 + np.exp(-logit))
    res = feat[:, 3:4]
    col = (1.0 - res) * feat[:, :3] + res * s
    diff = col - tgt
    gc = 2.0 * diff / N
    dfeat = np.zeros_like(feat)
    dfeat[:, :3] = (1.0 - res) * gc
    dfeat[:, 3] = ((s - feat[:, :3]) * gc).sum(axis=1)
    dz = res * gc * s * (1.0 - s)
    grads = [None] * len(mlp)
    grads[-1] = (bf16(dz).T @ acts[-1], dz.sum(axis=0))
    d = (bf16(dz) @ Wr[-1]) * (acts[-1] > 0)
    for l in range(len(mlp) - 2, -1, -1):
        dr = bf16(d)
        grads[l] = (dr.T @ acts[l], d.sum(axis=0))
        if l > 0:
            d = (dr @ Wr[l]) * (acts[l] > 0)
        else:
            dfeat += (dr @ Wr[0])[:, :C]
    return col, dfeat, grads, float((diff ** 2).sum())


def train_step(inp: StepInputs, precision: str = "f64", rast_in: Optional[List[np.ndarray]] = None,
               pos32: Optional[np.ndarray] = None, alpha32: Optional[np.ndarray] = None,
               mlp_rounding: str = "none") -> StepResult:
    """One forward+backward.  rast_in / pos32 / alpha32 let a caller supply the
    FP32 rasterization inputs of the device under test (they are recomputed
    here otherwise)."""
    f64 = precision == "f64"
    assert mlp_rounding in ("none", "bf16") and (mlp_rounding == "none" or f64)
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
        vdir = cpu.encode_view(rast, inp.inv_mvps[b:b + 1], sh=inp.view_enc == "sh2",
                               precision="f64" if f64 else "f32")
        if mlp_rounding == "bf16":
            feat = cpu.multires_color(rast, hi, hi, bf16(f_acc), "f64")
            m = rast[0, ..., 3] > 0
            tg = inp.targets[b].astype(np.float64)
            col = np.ones((H, W, 3))
            dfeat = np.zeros((H, W, feat.shape[-1]))
            cm, dfm, gm, sq = _mlp_bf16(feat[0][m], vdir[0][m], inp.mlp, tg[m], N)
            col[m] = cm
            dfeat[m] = dfm
            loss += (sq + float(((1.0 - tg[~m]) ** 2).sum())) / N
            for (W, bb), (gW, gb) in zip(mlp_t, gm):
                W.grad = (W.grad if W.grad is not None else 0) + torch.from_numpy(gW)
                bb.grad = (bb.grad if bb.grad is not None else 0) + torch.from_numpy(gb)
            colors.append(col)
            gcol = (2.0 * (col - tg) / N)[None]
            grad_f_acc += cpu.multires_color_backward(rast, hi, hi, T, dfeat[None])
            grad_pos[b:b + 1] += cpu.edge_grad(col[None], gcol, rast, pos[b:b + 1], inp.tri, precision="f64")
            grad_a_acc += cpu.opacity_aux(col[None], tg[None], rast, pos32[b:b + 1], inp.tri, hi, a_acc,
                                          precision="f64") / N
            continue
        feat = cpu.multires_color(rast, hi, hi, f_acc, "f64" if f64 else "f32")
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

"""The batched training step against the reference's own CUDA kernels, on
the reference's own shading model at full size, and the throughput of both.

The benchmark soup (15,000 triangles, 8 views of 800x800) shaded with the
reference's model (7 features + SH2 -> 16 -> 16 -> 3, examples/02_synthetic.py
:289-306) and a deterministic 0.5 opacity threshold: diffsoup_b200's step in
split-BF16 precision, one launch sequence for the 8 views, against
oracle/ref_step.py, which runs the reference's CUDA sources (compiled
unmodified into oracle/_ref) view after view with torch for the MLP, as the
reference's Python layer does.  Checked: the ID buffers bit for bit (except
the exact depth-key ties the reference breaks by scheduling order), the
loss, colours and every gradient group.  Printed: views per second of both
on this GPU (the step as a replayed CUDA graph; the reference path with its
own host synchronisations where it reads counts back).  Skipped where
oracle/_ref was not built.
"""

import numpy as np
import pytest
import torch

import bench
from diffsoup_b200 import scenes
from diffsoup_b200.step import TrainStep
from oracle import ref as oref
from oracle.ref_step import ref_train_step

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oref.available("fma"), reason="oracle/_ref not built")]
DEV = "cuda"


def rel(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def test_batched_step_vs_reference_kernels_reference_model_full_size():
    sc = scenes.make_scene(2, seed=0, shading="reference")
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=0)
    hw = [(v.height, v.width) for v in sc.views]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    verts, tri = t(sc.verts), t(sc.tri)
    mvp, inv = t(sc.mvps()), t(sc.inv_mvps())
    feat_src, alpha_src = t(sc.feat_src), t(sc.alpha_src[..., 0])
    targets = [t(x) for x in sc.targets]
    kw = dict(verts=verts, tri=tri, mvp=mvp, inv_mvp=inv, feat_src=feat_src, alpha_src=alpha_src,
              mlp_params=t(bench.mlp_flat(mlp)), target=torch.cat([x.reshape(-1, 3) for x in targets]))
    step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=False, device=DEV, precision="split", view_enc="sh2")
    step.fit_capacity(**kw)
    rast = torch.empty(step.num_pixels, 4, device=DEV)
    color = torch.empty(step.num_pixels, 3, device=DEV)
    loss = float(step.run(**kw, rast_out=rast, color_out=color).item())

    # the reference's kernels on the step's own clip positions and opacities (their last bits come from
    # the step's projection and sigmoid, which the reference computes in torch)
    R = oref.Ref("fma", sync=False)
    mlp_t = [(t(W), t(b)) for W, b in mlp]
    ST = scenes.feats_at_level(sc.max_level)
    pos = step.intermediate("pos").clone()
    alpha_rast = step.intermediate("alpha_acc")[:, :ST].contiguous().clone()
    args = (verts, tri, mvp, inv, hw, feat_src, alpha_src, mlp_t, targets, sc.min_level, sc.max_level,
            scenes.feats_at_level)
    rloss, rcols, rgv, rgf, rga, rgm, rrasts = ref_train_step(R, *args, pos=pos, alpha_rast=alpha_rast)
    torch.cuda.synchronize()

    # ID buffers
    ties = 0
    for b, (H, W) in enumerate(hw):
        o = step.pix_offsets[b]
        x = rast[o:o + H * W].reshape(H, W, 4).cpu().numpy()
        y = rrasts[b].cpu().numpy()
        diff = (x.view(np.uint32) != y.view(np.uint32)).any(-1)
        zx = (x[..., 2] + np.float32(2.0)).astype(np.float32).view(np.uint32)
        zy = (y[..., 2] + np.float32(2.0)).astype(np.float32).view(np.uint32)
        tie = diff & (zx == zy) & (x[..., 3] > 0) & (y[..., 3] > 0)
        assert not (diff & ~tie).any(), f"view {b}: {int((diff & ~tie).sum())} pixels differ beyond key ties"
        ties += int(tie.sum())
    assert ties <= 1e-4 * step.num_pixels

    sq = sum(float(((color[step.pix_offsets[b]:step.pix_offsets[b] + H * W] - rcols[b].reshape(-1, 3)) ** 2).sum())
             for b, (H, W) in enumerate(hw))
    flat_ref = torch.cat([torch.cat([W.reshape(-1), bb]) for W, bb in rgm])
    errs = {
        "loss": abs(loss - float(rloss)) / float(rloss),
        "image_rms": (sq / (step.num_pixels * 3)) ** 0.5,
        "grad_verts": rel(step.grad_verts, rgv),
        "grad_feat_src": rel(step.grad_feat_src, rgf),
        "grad_alpha_src": rel(step.grad_alpha_src, rga),
        "mlp": rel(step.grad_mlp, flat_ref),
    }

    # throughput: the step as a replayed graph, the reference path as its Python layer runs it
    g = step.capture(**kw)
    for _ in range(3):
        g.replay()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(20):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    ours = 20 * len(hw) / (e0.elapsed_time(e1) / 1000.0)
    ref_train_step(R, *args)  # the reference path on its own inputs (projection and opacities in torch)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(2):
        ref_train_step(R, *args)
    e1.record()
    torch.cuda.synchronize()
    theirs_vps = 2 * len(hw) / (e0.elapsed_time(e1) / 1000.0)
    print(f"reference model, 8 views of 800x800, 15,000 triangles: batched step (split-BF16) {ours:.1f} views/s, "
          f"the reference's CUDA kernels view by view {theirs_vps:.1f} views/s ({ours / theirs_vps:.1f}x); "
          f"{ties} key ties; vs the reference: " + ", ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v <= 1e-3, (k, v)

"""Parity of the training step at full size against the FP64 oracle.

  * the benchmark workload exactly as bench.py builds and tunes it: 15,000
    triangles on the noisy sphere shell, 8 views of 800x800, levels 0..2 x 8
    channels, MLP 11-16-3, stochastic opacity, the autotuned pixel block,
    tile-list capacity and fragment-record store.  All 8 ID buffers bit for
    bit against the oracle's rasterization; image RMS, loss and every
    gradient group within 1e-3 of the FP64 oracle in split precision, and of
    the FP64 oracle that rounds the same operands to BF16 in BF16 precision;
  * configurations 3 and 5 at their full triangle counts and resolutions on
    a subset of their views (the smallest and the largest view of the 64
    uneven ones of configuration 3; two 1920x1080 views of configuration 5,
    200,000 triangles, MLP 19-64-64-3): the same checks, split precision,
    except for the vertex gradients.  There the reference's own FP32
    estimator (the FP32 oracle, run on the same ID buffers) is itself about
    2e-3 from FP64 on these views: its case decisions (is the neighbour's
    centre inside the triangle, which edge does the pair cross) flip near
    edges between FP32 and FP64.  The step's vertex gradients must be within
    max(1e-3, 1.5 x that error) of FP64, and close to the FP32 oracle.
    Configuration 5 also in BF16 precision on the tcgen05 shading kernel
    (32,400 tiles of 128 pixels, two CTAs per SM), against the FP64 oracle
    that rounds the same MLP operands to BF16.

The oracle (oracle/pipeline.py) restates the reference's kernels
(rasterize.cu:653-992 for the edge and opacity estimators) and runs the
shading MLP in float64.
"""

import numpy as np
import pytest
import torch

import bench
from diffsoup_b200 import scenes
from diffsoup_b200.step import TrainStep
from oracle import cpu
from oracle import pipeline as P

pytestmark = pytest.mark.gpu
DEV = "cuda"


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _check(sc_like, hw, tri, mvps, step, kw, inp, seed, mlp_rounding="none", with_f32=False):
    rast = torch.empty(step.num_pixels, 4, device=DEV)
    color = torch.empty(step.num_pixels, 3, device=DEV)
    step.rng[1] = 0
    step.status.zero_()
    loss = float(step.run(**kw, rast_out=rast, color_out=color).item())
    torch.cuda.synchronize()
    assert not step.overflowed()
    pos = step.intermediate("pos").cpu().numpy()
    assert np.array_equal(pos.view(np.uint32), cpu.project(sc_like.verts, mvps).view(np.uint32))
    alpha32 = step.intermediate("alpha_acc").cpu().numpy()
    r = rast.cpu().numpy()
    rasts = []
    for b, (H, W) in enumerate(hw):
        o = step.pix_offsets[b]
        got = r[o:o + H * W].reshape(1, H, W, 4)
        want, _ = cpu.rasterize_alpha(H, W, pos[b:b + 1], tri, sc_like.max_level, alpha32, True, seed, 0, view0=b)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"view {b} ID buffer differs"
        rasts.append(got)
    ref = P.train_step(inp, "f64", rast_in=rasts, pos32=pos, alpha32=alpha32, mlp_rounding=mlp_rounding)
    c = color.cpu().numpy()
    sq = [(c[step.pix_offsets[b]:step.pix_offsets[b] + H * W] - ref.color[b].reshape(-1, 3)) ** 2
          for b, (H, W) in enumerate(hw)]
    errs = {
        "loss": abs(loss - ref.loss) / ref.loss,
        "image_rms": float(np.sqrt(np.concatenate(sq).mean())),
        "grad_verts": rel(step.grad_verts.cpu().numpy(), ref.grad_verts),
        "grad_feat_src": rel(step.grad_feat_src.cpu().numpy(), ref.grad_feat_src),
        "grad_alpha_src": rel(step.grad_alpha_src.cpu().numpy(), ref.grad_alpha_src),
        "mlp": rel(step.grad_mlp.cpu().numpy(),
                   np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in ref.grad_mlp])),
    }
    if not with_f32:
        return errs
    # the reference's FP32 arithmetic on the same ID buffers
    r32 = P.train_step(inp, "f32", rast_in=rasts, pos32=pos, alpha32=alpha32)
    return errs, {"f32_vs_f64": rel(r32.grad_verts, ref.grad_verts),
                  "step_vs_f32": rel(step.grad_verts.cpu().numpy(), r32.grad_verts)}


@pytest.mark.parametrize("precision", ["split", "bf16"])
def test_benchmark_workload_full_size(precision):
    sc, mlp, sets = bench.make_inputs(0)
    mvp, inv, tgt = sets[0]
    B = mvp.shape[0]
    hw = [(800, 800)] * B
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    kw = dict(verts=t(sc.verts), tri=t(sc.tri), mvp=t(mvp), inv_mvp=t(inv), feat_src=t(sc.feat_src),
              alpha_src=t(sc.alpha_src[..., 0]), mlp_params=t(bench.mlp_flat(mlp)), target=t(tgt))
    assert tgt.dtype == np.uint8  # the benchmark's 8-bit targets
    seed = 1234
    step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=True, seed=seed, device=DEV, precision=precision, target_u8=True)
    tuned = step.autotune(**kw)
    assert step.record_capacity > 0
    inp = P.StepInputs(verts=sc.verts, tri=sc.tri, mvps=mvp, inv_mvps=inv, hw=hw, feat_src=sc.feat_src,
                       alpha_src=sc.alpha_src[..., 0], mlp=mlp,
                       targets=list(bench.target_f32(tgt).reshape(B, 800, 800, 3)),
                       min_level=sc.min_level, max_level=sc.max_level, stochastic=True, seed=seed, iteration=0)
    errs = _check(sc, hw, sc.tri, mvp, step, kw, inp, seed, "none" if precision == "split" else "bf16")
    assert not step.record_fallback()
    print(f"benchmark workload ({precision}, block {tuned['block']}, list capacity {tuned['list_capacity']}, "
          f"{tuned['frag_records']:.3f} records/px) vs the {'FP64' if precision == 'split' else 'BF16-rounding FP64'}"
          " oracle: " + ", ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v <= 1e-3, (k, v)


@pytest.mark.parametrize("config,precision", [(3, "split"), (5, "split"), (5, "bf16")])
def test_full_size_subset_gradients(config, precision):
    full = scenes.make_scene(config, seed=0)
    sizes = [v.height * v.width for v in full.views]
    pick = sorted({int(np.argmin(sizes)), int(np.argmax(sizes))}) if config == 3 else [0, 5]
    views = [full.views[i] for i in pick]
    hw = [(v.height, v.width) for v in views]
    mvp = np.stack([v.mvp for v in views]).astype(np.float32)
    inv = np.stack([v.inv_mvp for v in views]).astype(np.float32)
    targets = [full.targets[i] for i in pick]
    mlp = scenes.mlp_weights(full.mlp_input_dim, 3, full.hidden_dim, full.n_layers, seed=0)
    flat = np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp]).astype(np.float32)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    kw = dict(verts=t(full.verts), tri=t(full.tri), mvp=t(mvp), inv_mvp=t(inv), feat_src=t(full.feat_src),
              alpha_src=t(full.alpha_src[..., 0]), mlp_params=t(flat),
              target=t(np.concatenate([x.reshape(-1, 3) for x in targets])))
    seed = 321
    step = TrainStep(full.T, full.verts.shape[0], hw, full.feat_dim, full.min_level, full.max_level,
                     full.hidden_dim, full.n_layers, stochastic=True, seed=seed, device=DEV, precision=precision)
    if precision == "bf16":
        assert step.tcgen05_shading()
        step.cfg.shade_mode = 1
    step.fit_capacity(**kw)
    inp = P.StepInputs(verts=full.verts, tri=full.tri, mvps=mvp, inv_mvps=inv, hw=hw, feat_src=full.feat_src,
                       alpha_src=full.alpha_src[..., 0], mlp=mlp, targets=targets, min_level=full.min_level,
                       max_level=full.max_level, stochastic=True, seed=seed, iteration=0)
    rounding = "bf16" if precision == "bf16" else "none"
    errs, ref32 = _check(full, hw, full.tri, mvp, step, kw, inp, seed, rounding, with_f32=True)
    assert int(step.status.item()) & 8 == 0  # no tensor-core stage timed out
    print(f"config{config}: views {pick} ({', '.join(f'{w}x{h}' for h, w in hw)}), {full.T} triangles, {precision} "
          f"precision vs {'BF16-rounding ' if precision == 'bf16' else ''}FP64 oracle: "
          + ", ".join(f"{k}={v:.2e}" for k, v in errs.items())
          + f"; vertex gradients of the FP32 oracle vs FP64 {ref32['f32_vs_f64']:.2e}, step vs FP32 oracle "
          f"{ref32['step_vs_f32']:.2e}")
    for k, v in errs.items():
        if k != "grad_verts":
            assert v <= 1e-3, (k, v)
    assert errs["grad_verts"] <= max(1e-3, 1.5 * ref32["f32_vs_f64"]), (errs["grad_verts"], ref32)
    if precision == "split":  # the FP32 oracle does not round the MLP operands to BF16
        assert ref32["step_vs_f32"] <= max(1e-3, 1.5 * ref32["f32_vs_f64"]), ref32

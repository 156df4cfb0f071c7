"""The batched training step against the FP64 oracle of the same step.

Discrete outputs (clip positions, ID buffer) must match the oracle bit for bit
given the step's own FP32 opacities.  Continuous outputs are compared with the
FP64 oracle: image RMS error <= 1e-3, loss to 1e-3 relative, and each
gradient group as a relative L2 error:

  * precision "split" (the benchmark's mode): every group <= 1e-3;
  * precision "bf16": against the plain FP64 oracle, vertex and opacity
    gradients <= 1e-3, feature and MLP gradients within BF16_INPUT_TOL (the
    rounding of the BF16 operands alone flips ReLU masks; the values are
    printed for the report); against the FP64 oracle that rounds the same
    operands to BF16 (pipeline.train_step(mlp_rounding="bf16")), every group
    <= 1e-3 -- the kernel's own arithmetic.
"""

import numpy as np
import pytest
import torch

from diffsoup_b200 import scenes
from diffsoup_b200.step import TrainStep, pack_mlp
from oracle import cpu
from oracle import pipeline as P

pytestmark = pytest.mark.gpu
DEV = "cuda"
BF16_INPUT_TOL = {"grad_verts": 1e-3, "grad_feat_src": 2e-2, "grad_alpha_src": 1e-3, "mlp": 1e-2}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _mlp_flat(mlp):
    return torch.from_numpy(np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp])).float()


def _setup(config, seed, precision="bf16", **kw):
    sc = scenes.make_scene(config, seed=seed, **kw)
    assert (sc.view_enc == "sh2") == (kw.get("shading") == "reference")
    hw = [(v.height, v.width) for v in sc.views]
    # per-view projection (views may have different aspect ratios)
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=seed)
    inp = P.StepInputs(verts=sc.verts, tri=sc.tri, mvps=sc.mvps(), inv_mvps=sc.inv_mvps(), hw=hw,
                       feat_src=sc.feat_src, alpha_src=sc.alpha_src[..., 0], mlp=mlp, targets=sc.targets,
                       min_level=sc.min_level, max_level=sc.max_level, stochastic=True, seed=4242, iteration=0,
                       view_enc=sc.view_enc)
    step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=True, seed=4242, precision=precision, view_enc=sc.view_enc)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    dev_inputs = dict(verts=t(sc.verts), tri=t(sc.tri), mvp=t(sc.mvps()), inv_mvp=t(sc.inv_mvps()),
                      feat_src=t(sc.feat_src), alpha_src=t(sc.alpha_src[..., 0]), mlp_params=_mlp_flat(mlp).to(DEV),
                      target=t(np.concatenate([x.reshape(-1, 3) for x in sc.targets])))
    return sc, hw, inp, step, dev_inputs


STEP_CASES = [
    (1, 0, dict(num_tris=1500, num_views=2, resolution=(96, 128))),
    (2, 1, dict(num_tris=3000, num_views=3, resolution=(160, 160))),
    (3, 2, dict(num_tris=2000, num_views=3)),
    (4, 3, dict(num_tris=800, num_views=2, resolution=(80, 96))),
    # the reference's own shading model: 7 features + SH2 -> 16 -> 16 -> 3
    (1, 8, dict(num_tris=1500, num_views=2, resolution=(96, 128), shading="reference")),
    (2, 9, dict(num_tris=3000, num_views=3, resolution=(160, 160), shading="reference")),
]
# precision "split": every MLP operand as bf16 hi + lo -- the image and every
# gradient group within 1e-3 of the FP64 oracle
SPLIT_TOL = {"grad_verts": 1e-3, "grad_feat_src": 1e-3, "grad_alpha_src": 1e-3, "mlp": 1e-3}


def _run_and_check_ids(sc, hw, step, d):
    """One step; positions and every view's ID buffer bit-exact against the
    oracle.  Returns (loss, colour, rasts, pos, alpha32)."""
    rast = torch.empty(step.num_pixels, 4, device=DEV)
    color = torch.empty(step.num_pixels, 3, device=DEV)
    loss = step.run(**d, rast_out=rast, color_out=color)
    torch.cuda.synchronize()
    assert not step.overflowed()
    pos = step.intermediate("pos").cpu().numpy()
    assert np.array_equal(pos.view(np.uint32), cpu.project(sc.verts, sc.mvps()).view(np.uint32))
    alpha32 = step.intermediate("alpha_acc").cpu().numpy()
    r = rast.cpu().numpy()
    rasts = []
    for b, (H, W) in enumerate(hw):
        o = step.pix_offsets[b]
        got = r[o:o + H * W].reshape(1, H, W, 4)
        want, _ = cpu.rasterize_alpha(H, W, pos[b:b + 1], sc.tri, sc.max_level, alpha32, True, 4242, 0, view0=b)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"view {b} ID buffer differs"
        rasts.append(got)
    return float(loss.item()), color.cpu().numpy(), rasts, pos, alpha32


def _errors(step, hw, loss, c, ref):
    sq = [(c[step.pix_offsets[b]:step.pix_offsets[b] + H * W] - ref.color[b].reshape(-1, 3)) ** 2
          for b, (H, W) in enumerate(hw)]
    return {
        "loss": abs(loss - ref.loss) / ref.loss,
        "image_rms": float(np.sqrt(np.concatenate(sq).mean())),
        "grad_verts": rel(step.grad_verts.cpu().numpy(), ref.grad_verts),
        "grad_feat_src": rel(step.grad_feat_src.cpu().numpy(), ref.grad_feat_src),
        "grad_alpha_src": rel(step.grad_alpha_src.cpu().numpy(), ref.grad_alpha_src),
        "mlp": rel(step.grad_mlp.cpu().numpy(), np.concatenate([np.concatenate([W.reshape(-1), b])
                                                               for W, b in ref.grad_mlp])),
    }


@pytest.mark.parametrize("config,seed,kw", STEP_CASES)
def test_bf16_step_matches_the_bf16_rounding_oracle(config, seed, kw):
    """BF16 mode against the FP64 oracle fed the same BF16-rounded operands
    (feature table, MLP inputs, weights, activations, back-propagated
    gradients): the kernel's own arithmetic, every group within 1e-3."""
    sc, hw, inp, step, d = _setup(config, seed, "bf16", **kw)
    loss, c, rasts, pos, alpha32 = _run_and_check_ids(sc, hw, step, d)
    ref = P.train_step(inp, "f64", rast_in=rasts, pos32=pos, alpha32=alpha32, mlp_rounding="bf16")
    errs = _errors(step, hw, loss, c, ref)
    print(f"config{config}{'-ref' if kw.get('shading') else ''} bf16 vs BF16-rounding FP64 oracle: "
          + ", ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    assert errs["image_rms"] <= 1e-3 and errs["loss"] <= 1e-3
    for k in ("grad_verts", "grad_feat_src", "grad_alpha_src", "mlp"):
        assert errs[k] <= 1e-3, (k, errs[k])


@pytest.mark.parametrize("precision", ["bf16", "split"])
@pytest.mark.parametrize("config,seed,kw", STEP_CASES)
def test_train_step_matches_fp64_oracle(config, seed, kw, precision):
    sc, hw, inp, step, d = _setup(config, seed, precision, **kw)
    loss, c, rasts, pos, alpha32 = _run_and_check_ids(sc, hw, step, d)
    want_alpha = cpu.accumulate_sigmoid_f32(sc.min_level, sc.max_level, sc.max_level, sc.alpha_src)[..., 0]
    np.testing.assert_allclose(alpha32, want_alpha, rtol=0, atol=3e-7)
    # continuous path against the FP64 oracle on the same ID buffer
    ref = P.train_step(inp, "f64", rast_in=rasts, pos32=pos, alpha32=alpha32)
    errs = _errors(step, hw, loss, c, ref)
    print(f"config{config}{'-ref' if kw.get('shading') else ''} {precision} errors vs FP64 oracle: "
          + ", ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    assert errs["image_rms"] <= 1e-3
    assert errs["loss"] <= 1e-3
    for k, tol in (SPLIT_TOL if precision == "split" else BF16_INPUT_TOL).items():
        assert errs[k] <= tol, (k, errs[k])


@pytest.mark.parametrize("config,seed,kw", [
    (4, 3, dict(num_tris=800, num_views=2, resolution=(80, 96))),
    (4, 13, dict(num_tris=1500, num_views=3, resolution=(120, 136))),
    (5, 0, dict(num_tris=4000, num_views=2, resolution=(90, 160))),
])
def test_tcgen05_shading_matches_the_bf16_rounding_oracle(config, seed, kw):
    """The tcgen05 kernel of the wide BF16 MLP (shade_mode 1: 128-pixel
    tiles, accumulators and the launch's weight gradients in tensor memory)
    against the FP64 oracle with the same BF16 operand rounding (every group
    within 1e-3) and against the mma.sync kernel of the same step."""
    sc, hw, inp, step, d = _setup(config, seed, "bf16", **kw)
    assert step.tcgen05_shading()
    step.cfg.shade_mode = 1
    loss, c, rasts, pos, alpha32 = _run_and_check_ids(sc, hw, step, d)
    ref = P.train_step(inp, "f64", rast_in=rasts, pos32=pos, alpha32=alpha32, mlp_rounding="bf16")
    errs = _errors(step, hw, loss, c, ref)
    print(f"config{config} tcgen05 shading vs BF16-rounding FP64 oracle: "
          + ", ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    assert not (int(step.status.item()) & 8)  # DS_STATUS_MMA_TIMEOUT
    for k, v in errs.items():
        assert v <= 1e-3, (k, v)
    got = {k: getattr(step, k).clone() for k in ("grad_feat_src", "grad_mlp", "grad_verts")}
    step.cfg.shade_mode = 0
    step.rng[1] = 0
    c0 = torch.empty(step.num_pixels, 3, device=DEV)
    step.run(**d, color_out=c0)
    torch.cuda.synchronize()
    assert float(np.abs(c0.cpu().numpy() - c).max()) < 1e-5
    for k, v in got.items():
        assert rel(v.cpu().numpy(), getattr(step, k).cpu().numpy()) < 1e-3, k


def test_eight_bit_targets_equal_their_fp32_quotients():
    """target_u8: 8-bit targets read as value / 255 give the step that the
    same quotients in fp32 give (colours bit for bit; loss and gradients up to
    the order of the floating-point atomics)."""
    sc, hw, inp, _, d = _setup(2, 4, "split", num_tris=2000, num_views=2, resolution=(96, 112))
    P_ = sum(h * w for h, w in hw)
    u8 = np.random.default_rng(5).integers(0, 256, size=(P_, 3), dtype=np.uint8)
    f32 = u8.astype(np.float32) / np.float32(255)
    outs = []
    for is_u8, tgt in ((False, f32), (True, u8)):
        step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                         sc.n_layers, stochastic=True, seed=4242, precision="split", target_u8=is_u8)
        color = torch.empty(step.num_pixels, 3, device=DEV)
        loss = float(step.run(**dict(d, target=torch.from_numpy(tgt).to(DEV)), color_out=color).item())
        torch.cuda.synchronize()
        outs.append((loss, color.cpu().numpy(), step.grad_verts.cpu().numpy(), step.grad_feat_src.cpu().numpy(),
                     step.grad_mlp.cpu().numpy()))
    (l0, c0, v0, f0, m0), (l1, c1, v1, f1, m1) = outs
    assert np.array_equal(c0.view(np.uint32), c1.view(np.uint32))
    assert abs(l0 - l1) <= 1e-6 * l0
    for a, b in ((v0, v1), (f0, f1), (m0, m1)):
        assert rel(b, a) < 1e-5
    with pytest.raises(ValueError):
        step.run(**dict(d, target=torch.from_numpy(f32).to(DEV)))  # fp32 target given to an 8-bit step


def test_train_step_graph_replay():
    sc, hw, inp, step, d = _setup(1, 5, num_tris=1000, num_views=2, resolution=(64, 64))
    step.run(**d)
    torch.cuda.synchronize()
    l0 = float(step.loss.item())
    it0 = int(step.rng[1].item())
    g = step.capture(**d)
    losses = []
    for _ in range(3):
        g.replay()
        torch.cuda.synchronize()
        losses.append(float(step.loss.item()))
    # the warm-up inside capture() advances the iteration once; capture itself runs nothing
    assert int(step.rng[1].item()) == it0 + 4
    assert all(np.isfinite(losses)) and abs(losses[0] - l0) / l0 < 0.05
    # a replay equals an eager step with the same RNG state
    step.rng[1] = 77
    g.replay()
    torch.cuda.synchronize()
    gv_graph = step.grad_verts.clone()
    step.rng[1] = 77
    step.run(**d)
    torch.cuda.synchronize()
    assert rel(step.grad_verts.cpu().numpy(), gv_graph.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("config,kw", [
    (2, dict(num_tris=3000, num_views=2, resolution=(128, 128))),
    (4, dict(num_tris=800, num_views=2, resolution=(80, 96))),
    (2, dict(num_tris=3000, num_views=2, resolution=(128, 128), shading="reference")),  # 7 channels, stride 8
])
def test_level_accumulation_matches_oracle(config, kw):
    """Opacity and feature accumulation + sigmoid (forward; the sums bit for
    bit, so only CUDA's and the host's expf may differ) and its adjoint
    (given the step's own gradients of the accumulated values) against the
    oracle's accumulate_to_level."""
    sc, hw, inp, step, d = _setup(config, 7, **kw)
    step.run(**d)
    torch.cuda.synchronize()
    lo, hi = sc.min_level, sc.max_level
    a = step.intermediate("alpha_acc").cpu().numpy()
    fp = step.intermediate("feat_acc").cpu().numpy()
    C = sc.feat_dim
    assert fp.shape[-1] == step.CP and not fp[..., C:].any()  # padding channels stay zero
    f = np.ascontiguousarray(fp[..., :C])
    want_a = cpu.accumulate_sigmoid_f32(lo, hi, hi, sc.alpha_src)[..., 0]
    want_f = cpu.accumulate_sigmoid_f32(lo, hi, hi, sc.feat_src)
    np.testing.assert_allclose(a, want_a, rtol=0, atol=3e-7)
    np.testing.assert_allclose(f, want_f, rtol=0, atol=3e-7)
    bf = step.intermediate("feat_bf16").float().cpu().numpy()[..., :C]
    assert np.array_equal(bf, torch.from_numpy(f).bfloat16().float().numpy())
    ga = step.intermediate("grad_alpha_acc").cpu().numpy().astype(np.float64)
    gf = step.intermediate("grad_feat_acc").cpu().numpy().astype(np.float64)[..., :C]
    want_ga = cpu.accumulate_backward(lo, hi, hi, sc.T, (ga * a * (1 - a))[..., None])[..., 0]
    want_gf = cpu.accumulate_backward(lo, hi, hi, sc.T, gf * f * (1 - f))
    assert rel(step.grad_alpha_src.cpu().numpy(), want_ga) < 1e-5
    assert rel(step.grad_feat_src.cpu().numpy(), want_gf) < 1e-5


@pytest.mark.parametrize("config", [1, 5])
def test_train_step_gradients_match_central_differences(config):
    """The split-precision step's feature and MLP gradients against FP64
    central differences (step 1e-4) of the oracle's loss over the step's own
    ID buffer: relative L2 over the sampled entries within 1e-3.  (BF16
    precision is pinned by the BF16-rounding oracle above: the rounding of its
    operands alone puts it 5e-3..2e-2 from the exact gradients.)"""
    from test_fd_gradients import fd_feature, fd_mlp, fd_scene, feature_entries

    sc, inp, _ = fd_scene(2, config)
    hw = list(inp.hw)
    step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=True, seed=inp.seed, precision="split")
    tol = SPLIT_TOL
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    mlp32 = [(W.astype(np.float32), b.astype(np.float32)) for W, b in inp.mlp]
    rast = torch.empty(step.num_pixels, 4, device=DEV)
    step.run(verts=t(sc.verts), tri=t(sc.tri), mvp=t(sc.mvps()), inv_mvp=t(sc.inv_mvps()),
             feat_src=t(sc.feat_src), alpha_src=t(sc.alpha_src[..., 0]), mlp_params=_mlp_flat(mlp32).to(DEV),
             target=t(np.concatenate([x.reshape(-1, 3) for x in sc.targets])), rast_out=rast)
    torch.cuda.synchronize()
    rasts = [rast.cpu().numpy()[step.pix_offsets[b]:step.pix_offsets[b] + h * w].reshape(1, h, w, 4)
             for b, (h, w) in enumerate(hw)]
    gf = step.grad_feat_src.cpu().numpy().astype(np.float64)
    gm = step.grad_mlp.cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(1)
    got, want = [], []
    for idx in feature_entries(gf, 12, rng):
        got.append(gf[idx])
        want.append(fd_feature(inp, rasts, idx))
    r = rel(got, want)
    print(f"config{config} split feature gradients vs FP64 central differences: {r:.2e}")
    assert r <= tol["grad_feat_src"], (r, got, want)
    # MLP parameters, packed as [W0, b0, (W, b)..., Wo, bo] like the step's grad_mlp
    got, want, off = [], [], 0
    for layer, (W, b) in enumerate(inp.mlp):
        for which, arr in ((0, W), (1, b)):
            g = gm[off:off + arr.size].reshape(arr.shape)
            for idx in feature_entries(g, 4, rng):
                got.append(g[idx])
                want.append(fd_mlp(inp, rasts, layer, which, idx))
            off += arr.size
    r = rel(got, want)
    print(f"config{config} split MLP gradients vs FP64 central differences: {r:.2e}")
    assert r <= tol["mlp"], (r, got, want)


def test_block_shapes_give_identical_results_and_autotune_picks_one():
    """The three pixel-block shapes of the rasterizer warps (8x4, 16x2, 4x8)
    give bit-identical ID buffers, the same loss and the same opacity gradients
    (which read the rasterizer's fragment records); the autotuner times them,
    keeps one and leaves the RNG iteration where it was."""
    sc, hw, inp, step, d = _setup(2, 6, num_tris=3000, num_views=2, resolution=(128, 160))
    outs = []
    for shape in (0, 1, 2):
        step.cfg.block_shape = shape
        step.rng[1] = 0
        rast = torch.empty(step.num_pixels, 4, device=DEV)
        loss = float(step.run(**d, rast_out=rast).item())
        torch.cuda.synchronize()
        outs.append((rast.cpu().numpy().view(np.uint32), loss, step.grad_alpha_src.clone()))
    for r, l, ga in outs[1:]:
        assert np.array_equal(r, outs[0][0])
        assert abs(l - outs[0][1]) <= 1e-6 * outs[0][1]
        assert rel(ga.cpu().numpy(), outs[0][2].cpu().numpy()) < 1e-5
    step.rng[1] = 3
    choice = step.autotune(**d, steps=2)
    assert choice["block_shape"] in (0, 1, 2)
    assert set(choice["ms_per_step"]) == {"8x4", "16x2", "4x8"}
    assert int(step.rng[1].item()) == 3
    assert step.autotune(**d, steps=2)["block_shape"] == choice["block_shape"]  # cached

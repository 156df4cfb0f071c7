"""The headless renderer (diffsoup_b200.viewer, csrc/render.cu) against the
oracle of the viewer's deferred shading.

  * the LUT opacity decode equals c / 255 in FP32, bit for bit;
  * the projection equals the oracle's, bit for bit;
  * the G-buffer (triangle ID buffer with barycentrics and depth) equals the
    oracle rasterizer with the deterministic threshold 0.5 on the LUT opacity,
    bit for bit, for every view of a batch;
  * the FP32 colour is within 2e-5 of the FP64 restatement of the shader on
    the same G-buffer, and the RGBA8 image is the GL_RGBA8 rounding of it;
  * a CUDA-graph replay with new MVPs equals an eager render of them;
  * an off-screen soup gives the background everywhere;
  * benchmark() writes the viewer's summary files and screenshots.
"""

import os

import numpy as np
import pytest
import torch

from diffsoup_b200 import scenes, viewer
from oracle import cpu
from oracle import viewer as oviewer

pytestmark = pytest.mark.gpu
RGB_TOL = 2e-5  # FP32 shader arithmetic against FP64, absolute, per channel


@pytest.fixture(scope="module")
def inputs():
    return scenes.make_viewer_inputs(2, seed=5, level=5, num_tris=3000, num_views=3, resolution=(96, 128))


@pytest.fixture(scope="module")
def renderer(inputs):
    (W1, b1), (W2, b2), (W3, b3) = inputs.mlp
    return viewer.Renderer(inputs.verts, inputs.faces, inputs.lut0, inputs.lut1, W1, b1, W2, b2, W3, b3,
                           level=inputs.level, background=(1.0, 0.9, 0.8))


def test_lut_opacity_decode(renderer, inputs):
    want = inputs.lut1.reshape(-1, 4)[:, 3].astype(np.float32) / np.float32(255)
    assert np.array_equal(renderer.alpha.cpu().numpy(), want)


def test_render_matches_oracle(renderer, inputs):
    H, W = inputs.height, inputs.width
    rgba, rgb, gbuf = renderer.render(inputs.mvps, H, W, rgb=True, gbuf=True)
    rgba, rgb, gbuf = rgba.cpu().numpy(), rgb.cpu().numpy(), gbuf.cpu().numpy()
    B = inputs.mvps.shape[0]
    f = renderer.frame(inputs.mvps, H, W)
    pos = f.workspace[:B * renderer.V * 16].view(torch.float32).view(B, renderer.V, 4).cpu().numpy()
    assert np.array_equal(pos.view(np.uint32), cpu.project(inputs.verts, inputs.mvps).view(np.uint32))
    S = renderer.S
    alpha = renderer.alpha.cpu().numpy()[:renderer.T * S].reshape(renderer.T, S)
    covered = 0
    for b in range(B):
        want, _ = cpu.rasterize_alpha(H, W, pos[b:b + 1], inputs.faces, inputs.level, alpha, False, view0=b)
        assert np.array_equal(gbuf[b:b + 1].view(np.uint32), want.view(np.uint32)), b
        covered += int((want[..., 3] > 0).sum())
    assert 0.05 * B * H * W < covered < B * H * W
    inv = np.linalg.inv(inputs.mvps.astype(np.float64)).astype(np.float32)
    mlp = [a for wb in inputs.mlp for a in wb]
    ref = oviewer.post_pass(gbuf, inv, inputs.level, inputs.lut0, inputs.lut1, mlp, background=(1.0, 0.9, 0.8))
    err = np.abs(rgb.astype(np.float64) - ref).max()
    assert err <= RGB_TOL, err
    assert np.array_equal(rgba, oviewer.to_rgba8(rgb))
    q = oviewer.to_rgba8(ref.astype(np.float32)).astype(np.int32)
    assert np.abs(rgba.astype(np.int32) - q).max() <= 1
    print(f"viewer render: max |rgb - fp64| = {err:.2e}, covered {covered / (B * H * W):.1%}")


def test_graph_replay_equals_eager(renderer, inputs):
    H, W = inputs.height, inputs.width
    f = renderer.frame(inputs.mvps[:1], H, W)
    g = f.capture()
    for b in range(inputs.mvps.shape[0]):
        f.set_views(torch.from_numpy(inputs.mvps[b:b + 1]))
        g.replay()
        torch.cuda.synchronize()
        got = f.rgba8.view(H, W, 4).clone()
        want = renderer.render(inputs.mvps[b:b + 1], H, W)[0]
        assert torch.equal(got, want), b
    del g


def test_offscreen_soup_is_background(inputs):
    (W1, b1), (W2, b2), (W3, b3) = inputs.mlp
    far = inputs.verts + np.float32(1e3)
    r = viewer.Renderer(far, inputs.faces, inputs.lut0, inputs.lut1, W1, b1, W2, b2, W3, b3, level=inputs.level)
    rgba, rgb = r.render(inputs.mvps[:1], 40, 56, rgb=True)
    assert bool((rgb == 1.0).all()) and bool((rgba == 255).all())


def test_lut_too_small_is_rejected(inputs):
    (W1, b1), (W2, b2), (W3, b3) = inputs.mlp
    with pytest.raises(RuntimeError, match="smaller than"):
        viewer.Renderer(inputs.verts, inputs.faces, inputs.lut0[:1, :8], inputs.lut1[:1, :8], W1, b1, W2, b2, W3,
                        b3, level=inputs.level)


def test_benchmark_writes_viewer_outputs(inputs, tmp_path):
    (W1, b1), (W2, b2), (W3, b3) = inputs.mlp
    col = np.ascontiguousarray(np.transpose(inputs.mvps, (0, 2, 1)))
    times = viewer.benchmark(inputs.verts, inputs.faces, inputs.lut0, inputs.lut1, W1, b1, W2, b2, W3, b3, col,
                             width=inputs.width, height=inputs.height, warmup=2, save_every=2,
                             output_dir=str(tmp_path), repeat=5, level=inputs.level)
    assert len(times) == inputs.mvps.shape[0] and all(t > 0 for t in times)
    summary = open(os.path.join(tmp_path, "benchmark_summary.txt")).read()
    assert summary.startswith("frames: 3") and "fps:" in summary
    assert len(open(os.path.join(tmp_path, "benchmark_frames.txt")).read().splitlines()) == 3
    shots = sorted(os.listdir(os.path.join(tmp_path, "screenshots")))
    assert shots == ["benchmark_00000.png", "benchmark_00002.png"]
    with open(os.path.join(tmp_path, "screenshots", shots[0]), "rb") as fh:
        assert fh.read(8) == b"\x89PNG\r\n\x1a\n"


def test_bin_list_overflow_stays_exact(renderer, inputs):
    H, W = inputs.height, inputs.width
    want = renderer.render(inputs.mvps, H, W)
    f = renderer._frame(inputs.mvps.shape[0], H, W)
    f.capacity = 4096  # far fewer (triangle, tile) entries than the views need
    f._alloc()
    got = renderer.render(inputs.mvps, H, W)
    assert torch.equal(got, want)
    assert f.capacity == 8192  # grown after the overflowing frame
    f.fit()
    assert not f.overflowed()


def test_batched_frames_equal_single_view_frames(renderer, inputs):
    """Views rendered in one call equal the same views rendered one by one
    (view table offsets, per-view inverse MVPs)."""
    H, W = inputs.height, inputs.width
    batch = renderer.render(inputs.mvps, H, W)
    for b in range(inputs.mvps.shape[0]):
        assert torch.equal(batch[b], renderer.render(inputs.mvps[b:b + 1], H, W)[0]), b


def test_post_pass_entry_point_equals_the_frame(renderer, inputs):
    """ds_render_deferred on a frame's G-buffer gives that frame's image."""
    from diffsoup_b200 import _core

    H, W = inputs.height, inputs.width
    f = renderer.frame(inputs.mvps, H, W)
    f.run(want_rgb=True)
    torch.cuda.synchronize()
    rgb = torch.empty_like(f.rgb)
    rgba = torch.empty_like(f.rgba8)
    bg = renderer.background
    _core.check(_core.lib.ds_render_deferred(f.B, _core.ptr(f.views), f.num_pixels, _core.ptr(f.gbuf), renderer.level,
                                             _core.ptr(renderer.lut0), _core.ptr(renderer.lut1),
                                             renderer.lut0.shape[0], _core.ptr(f.inv_mvp), _core.ptr(renderer.mlp),
                                             bg[0], bg[1], bg[2], _core.ptr(rgb), _core.ptr(rgba), _core.stream()))
    torch.cuda.synchronize()
    assert torch.equal(rgb, f.rgb) and torch.equal(rgba, f.rgba8)

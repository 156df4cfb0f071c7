"""GPU parity of every operator against the reference's outputs and the oracle.

Integer outputs, fragments, opacities and ID buffers must match bit for bit;
accumulated gradients (float atomics, order-dependent in the reference too)
within a relative L2 error of 1e-5.
"""

import numpy as np
import pytest
import torch

from oracle import cpu
from diffsoup_b200 import _core, scenes, tiles
import diffsoup_b200 as ds

pytestmark = pytest.mark.gpu
CASES = ["config1_small", "config2_small", "edge_cases"]
DEV = "cuda"


def T_(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(DEV)


def bits(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    if isinstance(b, torch.Tensor):
        b = b.detach().cpu().numpy()
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("case", CASES)
def test_fragment_ops_match_reference(golden, case):
    g = golden[case]
    H, W, lvl = int(g["H"]), int(g["W"]), int(g["level"])
    pos, tri = T_(g["pos"]), T_(g["tri"])
    B, T = pos.shape[0], tri.shape[0]
    rects = torch.empty((B * T, 4), dtype=torch.int32, device=DEV)
    prefix = torch.empty(B * T, dtype=torch.int32, device=DEV)
    n = _core.compute_triangle_rects(H, W, pos, tri, rects, prefix)
    assert n == int(g["fma_prefix"][-1])
    assert (rects.cpu().numpy() == g["fma_rects"]).all() and (prefix.cpu().numpy() == g["fma_prefix"]).all()
    from diffsoup_b200.rasterize import _compute_fragments, _depth_test

    fp, fa = _compute_fragments((H, W), pos, tri)
    # order preserving compaction == (view, triangle, y, x) order of the fixtures
    assert (fp.cpu().numpy() == g["fma_frag_pix"]).all()
    assert (bits(fa) == bits(g["fma_frag_attrs"])).all()
    alpha = torch.zeros(fp.shape[0], device=DEV)
    _core.multires_triangle_alpha(fa, lvl, lvl, T_(g["alpha_src"]), alpha)
    assert (bits(alpha) == bits(g["fma_frag_alpha"])).all()
    rast = _depth_test((H, W), pos, fp, fa, alpha, torch.full_like(alpha, 0.5))
    assert (bits(rast) == bits(g["fma_rast"])).all()
    # alpha backward against the oracle's double accumulation
    gfa = np.random.default_rng(0).normal(size=fp.shape[0]).astype(np.float32)
    ga = torch.zeros(T, g["alpha_src"].shape[1], device=DEV)
    _core.backward_multires_triangle_alpha(fa, lvl, lvl, ga, T_(gfa))
    assert rel(ga, cpu.multires_alpha_backward(g["fma_frag_attrs"], lvl, lvl, T, gfa)) < 1e-5


@pytest.mark.parametrize("case", CASES)
def test_pixel_ops_match_reference(golden, case):
    g = golden[case]
    lvl, lo, hi = int(g["level"]), int(g["lo"]), int(g["hi"])
    rast = T_(g["fma_rast"])
    B, H, W, _ = rast.shape
    T = g["tri"].shape[0]
    feat = T_(g["feat_lvl"])
    out = torch.zeros(B, H, W, feat.shape[2], device=DEV)
    _core.multires_triangle_color(rast, lvl, lvl, feat, out)
    assert (bits(out) == bits(g["fma_color_lvl"])).all()
    featml = T_(g["feat_ml"])
    outml = torch.zeros(B, H, W, featml.shape[2], device=DEV)
    _core.multires_triangle_color(rast, lo, hi, featml, outml)
    assert (bits(outml) == bits(g["fma_color_ml"])).all()
    gf = torch.zeros_like(feat)
    _core.backward_multires_triangle_color(rast, lvl, lvl, gf, T_(g["fma_grad_out"]))
    assert rel(gf, g["fma_grad_feat"]) < 1e-5
    enc = torch.zeros(B, H, W, 9, device=DEV)
    _core.encode_view_dir_sh2(rast, T_(g["inv_mvp"]), enc)
    np.testing.assert_allclose(enc.cpu().numpy(), g["fma_sh2"], atol=2e-6)
    gp = torch.zeros(T_(g["pos"]).shape, device=DEV)
    _core.backward_edge_grad(T_(g["fma_color"]), T_(g["fma_grad_color"]), rast, T_(g["pos"]), gp, T_(g["tri"]))
    assert rel(gp, g["fma_grad_pos"]) < 1e-5
    ST = scenes.feats_at_level(hi)
    acc = torch.empty(T, ST, featml.shape[2], device=DEV)
    _core.accumulate_to_level_forward(lo, hi, hi, featml, acc)
    assert (bits(acc) == bits(g["fma_acc"])).all()
    accg = torch.zeros_like(featml)
    _core.accumulate_to_level_backward(lo, hi, hi, accg, T_(g["fma_acc_grad_out"]))
    assert rel(accg, g["fma_acc_grad"]) < 1e-5


@pytest.mark.parametrize("case", CASES)
def test_aux_fragment_kernel_matches_reference(golden, case):
    g = golden[case]
    H, W, lvl = int(g["H"]), int(g["W"]), int(g["level"])
    from diffsoup_b200.rasterize import _compute_fragments

    fp, fa = _compute_fragments((H, W), T_(g["pos"]), T_(g["tri"]))
    alpha = torch.zeros(fp.shape[0], device=DEV)
    _core.multires_triangle_alpha(fa, lvl, lvl, T_(g["alpha_src"]), alpha)
    gfa = torch.zeros_like(alpha)
    _core.backward_opacity_aux_loss(T_(g["fma_color"]), T_(g["fma_target"]), T_(g["fma_rast"]), fp, fa, alpha, gfa)
    assert rel(gfa, g["fma_aux_grad_frag"]) < 1e-5


@pytest.mark.parametrize("case", CASES)
def test_tiled_rasterizer_matches_reference(golden, case):
    g = golden[case]
    H, W, lvl = int(g["H"]), int(g["W"]), int(g["level"])
    alpha = T_(g["alpha_src"]).unsqueeze(-1).contiguous()
    rast = ds.rasterize_multires_triangle_alpha((H, W), T_(g["pos"]), T_(g["tri"]), lvl, alpha, stochastic=False)
    assert (bits(rast) == bits(g["fma_rast"])).all()


def _scene_inputs(config, seed, **kw):
    sc = scenes.make_scene(config, seed=seed, with_targets=False, **kw)
    lvl = sc.max_level
    S = scenes.feats_at_level(lvl)
    alpha = (1.0 / (1.0 + np.exp(-sc.alpha_src[:, :S, 0]))).astype(np.float32)
    return sc, lvl, alpha


@pytest.mark.parametrize("config,seed,kw", [
    (1, 0, {}),
    (1, 1, dict(num_views=3, resolution=(97, 131))),
    (2, 0, dict(num_views=2, resolution=(800, 800))),
    (3, 0, dict(num_tris=6000, num_views=2, resolution=(300, 400))),
])
def test_tiled_rasterizer_matches_oracle(config, seed, kw):
    sc, lvl, alpha = _scene_inputs(config, seed, **kw)
    H, W = sc.uniform_resolution
    pos = sc.clip_positions()
    rast = ds.rasterize_multires_triangle_alpha((H, W), T_(pos), T_(sc.tri), lvl, T_(alpha[..., None]),
                                                stochastic=False)
    ref, nf = cpu.rasterize_alpha(H, W, pos, sc.tri, lvl, alpha, stochastic=False)
    assert nf > 0
    assert (bits(rast) == bits(ref)).all()
    # stochastic threshold with an explicit (seed, iteration)
    bins = tiles.bin_views(T_(pos), T_(sc.tri), [(H, W)] * pos.shape[0])
    rs = torch.empty_like(rast)
    rng = torch.tensor([987654321, 3], dtype=torch.int64, device=DEV)
    tiles.rasterize(bins, lvl, T_(alpha), rs, thr_mode=1, rng=rng)
    ref_s, _ = cpu.rasterize_alpha(H, W, pos, sc.tri, lvl, alpha, stochastic=True, seed=987654321, iteration=3)
    assert (bits(rs) == bits(ref_s)).all()


@pytest.mark.parametrize("hw", [
    [(1000, 1000)],            # 3,969 tiles: scanned in one launch, the last busy thread holds one count
    [(1024, 1024)],            # 4,096 tiles: one launch, 4 counts in every thread
    [(1024, 1024), (16, 16)],  # 4,097 tiles: the three-launch scan
])
def test_tile_count_scans_bin_alike(hw):
    """Both scans of the per-tile counts (one launch up to 4,096 tiles, three
    launches above) give the tile lists of view 0 its oracle ID buffer."""
    sc, lvl, alpha = _scene_inputs(1, 4)
    pos = np.repeat(sc.clip_positions()[:1], len(hw), axis=0)
    bins = tiles.bin_views(T_(pos), T_(sc.tri), hw, reuse=False)
    assert bins.num_tiles == sum(((h + 15) // 16) * ((w + 15) // 16) for h, w in hw)
    rast = torch.empty(bins.num_pixels, 4, device=DEV)
    tiles.rasterize(bins, lvl, T_(alpha), rast, thr_mode=0, thr_const=0.5)
    H, W = hw[0]
    ref, nf = cpu.rasterize_alpha(H, W, pos[:1], sc.tri, lvl, alpha, stochastic=False)
    assert nf > 0
    got = rast.cpu().numpy()[: H * W].reshape(1, H, W, 4)
    assert (bits(got) == bits(ref)).all()


def test_tiled_rasterizer_uneven_views_and_overflow():
    sc, lvl, alpha = _scene_inputs(3, 1, num_tris=3000, num_views=4)
    hw = [(v.height, v.width) for v in sc.views]
    assert len(set(hw)) > 1
    pos = sc.clip_positions().copy()
    # per-view projection with each view's own aspect: recompute clip positions
    vh = np.concatenate([sc.verts, np.ones_like(sc.verts[:, :1])], axis=1)
    pos = np.stack([vh @ v.mvp.T for v in sc.views]).astype(np.float32)
    posd, trid = T_(pos), T_(sc.tri)
    for cap_override in (None, 512):
        if cap_override is not None:
            tiles._capacity.clear()
            tiles._pending_status.clear()
            orig = tiles._capacity_for
            tiles._capacity_for = lambda dev, B, T: cap_override
        try:
            bins = tiles.bin_views(posd, trid, hw, reuse=False)
            rast = torch.empty(bins.num_pixels, 4, device=DEV)
            tiles.rasterize(bins, lvl, T_(alpha), rast, thr_mode=0, thr_const=0.5)
            torch.cuda.synchronize()
            if cap_override is not None:
                assert int(bins.status.item()) & tiles.DS_STATUS_LIST_OVERFLOW
        finally:
            if cap_override is not None:
                tiles._capacity_for = orig
        r = rast.cpu().numpy()
        for b, (h, w) in enumerate(hw):
            ref, _ = cpu.rasterize_alpha(h, w, pos[b:b + 1], sc.tri, lvl, alpha, stochastic=False)
            got = r[bins.pix_offsets[b]: bins.pix_offsets[b] + h * w].reshape(1, h, w, 4)
            assert (bits(got) == bits(ref)).all(), (cap_override, b)


def test_tiled_rasterizer_adversarial_edges():
    """Edges through pixel centres, shared edges, slivers, vertices at pixel
    centres with varied w and huge triangles: the block-level rejection and
    the per-pixel test must keep every fragment the reference keeps."""
    H, W = 64, 96
    rng = np.random.default_rng(17)
    cx = lambda i: -1.0 + (2.0 * i + 1.0) / W  # noqa: E731
    cy = lambda j: -1.0 + (2.0 * j + 1.0) / H  # noqa: E731
    tris = []
    for _ in range(300):  # vertices on pixel centres, random depth and w
        ij = rng.integers(0, [W, H], size=(3, 2))
        w = rng.uniform(0.3, 3.0, size=3)
        z = rng.uniform(-0.9, 0.9, size=3)
        tris.append([[cx(i) * wk, cy(j) * wk, zk * wk, wk] for (i, j), wk, zk in zip(ij, w, z)])
    for _ in range(100):  # slivers along a line through pixel centres
        i0, j0 = rng.integers(0, [W, H])
        di, dj = rng.integers(-20, 21, size=2)
        e = rng.uniform(-1e-6, 1e-6)
        tris.append([[cx(i0), cy(j0), 0.1, 1.0], [cx(i0 + di), cy(j0 + dj), 0.2, 1.0],
                     [cx(i0 + di) + e, cy(j0 + dj) - e, 0.3, 1.0]])
    for _ in range(50):  # pairs sharing an edge through pixel centres
        a, b, c, d = (rng.integers(0, [W, H], size=2) for _ in range(4))
        z = float(rng.uniform(-0.5, 0.5))
        pa, pb = [cx(a[0]), cy(a[1]), z, 1.0], [cx(b[0]), cy(b[1]), z, 1.0]
        tris.append([pa, pb, [cx(c[0]), cy(c[1]), z, 1.0]])
        tris.append([pb, pa, [cx(d[0]), cy(d[1]), z, 1.0]])
    for _ in range(20):  # huge triangles, far vertices
        v = rng.uniform(-50.0, 50.0, size=(3, 2))
        w = rng.uniform(0.05, 2.0, size=3)
        tris.append([[v[k, 0], v[k, 1], rng.uniform(-0.5, 0.5) * w[k], w[k]] for k in range(3)])
    pos = np.asarray(tris, np.float32).reshape(1, -1, 4)
    T = pos.shape[1] // 3
    tri = np.arange(3 * T, dtype=np.int32).reshape(T, 3)
    alpha = np.ones((T, 3), np.float32)
    rast = ds.rasterize_multires_triangle_alpha((H, W), T_(pos), T_(tri), 0, T_(alpha[..., None]), stochastic=False)
    ref, nf = cpu.rasterize_alpha(H, W, pos, tri, 0, alpha, stochastic=False)
    assert nf > 0
    assert (bits(rast) == bits(ref)).all()


def test_tiled_empty_and_culled():
    H, W = 40, 56
    tri = torch.zeros((0, 3), dtype=torch.int32, device=DEV)
    pos = torch.zeros((2, 0, 4), device=DEV)
    alpha = torch.zeros((0, 3, 1), device=DEV)
    rast = ds.rasterize_multires_triangle_alpha((H, W), pos, tri, 0, alpha, stochastic=False)
    assert rast.shape == (2, H, W, 4) and float(rast.abs().sum()) == 0.0
    # every triangle behind the camera or off screen
    p = torch.tensor([[[-0.2, -0.2, 0.5, -1.0], [0.3, -0.1, 0.5, -1.0], [0.0, 0.3, 0.5, -1.0],
                       [2.0, 2.0, 0.0, 1.0], [3.0, 2.0, 0.0, 1.0], [2.5, 3.0, 0.0, 1.0]]], device=DEV)
    t = torch.arange(6, dtype=torch.int32, device=DEV).view(2, 3)
    a = torch.ones((2, 3, 1), device=DEV)
    rast = ds.rasterize_multires_triangle_alpha((H, W), p, t, 0, a, stochastic=True)
    assert float(rast.abs().sum()) == 0.0


@pytest.mark.parametrize("config,seed,kw", [(1, 2, {}), (2, 1, dict(num_views=2, resolution=(200, 200)))])
def test_tiled_opacity_aux_matches_oracle(config, seed, kw):
    sc, lvl, alpha = _scene_inputs(config, seed, **kw)
    H, W = sc.uniform_resolution
    pos = sc.clip_positions()
    B = pos.shape[0]
    ref_rast, _ = cpu.rasterize_alpha(H, W, pos, sc.tri, lvl, alpha, stochastic=True, seed=5, iteration=1)
    rng = np.random.default_rng(seed)
    color = rng.uniform(0, 1, size=(B, H, W, 3)).astype(np.float32)
    target = rng.uniform(0, 1, size=(B, H, W, 3)).astype(np.float32)
    a3 = T_(alpha[..., None]).requires_grad_(True)
    aux = ds.opacity_aux_loss(T_(color), T_(target), T_(ref_rast), T_(pos), T_(sc.tri), lvl, a3)
    assert float(aux.item()) == 0.0
    aux.backward()
    want = cpu.opacity_aux(color, target, ref_rast, pos, sc.tri, lvl, alpha, precision="f32") / color.size
    assert rel(a3.grad[..., 0], want) < 1e-5


def test_autograd_wrappers_match_oracle():
    sc, lvl, alpha = _scene_inputs(1, 4, num_views=2, resolution=(64, 80))
    H, W = sc.uniform_resolution
    pos = sc.clip_positions()
    rast, _ = cpu.rasterize_alpha(H, W, pos, sc.tri, lvl, alpha, stochastic=False)
    S = scenes.feats_at_level(lvl)
    feat = np.random.default_rng(1).uniform(0, 1, size=(sc.T, S, 8)).astype(np.float32)
    fd = T_(feat).requires_grad_(True)
    out = ds.multires_triangle_color(T_(rast), lvl, fd)
    go = np.random.default_rng(2).normal(size=out.shape).astype(np.float32)
    out.backward(T_(go))
    np.testing.assert_array_equal(bits(out), bits(cpu.multires_color(rast, lvl, lvl, feat, precision="f32")))
    assert rel(fd.grad, cpu.multires_color_backward(rast, lvl, lvl, sc.T, go)) < 1e-5
    # edge_grad: identity forward, pos gradient in backward
    color = out.detach()[..., :3].contiguous()
    pd = T_(pos).requires_grad_(True)
    c2 = ds.edge_grad(color, T_(rast), pd, T_(sc.tri))
    gc = np.random.default_rng(3).normal(size=c2.shape).astype(np.float32) * 1e-3
    c2.backward(T_(gc))
    want = cpu.edge_grad(color.cpu().numpy(), gc, rast, pos, sc.tri, precision="f32")
    assert rel(pd.grad, want) < 1e-5
    # accumulate_to_level over levels 0..2
    src = np.random.default_rng(4).normal(size=(sc.T, sc.S, 8)).astype(np.float32)
    sd = T_(src).requires_grad_(True)
    acc = ds.accumulate_to_level(0, 2, sd)
    np.testing.assert_array_equal(bits(acc), bits(cpu.accumulate_forward(0, 2, 2, src, precision="f32")))
    ga = np.random.default_rng(5).normal(size=acc.shape).astype(np.float32)
    acc.backward(T_(ga))
    assert rel(sd.grad, cpu.accumulate_backward(0, 2, 2, sc.T, ga)) < 1e-5
    # view direction encodings
    inv = sc.inv_mvps()
    sh = ds.encode_view_dir_sh2(T_(rast), T_(inv))
    np.testing.assert_allclose(sh.cpu().numpy(), cpu.encode_view(rast, inv, sh=True), atol=2e-6)
    d3 = ds.encode_view_dir(T_(rast), T_(inv))
    np.testing.assert_allclose(d3.cpu().numpy(), cpu.encode_view(rast, inv, sh=False), atol=2e-6)


def test_shape_errors_raise():
    rast = torch.zeros(1, 4, 4, 4, device=DEV)
    feat = torch.zeros(5, 7, 3, device=DEV)
    with pytest.raises(RuntimeError, match="Invalid feature size"):
        _core.multires_triangle_color(rast, 1, 1, feat, torch.zeros(1, 4, 4, 3, device=DEV))

"""Synthetic workloads: seeded, with the benchmark configurations' shapes."""

import numpy as np

from diffsoup_b200 import scenes


def test_config_shapes():
    s = scenes.make_scene(2, seed=0, with_targets=False)
    assert s.T == 15000 and s.verts.shape == (45000, 3)
    assert len(s.views) == 8 and s.uniform_resolution == (800, 800)
    assert s.S == 24 and s.feat_src.shape == (15000, 24, 8) and s.alpha_src.shape == (15000, 24, 1)
    assert s.mlp_input_dim == 11 and s.hidden_dim == 16 and s.n_layers == 1
    s1 = scenes.make_scene(1, seed=0)
    assert s1.T == 5000 and s1.uniform_resolution == (256, 256) and len(s1.targets) == 1
    s4 = scenes.make_scene(4, seed=0, with_targets=False)
    assert s4.S == 69 and s4.feat_dim == 16 and s4.mlp_input_dim == 19 and s4.hidden_dim == 64
    s3 = scenes.make_scene(3, seed=0, num_views=64, with_targets=False)
    assert s3.T == 60000 and len(s3.views) == 64 and s3.uniform_resolution is None
    widths = [v.width for v in s3.views]
    assert min(widths) >= 400 and max(widths) <= 1200


def test_seeded_and_projected():
    a = scenes.make_scene(1, seed=3, num_tris=100, with_targets=False)
    b = scenes.make_scene(1, seed=3, num_tris=100, with_targets=False)
    c = scenes.make_scene(1, seed=4, num_tris=100, with_targets=False)
    assert np.array_equal(a.verts, b.verts) and not np.array_equal(a.verts, c.verts)
    clip = a.clip_positions()
    assert clip.shape == (1, 300, 4)
    # the camera looks at the origin: the origin projects to the image centre
    o = a.mvps()[0] @ np.array([0, 0, 0, 1.0], np.float32)
    assert abs(o[0] / o[3]) < 1e-5 and abs(o[1] / o[3]) < 1e-5 and o[3] > 0
    # inverse MVP is the inverse
    np.testing.assert_allclose(a.mvps()[0] @ a.inv_mvps()[0], np.eye(4), atol=1e-4)


def test_mlp_init_matches_reference_distributions():
    ws = scenes.mlp_weights(11, 3, 16, 1, seed=0)
    assert [w.shape for w, _ in ws] == [(16, 11), (3, 16)]
    assert np.abs(ws[0][0]).max() <= np.sqrt(6.0 / 11) + 1e-6
    assert np.abs(ws[1][0]).max() <= np.sqrt(6.0 / 19) + 1e-6

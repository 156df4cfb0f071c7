"""Visibility counting (count_triangle_ids, count_visible_triangles) against
the oracle's rasterization with the deterministic threshold: exact counts."""

import numpy as np
import pytest
import torch

import diffsoup_b200 as ds
from diffsoup_b200 import scenes
from oracle import cpu

pytestmark = pytest.mark.gpu


def test_count_visible_triangles_matches_oracle():
    sc = scenes.make_scene(2, seed=4, num_tris=3000, num_views=5, resolution=(96, 128))
    H, W = 96, 128
    alpha = cpu.accumulate_sigmoid_f32(sc.min_level, sc.max_level, sc.max_level, sc.alpha_src)
    pos = cpu.project(sc.verts, sc.mvps())
    want = np.zeros(sc.T, np.int64)
    for b in range(len(sc.views)):
        rast, _ = cpu.rasterize_alpha(H, W, pos[b:b + 1], sc.tri, sc.max_level, alpha[..., 0], False)
        ids = rast[..., 3].astype(np.int64).ravel()
        want += np.bincount(ids[ids > 0] - 1, minlength=sc.T)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got = ds.visibility.count_visible_triangles((H, W), t(sc.mvps()), t(sc.verts), t(sc.tri), sc.max_level,
                                                t(alpha), batch_size=2)
    assert got.dtype == torch.int64
    assert np.array_equal(got.cpu().numpy(), want)
    assert int(want.sum()) > 0


def test_count_triangle_ids_matches_bincount():
    g = torch.Generator().manual_seed(0)
    ids = torch.randint(0, 50, (3, 40, 70), generator=g)
    ids[:, :5] = 7  # runs of equal ids inside a warp
    rast = torch.zeros(3, 40, 70, 4)
    rast[..., 3] = ids.float()
    got = ds.count_triangle_ids(rast.cuda(), 49)
    want = torch.bincount(ids[ids > 0] - 1, minlength=49)
    assert torch.equal(got.cpu(), want)
    with pytest.raises(AssertionError):
        ds.count_triangle_ids(rast.cuda(), 10)

"""The GPU soup subdivision (csrc/remesh.cu through diffsoup_b200.remesh)
against its oracle.

* bit for bit the arrays of the restatement (oracle/remesh.py, pinned to the
  reference's remeshers on CPU), which numbers the output as the GPU does:
  vertices, faces, face mapping and flags, world and screen-space lengths,
  masked faces and corners outside the NDC cube;
* at the benchmark soup's size (15,000 faces, one 800x800 view), the same
  triangles per input face as the reference's own compiled remesher;
* the resampling step of training (several views in turn) keeps the face
  mapping consistent with the faces' geometry.
"""

import numpy as np
import pytest
import torch

from diffsoup_b200 import remesh, scenes
from oracle import remesh as R

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _np(q):
    return tuple(x.cpu().numpy() for x in q)


def _soup(T, seed, spread=0.15):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, (T, 3))
    v = (c[:, None, :] + rng.normal(0, spread, (T, 3, 3))).reshape(-1, 3).astype(np.float32)
    return v, np.arange(3 * T, dtype=np.int32).reshape(T, 3)


def _equal(got, want):
    for g, w in zip(got, want):
        assert g.shape == w.shape
        assert np.array_equal(g.view(np.uint32) if g.dtype == np.float32 else g, w.view(np.uint32)
                              if w.dtype == np.float32 else w)


@pytest.mark.parametrize("tau", [0.05, 0.2])
def test_world_split_equals_oracle(tau):
    v, f = _soup(200, seed=7)
    got = _np(remesh.split_triangle_soup_until(torch.from_numpy(v).to(DEV), torch.from_numpy(f).to(DEV), tau))
    _equal(got, R.restated_split(v, f, tau))


def test_clip_split_equals_oracle():
    sc = scenes.make_scene(2, seed=3, num_tris=300, num_views=1, resolution=(600, 800), with_targets=False)
    rng = np.random.default_rng(3)
    valid = (rng.random(sc.T) < 0.7).astype(np.int32)
    verts = sc.verts.copy()
    verts[:40] *= 6.0
    mvp = sc.mvps()[0]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    got = _np(remesh.split_triangle_soup_clip_until((600, 800), t(mvp), t(verts), t(sc.tri), t(valid), 0.01))
    want = R.restated_split(verts, sc.tri, 0.01, mvp=mvp, valid=valid, aspect_wh=800 / 600)
    assert want[1].shape[0] > sc.T
    _equal(got, want)


@pytest.mark.skipif(not R.reference_available(), reason="oracle/_ref/libremesh_ref.so not built")
def test_benchmark_soup_matches_reference():
    sc = scenes.make_scene(2, seed=0, num_views=1, with_targets=False)
    mvp = sc.mvps()[0]
    valid = np.ones(sc.T, np.int32)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    got = _np(remesh.split_triangle_soup_clip_until((800, 800), t(mvp), t(sc.verts), t(sc.tri), t(valid), 0.004))
    ref = R.reference_split(sc.verts, sc.tri, -1, 0.004, mvp=mvp, valid=valid, aspect_wh=1.0)
    assert got[1].shape == ref[1].shape and ref[1].shape[0] > 2 * sc.T
    assert R.families(*got) == R.families(*ref)
    print(f"clip split of {sc.T} faces: {ref[1].shape[0] - sc.T} splits, same triangles as the reference")


def test_resampling_step_keeps_the_mapping():
    sc = scenes.make_scene(2, seed=2, num_tris=2000, num_views=4, resolution=(200, 200), with_targets=False)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    torch.manual_seed(0)
    S = 15  # level 2
    alpha = torch.full((sc.T, S), 0.9, device=DEV)
    V, F, fmap = remesh.split_edges_from_training_views((200, 200), t(sc.mvps()), t(sc.verts), t(sc.tri), 2, alpha,
                                                        tau_ratio=0.02, num_views_cap=3)
    assert F.shape[0] > sc.T and fmap.shape[0] == F.shape[0]
    assert int(fmap.min()) >= 0 and int(fmap.max()) < sc.T
    # every output face lies in the plane of the input face it maps to
    v0 = t(sc.verts)[t(sc.tri).long()]  # [T,3,3]
    n = torch.linalg.cross(v0[:, 1] - v0[:, 0], v0[:, 2] - v0[:, 0])
    n = n / n.norm(dim=1, keepdim=True)
    pts = V[F.long()]  # [M',3,3]
    d = ((pts - v0[fmap][:, :1]) * n[fmap][:, None, :]).sum(-1)
    assert float(d.abs().max()) < 1e-4


@pytest.mark.skipif(not R.reference_available(), reason="oracle/_ref/libremesh_ref.so not built")
@pytest.mark.parametrize("mode,K,tau", [("world", 500, 0.0), ("world", 300, 0.1), ("world", 10 ** 6, 0.2),
                                        ("clip", 1000, 0.005), ("clip", 40, 0.0)])
def test_split_budget_matches_reference(mode, K, tau):
    """num_splits > 0: the K longest splits over all faces, as the reference's
    queue pops them (stopping early at the threshold when tau > 0)."""
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    if mode == "world":
        v, f = _soup(200, seed=11)
        got = _np(remesh.split_triangle_soup(t(v), t(f), K, tau=tau))
        ref = R.reference_split(v, f, K, tau)
    else:
        sc = scenes.make_scene(2, seed=5, num_tris=300, num_views=1, resolution=(600, 800), with_targets=False)
        valid = (np.random.default_rng(5).random(sc.T) < 0.8).astype(np.int32)
        mvp = sc.mvps()[0]
        got = _np(remesh.split_triangle_soup_clip((600, 800), t(mvp), t(sc.verts), t(sc.tri), t(valid), K,
                                                  tau_ratio=tau))
        ref = R.reference_split(sc.verts, sc.tri, K, tau, mvp=mvp, valid=valid, aspect_wh=800 / 600)
    assert got[1].shape == ref[1].shape and got[0].shape == ref[0].shape
    assert R.families(*got) == R.families(*ref)


def test_split_budget_with_equal_edges():
    """Congruent faces tie at every length: the budget is met exactly and the
    ties go to the lower faces first."""
    base = np.array([[0, 0, 0], [1, 0, 0], [0, 0.7, 0]], np.float32)
    v = np.concatenate([base + np.float32(2 * i) for i in range(10)]).astype(np.float32)
    f = np.arange(30, dtype=np.int32).reshape(10, 3)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    got = _np(remesh.split_triangle_soup(t(v), t(f), 15, tau=0.0))
    assert got[1].shape[0] == 10 + 15 and got[0].shape[0] == 30 + 3 * 15
    if R.reference_available():
        ref = R.reference_split(v, f, 15, 0.0)
        assert ref[1].shape == got[1].shape
    # every face splits its hypotenuse (10 splits), then the next longest edges (one leg per face, all
    # equal) take the remaining 5 in face order: faces 0..4 end with 3 triangles, faces 5..9 with 2
    per_face = np.bincount(got[2], minlength=10)
    assert per_face.tolist() == [3] * 5 + [2] * 5


def test_degenerate_and_empty_soups():
    v, f = _soup(40, seed=9)
    v[0:3] = v[0]
    v[3:6] = [[0, 0, 0], [1, 0.001, 0.0003], [2.7, 0.002, 0.0001]]
    f[10] = f[9]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    for tau in (0.05, 0.3):
        _equal(_np(remesh.split_triangle_soup_until(t(v), t(f), tau)), R.restated_split(v, f, tau))
    got = _np(remesh.split_triangle_soup_until(t(np.zeros((0, 3), np.float32)), t(np.zeros((0, 3), np.int32)), 0.1))
    assert got[0].shape == (0, 3) and got[1].shape == (0, 3)
    # no face valid: nothing splits, everything is flagged as original
    sc = scenes.make_scene(1, seed=9, num_tris=30, num_views=1, resolution=(64, 64), with_targets=False)
    got = _np(remesh.split_triangle_soup_clip_until((64, 64), t(sc.mvps()[0]), t(sc.verts), t(sc.tri),
                                                    t(np.zeros(sc.T, np.int32)), 0.01))
    assert got[1].shape == sc.tri.shape and (got[3] == 1).all() and np.array_equal(got[1], sc.tri)
    # CPU tensors in, CPU tensors out (computed on the GPU)
    cpu = remesh.split_triangle_soup_until(torch.from_numpy(v), torch.from_numpy(f), 0.3)
    assert cpu[0].device.type == "cpu"
    _equal(tuple(x.numpy() for x in cpu), R.restated_split(v, f, 0.3))


def test_core_bindings_take_numpy():
    """ds._core.split_triangle_soup(_clip): the reference binding's numpy
    arguments and results (src/main.cpp:308-388)."""
    from diffsoup_b200 import _core
    v, f = _soup(50, seed=12)
    got = _core.split_triangle_soup(v, f, -1, 0.1)
    assert all(isinstance(x, np.ndarray) for x in got)
    _equal(got, R.restated_split(v, f, 0.1))
    sc = scenes.make_scene(2, seed=12, num_tris=100, num_views=1, resolution=(300, 400), with_targets=False)
    valid = np.ones(sc.T, np.int32)
    got = _core.split_triangle_soup_clip(sc.mvps()[0], sc.verts, sc.tri, valid, -1, 0.02, 400 / 300)
    _equal(got, R.restated_split(sc.verts, sc.tri, 0.02, mvp=sc.mvps()[0], valid=valid, aspect_wh=400 / 300))

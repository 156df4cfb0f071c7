"""The soup subdivision's oracle against the reference's own remeshers (CPU).

oracle/remesh.py restates src/remesh.cpp and src/remesh_clip.cpp in threshold
mode with the GPU remesher's numbering; here it is compared with the
reference's compiled sources (oracle/_ref/libremesh_ref.so) as the set of
triangles each input face becomes, bit for bit, with the same counts and
flags.  Cases: world-space and screen-space lengths, faces masked out, corners
outside the NDC cube and behind the camera, thresholds that split nothing.
The product's host-side argument checks run here too (no GPU needed).
"""

import numpy as np
import pytest
import torch

from diffsoup_b200 import remesh, scenes
from oracle import remesh as R

pytestmark = pytest.mark.skipif(not R.reference_available(), reason="oracle/_ref/libremesh_ref.so not built")


def _soup(T, seed, spread=0.15):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, (T, 3))
    v = (c[:, None, :] + rng.normal(0, spread, (T, 3, 3))).reshape(-1, 3).astype(np.float32)
    return v, np.arange(3 * T, dtype=np.int32).reshape(T, 3)


def _same(ref, res, n):
    assert ref[0].shape == res[0].shape and ref[1].shape == res[1].shape
    assert np.array_equal(ref[0][:n].view(np.uint32), res[0][:n].view(np.uint32))  # the inputs, in place
    assert R.families(*ref) == R.families(*res)


@pytest.mark.parametrize("tau", [0.05, 0.12, 0.4])
def test_world_split_matches_reference(tau):
    v, f = _soup(150, seed=int(tau * 100))
    ref = R.reference_split(v, f, -1, tau)
    res = R.restated_split(v, f, tau)
    _same(ref, res, v.shape[0])


@pytest.mark.parametrize("seed,tau", [(1, 0.01), (2, 0.03)])
def test_clip_split_matches_reference(seed, tau):
    sc = scenes.make_scene(2, seed=seed, num_tris=250, num_views=1, resolution=(600, 800), with_targets=False)
    rng = np.random.default_rng(seed)
    valid = (rng.random(sc.T) < 0.8).astype(np.int32)
    verts = sc.verts.copy()
    verts[:30] *= 6.0  # some corners leave the NDC cube, some pass behind the camera
    mvp = sc.mvps()[0]
    ref = R.reference_split(verts, sc.tri, -1, tau, mvp=mvp, valid=valid, aspect_wh=800 / 600)
    res = R.restated_split(verts, sc.tri, tau, mvp=mvp, valid=valid, aspect_wh=800 / 600)
    assert ref[1].shape[0] > sc.T  # something was split
    _same(ref, res, verts.shape[0])
    # masked faces are never split
    split_fams = {int(m) for m, fl in zip(res[2], res[3]) if fl == 0}
    assert all(valid[t] > 0 for t in split_fams)


def test_thresholds_that_split_nothing():
    v, f = _soup(20, seed=3)
    for tau in (0.0, -1.0, 100.0):
        ref = R.reference_split(v, f, -1, tau)
        res = R.restated_split(v, f, tau)
        _same(ref, res, v.shape[0])
        assert res[1].shape == f.shape and (res[3] == 1).all()


def test_product_argument_checks():
    v, f = _soup(4, seed=4)
    src = torch.arange(5.0)
    assert torch.equal(remesh.expand_by_index(src, torch.tensor([4, 0, 0])), torch.tensor([4.0, 0.0, 0.0]))
    with pytest.raises(ValueError):
        remesh.expand_by_index(src, torch.tensor([5]))
    with pytest.raises(TypeError):
        remesh.expand_by_index(src, [1])


def test_degenerate_faces_match_reference():
    """A point face (every edge of length 0), a sliver, two faces on the same
    vertices and an empty soup, in both metrics.  (A face with two edges of
    equal float length, such as one with a vanishing edge, is split at either
    in the reference, by its heap's order; such faces are left out.)"""
    rng = np.random.default_rng(9)
    v, f = _soup(40, seed=9)
    v[0:3] = v[0]                        # a point face
    v[3:6] = [[0, 0, 0], [1, 0.001, 0.0003], [2.7, 0.002, 0.0001]]  # a sliver (exactly collinear corners give exact ties, unordered in the reference)
    f[10] = f[9]                          # two faces on the same vertices
    for tau in (0.05, 0.3):
        _same(R.reference_split(v, f, -1, tau), R.restated_split(v, f, tau), v.shape[0])
    sc = scenes.make_scene(1, seed=9, num_tris=30, num_views=1, resolution=(64, 64), with_targets=False)
    valid = np.ones(sc.T, np.int32)
    verts = sc.verts.copy()
    verts[0:3] = verts[0]
    ref = R.reference_split(verts, sc.tri, -1, 0.05, mvp=sc.mvps()[0], valid=valid, aspect_wh=1.0)
    res = R.restated_split(verts, sc.tri, 0.05, mvp=sc.mvps()[0], valid=valid, aspect_wh=1.0)
    _same(ref, res, verts.shape[0])
    empty = (np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
    e_ref = R.reference_split(*empty, -1, 0.1)
    e_res = R.restated_split(*empty, 0.1)
    assert e_ref[1].shape == e_res[1].shape == (0, 3)

"""ds_depth_test_noalloc: the depth test for callers that cannot allocate.

Some callers of this library cannot hand it device memory: an application
whose own allocator owns all device memory, code held to a fixed memory
budget, or a loop that cannot pay for cudaMalloc/cudaFree.  For them the
depth test has a variant whose depth-key scratch is a fixed buffer inside the
library (at most 2^21 pixels per call).  These tests call it through the C ABI
and check that two calls in a row give exactly what the workspace version
(ds_depth_test) gives on the same fragments, so a call sees none of the
previous call's depth keys.  The file runs last so that a stop at the first
failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from diffsoup_b200 import _core, scenes
from diffsoup_b200.rasterize import _compute_fragments

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _entry():
    f = _core.lib.ds_depth_test_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int] * 4 + [C.c_void_p] * 6
    return f


def _fragments(config, seed, views, res):
    sc = scenes.make_scene(config, seed=seed, num_views=views, resolution=res, with_targets=False)
    H, W = res
    pos = torch.from_numpy(sc.clip_positions()).to(DEV)
    tri = torch.from_numpy(sc.tri).to(DEV)
    fp, fa = _compute_fragments((H, W), pos, tri)
    lvl = sc.max_level
    S = scenes.feats_at_level(lvl)
    alpha_src = torch.sigmoid(torch.from_numpy(sc.alpha_src[:, :S, 0]).to(DEV)).contiguous()
    alpha = torch.zeros(fp.shape[0], device=DEV)
    _core.multires_triangle_alpha(fa, lvl, lvl, alpha_src, alpha)
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    thresh = torch.rand(fp.shape[0], device=DEV, generator=g)
    return fp, fa, alpha, thresh, pos.shape[0], H, W


def test_noalloc_depth_test_matches_workspace_version_twice():
    f = _entry()
    # two different batches in a row: the second must not see the first's keys
    for config, seed, views, res in ((2, 3, 2, (512, 640)), (1, 8, 3, (300, 400))):
        fp, fa, alpha, thresh, B, H, W = _fragments(config, seed, views, res)
        assert fp.shape[0] > 10000
        want = torch.zeros(B, H, W, 4, device=DEV)
        _core.depth_test(fp, fa, alpha, thresh, want)
        got = torch.zeros(B, H, W, 4, device=DEV)
        p = _core.ptr
        rc = f(B, H, W, fp.shape[0], p(fp), p(fa), p(alpha), p(thresh), p(got), _core.stream())
        _core.check(rc)
        torch.cuda.synchronize()
        assert int((want[..., 3] > 0).sum()) > 1000
        assert torch.equal(got.view(torch.int32), want.view(torch.int32))


def test_noalloc_same_shape_again_and_untouched_pixels():
    """Three calls in a row, the third with the first call's shape but other
    fragments: each equals the workspace version, and pixels that no fragment
    wins keep the value the caller put there."""
    f = _entry()
    p = _core.ptr
    for config, seed, views, res in ((2, 3, 2, (512, 640)), (1, 8, 3, (300, 400)), (2, 11, 2, (512, 640))):
        fp, fa, alpha, thresh, B, H, W = _fragments(config, seed, views, res)
        want = torch.full((B, H, W, 4), 7.0, device=DEV)
        _core.depth_test(fp, fa, alpha, thresh, want)
        got = torch.full((B, H, W, 4), 7.0, device=DEV)
        _core.check(f(B, H, W, fp.shape[0], p(fp), p(fa), p(alpha), p(thresh), p(got), _core.stream()))
        torch.cuda.synchronize()
        empty = (want == 7.0).all(dim=-1)  # pixels no fragment won (every channel as the caller left it)
        assert int(empty.sum()) > 1000
        assert bool((got[empty] == 7.0).all())
        assert torch.equal(got.view(torch.int32), want.view(torch.int32))


def test_noalloc_skips_fragments_outside_the_batch():
    """Fragments whose batch index or pixel lies outside the call's B x H x W
    are skipped: the result equals the workspace version on the valid
    fragments alone, and the next call is unaffected."""
    f = _entry()
    p = _core.ptr
    fp, fa, alpha, thresh, B, H, W = _fragments(1, 5, 2, (200, 240))
    n = fp.shape[0]
    assert (B + 1) * H * W < (1 << 21)
    # a winning fragment (in front of everything, opacity above its threshold) at
    # batch B, and one at column W of row 0 (which would alias pixel (1, 0))
    bad_pix = torch.tensor([[B, 3, 4], [0, 0, W]], dtype=torch.int32, device=DEV)
    bad_attr = torch.tensor([[0.3, 0.3, -0.99, 1.0], [0.3, 0.3, -0.99, 1.0]], device=DEV)
    fp2 = torch.cat([fp, bad_pix]).contiguous()
    fa2 = torch.cat([fa, bad_attr]).contiguous()
    al2 = torch.cat([alpha, torch.ones(2, device=DEV)]).contiguous()
    th2 = torch.cat([thresh, torch.zeros(2, device=DEV)]).contiguous()
    want = torch.zeros(B, H, W, 4, device=DEV)
    _core.depth_test(fp, fa, alpha, thresh, want)  # the valid fragments only
    got = torch.zeros(B, H, W, 4, device=DEV)
    _core.check(f(B, H, W, n + 2, p(fp2), p(fa2), p(al2), p(th2), p(got), _core.stream()))
    torch.cuda.synchronize()
    assert torch.equal(got.view(torch.int32), want.view(torch.int32))
    # the next call, one batch larger, sees nothing of the skipped fragments
    fp3, fa3, alpha3, thresh3, B3, H3, W3 = _fragments(1, 6, 3, (200, 240))
    want3 = torch.zeros(B3, H3, W3, 4, device=DEV)
    _core.depth_test(fp3, fa3, alpha3, thresh3, want3)
    got3 = torch.zeros(B3, H3, W3, 4, device=DEV)
    _core.check(f(B3, H3, W3, fp3.shape[0], p(fp3), p(fa3), p(alpha3), p(thresh3), p(got3), _core.stream()))
    torch.cuda.synchronize()
    assert torch.equal(got3.view(torch.int32), want3.view(torch.int32))


def test_noalloc_rejects_batches_beyond_its_buffer():
    f = _entry()
    null = C.c_void_p(0)
    rc = f(3, 1024, 1024, 1, null, null, null, null, null, _core.stream())
    assert rc == 1
    assert b"exceed" in _core.lib.ds_last_error()

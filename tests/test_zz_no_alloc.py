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


def test_noalloc_rejects_batches_beyond_its_buffer():
    f = _entry()
    null = C.c_void_p(0)
    rc = f(3, 1024, 1024, 1, null, null, null, null, null, _core.stream())
    assert rc == 1
    assert b"exceed" in _core.lib.ds_last_error()

"""The point-cloud helpers on the GPU: the spacing search (a blocked
all-pairs search on the device) against the reference's results, and the
initial soup and vertex compaction on CUDA tensors."""

import os

import numpy as np
import pytest
import torch

from diffsoup_b200 import point3d

pytestmark = pytest.mark.gpu
GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "point3d.npz"))


@pytest.mark.parametrize("name", ["uniform", "clustered", "duplicates"])
def test_nn_spacing_on_gpu(name):
    P = GOLDEN[f"{name}_points"]
    for red in ("median", "mean"):
        want = float(GOLDEN[f"{name}_{red}"])
        got = point3d.nn_spacing(torch.from_numpy(P).cuda(), red)
        assert abs(got - want) <= 1e-6 * max(want, 1e-12) + 1e-12, (red, got, want)


def test_soup_helpers_on_cuda_tensors():
    xyz = torch.randn(500, 3, device="cuda")
    V, F = point3d.triangle_soup_from_points(xyz, scale=0.1)
    assert V.is_cuda and F.is_cuda and V.shape == (1500, 3)
    assert torch.allclose(V.reshape(-1, 3, 3).mean(1), xyz, atol=1e-6)
    keep = F[::2]
    nv, nf = point3d.remove_unreferenced_vertices_from_soup(V, keep)
    assert nv.shape == (3 * keep.shape[0], 3) and torch.equal(nv[nf.long()], V[keep.long()])

"""The point-cloud helpers (diffsoup_b200/point3d.py) against the reference's
own results (tests/golden/make_golden_point3d.py) and the properties of the
random initial soup."""

import os

import numpy as np
import pytest
import torch

from diffsoup_b200 import point3d

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "point3d.npz"))


@pytest.mark.parametrize("name", ["uniform", "clustered", "duplicates"])
def test_nn_spacing_matches_reference(name):
    P = GOLDEN[f"{name}_points"]
    for red in ("median", "mean"):
        want = float(GOLDEN[f"{name}_{red}"])
        got = point3d.nn_spacing(P, red)
        assert abs(got - want) <= 1e-6 * max(want, 1e-12) + 1e-12, (red, got, want)
    assert point3d.nn_spacing(P[:1]) == 0.0
    with pytest.raises(ValueError):
        point3d.nn_spacing(P, "max")


def test_remove_unreferenced_matches_reference():
    V, F = torch.from_numpy(GOLDEN["ru_verts"]), torch.from_numpy(GOLDEN["ru_faces"])
    nv, nf = point3d.remove_unreferenced_vertices_from_soup(V, F)
    assert np.array_equal(nv.numpy(), GOLDEN["ru_new_verts"])
    assert np.array_equal(nf.numpy(), GOLDEN["ru_new_faces"]) and nf.dtype == torch.int32


def test_triangle_soup_from_points_geometry():
    torch.manual_seed(0)
    xyz = torch.randn(2000, 3, dtype=torch.float64)
    V, F = point3d.triangle_soup_from_points(xyz, scale=0.3)
    assert V.shape == (6000, 3) and F.dtype == torch.int32 and torch.equal(F.reshape(-1), torch.arange(6000,
                                                                                                        dtype=torch.int32))
    T = V.reshape(-1, 3, 3)
    assert torch.allclose(T.mean(1), xyz, atol=1e-12)                       # centroid on the point
    assert torch.allclose((T - xyz[:, None]).norm(dim=-1), torch.full((2000, 3), 0.3, dtype=torch.float64))
    e = torch.stack([(T[:, 1] - T[:, 0]).norm(dim=-1), (T[:, 2] - T[:, 1]).norm(dim=-1),
                     (T[:, 0] - T[:, 2]).norm(dim=-1)], -1)
    assert torch.allclose(e, torch.full_like(e, 0.3 * 3 ** 0.5))              # equilateral
    n = torch.linalg.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    n = n / n.norm(dim=-1, keepdim=True)
    assert abs(float(n.mean(0).norm())) < 0.1 and abs(float((n[:, 2] ** 2).mean()) - 1 / 3) < 0.05  # uniform
    V0, F0 = point3d.triangle_soup_from_points(xyz[:0], scale=1.0)
    assert V0.shape == (0, 3) and F0.shape == (0, 3)

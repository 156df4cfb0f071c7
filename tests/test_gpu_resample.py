"""A training run with the resampling step in the middle, all on the GPU:
TrainStep + the fused optimisers, the visibility count of the resampling
heuristics (examples/utils.py:445-482), the split of the faces seen in the
training views (examples/utils.py:493-545) with per-face parameters carried
to the children (expand_by_index), and training resumed on the new soup."""

import numpy as np
import pytest
import torch

from diffsoup_b200 import remesh, scenes, visibility
from diffsoup_b200.optimize import Adam, VectorAdam
from diffsoup_b200.step import TrainStep

pytestmark = pytest.mark.gpu


def _train(sc_hw, verts, tri, feat, alpha, params, d_extra, sc, iters):
    step = TrainStep(tri.shape[0], verts.shape[0], sc_hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=True, seed=9)
    d = dict(verts=verts, tri=tri, feat_src=feat, alpha_src=alpha, mlp_params=params, **d_extra)
    for p, g in ((verts, step.grad_verts), (feat, step.grad_feat_src), (alpha, step.grad_alpha_src),
                 (params, step.grad_mlp)):
        p.grad = g
    opts = [Adam([{"params": [feat], "lr": 5e-2}, {"params": [alpha], "lr": 5e-2}]), VectorAdam([verts], lr=1e-3),
            Adam([params], lr=1e-2)]
    step.fit_capacity(**d)
    losses = []
    for _ in range(iters):
        step.run(**d)
        for o in opts:
            o.step()
        losses.append(float(step.loss.item()))
    return step, losses


def test_training_with_resampling():
    sc = scenes.make_scene(1, seed=4, num_tris=1500, num_views=4, resolution=(96, 96))
    hw = [(v.height, v.width) for v in sc.views]
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=4)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    verts, tri = t(sc.verts), t(sc.tri)
    feat, alpha = t(sc.feat_src), t(sc.alpha_src[..., 0])
    params = t(np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp]))
    mvps = t(sc.mvps())
    extra = dict(mvp=mvps, inv_mvp=t(sc.inv_mvps()), target=t(np.concatenate([x.reshape(-1, 3) for x in sc.targets])))
    step, losses = _train(hw, verts, tri, feat, alpha, params, extra, sc, 25)
    assert np.mean(losses[-5:]) < np.mean(losses[:3])

    # resampling: visibility, then the split of the faces the views see
    alpha_acc = step.intermediate("alpha_acc").clone()  # [T, S at max_level], after the sigmoid
    counts = visibility.count_visible_triangles((96, 96), mvps, verts.detach(), tri, sc.max_level, alpha_acc)
    assert counts.shape == (sc.T,) and int(counts.sum()) > 0
    torch.manual_seed(0)
    V2, F2, fmap = remesh.split_edges_from_training_views((96, 96), mvps, verts.detach(), tri, sc.max_level,
                                                          alpha_acc, tau_ratio=0.03, num_views_cap=2)
    assert F2.shape[0] > sc.T and fmap.shape[0] == F2.shape[0]
    # faces never seen by the views keep their parameters and are not split
    seen = counts > 0
    assert bool(seen[fmap[sc.T:]].all())

    # per-face parameters carried to the children; training resumes on the new soup
    feat2 = remesh.expand_by_index(feat.detach(), fmap).contiguous()
    alpha2 = remesh.expand_by_index(alpha.detach(), fmap).contiguous()
    verts2 = V2.contiguous()
    _, losses2 = _train(hw, verts2, F2.contiguous(), feat2, alpha2, params.detach().clone(), extra, sc, 15)
    assert all(np.isfinite(losses2))
    assert losses2[0] < 2.0 * losses[-1], (losses[-1], losses2[:3])
    assert np.mean(losses2[-5:]) < 1.1 * np.mean(losses2[:3]), losses2

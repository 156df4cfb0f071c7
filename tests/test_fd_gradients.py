"""FP64 central finite differences of the training-step loss.

The loss of one step (examples/02_synthetic.py:354-385, MSE photometric term)
is a smooth function of the neural features and the shading-MLP parameters
once the triangle-ID buffer is fixed, so their gradients are derivatives and
are checked against central differences of the FP64 oracle's loss (step
1e-4) on 100-triangle scenes of configuration 1 (8 channels, levels 0..2,
MLP 11-16-3) and of configuration 5 (16 channels, levels 0..3, MLP
19-64-64-3; the config-5 protocol):

  * the FP64 oracle's own backward (oracle/pipeline.py) on CPU, here;
  * the batched BF16 step on the GPU (tests/test_gpu_step.py), which is
    compared with the same differences.

Vertex positions and opacity logits enter the loss only through the
discrete rasterization: with the ID buffer fixed the loss does not depend on
them at all (the edge gradient and the opacity auxiliary loss are estimators
whose forward is the identity and zero, rasterize.py:190, :263-265), which
test_loss_is_flat_in_positions_and_opacity checks; their gradients are
pinned to the FP64 restatement of the estimators and to the reference's own
outputs instead (tests/test_oracle_golden.py, tests/test_gpu_reference.py).
"""

import numpy as np
import pytest

from diffsoup_b200 import scenes
from oracle import cpu
from oracle import pipeline as P

H = 1e-4


def fd_scene(seed: int = 0, config: int = 1):
    sc = scenes.make_scene(config, seed=seed, num_tris=100, num_views=1, resolution=(40, 48))
    hw = [(v.height, v.width) for v in sc.views]
    mlp = [(W.astype(np.float64), b.astype(np.float64))
           for W, b in scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=seed)]
    inp = P.StepInputs(verts=sc.verts, tri=sc.tri, mvps=sc.mvps(), inv_mvps=sc.inv_mvps(), hw=hw,
                       feat_src=sc.feat_src.astype(np.float64), alpha_src=sc.alpha_src[..., 0].astype(np.float64),
                       mlp=mlp, targets=sc.targets, min_level=sc.min_level, max_level=sc.max_level,
                       stochastic=True, seed=11, iteration=0)
    pos = cpu.project(sc.verts, sc.mvps())
    alpha32 = cpu.accumulate_sigmoid_f32(sc.min_level, sc.max_level, sc.max_level, sc.alpha_src)[..., 0]
    rasts = [cpu.rasterize_alpha(h, w, pos[b:b + 1], sc.tri, sc.max_level, alpha32, True, 11, 0, view0=b)[0]
             for b, (h, w) in enumerate(hw)]
    return sc, inp, rasts


def loss_of(inp, rasts, **changes) -> float:
    d = dict(inp.__dict__)
    d.update(changes)
    return P.train_step(P.StepInputs(**d), "f64", rast_in=rasts).loss


def feature_entries(grad: np.ndarray, n: int, rng: np.random.Generator):
    """The n/2 largest-|gradient| entries and n/2 random entries with a nonzero gradient."""
    flat = np.abs(grad).ravel()
    top = list(np.argsort(flat)[::-1][: n // 2])
    nz = np.flatnonzero(flat)
    top += list(rng.choice(nz, size=n - len(top), replace=False))
    return [np.unravel_index(i, grad.shape) for i in top]


def fd_feature(inp, rasts, idx) -> float:
    fp, fm = inp.feat_src.copy(), inp.feat_src.copy()
    fp[idx] += H
    fm[idx] -= H
    return (loss_of(inp, rasts, feat_src=fp) - loss_of(inp, rasts, feat_src=fm)) / (2 * H)


def fd_mlp(inp, rasts, layer: int, which: int, idx) -> float:
    def shifted(s):
        out = []
        for i, (W, b) in enumerate(inp.mlp):
            W, b = W.copy(), b.copy()
            if i == layer:
                (W if which == 0 else b)[idx] += s
            out.append((W, b))
        return out
    return (loss_of(inp, rasts, mlp=shifted(H)) - loss_of(inp, rasts, mlp=shifted(-H))) / (2 * H)


@pytest.mark.parametrize("config", [1, 5])
def test_oracle_feature_and_mlp_gradients_match_central_differences(config):
    sc, inp, rasts = fd_scene(0, config)
    ref = P.train_step(inp, "f64", rast_in=rasts)
    rng = np.random.default_rng(0)
    got, want = [], []
    for idx in feature_entries(ref.grad_feat_src, 12, rng):
        got.append(ref.grad_feat_src[idx])
        want.append(fd_feature(inp, rasts, idx))
    for layer, (gW, gb) in enumerate(ref.grad_mlp):
        for which, g in ((0, gW), (1, gb)):
            for idx in feature_entries(g, 4, rng):
                got.append(g[idx])
                want.append(fd_mlp(inp, rasts, layer, which, idx))
    got, want = np.array(got), np.array(want)
    scale = np.abs(want).max()
    assert scale > 0
    err = np.abs(got - want)
    # FP64 central differences with h = 1e-4: truncation O(h^2), rounding O(eps / h)
    assert (err <= 1e-7 * scale + 1e-5 * np.abs(want)).all(), np.c_[got, want, err]


def test_loss_is_flat_in_positions_and_opacity():
    sc, inp, rasts = fd_scene(1)
    base = loss_of(inp, rasts)
    v = inp.verts.copy()
    v[:, 0] += 1e-3
    a = inp.alpha_src + 0.5
    assert loss_of(inp, rasts, verts=v) == pytest.approx(base, rel=0, abs=0)
    assert loss_of(inp, rasts, alpha_src=a) == pytest.approx(base, rel=0, abs=0)

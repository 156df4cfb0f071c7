"""Fused optimiser updates (csrc/optim.cu through diffsoup_b200.optimize)
against the reference's VectorAdam and torch.optim.Adam (tests/golden/optim.npz,
pinned by tests/test_optim_oracle.py): FP32 within 1e-6 after five steps, and a
graph-captured update equal to the eager one."""

import os

import numpy as np
import pytest
import torch

from diffsoup_b200.optimize import Adam, VectorAdam

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "optim.npz"))


def test_vector_adam_matches_reference():
    p = torch.tensor(G["va_p0"], device="cuda", requires_grad=True)
    opt = VectorAdam([p], lr=1e-3, betas=(0.9, 0.999))
    for grad in G["va_grads"]:
        p.grad = torch.tensor(grad, device="cuda")
        opt.step()
    st = opt.state[p]
    assert int(st["step"].item()) == len(G["va_grads"])
    np.testing.assert_allclose(p.detach().cpu().numpy(), G["va_p"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(st["g1"].cpu().numpy(), G["va_g1"], rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(st["g2"].cpu().numpy(), G["va_g2"], rtol=1e-5, atol=1e-12)


@pytest.mark.parametrize("name", ["adam_feat", "adam_mlp"])
def test_adam_matches_torch(name):
    p = torch.tensor(G[f"{name}_p0"], device="cuda", requires_grad=True)
    opt = Adam([p], lr=float(G[f"{name}_lr"]))
    for grad in G[f"{name}_grads"]:
        p.grad = torch.tensor(grad, device="cuda")
        opt.step()
    st = opt.state[p]
    np.testing.assert_allclose(p.detach().cpu().numpy(), G[f"{name}_p"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(st["exp_avg"].cpu().numpy(), G[f"{name}_m"], rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(st["exp_avg_sq"].cpu().numpy(), G[f"{name}_v"], rtol=1e-5, atol=1e-12)


def test_captured_update_equals_eager():
    torch.manual_seed(0)
    p0 = torch.randn(1000, 3, device="cuda")
    grads = [torch.randn(1000, 3, device="cuda") * 1e-2 for _ in range(3)]
    a = p0.clone().requires_grad_(True)
    b = p0.clone().requires_grad_(True)
    oa, ob = VectorAdam([a], lr=1e-2), VectorAdam([b], lr=1e-2)
    for g in grads:
        a.grad = g.clone()
        oa.step()
    b.grad = grads[0].clone()
    ob.step()  # state created eagerly, outside the capture
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s), torch.cuda.graph(graph, stream=s):
        ob.step()
    torch.cuda.current_stream().wait_stream(s)
    for g in grads[1:]:
        b.grad.copy_(g)
        graph.replay()
    torch.cuda.synchronize()
    assert int(ob.state[b]["step"].item()) == 3
    assert torch.equal(a, b)


def test_training_loop_in_one_graph_reduces_the_loss():
    """TrainStep and the optimiser updates of examples/02_synthetic.py:310-315
    (Adam on features and opacities, VectorAdam on vertices, Adam on the MLP)
    captured in one CUDA graph and replayed: the loss decreases."""
    from diffsoup_b200 import scenes
    from diffsoup_b200.step import TrainStep

    sc = scenes.make_scene(1, seed=3, num_tris=800, num_views=4, resolution=(64, 64))
    hw = [(v.height, v.width) for v in sc.views]
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=3)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    verts, feat, alpha = t(sc.verts), t(sc.feat_src), t(sc.alpha_src[..., 0])
    params = t(np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp]))
    step = TrainStep(sc.T, verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim, sc.n_layers,
                     stochastic=True, seed=5)
    d = dict(verts=verts, tri=t(sc.tri), mvp=t(sc.mvps()), inv_mvp=t(sc.inv_mvps()), feat_src=feat, alpha_src=alpha,
             mlp_params=params, target=t(np.concatenate([x.reshape(-1, 3) for x in sc.targets])))
    for p, g in ((verts, step.grad_verts), (feat, step.grad_feat_src), (alpha, step.grad_alpha_src),
                 (params, step.grad_mlp)):
        p.grad = g
    soup = Adam([{"params": [feat], "lr": 5e-2}, {"params": [alpha], "lr": 5e-2}])
    vert = VectorAdam([verts], lr=1e-3)
    shader = Adam([params], lr=1e-2)

    def iteration():
        step.run(**d)
        soup.step()
        vert.step()
        shader.step()

    step.fit_capacity(**d)
    iteration()  # optimiser state created outside the capture
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s), torch.cuda.graph(graph, stream=s):
        iteration()
    torch.cuda.current_stream().wait_stream(s)
    losses = []
    for _ in range(60):
        graph.replay()
        losses.append(float(step.loss.item()))
    assert all(np.isfinite(losses))
    assert np.mean(losses[-10:]) < 0.9 * np.mean(losses[:5]), (losses[:5], losses[-10:])

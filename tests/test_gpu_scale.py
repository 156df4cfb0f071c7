"""The batched step at the full sizes of the batching and scale workloads.

  * configuration 3: 60,000 triangles (20 Gaussian clusters + a shell of
    radius 10), 64 views of uneven resolution (widths 400..1200, aspect
    4:3, 16:9 or 1:1) in one launch, captured in a CUDA graph;
  * configuration 5: 200,000 triangles, 16 views of 1920x1080, features 16
    channels at levels 0..3, MLP 19-64-64-3.

The CPU oracle cannot run the whole continuous step at these sizes in a test,
so parity is checked through what does not depend on size: the ID buffer of
the smallest and the largest view against the oracle's rasterization bit for
bit, the loss against an FP64 reduction of the step's own colours, finite
gradients, graph replay equal to the eager step, and the same opacity
gradients whether the auxiliary pass reads the rasterizer's fragment records
or re-enumerates the tiles.  Peak device memory of both modes is printed.
"""

import numpy as np
import pytest
import torch

from diffsoup_b200 import scenes
from diffsoup_b200.step import TrainStep
from oracle import cpu

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _flat(mlp):
    return torch.from_numpy(np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp])).float()


def _run(sc, hw, d, frag_records):
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=True, seed=321, frag_records=frag_records)
    rast = torch.empty(step.num_pixels, 4, device=DEV)
    color = torch.empty(step.num_pixels, 3, device=DEV)
    step.fit_capacity(**d, rast_out=rast, color_out=color)
    step.rng[1] = 0
    loss = float(step.run(**d, rast_out=rast, color_out=color).item())
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() - base
    return step, rast, color, loss, peak


@pytest.mark.parametrize("config", [3, 5])
def test_full_size_step(config):
    sc = scenes.make_scene(config, seed=0)
    hw = [(v.height, v.width) for v in sc.views]
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    target = np.concatenate([x.reshape(-1, 3) for x in sc.targets])
    d = dict(verts=t(sc.verts), tri=t(sc.tri), mvp=t(sc.mvps()), inv_mvp=t(sc.inv_mvps()), feat_src=t(sc.feat_src),
             alpha_src=t(sc.alpha_src[..., 0]), mlp_params=_flat(mlp).to(DEV), target=t(target))
    step, rast, color, loss, peak = _run(sc, hw, d, 2.0)
    assert not step.overflowed()

    # ID buffer of the smallest and the largest view, bit for bit
    pos = step.intermediate("pos").cpu().numpy()
    alpha32 = step.intermediate("alpha_acc").cpu().numpy()
    r = rast.cpu().numpy()
    sizes = [h * w for h, w in hw]
    for b in sorted({int(np.argmin(sizes)), int(np.argmax(sizes))}):
        H, W = hw[b]
        o = step.pix_offsets[b]
        want, _ = cpu.rasterize_alpha(H, W, pos[b:b + 1], sc.tri, sc.max_level, alpha32, True, 321, 0, view0=b)
        assert np.array_equal(r[o:o + H * W].reshape(1, H, W, 4).view(np.uint32), want.view(np.uint32)), b

    # the loss is the MSE of the step's own colours (FP64 reduction)
    c = color.cpu().numpy().astype(np.float64)
    mse = float(((c - target) ** 2).mean())
    assert abs(loss - mse) <= 1e-5 * mse, (loss, mse)
    grads = {"verts": step.grad_verts, "feat": step.grad_feat_src, "alpha": step.grad_alpha_src, "mlp": step.grad_mlp}
    for k, g in grads.items():
        assert bool(torch.isfinite(g).all()), k
        assert float(g.abs().max()) > 0, k
    ga_records = step.grad_alpha_src.clone()
    gv = step.grad_verts.clone()

    # a graph replay of the same iteration equals the eager step
    g = step.capture(**d, rast_out=rast, color_out=color)
    step.rng[1] = 0
    g.replay()
    torch.cuda.synchronize()
    assert torch.allclose(step.grad_verts, gv, rtol=1e-4, atol=1e-12)
    del g

    # tile-wise recomputation of the fragments instead of stored records: same gradients
    del step
    torch.cuda.empty_cache()
    step0, _, _, loss0, peak0 = _run(sc, hw, d, 0.0)
    assert abs(loss0 - loss) <= 1e-6 * loss, (loss0, loss)
    rel = float((step0.grad_alpha_src - ga_records).norm() / ga_records.norm())
    assert rel < 1e-5, rel
    print(f"config{config}: {len(hw)} views, {sum(sizes) / 1e6:.1f} M pixels, {sc.T} triangles; "
          f"peak device memory {peak / 2**30:.2f} GiB with fragment records, {peak0 / 2**30:.2f} GiB "
          f"recomputing them")

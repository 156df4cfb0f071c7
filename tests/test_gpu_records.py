"""Fragment records of the training step.

The rasterizer keeps every fragment in front of each pixel's surface and the
opacity auxiliary gradient reads them back; blocks whose records do not fit
are re-enumerated.  Both routes must give the same opacity gradient as
re-enumerating every block (frag_records=0), up to the order of the float
atomics.
"""

import numpy as np
import pytest
import torch

from diffsoup_b200 import scenes
from diffsoup_b200.step import TrainStep

pytestmark = pytest.mark.gpu
DEV = "cuda"


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _inputs(sc, mlp):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    flat = np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp]).astype(np.float32)
    return dict(verts=t(sc.verts), tri=t(sc.tri), mvp=t(sc.mvps()), inv_mvp=t(sc.inv_mvps()),
                feat_src=t(sc.feat_src), alpha_src=t(sc.alpha_src[..., 0]), mlp_params=t(flat),
                target=t(np.concatenate([x.reshape(-1, 3) for x in sc.targets])))


def _run(sc, d, frag_records):
    hw = [(v.height, v.width) for v in sc.views]
    step = TrainStep(sc.T, sc.verts.shape[0], hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim,
                     sc.n_layers, stochastic=True, seed=99, frag_records=frag_records)
    step.status.zero_()
    step.run(**d)
    torch.cuda.synchronize()
    return step


@pytest.mark.parametrize("config,kw", [
    (2, dict(num_tris=3000, num_views=3, resolution=(160, 160))),
    (3, dict(num_tris=2000, num_views=3)),
    (4, dict(num_tris=800, num_views=2, resolution=(80, 96))),
])
def test_records_match_reenumeration(config, kw):
    sc = scenes.make_scene(config, seed=11, **kw)
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=11)
    d = _inputs(sc, mlp)
    _compare(sc, d, [(2.0, False)])


def test_records_store_exhausted():
    """8 views of 800x800: with 0.02 records per pixel the store fills up and
    the blocks met after that are re-enumerated."""
    sc = scenes.make_scene(2, seed=12)
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=12)
    # at 2 records per pixel a few dense blocks still outgrow their 192-record buffer
    _compare(sc, _inputs(sc, mlp), [(2.0, None), (0.02, True)])


def _compare(sc, d, modes):
    ref = _run(sc, d, 0.0)
    runs = []
    for fr, fallback in modes:
        s = _run(sc, d, fr)
        assert fallback is None or s.record_fallback() == fallback, fr
        runs.append(s)
    ga = ref.intermediate("grad_alpha_acc").cpu().numpy()
    for s in runs:
        assert np.array_equal(s.intermediate("rast").cpu().numpy(), ref.intermediate("rast").cpu().numpy())
        e = rel(s.intermediate("grad_alpha_acc").cpu().numpy(), ga)
        assert e < 2e-6, e
        assert rel(s.grad_alpha_src.cpu().numpy(), ref.grad_alpha_src.cpu().numpy()) < 2e-6
        assert rel(s.grad_verts.cpu().numpy(), ref.grad_verts.cpu().numpy()) < 1e-6


def test_records_overflowing_block_buffer():
    """200 nearly transparent screen-filling triangles: every pixel keeps all
    of its fragments (none passes the opacity threshold), far more than a
    block's record buffer holds, so every block is re-enumerated."""
    sc = scenes.make_scene(1, seed=3, num_tris=4, num_views=1, resolution=(48, 64))
    n = 100
    z = np.linspace(-0.8, 0.8, n, dtype=np.float32)
    quad = np.array([[-1.2, -1.2], [1.2, -1.2], [1.2, 1.2], [-1.2, 1.2]], np.float32)
    verts = []
    for k in range(n):
        for a, b, c in ((0, 1, 2), (0, 2, 3)):
            for i in (a, b, c):
                verts.append([quad[i, 0], quad[i, 1], z[k]])
    sc.verts = np.asarray(verts, np.float32)
    T = sc.verts.shape[0] // 3
    sc.tri = np.arange(3 * T, dtype=np.int32).reshape(T, 3)
    S = sc.feat_src.shape[1]
    rng = np.random.default_rng(5)
    sc.feat_src = rng.normal(0.0, 0.1, size=(T, S, sc.feat_dim)).astype(np.float32)
    sc.alpha_src = np.full((T, S, 1), -4.0, np.float32)
    sc.alpha_src[150::7] = 2.0  # a few opaque layers behind 75 transparent ones
    eye = np.eye(4, dtype=np.float32)
    sc.views[0].mvp = eye
    sc.views[0].inv_mvp = eye
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=3)
    d = _inputs(sc, mlp)
    ref = _run(sc, d, 0.0)
    rec = _run(sc, d, 2.0)
    assert rec.record_fallback()
    ga = ref.intermediate("grad_alpha_acc").cpu().numpy()
    assert np.abs(ga).sum() > 0
    assert rel(rec.intermediate("grad_alpha_acc").cpu().numpy(), ga) < 2e-6


def test_records_are_the_fragments_in_front_of_the_surface():
    """One 800x800 view: outside the re-enumerated blocks, the records are
    exactly the oracle's fragments at or in front of each pixel's surface,
    each once, with the visible flag on the surface's own triangle."""
    from oracle import cpu
    sc = scenes.make_scene(2, seed=12, num_views=1)
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=12)
    st = _run(sc, _inputs(sc, mlp), 2.0)
    H, W = sc.views[0].height, sc.views[0].width
    rast = st.intermediate("rast").cpu().numpy()
    pos = st.intermediate("pos").cpu().numpy()
    reserved, nfb = st.intermediate("record_counters").cpu().numpy()
    fill = st.intermediate("chunk_fill").cpu().numpy()
    recs = st.intermediate("records").cpu().numpy()
    fb = set(st.intermediate("fallback_blocks").cpu().numpy()[:nfb].tolist())
    nch = min(int(reserved), st.record_capacity) // 256
    rl = np.concatenate([recs[c * 256:c * 256 + fill[c]] for c in range(nch)])
    fpix, fattr = cpu.compute_fragments(H, W, pos[0:1], sc.tri)
    pix = fpix[:, 1].astype(np.int64) * W + fpix[:, 2]
    t = fattr[:, 3].astype(np.int64) - 1
    tp = rast[pix, 3].astype(np.int64) - 1
    front = ~((tp >= 0) & (fattr[:, 2] > rast[pix, 2]))
    tiles_x = (W + 15) // 16

    def block_of(p):
        y, x = p // W, p % W
        return ((y // 16) * tiles_x + x // 16) * 8 + ((y % 16) // 4) * 2 + (x % 16) // 8

    keep = front & ~np.isin(block_of(pix), list(fb))
    want = np.sort(pix[keep] * sc.T + t[keep])
    rpix = rl[:, 0].astype(np.int64) & 0xFFFFFFFF
    rt = rl[:, 1].astype(np.int64) & 0x7FFFFFFF
    got = np.sort(rpix * sc.T + rt)
    assert len(got) == len(want) and np.array_equal(got, want)
    vis = (rl[:, 1].astype(np.int64) >> 31) & 1
    assert np.array_equal(vis == 1, (rast[rpix, 3].astype(np.int64) - 1) == rt)
    # the records carry the fragments' own barycentrics
    order = np.argsort(pix[keep] * sc.T + t[keep])
    rorder = np.argsort(rpix * sc.T + rt)
    b = rl[rorder, 2:4].view(np.float32)
    assert np.array_equal(b.view(np.uint32), fattr[keep][order, :2].view(np.uint32))

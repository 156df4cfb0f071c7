"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own CUDA sources (oracle/_ref/libdsref*.so, built from the
unmodified kenji-tojo/diffsoup src/cuda/*.cu by `make -C oracle ref`) on small
seeded scenes and records inputs and outputs of every `_core` operator
(src/main.cpp:30-304) for both builds: nvcc's default flags ("fma") and
-fmad=false ("nofma").  Needs a CUDA GPU.

    python tests/golden/make_golden.py OUT_DIR

The reference compacts fragments in a nondeterministic block order
(rasterize.cu:437-446), so fragment lists are stored sorted by
(view, triangle, y, x).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from diffsoup_b200 import scenes  # noqa: E402
from oracle import cpu as ocpu  # noqa: E402
from oracle.ref import Ref  # noqa: E402


def edge_case_scene(H: int = 40, W: int = 56):
    """Hand-made clip-space soup covering the reference's culling branches."""
    tris = []
    # ordinary front-facing and back-facing triangles
    tris.append([[-0.5, -0.5, 0.2, 1.0], [0.5, -0.4, 0.3, 1.0], [0.0, 0.6, 0.1, 1.0]])
    tris.append([[0.5, -0.4, 0.0, 1.0], [-0.5, -0.5, 0.0, 1.0], [0.1, 0.5, 0.0, 1.0]])
    # exact duplicate of the first triangle (equal depths: tie broken by index)
    tris.append(list(tris[0]))
    # vertex behind the camera (w <= 0): culled by the w > 0 test
    tris.append([[-0.2, -0.2, 0.5, 1.0], [0.3, -0.1, 0.5, -0.5], [0.0, 0.3, 0.5, 1.0]])
    # entirely off-screen (outcode reject)
    tris.append([[2.0, 2.0, 0.0, 1.0], [3.0, 2.0, 0.0, 1.0], [2.5, 3.0, 0.0, 1.0]])
    # beyond the far plane (z > w)
    tris.append([[-0.3, -0.3, 1.5, 1.0], [0.3, -0.3, 1.5, 1.0], [0.0, 0.3, 1.5, 1.0]])
    # screen-covering triangle, far
    tris.append([[-3.0, -3.0, 0.9, 1.0], [3.0, -3.0, 0.9, 1.0], [0.0, 3.0, 0.9, 1.0]])
    # zero-area (collinear) triangle
    tris.append([[-0.4, 0.0, 0.0, 1.0], [0.0, 0.0, 0.0, 1.0], [0.4, 0.0, 0.0, 1.0]])
    # sliver
    tris.append([[-0.9, -0.8, -0.2, 1.0], [0.9, -0.78, -0.2, 1.0], [0.9, -0.77, -0.2, 1.0]])
    # perspective triangle with varying w, partially off the right edge
    tris.append([[0.2, -0.6, 0.1, 0.8], [1.6, -0.2, 0.8, 2.0], [0.6, 0.7, 0.3, 1.2]])
    # intersecting pair (depth ordering switches inside the overlap)
    tris.append([[-0.8, 0.1, -0.5, 1.0], [-0.1, 0.1, 0.5, 1.0], [-0.45, 0.8, 0.0, 1.0]])
    tris.append([[-0.8, 0.4, 0.5, 1.0], [-0.1, 0.4, -0.5, 1.0], [-0.45, 0.9, 0.0, 1.0]])
    # vertices exactly on pixel centres
    cx = lambda i: -1.0 + 2.0 * (i + 0.5) / W  # noqa: E731
    cy = lambda j: -1.0 + 2.0 * (j + 0.5) / H  # noqa: E731
    tris.append([[cx(40), cy(5), 0.05, 1.0], [cx(50), cy(5), 0.05, 1.0], [cx(40), cy(15), 0.05, 1.0]])
    # straddling the near plane (one vertex z < -w, all w > 0)
    tris.append([[-0.2, 0.5, -1.5, 1.0], [0.3, 0.5, 0.2, 1.0], [0.0, 0.9, 0.2, 1.0]])
    pos = np.array(tris, np.float32).reshape(1, -1, 4)
    pos = np.concatenate([pos, pos * np.array([1.0, -1.0, 1.0, 1.0], np.float32)], axis=0)  # 2 views
    T = len(tris)
    tri = np.arange(3 * T, dtype=np.int32).reshape(T, 3)
    return pos, tri, H, W


def run_case(name: str, pos: np.ndarray, tri: np.ndarray, H: int, W: int, level: int, lo: int, hi: int, C: int,
             seed: int, inv_mvp: np.ndarray, out_dir: str) -> None:
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda")
    T = tri.shape[0]
    B = pos.shape[0]
    S_lvl = scenes.feats_at_level(level)
    S_tot = scenes.total_feats(lo, hi)
    alpha_src = (1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.0, size=(T, S_lvl))))).astype(np.float32)
    feat_lvl = rng.uniform(0.0, 1.0, size=(T, S_lvl, C)).astype(np.float32)
    feat_ml = rng.normal(0.0, 0.3, size=(T, S_tot, C)).astype(np.float32)
    rec = dict(pos=pos, tri=tri, H=H, W=W, level=level, lo=lo, hi=hi, alpha_src=alpha_src, feat_lvl=feat_lvl,
               feat_ml=feat_ml, inv_mvp=inv_mvp.astype(np.float32))
    tp = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    for build in ("fma", "nofma"):
        R = Ref(build)
        pos_t, tri_t = tp(pos), tp(tri)
        fpix, fattr = R.compute_fragments(H, W, pos_t, tri_t)
        rects = R.last_rects.cpu().numpy()
        prefix = R.last_prefix.cpu().numpy()
        alpha = R.multires_alpha(fattr, level, level, tp(alpha_src))
        rast, *_ = R.rasterize_alpha(H, W, pos_t, tri_t, level, tp(alpha_src))

        def thr_fn(fp, fa, _seed=1234, _it=7):
            return tp(ocpu.fragment_thresholds(fp.cpu().numpy(), fa.cpu().numpy(), W, True, _seed, _it))

        rast_st, *_ = R.rasterize_alpha(H, W, pos_t, tri_t, level, tp(alpha_src), thr_fn)
        col = R.multires_color(rast, level, level, tp(feat_lvl))
        col_ml = R.multires_color(rast, lo, hi, tp(feat_ml))
        g_out = tp(rng.normal(0.0, 1.0, size=(B, H, W, C)).astype(np.float32))
        gfeat = R.multires_color_backward(rast, level, level, (T, S_lvl, C), g_out)
        sh = R.encode_sh2(rast, tp(inv_mvp.astype(np.float32)))
        # a rendering-like colour: background 1, foreground from the features
        mask = (rast[..., 3:4] > 0).float()
        color = (mask * col[..., :3] + (1.0 - mask)).contiguous()
        gcol = tp(rng.normal(0.0, 1e-3, size=(B, H, W, 3)).astype(np.float32))
        gpos = R.edge_grad(color, gcol, rast, pos_t, tri_t)
        target = tp(rng.uniform(0.0, 1.0, size=(B, H, W, 3)).astype(np.float32))
        gas, afpix, afattr, aalpha, agfa = R.opacity_aux(color, target, rast, pos_t, tri_t, level, tp(alpha_src))
        acc = R.accumulate_forward(lo, hi, hi, tp(feat_ml), scenes.feats_at_level(hi))
        acc_g_out = tp(rng.normal(0.0, 1.0, size=acc.shape).astype(np.float32))
        acc_g = R.accumulate_backward(lo, hi, hi, (T, S_tot, C), acc_g_out)

        fp_np, fa_np, al_np = fpix.cpu().numpy(), fattr.cpu().numpy(), alpha.cpu().numpy()
        order = np.lexsort((fp_np[:, 2], fp_np[:, 1], fa_np[:, 3], fp_np[:, 0]))
        ap_np, aa_np, ag_np = afpix.cpu().numpy(), afattr.cpu().numpy(), agfa.cpu().numpy()
        aorder = np.lexsort((ap_np[:, 2], ap_np[:, 1], aa_np[:, 3], ap_np[:, 0]))
        k = build + "_"
        rec.update({
            k + "rects": rects, k + "prefix": prefix,
            k + "frag_pix": fp_np[order], k + "frag_attrs": fa_np[order], k + "frag_alpha": al_np[order],
            k + "rast": rast.cpu().numpy(), k + "rast_stoch": rast_st.cpu().numpy(),
            k + "color_lvl": col.cpu().numpy(), k + "color_ml": col_ml.cpu().numpy(),
            k + "grad_out": g_out.cpu().numpy(), k + "grad_feat": gfeat.cpu().numpy(),
            k + "sh2": sh.cpu().numpy(), k + "color": color.cpu().numpy(), k + "grad_color": gcol.cpu().numpy(),
            k + "grad_pos": gpos.cpu().numpy(), k + "target": target.cpu().numpy(),
            k + "aux_grad_alpha_src": gas.cpu().numpy(), k + "aux_grad_frag": ag_np[aorder],
            k + "acc": acc.cpu().numpy(), k + "acc_grad_out": acc_g_out.cpu().numpy(), k + "acc_grad": acc_g.cpu().numpy(),
        })
    path = os.path.join(out_dir, f"{name}.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {path}  T={T} B={B} {H}x{W}  frags={rec['fma_frag_pix'].shape[0]}")


def main(out_dir: str) -> None:
    os.makedirs(out_dir, exist_ok=True)
    # config 1 restated small: 200 triangles, 2 views of 48x40, levels 0..2
    sc = scenes.make_scene(1, seed=11, num_tris=200, num_views=2, resolution=(40, 48), with_targets=False)
    run_case("config1_small", sc.clip_positions(), sc.tri, 40, 48, level=2, lo=0, hi=2, C=8, seed=101,
             inv_mvp=sc.inv_mvps(), out_dir=out_dir)
    # config 2 restated small: 300 triangles on the shell, 2 ring views of 48x48
    sc = scenes.make_scene(2, seed=12, num_tris=300, num_views=2, resolution=(48, 48), with_targets=False)
    run_case("config2_small", sc.clip_positions(), sc.tri, 48, 48, level=1, lo=0, hi=3, C=4, seed=102,
             inv_mvp=sc.inv_mvps(), out_dir=out_dir)
    pos, tri, H, W = edge_case_scene()
    inv = np.stack([np.eye(4, dtype=np.float32)] * 2)
    inv[:, 2, 3] = 0.5
    run_case("edge_cases", pos, tri, H, W, level=0, lo=0, hi=1, C=3, seed=103, inv_mvp=inv, out_dir=out_dir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))

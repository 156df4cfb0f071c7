"""Generates tests/golden/viewer_lut.npz: the viewer's LUT packing and MLP
weight extraction as the reference's own benchmark script computes them.

pack_face_color_lut, level_size and extract_mlp_weights are taken from the
reference's examples/05_benchmark_fps.py (the module itself imports the
OpenGL viewer, so only these function definitions are executed); the RGBA8
conversion is the expression of its lines 316-317.  Three seeded cases: a
small soup whose texels fit one LUT row, one that spans several padded rows
(more than 4096 texels), and values outside [0, 1] that the conversion clips.
Run from the repository root:

    python tests/golden/make_golden_viewer.py /path/to/reference
"""

import ast
import os
import sys
from collections import OrderedDict

import numpy as np
import torch

WANTED = ("level_size", "pack_face_color_lut", "extract_mlp_weights")


def load_reference_functions(ref_root: str) -> dict:
    path = os.path.join(ref_root, "examples", "05_benchmark_fps.py")
    tree = ast.parse(open(path).read(), path)
    defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in WANTED]
    assert {d.name for d in defs} == set(WANTED), [d.name for d in defs]
    mod = ast.Module(body=defs, type_ignores=[])
    ns = {"np": np, "math": __import__("math")}
    exec(compile(mod, path, "exec"), ns)
    return ns


def reference_dir() -> str:
    """The reference checkout: $DIFFSOUP_REFERENCE, else a `reference`
    directory beside this repository."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    return os.environ.get("DIFFSOUP_REFERENCE") or os.path.join(os.path.dirname(root), "reference")


def main(ref_root: str) -> None:
    ns = load_reference_functions(ref_root)
    rng = np.random.default_rng(77)
    out = {}
    for name, (faces, level, lo, hi) in {"small": (6, 2, 0.0, 1.0), "rows": (95, 3, 0.0, 1.0),
                                         "clip": (40, 2, -0.3, 1.3)}.items():
        S = ns["level_size"](level)
        feat = rng.uniform(lo, hi, (faces, S, 7)).astype(np.float32)
        alpha = rng.uniform(lo, hi, (faces, S, 1)).astype(np.float32)
        lut = ns["pack_face_color_lut"](feat, alpha, faces, level)
        lut0 = (lut[..., :4] * 255).clip(0, 255).astype(np.uint8)
        lut1 = (lut[..., 4:] * 255).clip(0, 255).astype(np.uint8)
        out.update({f"{name}_feat": feat, f"{name}_alpha": alpha, f"{name}_level": np.int32(level),
                    f"{name}_lut": lut, f"{name}_lut0": lut0, f"{name}_lut1": lut1})
    # a ColorMLP-shaped state dict: Sequential of Linear(16,16) ReLU Linear(16,16) ReLU Linear(16,3) Sigmoid
    sd = OrderedDict()
    for i, (o, n) in zip((0, 2, 4), ((16, 16), (16, 16), (3, 16))):
        sd[f"mlp.{i}.weight"] = torch.from_numpy(rng.normal(0, 0.3, (o, n)).astype(np.float32))
        sd[f"mlp.{i}.bias"] = torch.from_numpy(rng.normal(0, 0.1, (o,)).astype(np.float32))
    W1, b1, W2, b2, W3, b3 = ns["extract_mlp_weights"](sd)
    for k, v in sd.items():
        out["sd_" + k] = v.numpy()
    out.update(mlp_W1=W1, mlp_b1=b1, mlp_W2=W2, mlp_b2=b2, mlp_W3=W3, mlp_b3=b3)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "viewer_lut.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, sorted(out))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_dir())

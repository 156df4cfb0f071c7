"""Generates tests/golden/point3d.npz: the reference's point-cloud helpers
(python/diffsoup/point3d.py, imported from its source file: it needs only
numpy, scipy and torch) on seeded inputs.  Run from the repository root:

    python tests/golden/make_golden_point3d.py /path/to/reference
"""

import importlib.util
import os
import sys

import numpy as np
import torch


def reference_dir() -> str:
    """The reference checkout: $DIFFSOUP_REFERENCE, else a `reference`
    directory beside this repository."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    return os.environ.get("DIFFSOUP_REFERENCE") or os.path.join(os.path.dirname(root), "reference")


def main(ref_root: str) -> None:
    spec = importlib.util.spec_from_file_location("ref_point3d", os.path.join(ref_root, "python", "diffsoup",
                                                                              "point3d.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rng = np.random.default_rng(31)
    out = {}
    clouds = {"uniform": rng.uniform(-1, 1, (3000, 3)).astype(np.float32),
              "clustered": np.concatenate([rng.normal(c, 0.05, (400, 3)) for c in rng.uniform(-2, 2, (5, 3))])
              .astype(np.float32),
              "duplicates": np.repeat(rng.uniform(0, 1, (50, 3)).astype(np.float32), 2, axis=0)}
    for name, P in clouds.items():
        out[f"{name}_points"] = P
        out[f"{name}_median"] = np.float64(mod.nn_spacing(P, "median"))
        out[f"{name}_mean"] = np.float64(mod.nn_spacing(P, "mean"))
    V = torch.from_numpy(rng.normal(0, 1, (60, 3)).astype(np.float32))
    F = torch.from_numpy(rng.choice(60, (25, 3)).astype(np.int32))
    nv, nf = mod.remove_unreferenced_vertices_from_soup(V, F)
    out.update(ru_verts=V.numpy(), ru_faces=F.numpy(), ru_new_verts=nv.numpy(), ru_new_faces=nf.numpy())
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "point3d.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_dir())

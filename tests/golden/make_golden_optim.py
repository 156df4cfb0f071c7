"""Generates tests/golden/optim.npz: the reference's own optimisers run on CPU.

VectorAdam is imported from the reference's source file
(python/diffsoup/optimize.py; the package itself needs its compiled
extension, this module only needs torch), Adam is torch.optim.Adam with the
reference's usage (examples/02_synthetic.py:310-315).  Five steps each with
seeded gradients; run from the repository root:

    python tests/golden/make_golden_optim.py /path/to/reference
"""

import importlib.util
import os
import sys

import numpy as np
import torch

STEPS = 5


def reference_dir() -> str:
    """The reference checkout: $DIFFSOUP_REFERENCE, else a `reference`
    directory beside this repository."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    return os.environ.get("DIFFSOUP_REFERENCE") or os.path.join(os.path.dirname(root), "reference")


def main(ref_root: str) -> None:
    spec = importlib.util.spec_from_file_location("ref_optimize", os.path.join(ref_root, "python", "diffsoup",
                                                                               "optimize.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rng = np.random.default_rng(2024)
    out = {}
    # VectorAdam on vertex positions [V, 3]
    p0 = rng.normal(0, 1, (200, 3)).astype(np.float32)
    grads = rng.normal(0, 1e-2, (STEPS, 200, 3)).astype(np.float32)
    grads[:, :5] = 0.0  # rows without gradient (the state still decays)
    p = torch.tensor(p0, requires_grad=True)
    opt = mod.VectorAdam([p], lr=1e-3, betas=(0.9, 0.999))
    for s in range(STEPS):
        p.grad = torch.tensor(grads[s])
        opt.step()
    st = opt.state[p]
    out.update(va_p0=p0, va_grads=grads, va_p=p.detach().numpy(), va_g1=st["g1"].numpy(), va_g2=st["g2"].numpy())
    # Adam on a feature tensor (n % 4 != 0) and an MLP weight (n % 4 == 0)
    for name, shape, lr in (("adam_feat", (37, 5), 5e-2), ("adam_mlp", (16, 12), 1e-2)):
        q0 = rng.normal(0, 0.5, shape).astype(np.float32)
        qg = rng.normal(0, 1e-1, (STEPS,) + shape).astype(np.float32)
        q = torch.tensor(q0, requires_grad=True)
        opt = torch.optim.Adam([q], lr=lr, foreach=False)
        for s in range(STEPS):
            q.grad = torch.tensor(qg[s])
            opt.step()
        st = opt.state[q]
        out.update({f"{name}_p0": q0, f"{name}_grads": qg, f"{name}_p": q.detach().numpy(),
                    f"{name}_m": st["exp_avg"].numpy(), f"{name}_v": st["exp_avg_sq"].numpy(),
                    f"{name}_lr": np.float32(lr)})
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "optim.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_dir())

"""Optimiser updates restated in NumPy FP64: the checker of the fused CUDA
updates (diffsoup_b200/csrc/optim.cu).

TEST INFRASTRUCTURE ONLY: used by tests/ to check the product's kernels.

  vector_adam_step  python/diffsoup/optimize.py:36-68 (VectorAdam.step)
  adam_step         torch.optim.Adam's update without weight decay or amsgrad
                    (the optimiser examples/02_synthetic.py:310-315 uses)

Pinned against the reference's own VectorAdam and torch.optim.Adam run on CPU
(tests/golden/make_golden_optim.py -> tests/golden/optim.npz).
"""

from __future__ import annotations

import numpy as np


def vector_adam_step(p, g, g1, g2, t: int, lr: float, b1: float, b2: float):
    """One VectorAdam update of p [..., D] at step t (1-based); returns (p, g1, g2)."""
    p, g, g1, g2 = (np.asarray(x, np.float64) for x in (p, g, g1, g2))
    g1 = b1 * g1 + (1.0 - b1) * g
    g2 = b2 * g2 + (1.0 - b2) * (g * g).sum(axis=-1, keepdims=True)
    m1 = g1 / (1.0 - b1 ** t)
    m2 = g2 / (1.0 - b2 ** t)
    return p - lr * m1 / (np.sqrt(m2) + 1e-8), g1, g2


def adam_step(p, g, m, v, t: int, lr: float, b1: float, b2: float, eps: float):
    """One Adam update at step t (1-based); returns (p, exp_avg, exp_avg_sq)."""
    p, g, m, v = (np.asarray(x, np.float64) for x in (p, g, m, v))
    m = m + (1.0 - b1) * (g - m)
    v = b2 * v + (1.0 - b2) * g * g
    denom = np.sqrt(v) / np.sqrt(1.0 - b2 ** t) + eps
    return p - lr / (1.0 - b1 ** t) * m / denom, m, v

"""The optimiser oracle (oracle/optim.py) against the reference's own
VectorAdam and torch.optim.Adam (tests/golden/optim.npz)."""

import os

import numpy as np

from oracle import optim

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "optim.npz"))


def test_vector_adam_restatement_matches_reference():
    p, g1, g2 = G["va_p0"], np.zeros_like(G["va_p0"]), np.zeros(G["va_p0"].shape[:-1] + (1,))
    for s, grad in enumerate(G["va_grads"]):
        p, g1, g2 = optim.vector_adam_step(p, grad, g1, g2, s + 1, 1e-3, 0.9, 0.999)
    np.testing.assert_allclose(p, G["va_p"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(g1, G["va_g1"], rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(g2, G["va_g2"], rtol=1e-5, atol=1e-12)


def test_adam_restatement_matches_torch():
    for name in ("adam_feat", "adam_mlp"):
        p = G[f"{name}_p0"]
        m, v = np.zeros_like(p), np.zeros_like(p)
        for s, grad in enumerate(G[f"{name}_grads"]):
            p, m, v = optim.adam_step(p, grad, m, v, s + 1, float(G[f"{name}_lr"]), 0.9, 0.999, 1e-8)
        np.testing.assert_allclose(p, G[f"{name}_p"], rtol=0, atol=1e-6)
        np.testing.assert_allclose(m, G[f"{name}_m"], rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(v, G[f"{name}_v"], rtol=1e-5, atol=1e-12)

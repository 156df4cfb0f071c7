"""The packed MLP parameter layout of the training step, on the host.

ds_train_step reads the ColorMLP's parameters as one fp32 vector
[W0, b0, (W1, b1), Wout, bout] (torch.nn.Linear order) and writes their
gradients in the same layout.  pack_mlp flattens a ColorMLP that way and
unpack_mlp_grads writes such a gradient back into the module's .grad, so a
torch optimiser can take the step's MLP gradients.
"""

import pytest
import torch

from diffsoup_b200.multires import ColorMLP
from diffsoup_b200.step import _L, pack_mlp, unpack_mlp_grads


@pytest.mark.parametrize("C_,enc,hidden,n_layers", [(8, 3, 16, 1), (7, 9, 16, 2), (16, 3, 64, 2)])
def test_pack_and_unpack_follow_the_step_layout(C_, enc, hidden, n_layers):
    torch.manual_seed(0)
    mlp = ColorMLP(C_ + enc, 3, hidden_dim=hidden, n_layers=n_layers)
    flat = pack_mlp(mlp)
    # the library's count (its W0 has C + 3 columns; SH2 adds 6 more inputs)
    assert flat.numel() == _L.ds_mlp_param_count(C_ + enc - 3, hidden, n_layers)
    assert flat.dtype == torch.float32 and flat.is_contiguous()
    lins = [m for m in mlp.modules() if isinstance(m, torch.nn.Linear)]
    assert [tuple(l.weight.shape) for l in lins] == (
        [(hidden, C_ + enc)] + [(hidden, hidden)] * (n_layers - 1) + [(3, hidden)])
    o = 0
    for lin in lins:
        for p in (lin.weight, lin.bias):
            assert torch.equal(flat[o:o + p.numel()], p.detach().reshape(-1))
            o += p.numel()
    assert o == flat.numel()
    # a packed gradient lands in .grad of the matching parameter
    grad = torch.arange(flat.numel(), dtype=torch.float32)
    unpack_mlp_grads(grad, mlp)
    o = 0
    for lin in lins:
        for p in (lin.weight, lin.bias):
            assert p.grad.shape == p.shape
            assert torch.equal(p.grad.reshape(-1), grad[o:o + p.numel()])
            o += p.numel()
    # .grad holds copies: the packed vector can be reused by the next step
    grad.zero_()
    assert float(lins[-1].bias.grad.sum()) > 0

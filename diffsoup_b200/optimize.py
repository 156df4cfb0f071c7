"""Optimisers of the training loop, as fused CUDA updates.

`VectorAdam` keeps the interface of the reference's optimiser
(python/diffsoup/optimize.py:7-68: VectorAdam(params, lr=1e-3,
betas=(0.9, 0.999)), step()) and `Adam` that of torch.optim.Adam as
examples/02_synthetic.py:310-315 uses it (lr, betas, eps; no weight decay or
amsgrad).  Each parameter is updated by one kernel of libdiffsoup_b200.so
(ds_vector_adam_step / ds_adam_step) on torch's current stream.  The step
count is a device int32 in the parameter's state (state["step"]), advanced by
the kernel, so an update can be captured in a CUDA graph together with the
training step; the reference keeps it as a Python int.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _core

_L = _core.lib
_L.ds_adam_step.restype = C.c_int
_L.ds_adam_step.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                               C.c_void_p, C.c_void_p]
_L.ds_vector_adam_step.restype = C.c_int
_L.ds_vector_adam_step.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int, C.c_double, C.c_double, C.c_double,
                                                      C.c_void_p, C.c_void_p]


def _check(p: torch.Tensor, g: torch.Tensor) -> None:
    if not (p.is_cuda and p.dtype == torch.float32 and p.is_contiguous()):
        raise RuntimeError("diffsoup_b200.optimize: parameters must be contiguous float32 CUDA tensors")
    if not (g.is_cuda and g.dtype == torch.float32 and g.is_contiguous() and g.shape == p.shape):
        raise RuntimeError("diffsoup_b200.optimize: the gradient must be a contiguous float32 CUDA tensor "
                           "of the parameter's shape")


class VectorAdam(torch.optim.Optimizer):
    """Adam with one second moment per vector of the last dimension
    (Ling, Sharp and Jacobson, "VectorAdam for Rotation Equivariant Geometry
    Optimization", NeurIPS 2022), as python/diffsoup/optimize.py:7-68."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999)):
        defaults = dict(lr=lr, betas=betas)
        super().__init__(params, defaults)

    @torch.no_grad()
    def step(self):
        for group in self.param_groups:
            lr = group["lr"]
            b1, b2 = group["betas"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                g = p.grad
                _check(p, g)
                state = self.state[p]
                if len(state) == 0:
                    state["step"] = torch.zeros(1, dtype=torch.int32, device=p.device)
                    state["g1"] = torch.zeros_like(p)
                    state["g2"] = torch.zeros_like(p[..., :1])
                dim = p.shape[-1] if p.dim() > 0 else 1
                _core.check(_L.ds_vector_adam_step(_core.ptr(p), _core.ptr(g), _core.ptr(state["g1"]),
                                                   _core.ptr(state["g2"]), p.numel() // dim, dim, lr, b1, b2,
                                                   _core.ptr(state["step"]), _core.stream()))


class Adam(torch.optim.Optimizer):
    """torch.optim.Adam's update (no weight decay, no amsgrad) as one fused
    kernel per parameter."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        defaults = dict(lr=lr, betas=betas, eps=eps)
        super().__init__(params, defaults)

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        for group in self.param_groups:
            lr, eps = group["lr"], group["eps"]
            b1, b2 = group["betas"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                g = p.grad
                _check(p, g)
                state = self.state[p]
                if len(state) == 0:
                    state["step"] = torch.zeros(1, dtype=torch.int32, device=p.device)
                    state["exp_avg"] = torch.zeros_like(p)
                    state["exp_avg_sq"] = torch.zeros_like(p)
                _core.check(_L.ds_adam_step(_core.ptr(p), _core.ptr(g), _core.ptr(state["exp_avg"]),
                                            _core.ptr(state["exp_avg_sq"]), p.numel(), lr, b1, b2, eps,
                                            _core.ptr(state["step"]), _core.stream()))
        return loss

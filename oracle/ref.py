"""ctypes wrapper of oracle/_ref/libdsref*.so: the reference's own CUDA
launchers (kenji-tojo/diffsoup src/cuda/*.cu, unmodified) behind the plain C
entry points of oracle/ref_capi.cu.

TEST INFRASTRUCTURE ONLY.  It reproduces the reference's `_core` calls
(src/main.cpp:30-304) on torch CUDA tensors so that tests and the golden
fixture script can run the reference path itself.  The libraries are built in
the development container by `make -C oracle ref` and travel with the tree.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Tuple

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
BUILDS = {"fma": os.path.join(HERE, "_ref", "libdsref.so"), "nofma": os.path.join(HERE, "_ref", "libdsref_nofma.so")}
_libs = {}


def available(build: str = "fma") -> bool:
    return os.path.exists(BUILDS[build])


def lib(build: str = "fma") -> C.CDLL:
    if build not in _libs:
        L = C.CDLL(BUILDS[build])
        vp, i = C.c_void_p, C.c_int
        L.dsref_compute_triangle_rects.restype = i
        L.dsref_compute_triangle_rects.argtypes = [i, i, i, i, vp, i, vp, vp, vp]
        L.dsref_compute_fragments.argtypes = [i, i, i, i, vp, i, vp, vp, vp, i, vp, vp]
        L.dsref_depth_test.argtypes = [i, i, i, i, vp, vp, vp, vp, vp]
        L.dsref_filter_valid_fragments.restype = i
        L.dsref_filter_valid_fragments.argtypes = [i, vp, vp, vp, vp]
        L.dsref_backward_edge_grad.argtypes = [i, i, i, i, vp, vp, vp, i, vp, vp, vp]
        L.dsref_backward_opacity_aux_loss.argtypes = [i, i, i, i, vp, vp, vp, i, vp, vp, vp, vp]
        L.dsref_encode_view_dir_sh2.argtypes = [i, i, i, vp, vp, vp]
        L.dsref_multires_triangle_alpha.argtypes = [i, vp, i, i, vp, vp]
        L.dsref_backward_multires_triangle_alpha.argtypes = [i, vp, i, i, vp, vp]
        L.dsref_multires_triangle_color.argtypes = [i, i, i, vp, i, i, i, vp, vp]
        L.dsref_backward_multires_triangle_color.argtypes = [i, i, i, vp, i, i, i, vp, vp]
        L.dsref_accumulate_to_level_forward.argtypes = [i, i, i, i, i, vp, vp]
        L.dsref_accumulate_to_level_backward.argtypes = [i, i, i, i, i, vp, vp]
        L.dsref_device_synchronize.restype = i
        _libs[build] = L
    return _libs[build]


def _p(t: torch.Tensor) -> C.c_void_p:
    assert t.is_cuda and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def _sync(build: str) -> None:
    torch.cuda.synchronize()
    rc = lib(build).dsref_device_synchronize()
    assert rc == 0, f"reference CUDA error {rc}"


class Ref:
    """The reference's Python-level composites (rasterize.py, multires.py) over
    one build of its CUDA sources."""

    def __init__(self, build: str = "fma", sync: bool = True):
        """sync=False leaves out the device synchronisation after each launch
        (kept where the reference itself reads a count back), for timing the
        reference's path as its Python layer runs it: the launchers and torch
        share the legacy default stream, so the order holds without it."""
        self.build = build
        self.L = lib(build)
        self.sync = sync

    def _done(self) -> None:
        if self.sync:
            _sync(self.build)

    def compute_fragments(self, H: int, W: int, pos: torch.Tensor, tri: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        """rasterize.py:40-76"""
        torch.cuda.synchronize()
        B, V, _ = pos.shape
        T = tri.shape[0]
        dev = pos.device
        rects = torch.empty((B * T, 4), dtype=torch.int32, device=dev)
        prefix = torch.empty(B * T, dtype=torch.int32, device=dev)
        n = self.L.dsref_compute_triangle_rects(H, W, B, V, _p(pos), T, _p(tri), _p(rects), _p(prefix)) if B * T else 0
        fpix = torch.full((n, 3), -1, dtype=torch.int32, device=dev)
        fattr = torch.empty((n, 4), dtype=torch.float32, device=dev)
        if n:
            self.L.dsref_compute_fragments(H, W, B, V, _p(pos), T, _p(tri), _p(prefix), _p(rects), n, _p(fpix), _p(fattr))
        po = torch.empty_like(fpix)
        ao = torch.empty_like(fattr)
        k = self.L.dsref_filter_valid_fragments(n, _p(fpix), _p(fattr), _p(po), _p(ao)) if n else 0
        self._done()
        self.last_rects, self.last_prefix = rects, prefix
        return po[:k].contiguous(), ao[:k].contiguous()

    def multires_alpha(self, frag_attrs, lo, hi, alpha_src_2d):
        out = torch.zeros(frag_attrs.shape[0], dtype=torch.float32, device=frag_attrs.device)
        if frag_attrs.shape[0]:
            self.L.dsref_multires_triangle_alpha(frag_attrs.shape[0], _p(frag_attrs), lo, hi, _p(alpha_src_2d), _p(out))
        self._done()
        return out

    def depth_test(self, B, H, W, frag_pix, frag_attrs, frag_alpha, thresh):
        rast = torch.zeros(B, H, W, 4, dtype=torch.float32, device=frag_pix.device)
        if frag_pix.shape[0]:
            self.L.dsref_depth_test(B, H, W, frag_pix.shape[0], _p(frag_pix), _p(frag_attrs), _p(frag_alpha),
                                    _p(thresh), _p(rast))
        self._done()
        return rast

    def rasterize_alpha(self, H, W, pos, tri, level, alpha_src, thresh_fn=None):
        """multires.py:52-102 with thresholds from thresh_fn(frag_pix, frag_attrs)
        (default 0.5, i.e. stochastic=False)."""
        fpix, fattr = self.compute_fragments(H, W, pos, tri)
        alpha = self.multires_alpha(fattr, level, level, alpha_src.reshape(tri.shape[0], -1).contiguous())
        if thresh_fn is None:
            thr = torch.full_like(alpha, 0.5)
        else:
            thr = thresh_fn(fpix, fattr)
        return self.depth_test(pos.shape[0], H, W, fpix, fattr, alpha, thr), fpix, fattr, alpha

    def multires_color(self, rast, lo, hi, feat):
        B, H, W, _ = rast.shape
        out = torch.zeros(B, H, W, feat.shape[2], dtype=torch.float32, device=rast.device)
        self.L.dsref_multires_triangle_color(B, H, W, _p(rast), lo, hi, feat.shape[2], _p(feat), _p(out))
        self._done()
        return out

    def multires_color_backward(self, rast, lo, hi, feat_shape, grad_out):
        B, H, W, _ = rast.shape
        g = torch.zeros(feat_shape, dtype=torch.float32, device=rast.device)
        self.L.dsref_backward_multires_triangle_color(B, H, W, _p(rast), lo, hi, feat_shape[2], _p(g), _p(grad_out))
        self._done()
        return g

    def encode_sh2(self, rast, inv_mvp):
        B, H, W, _ = rast.shape
        enc = torch.zeros(B, H, W, 9, dtype=torch.float32, device=rast.device)
        self.L.dsref_encode_view_dir_sh2(B, H, W, _p(rast), _p(inv_mvp), _p(enc))
        self._done()
        return enc

    def edge_grad(self, color, grad_color, rast, pos, tri):
        B, H, W, Cd = color.shape
        gp = torch.zeros_like(pos)
        self.L.dsref_backward_edge_grad(B, H, W, Cd, _p(color), _p(grad_color), _p(rast), pos.shape[1], _p(pos),
                                        _p(gp), _p(tri))
        self._done()
        return gp

    def opacity_aux(self, color, target, rast, pos, tri, level, alpha_src_2d):
        """_OpacityAuxLossFn.forward (rasterize.py:147-190), unscaled grad_alpha_src."""
        B, H, W, Cd = color.shape
        fpix, fattr = self.compute_fragments(H, W, pos, tri)
        nf = fpix.shape[0]
        alpha = self.multires_alpha(fattr, level, level, alpha_src_2d)
        gfa = torch.zeros_like(alpha)
        if nf:
            self.L.dsref_backward_opacity_aux_loss(B, H, W, Cd, _p(color), _p(target), _p(rast), nf, _p(fpix),
                                                   _p(fattr), _p(alpha), _p(gfa))
        gas = torch.zeros_like(alpha_src_2d)
        if nf:
            self.L.dsref_backward_multires_triangle_alpha(nf, _p(fattr), level, level, _p(gas), _p(gfa))
        self._done()
        return gas, fpix, fattr, alpha, gfa

    def accumulate_forward(self, lo, hi, target, feat, S_target):
        T, _, Cd = feat.shape
        out = torch.zeros(T, S_target, Cd, dtype=torch.float32, device=feat.device)
        self.L.dsref_accumulate_to_level_forward(T, lo, hi, target, Cd, _p(feat), _p(out))
        self._done()
        return out

    def accumulate_backward(self, lo, hi, target, feat_shape, grad_out):
        T, _, Cd = feat_shape
        g = torch.zeros(feat_shape, dtype=torch.float32, device=grad_out.device)
        self.L.dsref_accumulate_to_level_backward(T, lo, hi, target, Cd, _p(g), _p(grad_out))
        self._done()
        return g

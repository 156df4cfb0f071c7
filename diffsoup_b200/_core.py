"""ctypes binding of libdiffsoup_b200.so with the reference's `_core` names.

The reference exposes a nanobind module `_core` (kenji-tojo/diffsoup
src/main.cpp:24-304) whose functions take contiguous CUDA tensors.  This module
keeps those names, argument orders and shape checks, and calls the C ABI of
include/diffsoup_b200.h on torch's current CUDA stream.  Shape mismatches raise
RuntimeError("Invalid feature size.") like the reference; CUDA errors raise
RuntimeError instead of exiting the process.

There is no fallback: if the shared library is missing, importing this module
raises ImportError (build it with `python -c "import __graft_entry__ as g;
g.build()"` or `make -C diffsoup_b200/csrc`).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import torch

__version__ = "0.1.0"

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libdiffsoup_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"diffsoup_b200: {LIB_PATH} is missing; build the CUDA library first "
                      "(make -C diffsoup_b200/csrc)")

_lib = C.CDLL(LIB_PATH)

_vp, _i32, _i64, _f32, _sz = C.c_void_p, C.c_int, C.c_int64, C.c_float, C.c_size_t


class ViewDesc(C.Structure):
    _fields_ = [("H", C.c_int32), ("W", C.c_int32), ("tiles_x", C.c_int32), ("tiles_y", C.c_int32),
                ("pix_offset", C.c_int64), ("tile_base", C.c_int32), ("pad", C.c_int32)]


def _sig(name, restype, *args):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = list(args)
    return f


_sig("ds_last_error", C.c_char_p)
_sig("ds_version", C.c_char_p)
_sig("ds_compute_triangle_rects_workspace", _sz, _i32, _i32)
_sig("ds_compute_triangle_rects", _i32, _i32, _i32, _i32, _i32, _vp, _i32, _vp, _vp, _vp, C.POINTER(C.c_int), _vp,
     _sz, _vp)
_sig("ds_compute_fragments", _i32, _i32, _i32, _i32, _i32, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp)
_sig("ds_filter_valid_fragments_workspace", _sz, _i32)
_sig("ds_filter_valid_fragments", _i32, _i32, _vp, _vp, _vp, _vp, C.POINTER(C.c_int), _vp, _sz, _vp)
_sig("ds_depth_test_workspace", _sz, _i32, _i32, _i32)
_sig("ds_depth_test", _i32, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp)
_sig("ds_backward_edge_grad", _i32, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp)
_sig("ds_backward_opacity_aux_loss", _i32, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp)
_sig("ds_encode_view_dir_sh2", _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp)
_sig("ds_encode_view_dir", _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp)
_sig("ds_count_triangle_ids", _i32, _i64, _vp, _i32, _vp, _vp, _vp)
_sig("ds_multires_triangle_alpha", _i32, _i32, _vp, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("ds_backward_multires_triangle_alpha", _i32, _i32, _vp, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("ds_multires_triangle_color", _i32, _i32, _i32, _i32, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("ds_backward_multires_triangle_color", _i32, _i32, _i32, _i32, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("ds_accumulate_to_level_forward", _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("ds_accumulate_to_level_backward", _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("ds_make_view_table", _i32, _i32, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(ViewDesc),
     C.POINTER(C.c_int64))
_sig("ds_tiles_workspace_size", _sz, _i32, _i32, _i32, _i64)
_sig("ds_tiles_bin", _i32, _i32, _vp, _i32, _i32, _vp, _i32, _vp, _vp, _sz, _i64, _vp, _vp)
_sig("ds_tiles_rasterize", _i32, _i32, _vp, _i32, _i32, _vp, _i32, _vp, _i32, _i32, _vp, _i32, _f32, _vp, _vp, _vp,
     _sz, _i64, _vp)
_sig("ds_tiles_opacity_aux", _i32, _i32, _vp, _i32, _i32, _vp, _i32, _vp, _i32, _i32, _vp, _i32, _vp, _vp, _vp, _f32,
     _vp, _vp, _sz, _i64, _vp)
_sig("ds_project_vertices", _i32, _i32, _i32, _vp, _vp, _vp, _vp)
_sig("ds_split_soup_workspace_size", _sz, _i32)
_sig("ds_split_soup_count", _i32, _i32, _vp, _f32, _f32, _i32, _i32, _vp, _i32, _vp, _vp, _vp,
     C.POINTER(C.c_int64), _vp, _sz, _vp, _vp)
_sig("ds_split_soup_emit", _i32, _i32, _vp, _f32, _i32, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp)
_sig("ds_render_lut_opacity", _i32, _i64, _vp, _vp, _vp)
_sig("ds_render_deferred", _i32, _i32, _vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _f32, _f32, _f32, _vp, _vp, _vp)
_sig("ds_render_workspace_size", _sz, _i32, _i32, _i32, _i32, _i64)
_sig("ds_render_frame", _i32, _i32, _vp, _i32, _i64, _i32, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _i64, _vp, _vp,
     _f32, _f32, _f32, _vp, _vp, _vp, _vp, _sz, _i64, _vp, _vp)

lib = _lib


def version() -> str:
    return _lib.ds_version().decode()


def check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(_lib.ds_last_error().decode())


def ptr(t: Optional[torch.Tensor]) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    return C.c_void_p(t.data_ptr())


def stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _cuda_contig(name: str, t: torch.Tensor, dtype: torch.dtype, ndim: int) -> None:
    if not isinstance(t, torch.Tensor) or t.dtype != dtype or not t.is_contiguous() or not t.is_cuda or t.dim() != ndim:
        raise RuntimeError(f"{name}: expected a contiguous CUDA {dtype} tensor with {ndim} dims")


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def feats_at_level(level: int) -> int:
    return 3 if level == 0 else ((1 << (level - 1)) + 1) * ((1 << level) + 1)


def total_feats(lo: int, hi: int) -> int:
    return sum(feats_at_level(l) for l in range(lo, hi + 1))


# ---------------------------------------------------------------------------
# `_core` functions (src/main.cpp:30-304), same names and arguments.
# ---------------------------------------------------------------------------

def compute_triangle_rects(H: int, W: int, pos: torch.Tensor, tri: torch.Tensor, triangle_rects: torch.Tensor,
                           frag_prefix_sum: torch.Tensor) -> int:
    """main.cpp:30-48"""
    _cuda_contig("pos", pos, torch.float32, 3)
    _cuda_contig("tri", tri, torch.int32, 2)
    B, V, _ = pos.shape
    T = tri.shape[0]
    ws = workspace(_lib.ds_compute_triangle_rects_workspace(B, T), pos.device)
    n = C.c_int(0)
    check(_lib.ds_compute_triangle_rects(H, W, B, V, ptr(pos), T, ptr(tri), ptr(triangle_rects), ptr(frag_prefix_sum),
                                         C.byref(n), ptr(ws), ws.numel(), stream()))
    return int(n.value)


def compute_fragments(H: int, W: int, pos, tri, frag_prefix_sum, triangle_rects, frag_pix, frag_attrs) -> None:
    """main.cpp:50-76"""
    B, V, _ = pos.shape
    T = tri.shape[0]
    check(_lib.ds_compute_fragments(H, W, B, V, ptr(pos), T, ptr(tri), ptr(frag_prefix_sum), ptr(triangle_rects),
                                    frag_pix.shape[0], ptr(frag_pix), ptr(frag_attrs), stream()))


def depth_test(frag_pix, frag_attrs, frag_alpha, alpha_thresh, rast_out) -> None:
    """main.cpp:78-94"""
    B, H, W, _ = rast_out.shape
    n = frag_pix.shape[0]
    ws = workspace(_lib.ds_depth_test_workspace(B, H, W), rast_out.device)
    check(_lib.ds_depth_test(B, H, W, n, ptr(frag_pix), ptr(frag_attrs), ptr(frag_alpha), ptr(alpha_thresh),
                             ptr(rast_out), ptr(ws), ws.numel(), stream()))


def filter_valid_fragments(frag_pix, frag_attrs, frag_pix_out, frag_attrs_out) -> int:
    """main.cpp:96-108"""
    n = frag_pix.shape[0]
    ws = workspace(_lib.ds_filter_valid_fragments_workspace(n), frag_pix.device)
    k = C.c_int(0)
    check(_lib.ds_filter_valid_fragments(n, ptr(frag_pix), ptr(frag_attrs), ptr(frag_pix_out), ptr(frag_attrs_out),
                                         C.byref(k), ptr(ws), ws.numel(), stream()))
    return int(k.value)


def backward_edge_grad(color, grad_color, rast, pos, grad_pos, tri) -> None:
    """main.cpp:112-130"""
    B, H, W, Cd = color.shape
    check(_lib.ds_backward_edge_grad(B, H, W, Cd, ptr(color), ptr(grad_color), ptr(rast), pos.shape[1], ptr(pos),
                                     ptr(grad_pos), ptr(tri), stream()))


def backward_opacity_aux_loss(color, target, rast, frag_pix, frag_attrs, frag_alpha, grad_frag_alpha) -> None:
    """main.cpp:134-154"""
    B, H, W, Cd = color.shape
    check(_lib.ds_backward_opacity_aux_loss(B, H, W, Cd, ptr(color), ptr(target), ptr(rast), frag_pix.shape[0],
                                            ptr(frag_pix), ptr(frag_attrs), ptr(frag_alpha), ptr(grad_frag_alpha),
                                            stream()))


def encode_view_dir_sh2(rast, inv_mvp, encoding) -> None:
    """main.cpp:158-170"""
    B, H, W, _ = rast.shape
    check(_lib.ds_encode_view_dir_sh2(B, H, W, ptr(rast), ptr(inv_mvp), ptr(encoding), stream()))


def encode_view_dir(rast, inv_mvp, encoding) -> None:
    """Raw 3-D view direction (encoding.cu:28-53, not exported by the reference)."""
    B, H, W, _ = rast.shape
    check(_lib.ds_encode_view_dir(B, H, W, ptr(rast), ptr(inv_mvp), ptr(encoding), stream()))


def multires_triangle_alpha(frag_attrs, min_level: int, max_level: int, alpha_src, frag_alpha) -> None:
    """main.cpp:174-191"""
    check(_lib.ds_multires_triangle_alpha(frag_attrs.shape[0], ptr(frag_attrs), min_level, max_level,
                                          alpha_src.shape[1], ptr(alpha_src), ptr(frag_alpha), stream()))


def backward_multires_triangle_alpha(frag_attrs, min_level: int, max_level: int, grad_alpha_src,
                                     grad_frag_alpha) -> None:
    """main.cpp:193-210"""
    check(_lib.ds_backward_multires_triangle_alpha(frag_attrs.shape[0], ptr(frag_attrs), min_level, max_level,
                                                   grad_alpha_src.shape[1], ptr(grad_alpha_src),
                                                   ptr(grad_frag_alpha), stream()))


def multires_triangle_color(rast, min_level: int, max_level: int, features, out) -> None:
    """main.cpp:212-232"""
    B, H, W, _ = rast.shape
    check(_lib.ds_multires_triangle_color(B, H, W, ptr(rast), min_level, max_level, features.shape[1],
                                          features.shape[2], ptr(features), ptr(out), stream()))


def backward_multires_triangle_color(rast, min_level: int, max_level: int, grad_features, grad_out) -> None:
    """main.cpp:234-254"""
    B, H, W, _ = rast.shape
    check(_lib.ds_backward_multires_triangle_color(B, H, W, ptr(rast), min_level, max_level, grad_features.shape[1],
                                                   grad_features.shape[2], ptr(grad_features), ptr(grad_out),
                                                   stream()))


def accumulate_to_level_forward(min_level: int, max_level: int, target_level: int, feat_all, feat_max) -> None:
    """main.cpp:258-280"""
    T, S, Cd = feat_all.shape
    check(_lib.ds_accumulate_to_level_forward(T, min_level, max_level, target_level, S, feat_max.shape[1], Cd,
                                              ptr(feat_all), ptr(feat_max), stream()))


def accumulate_to_level_backward(min_level: int, max_level: int, target_level: int, grad_feat_all,
                                 grad_feat_max) -> None:
    """main.cpp:282-304"""
    T, S, Cd = grad_feat_all.shape
    check(_lib.ds_accumulate_to_level_backward(T, min_level, max_level, target_level, S, grad_feat_max.shape[1], Cd,
                                               ptr(grad_feat_all), ptr(grad_feat_max), stream()))


def split_triangle_soup(verts, faces, numSplits: int, tau: float):
    """_core.split_triangle_soup (src/main.cpp:308-340): numpy verts [N,3] f32,
    faces [M,3] i32 -> numpy (verts, faces, face_mapping, face_flags), split
    on the GPU (csrc/remesh.cu)."""
    import numpy as np
    from . import remesh
    out = remesh._split(0, torch.from_numpy(np.ascontiguousarray(verts, np.float32)),
                        torch.from_numpy(np.ascontiguousarray(faces, np.int32)), int(numSplits), float(tau))
    return tuple(x.numpy() for x in out)


def split_triangle_soup_clip(mvp, verts, faces, valid_faces, numSplits: int, tau_ratio: float, aspectWH: float):
    """_core.split_triangle_soup_clip (src/main.cpp:342-388): numpy arguments
    and results as the reference's binding, split on the GPU."""
    import numpy as np
    from . import remesh
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt))  # noqa: E731
    out = remesh._split(1, t(verts, np.float32), t(faces, np.int32), int(numSplits), float(tau_ratio),
                        mvp=t(mvp, np.float32), valid=t(valid_faces, np.int32), aspect_wh=float(aspectWH))
    return tuple(x.numpy() for x in out)

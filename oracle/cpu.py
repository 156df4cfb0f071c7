"""ctypes wrapper of liboracle.so (oracle/oracle.cpp) over numpy arrays.

TEST INFRASTRUCTURE ONLY (see oracle/oracle.cpp).  Every function mirrors one
reference kernel or Python composite; the docstrings cite it.

FP32 functions take `variant`, the FMA-contraction mask of oracle.cpp:
0 = every operation rounded (reference built with -fmad=false).
REF_VARIANT = the contraction pattern that reproduces the reference built with
nvcc's default flags (pinned against the reference's own outputs in
tests/golden/).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# Contraction pattern of the reference's default nvcc build (see oracle.cpp V_*),
# pinned bit for bit on the golden fixtures: q = fma(-ndc, p.w, p.xy),
# A_i = fma(a, b, -(c*d)), z = fma(b2,z2, fma(b1,z1, b0*z0)),
# w = fma(b2,w2, fma(b0,w0, b1*w1)), multires accumulation fused.
V_Q, V_CROSS, V_CROSS_ALT, V_DOT, V_INTERP = 1, 2, 4, 8, 64
REF_VARIANT = V_Q | V_CROSS | V_DOT | (0 << 4) | (1 << 7) | V_INTERP
NOFMA_VARIANT = 0

_lib = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return C.c_void_p(a.ctypes.data)


def _declare(L: C.CDLL) -> None:
    vp, i32, i64, u32, u64, f32 = C.c_void_p, C.c_int, C.c_int64, C.c_uint32, C.c_uint64, C.c_float
    L.orc_triangle_rects.restype = i64
    L.orc_triangle_rects.argtypes = [i32, i32, i32, i32, vp, i32, vp, vp, vp]
    L.orc_fragments.argtypes = [i32, i32, i32, i32, i32, vp, i32, vp, vp, vp, vp, vp]
    L.orc_filter_valid.restype = i64
    L.orc_filter_valid.argtypes = [i64, vp, vp, vp, vp]
    L.orc_multires_alpha.argtypes = [i32, i64, vp, i32, i32, vp, vp]
    L.orc_multires_alpha_backward.argtypes = [i64, vp, i32, i32, i32, vp, vp]
    L.orc_fragment_thresholds.argtypes = [i64, vp, vp, i32, i32, u64, u32, vp]
    L.orc_depth_test.argtypes = [i32, i32, i32, i64, vp, vp, vp, vp, vp]
    L.orc_rasterize_alpha.restype = i64
    L.orc_rasterize_alpha.argtypes = [i32, i32, i32, i32, i32, vp, i32, vp, i32, vp, i32, u64, u32, i32, vp]
    L.orc_project_f32.argtypes = [i32, i32, vp, vp, vp]
    L.orc_accumulate_sigmoid_f32.argtypes = [i32, i32, i32, i32, i32, vp, vp]
    L.orc_multires_color_f32.argtypes = [i32, i32, i32, i32, vp, i32, i32, i32, vp, vp]
    L.orc_multires_color_f64.argtypes = [i32, i32, i32, vp, i32, i32, i32, vp, vp]
    L.orc_multires_color_backward.argtypes = [i32, i32, i32, vp, i32, i32, i32, vp, vp]
    L.orc_accumulate_forward_f64.argtypes = [i32, i32, i32, i32, i32, vp, vp]
    L.orc_accumulate_forward_f32.argtypes = [i32, i32, i32, i32, i32, i32, vp, vp]
    L.orc_accumulate_backward.argtypes = [i32, i32, i32, i32, i32, vp, vp]
    L.orc_encode_view_f32.argtypes = [i32, i32, i32, vp, vp, vp, i32]
    L.orc_encode_view_f64.argtypes = [i32, i32, i32, vp, vp, vp, i32]
    L.orc_edge_grad_f32.argtypes = [i32, i32, i32, i32, i32, vp, vp, vp, i32, vp, vp, vp]
    L.orc_edge_grad_f64.argtypes = [i32, i32, i32, i32, vp, vp, vp, i32, vp, vp, vp]
    L.orc_aux_fragment_grad_f32.argtypes = [i32, i32, i32, vp, vp, vp, i64, vp, vp, vp, vp]
    L.orc_opacity_aux.argtypes = [i32, i32, i32, i32, i32, i32, vp, vp, vp, i32, vp, i32, vp, i32, vp, vp]
    L.orc_intersect.restype = i32
    L.orc_intersect.argtypes = [i32, f32, f32, vp, vp, vp, vp]
    L.orc_opacity_threshold.restype = f32
    L.orc_opacity_threshold.argtypes = [u64, u32, u32, u32, u32]
    L.orc_feats_at_level.restype = u32
    L.orc_feats_at_level.argtypes = [u32]
    L.orc_omp_threads.restype = i32
    L.orc_set_threads.argtypes = [i32]


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def omp_threads() -> int:
    return int(lib().orc_omp_threads())


# ---------------------------------------------------------------------------
# rasterize.cu
# ---------------------------------------------------------------------------

def triangle_rects(H: int, W: int, pos: np.ndarray, tri: np.ndarray) -> Tuple[np.ndarray, np.ndarray, int]:
    """compute_triangle_rects (rasterize.cu:43-168): rects [B*T,4], inclusive prefix [B*T]."""
    pos, tri = f32(pos), i32(tri)
    B, V, _ = pos.shape
    T = tri.shape[0]
    rects = np.zeros((B * T, 4), np.int32)
    prefix = np.zeros(B * T, np.int64)
    n = lib().orc_triangle_rects(H, W, B, V, _p(pos), T, _p(tri), _p(rects), _p(prefix))
    return rects, prefix, int(n)


def fragments(H: int, W: int, pos: np.ndarray, tri: np.ndarray, rects: np.ndarray, prefix: np.ndarray,
              variant: int = REF_VARIANT) -> Tuple[np.ndarray, np.ndarray]:
    """compute_fragments (rasterize.cu:208-305), uncompacted: frag_pix -1 where rejected."""
    pos, tri, rects = f32(pos), i32(tri), i32(rects)
    prefix = np.ascontiguousarray(prefix, np.int64)
    B, V, _ = pos.shape
    T = tri.shape[0]
    n = int(prefix[-1]) if prefix.size else 0
    fpix = np.full((n, 3), -1, np.int32)
    fattr = np.zeros((n, 4), np.float32)
    lib().orc_fragments(variant, H, W, B, V, _p(pos), T, _p(tri), _p(rects), _p(prefix), _p(fpix), _p(fattr))
    return fpix, fattr


def filter_valid(fpix: np.ndarray, fattr: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """filter_valid_fragments (rasterize.cu:402-487), order preserving."""
    fpix, fattr = i32(fpix), f32(fattr)
    n = fpix.shape[0]
    po = np.zeros_like(fpix)
    ao = np.zeros_like(fattr)
    k = lib().orc_filter_valid(n, _p(fpix), _p(fattr), _p(po), _p(ao))
    return po[:k].copy(), ao[:k].copy()


def compute_fragments(H: int, W: int, pos: np.ndarray, tri: np.ndarray, variant: int = REF_VARIANT):
    """_compute_fragments (rasterize.py:40-76): compacted fragments of all views."""
    rects, prefix, _ = triangle_rects(H, W, pos, tri)
    fpix, fattr = fragments(H, W, pos, tri, rects, prefix, variant)
    return filter_valid(fpix, fattr)


def multires_alpha(frag_attrs: np.ndarray, lo: int, hi: int, alpha_src: np.ndarray, variant: int = REF_VARIANT) -> np.ndarray:
    """multires_triangle_alpha (multires.cu:130-176)."""
    fa, asrc = f32(frag_attrs), f32(alpha_src)
    out = np.zeros(fa.shape[0], np.float32)
    lib().orc_multires_alpha(variant, fa.shape[0], _p(fa), lo, hi, _p(asrc), _p(out))
    return out


def multires_alpha_backward(frag_attrs: np.ndarray, lo: int, hi: int, T: int, grad_frag_alpha: np.ndarray) -> np.ndarray:
    """backward_multires_triangle_alpha (multires.cu:178-222), double accumulation."""
    fa, g = f32(frag_attrs), f64(grad_frag_alpha)
    S = sum(int(lib().orc_feats_at_level(l)) for l in range(lo, hi + 1))
    out = np.zeros((T, S), np.float64)
    lib().orc_multires_alpha_backward(fa.shape[0], _p(fa), lo, hi, T, _p(out), _p(g))
    return out


def fragment_thresholds(frag_pix: np.ndarray, frag_attrs: np.ndarray, W: int, stochastic: bool, seed: int = 0,
                        iteration: int = 0) -> np.ndarray:
    """Per-fragment opacity thresholds: 0.5, or Philox keyed by (view, pixel, triangle)."""
    fp, fa = i32(frag_pix), f32(frag_attrs)
    out = np.zeros(fp.shape[0], np.float32)
    lib().orc_fragment_thresholds(fp.shape[0], _p(fp), _p(fa), W, int(stochastic), seed, iteration, _p(out))
    return out


def depth_test(B: int, H: int, W: int, frag_pix, frag_attrs, frag_alpha, alpha_thresh) -> np.ndarray:
    """depth_test (rasterize.cu:307-400): rast [B,H,W,4]."""
    fp, fa, al, th = i32(frag_pix), f32(frag_attrs), f32(frag_alpha), f32(alpha_thresh)
    rast = np.zeros((B, H, W, 4), np.float32)
    lib().orc_depth_test(B, H, W, fp.shape[0], _p(fp), _p(fa), _p(al), _p(th), _p(rast))
    return rast


def project(verts, mvp) -> np.ndarray:
    """Clip positions [B,V,4] with the product step's fused evaluation order."""
    v, m = f32(verts), f32(mvp)
    B, V = m.shape[0], v.shape[0]
    out = np.zeros((B, V, 4), np.float32)
    lib().orc_project_f32(B, V, _p(v), _p(m), _p(out))
    return out


def accumulate_sigmoid_f32(lo: int, hi: int, target: int, feat) -> np.ndarray:
    """sigmoid(accumulate_to_level(lo, hi, feat, target)) in FP32."""
    ft = f32(feat)
    T, _, Cd = ft.shape
    out = np.zeros((T, int(lib().orc_feats_at_level(target)), Cd), np.float32)
    lib().orc_accumulate_sigmoid_f32(T, lo, hi, target, Cd, _p(ft), _p(out))
    return out


def rasterize_alpha(H: int, W: int, pos, tri, level: int, alpha_src, stochastic: bool = False, seed: int = 0,
                    iteration: int = 0, variant: int = REF_VARIANT, view0: int = 0) -> Tuple[np.ndarray, int]:
    """rasterize_multires_triangle_alpha (multires.py:52-102) with the opacity
    threshold of each fragment taken from `fragment_thresholds`.  Returns
    (rast [B,H,W,4], number of covered fragments)."""
    pos, tri, asrc = f32(pos), i32(tri), f32(alpha_src).reshape(tri.shape[0], -1)
    B, V, _ = pos.shape
    rast = np.zeros((B, H, W, 4), np.float32)
    nf = lib().orc_rasterize_alpha(variant, H, W, B, V, _p(pos), tri.shape[0], _p(tri), level, _p(asrc),
                                   int(stochastic), seed, iteration, view0, _p(rast))
    return rast, int(nf)


# ---------------------------------------------------------------------------
# multires.cu / encoding.cu
# ---------------------------------------------------------------------------

def multires_color(rast, lo: int, hi: int, feat, precision: str = "f64", variant: int = REF_VARIANT) -> np.ndarray:
    """multires_triangle_color (multires.cu:224-266)."""
    rast = f32(rast)
    B, H, W, _ = rast.shape
    Cd = feat.shape[-1]
    if precision == "f64":
        ft = f64(feat)
        out = np.zeros((B, H, W, Cd), np.float64)
        lib().orc_multires_color_f64(B, H, W, _p(rast), lo, hi, Cd, _p(ft), _p(out))
    else:
        ft = f32(feat)
        out = np.zeros((B, H, W, Cd), np.float32)
        lib().orc_multires_color_f32(variant, B, H, W, _p(rast), lo, hi, Cd, _p(ft), _p(out))
    return out


def multires_color_backward(rast, lo: int, hi: int, T: int, grad_out) -> np.ndarray:
    """backward_multires_triangle_color (multires.cu:268-311), double accumulation."""
    rast, g = f32(rast), f64(grad_out)
    B, H, W, _ = rast.shape
    Cd = g.shape[-1]
    S = sum(int(lib().orc_feats_at_level(l)) for l in range(lo, hi + 1))
    out = np.zeros((T, S, Cd), np.float64)
    lib().orc_multires_color_backward(B, H, W, _p(rast), lo, hi, Cd, _p(out), _p(g))
    return out


def accumulate_forward(lo: int, hi: int, target: int, feat, precision: str = "f64", variant: int = REF_VARIANT) -> np.ndarray:
    """accumulate_to_level_forward (multires.cu:329-389)."""
    T, _, Cd = feat.shape
    ST = int(lib().orc_feats_at_level(target))
    if precision == "f64":
        ft = f64(feat)
        out = np.zeros((T, ST, Cd), np.float64)
        lib().orc_accumulate_forward_f64(T, lo, hi, target, Cd, _p(ft), _p(out))
    else:
        ft = f32(feat)
        out = np.zeros((T, ST, Cd), np.float32)
        lib().orc_accumulate_forward_f32(variant, T, lo, hi, target, Cd, _p(ft), _p(out))
    return out


def accumulate_backward(lo: int, hi: int, target: int, T: int, grad_out) -> np.ndarray:
    """accumulate_to_level_backward (multires.cu:393-450)."""
    g = f64(grad_out)
    Cd = g.shape[-1]
    S = sum(int(lib().orc_feats_at_level(l)) for l in range(lo, hi + 1))
    out = np.zeros((T, S, Cd), np.float64)
    lib().orc_accumulate_backward(T, lo, hi, target, Cd, _p(out), _p(g))
    return out


def encode_view(rast, inv_mvp, sh: bool = True, precision: str = "f64") -> np.ndarray:
    """encode_view_dir_sh2 (encoding.cu:89-130); sh=False gives the raw
    normalised view direction (compute_view_direction, encoding.cu:28-53)."""
    rast = f32(rast)
    B, H, W, _ = rast.shape
    K = 9 if sh else 3
    if precision == "f64":
        m = f64(inv_mvp)
        out = np.zeros((B, H, W, K), np.float64)
        lib().orc_encode_view_f64(B, H, W, _p(rast), _p(m), _p(out), int(sh))
    else:
        m = f32(inv_mvp)
        out = np.zeros((B, H, W, K), np.float32)
        lib().orc_encode_view_f32(B, H, W, _p(rast), _p(m), _p(out), int(sh))
    return out


def edge_grad(color, grad_color, rast, pos, tri, precision: str = "f64", variant: int = REF_VARIANT) -> np.ndarray:
    """backward_edge_grad (rasterize.cu:653-921): grad_pos [B,V,4] (double)."""
    rast, tri = f32(rast), i32(tri)
    B, H, W, Cd = color.shape
    V = pos.shape[1]
    out = np.zeros((B, V, 4), np.float64)
    if precision == "f64":
        c, g, p = f64(color), f64(grad_color), f64(pos)
        lib().orc_edge_grad_f64(B, H, W, Cd, _p(c), _p(g), _p(rast), V, _p(p), _p(tri), _p(out))
    else:
        c, g, p = f32(color), f32(grad_color), f32(pos)
        lib().orc_edge_grad_f32(variant, B, H, W, Cd, _p(c), _p(g), _p(rast), V, _p(p), _p(tri), _p(out))
    return out


def aux_fragment_grad(color, target, rast, frag_pix, frag_attrs, frag_alpha) -> np.ndarray:
    """backward_opacity_aux_loss (rasterize.cu:923-992), FP32."""
    c, t, r = f32(color), f32(target), f32(rast)
    B, H, W, Cd = c.shape
    fp, fa, al = i32(frag_pix), f32(frag_attrs), f32(frag_alpha)
    out = np.zeros(fp.shape[0], np.float32)
    lib().orc_aux_fragment_grad_f32(H, W, Cd, _p(c), _p(t), _p(r), fp.shape[0], _p(fp), _p(fa), _p(al), _p(out))
    return out


def opacity_aux(color, target, rast, pos, tri, level: int, alpha_src, precision: str = "f64",
                variant: int = REF_VARIANT) -> np.ndarray:
    """_OpacityAuxLossFn.forward (rasterize.py:147-190): unscaled grad_alpha_src [T,S] (double)."""
    r, p, tr = f32(rast), f32(pos), i32(tri)
    B, H, W, Cd = color.shape
    V = p.shape[1]
    T = tr.shape[0]
    S = int(lib().orc_feats_at_level(level))
    out = np.zeros((T, S), np.float64)
    if precision == "f64":
        c, t, a = f64(color), f64(target), f64(alpha_src).reshape(T, S)
        lib().orc_opacity_aux(variant, 1, B, H, W, Cd, _p(c), _p(t), _p(r), V, _p(p), T, _p(tr), level, _p(a), _p(out))
    else:
        c, t, a = f32(color), f32(target), f32(alpha_src).reshape(T, S)
        lib().orc_opacity_aux(variant, 0, B, H, W, Cd, _p(c), _p(t), _p(r), V, _p(p), T, _p(tr), level, _p(a), _p(out))
    return out


def opacity_threshold(seed: int, iteration: int, view: int, pixel: int, tri: int) -> float:
    return float(lib().orc_opacity_threshold(seed, iteration, view, pixel, tri))


def intersect(variant: int, ndc_y: float, ndc_x: float, p0, p1, p2):
    """intersect_triangle (rasterize.cu:170-206) -> (hit, b0, b1, z, w)."""
    a, b, c = f32(p0), f32(p1), f32(p2)
    o = np.zeros(4, np.float32)
    hit = lib().orc_intersect(variant, C.c_float(ndc_y), C.c_float(ndc_x), _p(a), _p(b), _p(c), _p(o))
    return bool(hit), o

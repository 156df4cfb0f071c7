"""CPU restatement of the viewer's deferred shading, in FP64 numpy.

TEST INFRASTRUCTURE ONLY: the checker of diffsoup_b200.viewer / csrc/render.cu.
Nothing in the package imports it.

The reference runs this arithmetic as GLSL in an OpenGL context
(viewer/src/viewer.cpp:169-340), which cannot be created on these machines, so
the shading is restated from the shader source and its parity is unpinned
against the reference's own output.  The geometry pass's visibility is the
oracle rasterizer (oracle/cpu.py rasterize_alpha, pinned to the reference's
CUDA rasterizer) with the deterministic threshold 0.5 on the LUT opacity; the
LUT packing is pinned on fixtures made by the reference's own
pack_face_color_lut (tests/golden/make_golden_viewer.py).
"""

from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np

SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199
SH_C2 = (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396)


def level_size(L: int) -> int:
    """Texels per face at level L (viewer.cpp:186-191)."""
    return 3 if L == 0 else ((1 << (L - 1)) + 1) * ((1 << L) + 1)


def lattice_cell(b0: np.ndarray, b1: np.ndarray, level: int) -> Tuple[np.ndarray, np.ndarray]:
    """Texel indices [...,3] and weights [...,3] of the lattice cell of
    (b0, b1) (viewer.cpp:199-226), in the shader's FP32 arithmetic."""
    f = np.float32
    res = 1 << level
    b0l = b0.astype(f) * f(res)
    b1l = b1.astype(f) * f(res)
    x = np.clip(np.floor(b0l).astype(np.int64), 0, res - 1)
    y = np.clip(np.floor(b1l).astype(np.int64), 0, (res - 1) - x)
    b0l = (b0l - x.astype(f)).astype(f)
    b1l = (b1l - y.astype(f)).astype(f)
    flip = (b0l + b1l).astype(f) > f(1.0)
    fu = flip.astype(np.int64)
    x0, y0 = x + 1, y
    x1, y1 = x, y + 1
    x2 = x + fu
    y2 = np.minimum(y + fu, res - x2)
    tri = lambda a, b: (a + b) * (a + b + 1) // 2 + b  # noqa: E731
    idx = np.stack([tri(x0, y0), tri(x1, y1), tri(x2, y2)], -1)
    w0 = np.where(flip, f(1.0) - b1l, b0l).astype(f)
    w1 = np.where(flip, f(1.0) - b0l, b1l).astype(f)
    w2 = ((f(1.0) - w0).astype(f) - w1).astype(f)
    return idx, np.stack([w0, w1, w2], -1)


def geometry_pass(gbuf: np.ndarray, level: int, lut0: np.ndarray, lut1: np.ndarray):
    """FragA, FragB of the visible fragment of every pixel (viewer.cpp:
    193-237): the LUT texels c / 255 interpolated at the fragment's lattice
    cell.  gbuf [...,4] = (b0, b1, z/w, id + 1); returns A [...,4], B [...,3]
    and the covered mask."""
    S = level_size(level)
    l0 = lut0.reshape(-1, 4).astype(np.float64) / 255.0
    l1 = lut1.reshape(-1, 4).astype(np.float64) / 255.0
    ids = gbuf[..., 3].astype(np.int64) - 1
    mask = ids >= 0
    idx, w = lattice_cell(gbuf[..., 0], gbuf[..., 1], level)
    tex = np.where(mask[..., None], ids[..., None] * S + idx, 0)
    wd = w.astype(np.float64)
    A = (l0[tex] * wd[..., None]).sum(-2)
    Bv = (l1[tex] * wd[..., None]).sum(-2)
    return A, Bv[..., :3], mask


def view_dirs(B: int, H: int, W: int, inv_mvp: np.ndarray) -> np.ndarray:
    """normalize(near - far) through the inverse MVP at every pixel centre
    (viewer.cpp:279-309), rows in framebuffer order; [B,H,W,3]."""
    M = inv_mvp.reshape(B, 4, 4).astype(np.float64)
    xs = (np.arange(W) + 0.5) / W * 2.0 - 1.0
    ys = (np.arange(H) + 0.5) / H * 2.0 - 1.0
    nx, ny = np.meshgrid(xs, ys)
    out = []
    for b in range(B):
        pts = []
        for nz in (-1.0, 1.0):
            ndc = np.stack([nx, ny, np.full_like(nx, nz), np.ones_like(nx)], -1)
            c = ndc @ M[b].T
            w = np.where(np.abs(c[..., 3]) < 1e-20, 1e-20, c[..., 3])
            pts.append(c[..., :3] / w[..., None])
        d = pts[0] - pts[1]
        out.append(d / np.linalg.norm(d, axis=-1, keepdims=True))
    return np.stack(out)


def sh2(d: np.ndarray) -> np.ndarray:
    """Real SH basis to degree 2 (viewer.cpp:290-302); [...,9]."""
    x, y, z = d[..., 0], d[..., 1], d[..., 2]
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([np.full_like(x, SH_C0), -SH_C1 * y, SH_C1 * z, -SH_C1 * x, SH_C2[0] * x * y,
                     SH_C2[1] * y * z, SH_C2[2] * (2.0 * zz - xx - yy), SH_C2[3] * x * z, SH_C2[4] * (xx - yy)], -1)


def post_pass(gbuf: np.ndarray, inv_mvp: np.ndarray, level: int, lut0, lut1, mlp: Sequence[np.ndarray],
              background=(1.0, 1.0, 1.0)) -> np.ndarray:
    """Colour of every pixel (viewer.cpp:304-340): x = [A.rgba, B.rgb, SH2],
    16 -> 16 ReLU -> 16 ReLU -> 3 sigmoid, mix(A.rgb, mlp, A.a); background
    where no fragment was kept.  gbuf [B,H,W,4]; mlp = (W1, b1, W2, b2, W3,
    b3) with weights [out, in]; returns FP64 [B,H,W,3]."""
    B, H, W, _ = gbuf.shape
    A, Bv, mask = geometry_pass(gbuf, level, lut0, lut1)
    sh = sh2(view_dirs(B, H, W, inv_mvp))
    x = np.concatenate([A, Bv, sh], -1)
    W1, b1, W2, b2, W3, b3 = [np.asarray(a, np.float64) for a in mlp]
    y = np.maximum(x @ W1.T + b1, 0.0)
    z = np.maximum(y @ W2.T + b2, 0.0)
    m = 1.0 / (1.0 + np.exp(-(z @ W3.T + b3)))
    a = A[..., 3:4]
    col = A[..., :3] * (1.0 - a) + m * a
    return np.where(mask[..., None], col, np.asarray(background, np.float64))


def to_rgba8(rgb: np.ndarray) -> np.ndarray:
    """GL_RGBA8 conversion of an FP32 colour: round(clamp(c, 0, 1) * 255)
    to nearest even, alpha 255."""
    c = np.clip(rgb.astype(np.float32), 0, 1) * np.float32(255)
    q = np.rint(c).astype(np.uint8)
    return np.concatenate([q, np.full(q.shape[:-1] + (1,), 255, np.uint8)], -1)

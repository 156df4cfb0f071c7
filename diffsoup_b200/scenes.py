"""Seeded synthetic triangle-soup scenes.

The reference trains on NeRF-Synthetic / MipNeRF-360 / Shelly captures and
MobileNeRF meshes (examples/02_synthetic.py, examples/01_mip360.py).  Those
datasets are not available here, so these generators produce soups, cameras,
features and target images with the shapes and value distributions of the five
benchmark configurations.  Everything is drawn from numpy's PCG64 with an
explicit seed, so a (config, seed) pair names one exact scene on any machine.

Cameras follow the reference's conventions: OpenGL clip space with
NEAR, FAR = 0.1, 10 (examples/02_synthetic.py:61), the projection of
examples/02_synthetic.py:105-114 (horizontal field of view), MVP = P @ inv(c2w)
(:185-187), and per-view inverse MVPs (:269).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

NEAR, FAR = 0.1, 10.0


def feats_at_level(level: int) -> int:
    """Lattice sample count of one level (multires.py:16-23)."""
    assert level >= 0
    return 3 if level == 0 else ((1 << (level - 1)) + 1) * ((1 << level) + 1)


def total_feats(min_level: int, max_level: int) -> int:
    return sum(feats_at_level(l) for l in range(min_level, max_level + 1))


def projection_matrix(fov_x_deg: float, width: int, height: int) -> np.ndarray:
    """Perspective projection from a horizontal FOV (02_synthetic.py:105-114)."""
    fov_x = np.deg2rad(fov_x_deg)
    aspect = width / float(height)
    fovy = 2.0 * np.arctan((1.0 / aspect) * np.tan(fov_x / 2.0))
    f = 1.0 / np.tan(fovy / 2.0)
    return np.array(
        [
            [f / aspect, 0, 0, 0],
            [0, f, 0, 0],
            [0, 0, (FAR + NEAR) / (NEAR - FAR), (2 * FAR * NEAR) / (NEAR - FAR)],
            [0, 0, -1, 0],
        ],
        dtype=np.float64,
    )


def look_at_c2w(eye: np.ndarray, target: np.ndarray = None, up: np.ndarray = None) -> np.ndarray:
    """Camera-to-world matrix, camera looking down its -z axis (Blender/NeRF)."""
    target = np.zeros(3) if target is None else target
    up = np.array([0.0, 0.0, 1.0]) if up is None else up
    fwd = target - eye
    fwd = fwd / np.linalg.norm(fwd)
    if abs(np.dot(fwd, up)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    cup = np.cross(right, fwd)
    c2w = np.eye(4)
    c2w[:3, 0] = right
    c2w[:3, 1] = cup
    c2w[:3, 2] = -fwd
    c2w[:3, 3] = eye
    return c2w


@dataclass
class View:
    width: int
    height: int
    mvp: np.ndarray  # (4,4) float32
    inv_mvp: np.ndarray  # (4,4) float32


@dataclass
class Scene:
    """One synthetic workload: soup, views, parameters and targets."""

    name: str
    verts: np.ndarray  # (V,3) float32 world-space soup vertices, V = 3T
    tri: np.ndarray  # (T,3) int32
    views: List[View]
    min_level: int
    max_level: int
    feat_dim: int
    feat_src: np.ndarray  # (T, S, C) float32, pre-sigmoid
    alpha_src: np.ndarray  # (T, S, 1) float32, pre-sigmoid logits
    hidden_dim: int
    n_layers: int
    view_enc: str  # "dir3" or "sh2"
    precision: str  # "fp32" or "bf16"
    seed: int
    targets: Optional[List[np.ndarray]] = field(default=None)  # per view (H,W,3) float32

    @property
    def T(self) -> int:
        return int(self.tri.shape[0])

    @property
    def S(self) -> int:
        return total_feats(self.min_level, self.max_level)

    @property
    def uniform_resolution(self) -> Optional[Tuple[int, int]]:
        hw = {(v.height, v.width) for v in self.views}
        return next(iter(hw)) if len(hw) == 1 else None

    def mvps(self) -> np.ndarray:
        return np.stack([v.mvp for v in self.views]).astype(np.float32)

    def inv_mvps(self) -> np.ndarray:
        return np.stack([v.inv_mvp for v in self.views]).astype(np.float32)

    def clip_positions(self) -> np.ndarray:
        """(B,V,4) clip-space positions, as examples/utils.py:412-426 computes them."""
        vh = np.concatenate([self.verts, np.ones_like(self.verts[:, :1])], axis=1)
        return np.einsum("bij,nj->bni", self.mvps(), vh).astype(np.float32)

    @property
    def mlp_input_dim(self) -> int:
        return self.feat_dim + (3 if self.view_enc == "dir3" else 9)


def _soup_from_centres(rng: np.random.Generator, centres: np.ndarray, sigma: float = 0.05) -> np.ndarray:
    T = centres.shape[0]
    offs = rng.normal(0.0, sigma, size=(T, 3, 3))
    return (centres[:, None, :] + offs).reshape(-1, 3)


def _shell_centres(rng: np.random.Generator, n: int, radius: float, noise: float) -> np.ndarray:
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius + rng.normal(0.0, noise, size=(n, 1))
    return d * r


def _cluster_centres(rng: np.random.Generator, n: int, k: int, sigma: float, box: float) -> np.ndarray:
    cc = rng.uniform(-box, box, size=(k, 3))
    lab = rng.integers(0, k, size=n)
    return cc[lab] + rng.normal(0.0, sigma, size=(n, 3))


def _make_view(eye: np.ndarray, width: int, height: int, fov_x_deg: float = 40.0) -> View:
    P = projection_matrix(fov_x_deg, width, height)
    Vm = np.linalg.inv(look_at_c2w(eye))
    M = P @ Vm
    return View(width=width, height=height, mvp=M.astype(np.float32), inv_mvp=np.linalg.inv(M).astype(np.float32))


def _ring_views(n: int, radius: float, width: int, height: int, elevation: float = 0.3) -> List[View]:
    views = []
    for i in range(n):
        th = 2.0 * np.pi * i / n
        eye = np.array([radius * np.cos(th), radius * np.sin(th), elevation * radius])
        views.append(_make_view(eye, width, height))
    return views


def make_scene(config: int, seed: int = 0, *, num_tris: Optional[int] = None, num_views: Optional[int] = None,
               resolution: Optional[Tuple[int, int]] = None, with_targets: bool = True,
               shading: str = "config") -> Scene:
    """Build benchmark configuration `config` (1-5) with `seed`.

    num_tris / num_views / resolution shrink a configuration for fast parity
    tests while keeping its distributions.  shading="reference" keeps the
    configuration's soup, views and levels but shades it with the reference's
    own model (examples/02_synthetic.py:289-306, 364): 7 features, the SH2
    view encoding and ColorMLP(16, hidden 16, n_layers 2).
    """
    if shading not in ("config", "reference"):
        raise ValueError(f"shading must be 'config' or 'reference', not {shading!r}")
    rng = np.random.default_rng(np.random.PCG64(seed * 1000003 + config))
    if config in (1, 4):
        T = num_tris or 5000
        centres = rng.uniform(-1.0, 1.0, size=(T, 3))
        verts = _soup_from_centres(rng, centres)
        H, W = resolution or (256, 256)
        nv = num_views or 1
        views = []
        for _ in range(nv):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            views.append(_make_view(3.0 * d, W, H))
        if config == 1:
            lo, hi, C, hid, nl, prec = 0, 2, 8, 16, 1, "fp32"
        else:
            lo, hi, C, hid, nl, prec = 0, 3, 16, 64, 2, "bf16"
    elif config == 2:
        T = num_tris or 15000
        centres = _shell_centres(rng, T, 1.0, 0.1)
        verts = _soup_from_centres(rng, centres)
        H, W = resolution or (800, 800)
        views = _ring_views(num_views or 8, 4.0, W, H)
        lo, hi, C, hid, nl, prec = 0, 2, 8, 16, 1, "fp32"
    elif config == 3:
        Tc = num_tris or 50000
        Tb = max(Tc // 5, 1)
        centres = np.concatenate([_cluster_centres(rng, Tc, 20, 0.3, 3.0), _shell_centres(rng, Tb, 10.0, 0.0)])
        verts = _soup_from_centres(rng, centres)
        nv = num_views or 64
        views = []
        aspects = [(4, 3), (16, 9), (1, 1)]
        for _ in range(nv):
            if resolution is not None:
                H, W = resolution
            else:
                W = int(rng.integers(400, 1201))
                a = aspects[int(rng.integers(0, 3))]
                H = max(1, int(round(W * a[1] / a[0])))
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            views.append(_make_view(rng.uniform(4.0, 6.0) * d, W, H))
        lo, hi, C, hid, nl, prec = 0, 2, 8, 16, 1, "fp32"
    elif config == 5:
        T = num_tris or 200000
        n_shell = T * 15 // 200
        n_cl = T - n_shell
        centres = np.concatenate([_shell_centres(rng, n_shell, 1.0, 0.1), _cluster_centres(rng, n_cl, 20, 0.3, 3.0)])
        verts = _soup_from_centres(rng, centres)
        H, W = resolution or (1080, 1920)
        views = _ring_views(num_views or 16, 5.0, W, H)
        lo, hi, C, hid, nl, prec = 0, 3, 16, 64, 2, "bf16"
    else:
        raise ValueError(f"unknown config {config}")
    enc = "dir3"
    if shading == "reference":
        C, hid, nl, enc = 7, 16, 2, "sh2"

    T = verts.shape[0] // 3
    tri = np.arange(3 * T, dtype=np.int32).reshape(T, 3)
    S = total_feats(lo, hi)
    feat_src = rng.normal(0.0, 0.1, size=(T, S, C)).astype(np.float32)
    alpha_src = rng.normal(0.0, 1.0, size=(T, S, 1)).astype(np.float32)
    targets = None
    if with_targets:
        targets = [rng.uniform(0.0, 1.0, size=(v.height, v.width, 3)).astype(np.float32) for v in views]
    return Scene(
        name=f"config{config}" + ("-refmodel" if shading == "reference" else ""),
        verts=verts.astype(np.float32),
        tri=tri,
        views=views,
        min_level=lo,
        max_level=hi,
        feat_dim=C,
        feat_src=feat_src,
        alpha_src=alpha_src,
        hidden_dim=hid,
        n_layers=nl,
        view_enc=enc,
        precision=prec,
        seed=seed,
        targets=targets,
    )


def mlp_weights(in_dim: int, out_dim: int, hidden: int, n_layers: int, seed: int = 0) -> List[Tuple[np.ndarray, np.ndarray]]:
    """ColorMLP initial weights (multires.py:154-167): Kaiming-uniform hidden
    layers (ReLU gain, fan-in), Xavier-uniform output layer, zero biases.
    Returns [(W[out,in], b[out]), ...] as float32."""
    rng = np.random.default_rng(np.random.PCG64(seed + 7919))
    dims = [in_dim] + [hidden] * n_layers + [out_dim]
    out = []
    for i in range(len(dims) - 1):
        fi, fo = dims[i], dims[i + 1]
        if i < len(dims) - 2:
            bound = np.sqrt(2.0) * np.sqrt(3.0 / fi)
        else:
            bound = np.sqrt(6.0 / (fi + fo))
        out.append((rng.uniform(-bound, bound, size=(fo, fi)).astype(np.float32), np.zeros(fo, dtype=np.float32)))
    return out


@dataclass
class ViewerInputs:
    """A soup as the viewer takes it (examples/05_benchmark_fps.py:290-375):
    vertices, faces, the RGBA8 LUT pair at `level`, MLP 16 -> 16 -> 16 -> 3
    and row-major MVPs of its views."""

    verts: np.ndarray  # (V,3) float32
    faces: np.ndarray  # (T,3) int32
    lut0: np.ndarray  # (tex_h, tex_w, 4) uint8
    lut1: np.ndarray  # (tex_h, tex_w, 4) uint8
    mlp: List[Tuple[np.ndarray, np.ndarray]]
    mvps: np.ndarray  # (B,4,4) float32 row-major
    height: int
    width: int
    level: int


def make_viewer_inputs(config: int = 2, seed: int = 0, *, level: int = 5, num_tris: Optional[int] = None,
                       num_views: Optional[int] = None, resolution: Optional[Tuple[int, int]] = None) -> ViewerInputs:
    """Synthetic stand-in for a trained checkpoint rendered by the viewer: the
    soup and cameras of configuration `config`, per-texel features U[0,1]
    (7 channels) and opacities sigmoid(N(0.5, 2)) at `level`, packed and
    quantised to RGBA8 as 05_benchmark_fps.py:56-80 and :315-317 do, and a
    16 -> 16 -> 16 -> 3 ColorMLP with random biases."""
    sc = make_scene(config, seed, num_tris=num_tris, num_views=num_views, resolution=resolution, with_targets=False)
    hw = sc.uniform_resolution
    assert hw is not None, "the viewer renders views of one resolution"
    rng = np.random.default_rng(np.random.PCG64(seed * 7 + 104729))
    S = total_feats(level, level)
    N = sc.T * S
    feat = rng.uniform(0.0, 1.0, size=(N, 7)).astype(np.float32)
    alpha = (1.0 / (1.0 + np.exp(-rng.normal(0.5, 2.0, size=(N, 1))))).astype(np.float32)
    tex_w = min(4096, N)
    tex_h = -(-N // tex_w)
    lut = np.zeros((tex_h * tex_w, 8), np.float32)
    lut[:N, :7] = feat
    lut[:N, 7:] = alpha
    lut = lut.reshape(tex_h, tex_w, 8)
    lut0 = (lut[..., :4] * 255).clip(0, 255).astype(np.uint8)
    lut1 = (lut[..., 4:] * 255).clip(0, 255).astype(np.uint8)
    mlp = mlp_weights(16, 3, 16, 2, seed=seed)
    mlp = [(W, rng.normal(0.0, 0.1, size=b.shape).astype(np.float32)) for W, b in mlp]
    return ViewerInputs(sc.verts, sc.tri, lut0, lut1, mlp, sc.mvps(), hw[0], hw[1], level)

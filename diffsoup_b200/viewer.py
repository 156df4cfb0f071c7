"""Headless inference render of a trained soup: the frame of the DiffSoup
viewer (viewer/src/viewer.cpp:169-340) on sm_100a kernels, without a window or
a graphics API.

The reference viewer (`diffsoupviewer`, viewer/python/diffsoupviewer/
__init__.py) draws each frame with OpenGL: a geometry pass that keeps, per
pixel, the nearest fragment whose opacity interpolated from an 8-bit LUT is at
least 0.5, and a post pass that shades it with an SH2-encoded view direction
and a 16 -> 16 -> 16 -> 3 MLP.  Here one C call (ds_render_frame) does the
same for a batch of views: projection, screen-tile binning, the tiled
rasterizer with the deterministic threshold and the deferred-shading kernel
(csrc/render.cu), never synchronising with the host, so a frame captures into a
CUDA graph.

  * `pack_face_color_lut`, `quantize_lut`, `extract_mlp_weights`: the data
    preparation of examples/05_benchmark_fps.py:56-102 and :315-317.
  * `Renderer`: uploads a soup with its LUTs and MLP once; `render(mvps, H, W)`
    returns RGBA8 frames (and optionally FP32 colour and the G-buffer).
  * `benchmark(...)`: the signature of diffsoupviewer.benchmark; per view the
    mean time of `repeat` frames (viewer.cpp:925-937), written with the
    summary and optional PNG screenshots like the viewer's.

Image rows are returned in framebuffer order (row 0 at NDC y = -1, the order
glReadPixels gives); screenshots are flipped to top-down like the viewer's.
The interactive window (`launch_viewer`) needs a display and is not provided.
"""

from __future__ import annotations

import math
import os
import struct
import zlib
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from . import _core
from . import tiles as _tiles

DEFAULT_LEVEL = 5  # Viewer::m_level (viewer/src/viewer.h:102)
MLP_PARAMS = 16 * 16 + 16 + 16 * 16 + 16 + 3 * 16 + 3


def level_size(L: int) -> int:
    """Texels per face at lattice level L (05_benchmark_fps.py:45-51)."""
    return _core.feats_at_level(int(L))


def pack_face_color_lut(feat_acc, alpha_acc, num_faces: int, level: int) -> torch.Tensor:
    """Per-texel features + opacity as a float32 [H, W, 8] LUT
    (05_benchmark_fps.py:56-80): rows of min(4096, N) texels, N = faces x
    texels per face, zero padding after the last texel."""
    feat = torch.as_tensor(feat_acc, dtype=torch.float32)
    alpha = torch.as_tensor(alpha_acc, dtype=torch.float32)
    S = level_size(level)
    N = int(num_faces) * S
    if feat.dim() == 3:
        feat = feat.reshape(-1, feat.shape[-1])
    if alpha.dim() == 3:
        alpha = alpha.reshape(-1, alpha.shape[-1])
    assert feat.shape[0] >= N and alpha.shape[0] >= N
    assert feat.shape[-1] == 7, f"expected feat_dim=7, got {feat.shape[-1]}"
    tex_w = min(4096, N)
    tex_h = math.ceil(N / tex_w)
    out = torch.zeros(tex_h * tex_w, 8, dtype=torch.float32, device=feat.device)
    out[:N, :7] = feat[:N]
    out[:N, 7:] = alpha[:N]
    return out.reshape(tex_h, tex_w, 8)


def quantize_lut(face_color_lut) -> Tuple[torch.Tensor, torch.Tensor]:
    """The two RGBA8 textures of a float LUT: (lut * 255).clip(0, 255)
    truncated to uint8, channels 0-3 and 4-7 (05_benchmark_fps.py:316-317,
    diffsoupviewer/__init__.py:48-49)."""
    lut = torch.as_tensor(face_color_lut, dtype=torch.float32)
    q = (lut * 255).clamp(0, 255).to(torch.uint8)
    return q[..., :4].contiguous(), q[..., 4:].contiguous()


def extract_mlp_weights(state_dict: dict):
    """(W1, b1, W2, b2, W3, b3) of a ColorMLP state dict, the first three
    weights and biases in key order (05_benchmark_fps.py:83-102)."""
    weights, biases = [], []
    for k, v in state_dict.items():
        t = v.detach().cpu().float()
        if "weight" in k:
            weights.append(t)
        elif "bias" in k:
            biases.append(t)
    if len(weights) < 3 or len(biases) < 3:
        raise ValueError(f"Expected >=3 linear layers, found {len(weights)} weights / {len(biases)} biases.  "
                         f"Keys: {list(state_dict.keys())}")
    W1, W2, W3 = weights[0], weights[1], weights[2]
    b1, b2, b3 = biases[0], biases[1], biases[2]
    assert tuple(W1.shape) == (16, 16) and tuple(W2.shape) == (16, 16) and tuple(W3.shape) == (3, 16)
    return W1, b1, W2, b2, W3, b3


def pack_mlp(W1, b1, W2, b2, W3, b3) -> torch.Tensor:
    """The 595 floats of ds_render_frame's mlp_params: W1 b1 W2 b2 W3 b3,
    weights row-major [out, in]."""
    parts = [torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a, dtype=torch.float32)
             .reshape(-1).cpu() for a in (W1, b1, W2, b2, W3, b3)]
    sizes = [256, 16, 256, 16, 48, 3]
    for p, n in zip(parts, sizes):
        if p.numel() != n:
            raise ValueError("MLP weights must be W1 [16,16], b1 [16], W2 [16,16], b2 [16], W3 [3,16], b3 [3]")
    return torch.cat(parts)


class Renderer:
    """A soup, its LUT textures and its MLP resident on one GPU, rendered
    frame by frame like the viewer (Viewer::render, viewer.cpp:663-720).

    verts [V,3] float32, faces [F,3] int32, lut0/lut1 [H,W,4] uint8 (any
    shape whose flattened texels are in face-major lattice order), MLP
    weights as diffsoupviewer takes them.  `level` is the lattice level of the
    LUT (the viewer's uLevel, 5); `background` the clear colour."""

    def __init__(self, verts, faces, lut0, lut1, W1, b1, W2, b2, W3, b3, level: int = DEFAULT_LEVEL,
                 background: Sequence[float] = (1.0, 1.0, 1.0), device=None):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if dev.type != "cuda":
            raise RuntimeError("Renderer: the render path runs on the GPU only")
        self.device = dev
        t = lambda a, dt: torch.as_tensor(a if isinstance(a, torch.Tensor) else np.asarray(a), dtype=dt)  # noqa: E731
        self.verts = t(verts, torch.float32).to(dev).reshape(-1, 3).contiguous()
        self.faces = t(faces, torch.int32).to(dev).reshape(-1, 3).contiguous()
        l0 = t(lut0, torch.uint8).reshape(-1, 4)
        l1 = t(lut1, torch.uint8).reshape(-1, 4)
        if l0.shape != l1.shape:
            raise RuntimeError("LUT0 and LUT1 sizes must match")
        self.lut0 = l0.to(dev).contiguous()
        self.lut1 = l1.to(dev).contiguous()
        self.level = int(level)
        self.S = level_size(self.level)
        self.T = int(self.faces.shape[0])
        self.V = int(self.verts.shape[0])
        if self.T * self.S > self.lut0.shape[0]:
            raise RuntimeError(f"LUT of {self.lut0.shape[0]} texels is smaller than {self.T} faces x {self.S}")
        self.mlp = pack_mlp(W1, b1, W2, b2, W3, b3).to(dev)
        self.background = tuple(float(c) for c in background)
        self.alpha = torch.empty(self.lut1.shape[0], dtype=torch.float32, device=dev)
        with torch.cuda.device(dev):
            _core.check(_core.lib.ds_render_lut_opacity(self.lut1.shape[0], _core.ptr(self.lut1),
                                                        _core.ptr(self.alpha), _core.stream()))
        self._frames: Dict[Tuple, "_Frame"] = {}

    # -- one frame --------------------------------------------------------
    def _frame(self, B: int, H: int, W: int) -> "_Frame":
        f = self._frames.get((B, H, W))
        if f is None:
            f = _Frame(self, B, H, W)
            self._frames[(B, H, W)] = f
        return f

    def render(self, mvps, height: int, width: int, rgb: bool = False, gbuf: bool = False):
        """Frames of views mvps [B,4,4] (row-major, clip = mvp . (v, 1)) at
        height x width.  Returns rgba8 [B,H,W,4] uint8, plus the FP32 colour
        [B,H,W,3] and the G-buffer [B,H,W,4] (b0, b1, z/w, id + 1) when asked
        (as a tuple in that order)."""
        m = torch.as_tensor(mvps, dtype=torch.float32).reshape(-1, 4, 4)
        f = self._frame(m.shape[0], int(height), int(width))
        f.set_views(m)
        f.status.zero_()
        f.run(want_rgb=rgb)
        torch.cuda.current_stream(self.device).synchronize()
        if f.overflowed():
            f.grow()  # this frame is exact all the same; the next ones bin without overflow
        out = [f.rgba8.view(f.B, f.H, f.W, 4).clone()]
        if rgb:
            out.append(f.rgb.view(f.B, f.H, f.W, 3).clone())
        if gbuf:
            out.append(f.gbuf.view(f.B, f.H, f.W, 4).clone())
        return out[0] if len(out) == 1 else tuple(out)

    def frame(self, mvps, height: int, width: int) -> "_Frame":
        """The resident frame for these views, inputs set and its bin-list
        capacity fitted to them, for replaying (its `run()` launches the whole
        frame; `capture()` returns a CUDA graph of it)."""
        m = torch.as_tensor(mvps, dtype=torch.float32).reshape(-1, 4, 4)
        f = self._frame(m.shape[0], int(height), int(width))
        f.set_views(m)
        f.fit()
        return f


class _Frame:
    """Device buffers of one batch shape: view table, MVPs, G-buffer, outputs
    and the binning workspace.

    The number of (triangle, tile) bin entries depends on the views.  The
    workspace holds `capacity` of them (first 8 per triangle and view); a
    frame whose lists do not fit sets DS_STATUS_LIST_OVERFLOW and is still
    exact (its overflowing tiles test every triangle, slowly), and `fit()` /
    `grow()` double the capacity until the lists fit."""

    def __init__(self, r: Renderer, B: int, H: int, W: int):
        self.r, self.B, self.H, self.W = r, B, H, W
        dev = r.device
        with torch.cuda.device(dev):
            self.views, self.num_tiles, self.num_pixels, _ = _tiles.view_table([(H, W)] * B, dev)
            self.mvp = torch.zeros(B, 16, dtype=torch.float32, device=dev)
            self.inv_mvp = torch.zeros(B, 16, dtype=torch.float32, device=dev)
            self.gbuf = torch.empty(self.num_pixels, 4, dtype=torch.float32, device=dev)
            self.rgb = torch.empty(self.num_pixels, 3, dtype=torch.float32, device=dev)
            self.rgba8 = torch.empty(self.num_pixels, 4, dtype=torch.uint8, device=dev)
            self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.capacity = max(1 << 16, 8 * B * r.T)
        self._alloc()

    def _alloc(self) -> None:
        nbytes = _core.lib.ds_render_workspace_size(self.B, self.r.V, self.r.T, self.num_tiles, self.capacity)
        self.workspace = None
        self.workspace = _core.workspace(nbytes, self.r.device)

    def overflowed(self) -> bool:
        return bool(int(self.status.item()) & _tiles.DS_STATUS_LIST_OVERFLOW)

    def grow(self) -> None:
        """Doubles the bin-list capacity (a new workspace: graphs captured
        before hold the old one)."""
        if self.capacity >= 0x7FFFFFFF:
            raise RuntimeError("render: bin-list capacity exceeds the int32 range")
        self.capacity = min(2 * self.capacity, 0x7FFFFFFF)
        self._alloc()

    def fit(self) -> None:
        """Eager frames of the current views, doubling the capacity until no
        bin list overflows."""
        for _ in range(24):
            self.status.zero_()
            self.run()
            torch.cuda.current_stream(self.r.device).synchronize()
            if not self.overflowed():
                return
            self.grow()
        raise RuntimeError("render: bin-list capacity did not converge")

    def set_views(self, mvps: torch.Tensor) -> None:
        """Row-major MVPs [B,4,4] and their inverses (FP64 on the host, then
        FP32, as glm::inverse gives the viewer's uInvMVP)."""
        m = mvps.detach().to("cpu", torch.float64).reshape(self.B, 4, 4)
        inv = torch.linalg.inv(m)
        self.mvp.copy_(m.reshape(self.B, 16).float(), non_blocking=False)
        self.inv_mvp.copy_(inv.reshape(self.B, 16).float(), non_blocking=False)

    def run(self, want_rgb: bool = False) -> None:
        r = self.r
        bg = r.background
        _core.check(_core.lib.ds_render_frame(
            self.B, _core.ptr(self.views), self.num_tiles, self.num_pixels, r.V, _core.ptr(r.verts), r.T,
            _core.ptr(r.faces), _core.ptr(self.mvp), _core.ptr(self.inv_mvp), r.level, _core.ptr(r.lut0),
            _core.ptr(r.lut1), r.lut0.shape[0], _core.ptr(r.alpha), _core.ptr(r.mlp), bg[0], bg[1], bg[2],
            _core.ptr(self.gbuf), _core.ptr(self.rgb) if want_rgb else _core.ptr(None), _core.ptr(self.rgba8),
            _core.ptr(self.workspace), self.workspace.numel(), self.capacity, _core.ptr(self.status), _core.stream()))

    def capture(self) -> torch.cuda.CUDAGraph:
        """A CUDA graph of one frame (RGBA8 output), reading the MVPs from
        this frame's buffers, so `set_views` + `replay()` renders new views."""
        s = torch.cuda.Stream(self.r.device)
        s.wait_stream(torch.cuda.current_stream(self.r.device))
        with torch.cuda.stream(s):
            self.run()  # warm-up outside capture (occupancy queries, first launch)
        torch.cuda.current_stream(self.r.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        return g


# ---------------------------------------------------------------------------
# diffsoupviewer.benchmark
# ---------------------------------------------------------------------------

def _write_png(path: str, rgba: np.ndarray) -> None:
    """RGBA8 [H,W,4] as a PNG (8-bit RGBA, filter 0, zlib)."""
    h, w, _ = rgba.shape
    raw = b"".join(b"\x00" + rgba[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def benchmark(verts, faces, lut0, lut1, W1, b1, W2, b2, W3, b3, mvps, width: int = 1200, height: int = 1200,
              warmup: int = 10, save_every: int = 0, output_dir: str = "./results/viewer",
              up: Sequence[float] = (0, 0, 1), repeat: int = 100, level: int = DEFAULT_LEVEL) -> List[float]:
    """diffsoupviewer.benchmark (viewer/python/diffsoupviewer/__init__.py:
    71-130, Viewer::launch_benchmark, viewer.cpp:835-967): mvps [B,4,4]
    column-major as the viewer takes them.  `warmup` frames of the first view,
    then per view the mean device time of `repeat` frames (one CUDA graph
    replay each), written to benchmark_frames.txt and summarised in
    benchmark_summary.txt under output_dir; every `save_every`-th view is
    saved as screenshots/benchmark_NNNNN.png.  `up` only orients the
    interactive camera and is unused.  Returns the per-view milliseconds."""
    del up
    m_col = np.ascontiguousarray(np.asarray(mvps, dtype=np.float32).reshape(-1, 4, 4))
    m_row = np.ascontiguousarray(np.transpose(m_col, (0, 2, 1)))
    r = Renderer(verts, faces, lut0, lut1, W1, b1, W2, b2, W3, b3, level=level)
    H, W = int(height), int(width)
    for i in range(m_row.shape[0]):  # bin-list capacity that fits every view
        f = r.frame(m_row[i:i + 1], H, W)
    f.set_views(torch.from_numpy(m_row[:1]))
    for _ in range(max(int(warmup), 1)):
        f.run()
    torch.cuda.synchronize()
    graph = f.capture()
    times: List[float] = []
    out_dir = os.path.join(os.path.abspath(output_dir), "")
    if save_every > 0:
        os.makedirs(os.path.join(out_dir, "screenshots"), exist_ok=True)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(m_row.shape[0]):
        f.set_views(torch.from_numpy(m_row[i:i + 1]))
        torch.cuda.synchronize()
        start.record()
        for _ in range(int(repeat)):
            graph.replay()
        end.record()
        end.synchronize()
        times.append(start.elapsed_time(end) / int(repeat))
        if save_every > 0 and i % save_every == 0:
            img = f.rgba8.view(H, W, 4).cpu().numpy()[::-1]
            path = os.path.join(out_dir, "screenshots", f"benchmark_{i:05d}.png")
            _write_png(path, np.ascontiguousarray(img))
    del graph
    os.makedirs(out_dir, exist_ok=True)
    with open(out_dir + "benchmark_frames.txt", "w") as fh:
        for i, t in enumerate(times):
            fh.write(f"{i} {t}\n")
    mean = sum(times) / len(times)
    with open(out_dir + "benchmark_summary.txt", "w") as fh:
        fh.write(f"frames: {len(times)}\nmean_ms: {mean}\nmin_ms:  {min(times)}\nmax_ms:  {max(times)}\n"
                 f"fps:     {1000.0 / mean}\n")
    return times


def launch_viewer(*args, **kwargs) -> None:
    """The interactive window of diffsoupviewer.launch_viewer needs a display
    and a graphics API; this package renders headless (Renderer)."""
    raise RuntimeError("launch_viewer: no interactive window in the headless renderer; use Renderer.render")

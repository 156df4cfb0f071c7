"""Batched training step: the whole forward+backward of one DiffSoup
optimisation step for many views in one graph-capturable call.

`TrainStep` wraps ds_train_step (csrc/step.cu) of the C ABI.  It computes,
for a batch of views that may differ in resolution, what
examples/02_synthetic.py:354-385 computes with an MSE photometric loss:

    alpha = sigmoid(accumulate_to_level(lo, hi, alpha_src))
    feat  = sigmoid(accumulate_to_level(lo, hi, feat_src))
    pos   = project_vertices(verts, mvp)
    rast  = rasterize_multires_triangle_alpha((H, W), pos, tri, hi, alpha)
    x     = cat(multires_triangle_color(rast, hi, feat), enc(rast))
            enc = view direction (3) or encode_view_dir_sh2 (9)
    color = mask * ColorMLP(x, mask) + (1 - mask)
    loss  = opacity_aux_loss(...) + mse(edge_grad(color, ...), target)

and the gradients of loss with respect to verts, feat_src, alpha_src and the
MLP parameters.  The shading MLP runs on the BF16 tensor cores with FP32
accumulation, with BF16 operands (precision="bf16") or every operand split
into two BF16 planes (precision="split", gradients within ~1e-5 of FP64);
coverage, depth and the triangle-ID buffer are exact FP32 as in the
reference.  Shading MLPs with fused kernels: the reference's own model
(7 features + SH2 -> 16 -> 16 -> 3, examples/02_synthetic.py:289-306),
8 features + direction -> 16 -> 3 and 16 features + direction -> 64 -> 64 -> 3.
"""

from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence, Tuple

import torch
from torch import nn

from . import _core
from . import tiles as _tiles


class StepConfig(C.Structure):
    _fields_ = [("B", C.c_int32), ("T", C.c_int32), ("V", C.c_int32), ("C", C.c_int32), ("min_level", C.c_int32),
                ("max_level", C.c_int32), ("hidden", C.c_int32), ("n_layers", C.c_int32),
                ("stochastic", C.c_int32), ("thr_const", C.c_float), ("frag_records", C.c_float),
                ("precision", C.c_int32), ("block_shape", C.c_int32), ("view_enc", C.c_int32),
                ("target_u8", C.c_int32), ("shade_mode", C.c_int32)]


_L = _core.lib
_L.ds_mlp_param_count.restype = C.c_int
_L.ds_mlp_param_count.argtypes = [C.c_int, C.c_int, C.c_int]
_L.ds_step_mlp_param_count.restype = C.c_int
_L.ds_step_mlp_param_count.argtypes = [C.POINTER(StepConfig)]
_L.ds_train_step_workspace_size.restype = C.c_size_t
_L.ds_train_step_workspace_size.argtypes = [C.POINTER(StepConfig), C.c_int, C.c_int64, C.c_int64]
_L.ds_train_step_layout.restype = C.c_int
_L.ds_train_step_layout.argtypes = [C.POINTER(StepConfig), C.c_int, C.c_int64, C.c_int64, C.POINTER(C.c_int64)]
_vp = C.c_void_p
_L.ds_train_step.restype = C.c_int
# cfg, views, num_tiles, num_pixels, 17 device pointers (verts .. workspace), bytes, capacity, status, stream
_L.ds_train_step.argtypes = ([C.POINTER(StepConfig), _vp, C.c_int, C.c_int64] + [_vp] * 17
                             + [C.c_size_t, C.c_int64, _vp, _vp])

_L.ds_train_step_set_events.restype = C.c_int
_L.ds_train_step_set_events.argtypes = [C.c_void_p, C.c_int]

LAYOUT = ["pos", "alpha_acc", "feat_acc", "feat_bf16", "rast", "color", "grad_color", "l1", "grad_pos",
          "grad_alpha_acc", "grad_feat_acc", "records", "chunk_fill", "record_counters", "fallback_blocks"]


def mlp_param_count(C_: int, hidden: int, n_layers: int) -> int:
    return int(_L.ds_mlp_param_count(C_, hidden, n_layers))


def pack_mlp(mlp: nn.Module) -> torch.Tensor:
    """Flatten a ColorMLP's Linear layers as [W0, b0, ..., Wout, bout] (fp32)."""
    lins = [m for m in mlp.modules() if isinstance(m, nn.Linear)]
    return torch.cat([t.detach().reshape(-1).float() for lin in lins for t in (lin.weight, lin.bias)]).contiguous()


def unpack_mlp_grads(flat: torch.Tensor, mlp: nn.Module) -> None:
    """Write a packed gradient into the .grad of a ColorMLP's parameters."""
    o = 0
    for lin in [m for m in mlp.modules() if isinstance(m, nn.Linear)]:
        for p in (lin.weight, lin.bias):
            n = p.numel()
            p.grad = flat[o:o + n].view_as(p).clone()
            o += n


# Launch-layout choices of TrainStep.autotune, per (device, workload).
autotune_cache: Dict[Tuple, Dict[str, object]] = {}


class TrainStep:
    """Workspace and launch state of the batched training step for a fixed
    batch layout (triangle count, vertex count, view resolutions)."""

    def __init__(self, T: int, V: int, hw: Sequence[Tuple[int, int]], C_: int, min_level: int, max_level: int,
                 hidden: int, n_layers: int, stochastic: bool = True, seed: int = 0,
                 device: Optional[torch.device] = None, list_capacity: Optional[int] = None,
                 frag_records: float = 2.0, precision: str = "bf16", view_enc: str = "dir3",
                 target_u8: bool = False):
        self.device = torch.device(device or "cuda")
        self.hw = [(int(h), int(w)) for h, w in hw]
        self.B = len(self.hw)
        # frag_records: fragment records per pixel kept by the rasterizer for the
        # opacity auxiliary gradient (0: that pass re-enumerates the tiles)
        # precision: "bf16" (BF16 operands) or "split" (every MLP operand as bf16 hi + lo, three
        # tensor-core products each; gradients within ~1e-5 of FP64)
        # view_enc: "dir3" (the 3-D view direction) or "sh2" (encode_view_dir_sh2, 9 inputs)
        # target_u8: targets are 8-bit images [pixels,3] uint8 (read as value / 255) instead of fp32
        if precision not in ("bf16", "split"):
            raise ValueError(f"precision must be 'bf16' or 'split', not {precision!r}")
        if view_enc not in ("dir3", "sh2"):
            raise ValueError(f"view_enc must be 'dir3' or 'sh2', not {view_enc!r}")
        self.cfg = StepConfig(B=self.B, T=T, V=V, C=C_, min_level=min_level, max_level=max_level, hidden=hidden,
                              n_layers=n_layers, stochastic=int(stochastic), thr_const=0.5,
                              frag_records=float(frag_records), precision=1 if precision == "split" else 0,
                              block_shape=0, view_enc=1 if view_enc == "sh2" else 0, target_u8=int(bool(target_u8)),
                              shade_mode=0)
        self.views, self.num_tiles, self.num_pixels, self.pix_offsets = _tiles.view_table(self.hw, self.device)
        self.S = sum(_core.feats_at_level(l) for l in range(min_level, max_level + 1))
        self.nparam = int(_L.ds_step_mlp_param_count(C.byref(self.cfg)))
        self.CP = (C_ + 7) // 8 * 8  # channel stride of the step's accumulated feature tables
        self.rng = torch.tensor([seed, 0], dtype=torch.int64, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.grad_verts = torch.zeros(V, 3, device=self.device)
        self.grad_feat_src = torch.zeros(T, self.S, C_, device=self.device)
        self.grad_alpha_src = torch.zeros(T, self.S, device=self.device)
        self.grad_mlp = torch.zeros(self.nparam, device=self.device)
        self.capacity = int(list_capacity or max(1 << 16, 8 * self.B * T))
        self._alloc()
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def _alloc(self) -> None:
        nb = int(_L.ds_train_step_workspace_size(C.byref(self.cfg), self.num_tiles, self.num_pixels, self.capacity))
        self.workspace = torch.empty(nb, dtype=torch.uint8, device=self.device)
        offs = (C.c_int64 * 16)()
        _core.check(_L.ds_train_step_layout(C.byref(self.cfg), self.num_tiles, self.num_pixels, self.capacity, offs))
        self.offsets = {k: int(offs[i]) for i, k in enumerate(LAYOUT)}
        self.record_capacity = int(offs[15])

    def intermediate(self, name: str) -> torch.Tensor:
        """A view of one workspace intermediate (valid after a step)."""
        c = self.cfg
        ST = _core.feats_at_level(c.max_level)
        shapes: Dict[str, Tuple[torch.dtype, Tuple[int, ...]]] = {
            "pos": (torch.float32, (c.B, c.V, 4)), "alpha_acc": (torch.float32, (c.T, ST)),
            "feat_acc": (torch.float32, (c.T, ST, self.CP)), "feat_bf16": (torch.bfloat16, (c.T, ST, self.CP)),
            "rast": (torch.float32, (self.num_pixels, 4)), "color": (torch.float32, (self.num_pixels, 3)),
            "grad_color": (torch.float32, (self.num_pixels, 3)), "l1": (torch.float32, (self.num_pixels,)),
            "grad_pos": (torch.float64, (c.B, c.V, 4)), "grad_alpha_acc": (torch.float32, (c.T, ST)),
            "grad_feat_acc": (torch.float32, (c.T, ST, self.CP)),
            "records": (torch.int32, (self.record_capacity, 4)),
            "chunk_fill": (torch.int32, (self.record_capacity // 256,)),
            "record_counters": (torch.int32, (2,)), "fallback_blocks": (torch.int32, (self.num_tiles * 8 if self.record_capacity else 0,)),
        }
        dt, shp = shapes[name]
        n = 1
        for s in shp:
            n *= s
        o = self.offsets[name]
        nbytes = n * torch.tensor([], dtype=dt).element_size()
        return self.workspace[o:o + nbytes].view(dt).view(shp)

    def run(self, verts: torch.Tensor, tri: torch.Tensor, mvp: torch.Tensor, inv_mvp: torch.Tensor,
            feat_src: torch.Tensor, alpha_src: torch.Tensor, mlp_params: torch.Tensor, target: torch.Tensor,
            rast_out: Optional[torch.Tensor] = None, color_out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Enqueue one step on the current stream; returns the device loss."""
        want = torch.uint8 if self.cfg.target_u8 else torch.float32
        if target.dtype != want or target.numel() != self.num_pixels * 3 or not target.is_contiguous():
            raise ValueError(f"target must be a contiguous [{self.num_pixels}, 3] {want} tensor")
        p = _core.ptr
        _core.check(_L.ds_train_step(C.byref(self.cfg), p(self.views), self.num_tiles, self.num_pixels, p(verts),
                                     p(tri), p(mvp), p(inv_mvp), p(feat_src), p(alpha_src), p(mlp_params), p(target),
                                     p(self.rng), p(self.loss), p(self.grad_verts), p(self.grad_feat_src),
                                     p(self.grad_alpha_src), p(self.grad_mlp), p(rast_out), p(color_out),
                                     p(self.workspace), self.workspace.numel(), self.capacity, p(self.status),
                                     _core.stream()))
        return self.loss

    def overflowed(self) -> bool:
        """True when a tile list outgrew its capacity (results stay exact; the
        affected tiles ran the exhaustive path).  Synchronises on the status."""
        return bool(int(self.status.item()) & _tiles.DS_STATUS_LIST_OVERFLOW)

    def record_fallback(self) -> bool:
        """True when some blocks' fragment records did not fit and the opacity
        auxiliary gradient re-enumerated them (results are the same).
        Synchronises on the status."""
        return bool(int(self.status.item()) & _tiles.DS_STATUS_RECORD_FALLBACK)

    def fit_capacity(self, *args, **kwargs) -> None:
        """Run eager steps, doubling the tile-list capacity until it fits."""
        for _ in range(16):
            self.status.zero_()
            self.run(*args, **kwargs)
            if not self.overflowed():
                return
            self.capacity *= 2
            self._alloc()
        raise RuntimeError("tile list capacity did not converge")

    BLOCK_SHAPES = {0: "8x4", 1: "16x2", 2: "4x8"}
    SHADE_MODES = {0: "mma.sync", 1: "tcgen05"}

    def tcgen05_shading(self) -> bool:
        """Whether this step's MLP has the tcgen05 shading kernel (16 features +
        direction -> 64 -> 64 -> 3 in BF16)."""
        c = self.cfg
        return (c.C == 16 and c.hidden == 64 and c.n_layers == 2 and c.view_enc == 0 and c.precision == 0)

    def autotune(self, *args, steps: int = 5, shapes: Sequence[int] = (0, 1, 2), **kwargs) -> Dict[str, object]:
        """Chooses the launch layout of this step for its inputs (the step's own
        autotuner, run eagerly before training and before any capture):

          * the tile-list capacity (triangles per bin), doubled until no list
            overflows (fit_capacity);
          * the fragment-record store, sized to the records a step reserves
            plus a quarter, so that no block is re-enumerated;
          * the pixel block of a rasterizer warp (8x4, 16x2 or 4x8 pixels of a
            16x16 tile, 8 warps per tile) and, for the wide BF16 MLP, the
            shading kernel (warp-level mma.sync or tcgen05 with TMEM
            accumulators): each combination is timed with CUDA events over
            `steps` eager steps after a warm-up, and the fastest kept.

        Results do not depend on the choices.  The RNG iteration is restored,
        so tuning does not advance the training state.  Choices are cached per
        device and workload (`autotune_cache`).  Returns them."""
        key = (torch.cuda.get_device_name(self.device), self.B, tuple(self.hw), self.cfg.T, self.cfg.V, self.cfg.C,
               self.cfg.min_level, self.cfg.max_level, self.cfg.hidden, self.cfg.n_layers, self.cfg.precision,
               self.cfg.stochastic, self.cfg.view_enc, self.cfg.target_u8, self.cfg.frag_records > 0)
        it0 = self.rng[1].clone()
        hit = autotune_cache.get(key)
        if hit is not None:
            self.capacity = max(self.capacity, hit["list_capacity"])
            self.cfg.frag_records = hit["frag_records"]
            self.cfg.block_shape = hit["block_shape"]
            self.cfg.shade_mode = hit["shade_mode"]
            self._alloc()
            return dict(hit)
        self.fit_capacity(*args, **kwargs)
        # records reserved by one step -> records per pixel with a margin
        self.run(*args, **kwargs)
        counters = self.intermediate("record_counters").cpu() if self.record_capacity else None
        if counters is not None:
            need = (int(counters[0]) + int(counters[1]) * 256) / max(self.num_pixels, 1)
            self.cfg.frag_records = float(min(max(1.25 * need, 0.5), 16.0))
            self._alloc()
        times = {}
        shade_modes = (0, 1) if self.tcgen05_shading() else (0,)
        combos = [(int(sh), sm) for sm in shade_modes for sh in shapes]
        name = lambda c: (self.BLOCK_SHAPES[c[0]]  # noqa: E731
                          + (f"/{self.SHADE_MODES[c[1]]}" if len(shade_modes) > 1 else ""))
        for combo in combos:
            self.cfg.block_shape, self.cfg.shade_mode = combo
            for _ in range(2):
                self.run(*args, **kwargs)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                self.run(*args, **kwargs)
            e1.record()
            torch.cuda.synchronize()
            times[name(combo)] = e0.elapsed_time(e1) / steps
        best = min(combos, key=lambda c: times[name(c)])
        self.cfg.block_shape, self.cfg.shade_mode = best
        self.rng[1].copy_(it0)
        self.status.zero_()
        out = {"list_capacity": int(self.capacity), "frag_records": float(self.cfg.frag_records),
               "block_shape": best[0], "block": self.BLOCK_SHAPES[best[0]], "shade_mode": best[1],
               "shade": self.SHADE_MODES[best[1]],
               "ms_per_step": times}
        autotune_cache[key] = dict(out)
        return out

    def capture(self, *args, **kwargs) -> torch.cuda.CUDAGraph:
        """Capture one step over fixed buffers into a CUDA graph (replay with
        self.graph.replay() after refreshing the input buffers in place)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run(*args, **kwargs)  # warm-up outside capture (sets kernel attributes)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(*args, **kwargs)
        self.graph = g
        return g

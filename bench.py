#!/usr/bin/env python
"""Benchmark of the DiffSoup training step on B200.

Workload (the "plain method, object scale" benchmark configuration): 15,000
triangles on a noisy unit sphere shell, 8 views of 800x800 on a ring of radius
4, multires features at levels 0..2 x 8 channels, shading MLP 11 -> 16 -> 3,
stochastic binary opacity, MSE against a U[0,1] target, full forward+backward
(edge gradients, opacity auxiliary gradient, feature/opacity/MLP/vertex
gradients).  Synthetic, seeded inputs stand in for the reference's datasets.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is views/s of the batched step
(diffsoup_b200.step.TrainStep, one CUDA graph per step) in split-BF16
precision (every shading-MLP operand as two BF16 planes on the tensor cores;
image and gradients within 1e-3 of the FP64 oracle; --precision bf16 for
plain BF16 operands) with inputs resident in HBM; `e2e` is the same step
through the public API with each step's camera matrices and target images
copied from pinned host memory and the loss read back.  `side` holds the same
workload in the other precision, the reference's own shading model (7
features + SH2 -> 16 -> 16 -> 3) on the same soup, and the other benchmark
configurations (1, 3, 4, 5), each with its dominant kernel's roofline fraction
and a CPU sample.  N > 1 runs one independent replica per GPU (views are
independent; the reference has no multi-GPU exchange), timed as the max over
ranks.  --impl reference times the CPU restatement of the reference's step
(oracle/pipeline.py, FP32, all host threads) on a bounded sample.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd views/s @15K tris 800²: batched BF16 vs plain FP32 on one B200"
# kernels one training step launches (the ncu launch list of the bench shows them): level
# accumulation + sigmoid (opacity and features in one), project | bin_setup, 3 scan kernels, bin_fill,
# sort_lists | raster | shade | aux from records, aux of re-enumerated blocks | edge | accumulation
# adjoint, project backward, finish
KERNELS_PER_STEP = 16
# kernels one inference frame launches: project | bin_setup, 3 scan kernels, bin_fill, sort_lists |
# raster | deferred shade
RENDER_KERNELS_PER_FRAME = 9
WORKLOAD = "config2: 15K-tri sphere-shell soup, 8 views 800x800, levels 0..2 x 8 ch, MLP 11-16-3, stochastic opacity"
PRECISION_TEXT = {
    "split": "split bf16: every MLP operand as bf16 hi + lo on the BF16 tensor cores (hi*hi + hi*lo + lo*hi, FP32 "
             "accumulation), FP32 features; image and every gradient group within 1e-3 of the FP64 oracle",
    "bf16": "bf16: BF16 features and MLP operands on the tensor cores, FP32 accumulation; feature and MLP gradients "
            "up to ~1.6e-2 / ~5e-3 from the FP64 oracle (the rounding of the BF16 inputs)",
}
N_INPUT_SETS = 10  # rotating view batches: 10 x 15.4 MB of 8-bit targets, larger than the 126 MB L2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--precision", choices=["split", "bf16"], default="split",
                    help="shading precision of the headline step: split (every MLP operand as two BF16 planes on "
                         "the tensor cores; image and gradients within 1e-3 of FP64) or bf16 (BF16 operands)")
    ap.add_argument("--no-side", dest="side", action="store_false",
                    help="skip the side entries (the other precision, the reference's own shading model and the "
                         "other benchmark configurations)")
    ap.add_argument("--no-render", dest="render", action="store_false",
                    help="skip timing the inference render (the viewer's frame) beside the training step")
    ap.add_argument("--views", type=int, default=8, help="views per step (8 is the benchmark workload; "
                    "fewer only for small profiling cases)")
    ap.add_argument("--side-case", default=None, choices=[w[0] for w in SIDE_WORKLOADS],
                    help="profiling: time only this side workload (on --side-views views when given) and print "
                         "its entry")
    ap.add_argument("--side-views", type=int, default=None)
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except Exception:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), samples=len(sm))
        out["reasons"] = sorted(reasons)
        return out


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def load_scenes():
    """diffsoup_b200/scenes.py (numpy only: the seeded synthetic soups and
    cameras) loaded from its file, so that a caller can build the workload
    without importing the package, which loads libdiffsoup_b200.so."""
    import importlib.util

    name = "_bench_scenes"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "diffsoup_b200", "scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def bench_config(world: int, nviews: int = 8) -> dict:
    """The workload both arms report (`config`)."""
    return {"workload": WORKLOAD if nviews == 8 else WORKLOAD.replace("8 views", f"{nviews} views"),
            "views_per_step": nviews, "triangles": 15000, "resolution": "800x800",
            "parallelism": f"replicas x{world}",
            "targets": "8-bit images (value / 255), as the reference's datasets",
            "l2": f"{N_INPUT_SETS} rotating input sets ({N_INPUT_SETS} x 15.4 MB of targets) larger than L2"}


def make_inputs(rank: int, nviews: int = 8, scenes=None):
    if scenes is None:
        from diffsoup_b200 import scenes

    sc = scenes.make_scene(2, seed=0, with_targets=False)
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=0)
    sets = []
    rng = np.random.default_rng(1000 + rank)
    for r in range(N_INPUT_SETS):
        phase = 2 * math.pi * (rank * N_INPUT_SETS + r) / (8 * N_INPUT_SETS * 64)
        views = []
        for i in range(nviews):
            th = 2 * math.pi * i / 8 + phase
            eye = np.array([4 * math.cos(th), 4 * math.sin(th), 1.2])
            views.append(scenes._make_view(eye, 800, 800))
        mvp = np.stack([v.mvp for v in views]).astype(np.float32)
        inv = np.stack([v.inv_mvp for v in views]).astype(np.float32)
        # U[0,1] targets as 8-bit images (value / 255)
        tgt = rng.integers(0, 256, size=(nviews * 800 * 800, 3), dtype=np.uint8)
        sets.append((mvp, inv, tgt))
    return sc, mlp, sets


def target_f32(u8: np.ndarray) -> np.ndarray:
    """An 8-bit target as the fp32 values the step reads (value / 255, correctly rounded)."""
    return u8.astype(np.float32) / np.float32(255)


def mlp_flat(mlp):
    return np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in mlp]).astype(np.float32)


# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference's step on the host cores, rank 0 only: the oracle port of
    its kernels (oracle/, FP32, OpenMP over all host threads; the reference has
    no CPU implementation of the path and its own CUDA build is the parity
    checker, not a baseline), one 800x800 view of the workload per step.
    Neither this arm nor its inputs load libdiffsoup_b200.so."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import cpu, pipeline as P

    sc, mlp, sets = make_inputs(0, scenes=load_scenes())
    cores = cpu.omp_threads()
    torch.set_num_threads(max(1, os.cpu_count() or 1))

    def one_view(i):
        mvp, inv, tgt = sets[i % N_INPUT_SETS]
        b = i % 8
        inp = P.StepInputs(verts=sc.verts, tri=sc.tri, mvps=mvp[b:b + 1], inv_mvps=inv[b:b + 1], hw=[(800, 800)],
                           feat_src=sc.feat_src, alpha_src=sc.alpha_src[..., 0], mlp=mlp,
                           targets=[target_f32(tgt).reshape(8, 800, 800, 3)[b]], min_level=sc.min_level,
                           max_level=sc.max_level, stochastic=True, seed=7, iteration=i)
        P.train_step(inp, "f32")

    for i in range(args.warmup):
        one_view(i)
    t0 = time.perf_counter()
    for i in range(args.steps):
        one_view(args.warmup + i)
    dt = time.perf_counter() - t0
    n = args.steps
    v = n / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "views/s", "n_gpus": args.gpus,
        "steps": n, "warmup": args.warmup, "ms_per_step": 1000 * dt / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; stands in for the reference datasets)",
        "config": bench_config(args.gpus),
        "step_unit": "one 800x800 view of the workload per step (a bounded sample of the 8-view step)",
        "cpu_baseline": {"value": v, "unit": "views/s", "cores": cores, "kind": "port",
                         "sample": f"{n} views of the workload (800x800, 15K tris), FP32 oracle port, {cores} threads"},
        "e2e": {"value": v, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def algorithmic_bytes(phase: str, P_: int, B: int, T: int, V: int, ST: int, C_: int, feat_bytes: int = 2,
                      target_bytes: int = 12) -> float:
    """Minimal DRAM bytes of one launch of each step kernel: what the kernel must read and write
    once (per-pixel buffers, per-(view, triangle) records, lattice samples), no re-reads.  feat_bytes:
    2 when the shading kernel gathers BF16 features, 4 for FP32 (split precision); target_bytes: 12 per
    pixel for fp32 targets, 3 for 8-bit ones."""
    if phase == "shade":  # rast 16 R, target R, colour 12 W, dL/dcolour 12 W, |c-t| 4 W; features + fp32 grads
        return P_ * (44.0 + target_bytes) + T * ST * C_ * (feat_bytes + 8)
    # fragment records: 16 B each, about one per pixel on this workload (fragments in front of the surface)
    if phase == "raster":  # rast 16 W + records 16 W per pixel; triangle records 64 B per (view, tri); opacities
        return P_ * 32.0 + B * T * 64.0 + T * ST * 4.0
    if phase == "aux":  # records 16 R + |c-t| 4 R per record; opacity table + grads
        return P_ * 20.0 + T * ST * 12.0
    if phase == "edge":  # rast 16 + colour 12 + dL/dcolour 12 per pixel; clip positions + fp64 grads
        return P_ * 40.0 + B * V * (16.0 + 64.0)
    if phase == "bin":
        return B * T * (12.0 * 3 + 64.0 + 2 * 16.0)
    if phase == "prep":
        return T * ST * C_ * 10.0 + B * V * 28.0
    return 0.0


def step_algorithmic_bytes(B: int, T: int, V: int, S: int, C_: int, P_: int, target_bytes: int = 12) -> float:
    """Minimal DRAM bytes of a whole training step: 12 B per triangle, features and opacities read and
    their gradients written (8 B per lattice sample and channel, C + 1 channels), and per view the clip
    positions read and their gradients written (32 B per vertex) plus, per pixel, the ID buffer written
    (16 B), the colour written (12 B), the target read (12 B, or 3 B for 8-bit targets) and dL/dcolour read
    (12 B)."""
    return 12.0 * T + 8.0 * T * S * (C_ + 1) + B * 32.0 * V + P_ * (16.0 + 12.0 + target_bytes + 12.0)


def run_ours(args):
    from diffsoup_b200 import scenes, _core, replicas
    from diffsoup_b200.step import TrainStep
    import diffsoup_b200 as ds

    rep = replicas.init()  # one process per GPU, NCCL process group for N > 1
    world, rank, local, dev = rep.world, rep.rank, rep.local_rank, rep.device

    sc, mlp, sets = make_inputs(rank, args.views)
    B, T, V = args.views, sc.T, sc.verts.shape[0]
    hw = [(800, 800)] * B
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    verts, tri = t(sc.verts), t(sc.tri)
    feat_src, alpha_src = t(sc.feat_src), t(sc.alpha_src[..., 0])
    params = t(mlp_flat(mlp))
    dsets = [(t(m), t(i), t(g)) for m, i, g in sets]
    step = TrainStep(T, V, hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim, sc.n_layers,
                     stochastic=True, seed=1234 + rank, device=dev, precision=args.precision, target_u8=True)

    def kw(s):
        return dict(verts=verts, tri=tri, mvp=s[0], inv_mvp=s[1], feat_src=feat_src, alpha_src=alpha_src,
                    mlp_params=params, target=s[2])

    tuned = step.autotune(**kw(dsets[0]))  # list capacity, record store, warp pixel block
    for s in dsets[1:]:
        step.status.zero_()
        step.run(**kw(s))
        if step.overflowed():
            step.capacity *= 2
            step._alloc()
    # covered fragments per step (every (pixel, triangle) pair passing the coverage test, before the
    # depth test), counted by the library's fragment operators, averaged over the input sets
    nfrag = 0
    for s in dsets:
        step.run(**kw(s))
        pos = step.intermediate("pos").clone()
        for b in range(B):
            fp, _ = ds.rasterize._compute_fragments(hw[b], pos[b:b + 1].contiguous(), tri)
            nfrag += fp.shape[0]
    nfrag /= len(dsets)
    graphs = [step.capture(**kw(s)) for s in dsets]
    torch.cuda.synchronize()

    # ---------------- device-resident throughput ------------------------------
    for i in range(args.warmup):
        graphs[i % N_INPUT_SETS].replay()
    step.status.zero_()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.25)
    replicas.barrier(rep)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        graphs[i % N_INPUT_SETS].replay()
    e1.record()
    torch.cuda.synchronize()
    replicas.barrier(rep)
    clocks = sampler.stop()
    ms = replicas.max_over_ranks(rep, e0.elapsed_time(e1))
    overflow = step.overflowed()
    value = replicas.job_throughput(rep, B * args.steps, ms)
    # steadiness: four more back-to-back windows of the same K steps (not part of `value`)
    windows = []
    for _ in range(4):
        e0.record()
        for i in range(args.steps):
            graphs[i % N_INPUT_SETS].replay()
        e1.record()
        torch.cuda.synchronize()
        windows.append(replicas.max_over_ranks(rep, e0.elapsed_time(e1)) / args.steps)

    # ---------------- end to end through the public API -----------------------
    # pinned host inputs; each step copies its cameras and targets H2D on a copy
    # stream (double-buffered, overlapping the previous step) and reads the loss.
    host = [(torch.from_numpy(m).pin_memory(), torch.from_numpy(i).pin_memory(), torch.from_numpy(g).pin_memory())
            for m, i, g in sets]
    bufs = [tuple(x.clone() for x in dsets[0]) for _ in range(2)]
    egraphs = [step.capture(**kw(b)) for b in bufs]
    loss_host = torch.empty(max(args.steps, 1), dtype=torch.float32, pin_memory=True)
    comp = torch.cuda.current_stream()
    cs = torch.cuda.Stream(dev)
    copied = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    for d in done:
        d.record(comp)
    h2d = sum(x.numel() * x.element_size() for x in host[0])

    def issue_copy(i):
        j = i % 2
        cs.wait_event(done[j])
        with torch.cuda.stream(cs):
            for dst, src in zip(bufs[j], host[i % N_INPUT_SETS]):
                dst.copy_(src, non_blocking=True)
        copied[j].record(cs)

    def e2e_loop(n):
        issue_copy(0)
        for i in range(n):
            j = i % 2
            if i + 1 < n:
                issue_copy(i + 1)
            comp.wait_event(copied[j])
            egraphs[j].replay()
            loss_host[i].copy_(step.loss[0], non_blocking=True)
            done[j].record(comp)

    e2e_loop(min(args.warmup, 4) or 1)
    torch.cuda.synchronize()
    replicas.barrier(rep)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    cs.wait_event(f0)
    e2e_loop(args.steps)
    f1.record()
    torch.cuda.synchronize()
    ems = replicas.max_over_ranks(rep, f0.elapsed_time(f1))
    e2e = replicas.job_throughput(rep, B * args.steps, ems)
    assert np.isfinite(loss_host[: args.steps].numpy()).all()

    # ---------------- per-phase kernel time (roofline) ------------------------
    names = ["prep", "bin", "raster", "shade", "aux", "edge", "finish"]
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(8)]
    for e in evs:  # torch creates the CUDA event on first record
        e.record()
    torch.cuda.synchronize()
    handles = ctypes_void_p_array(evs)
    _core.check(_core.lib.ds_train_step_set_events(handles, 8))
    acc = {n: 0.0 for n in names}
    M = 20
    for i in range(M):
        step.run(**kw(dsets[i % N_INPUT_SETS]))
        torch.cuda.synchronize()
        for k, n in enumerate(names):
            acc[n] += evs[k].elapsed_time(evs[k + 1])
    _core.check(_core.lib.ds_train_step_set_events(None, 0))
    phase_ms = {n: acc[n] / M for n in names}
    dom = max(["raster", "shade", "aux", "edge"], key=lambda n: phase_ms[n])
    ST = _core.feats_at_level(sc.max_level)
    P_ = step.num_pixels
    alg = algorithmic_bytes(dom, P_, B, T, V, ST, sc.feat_dim, 4 if args.precision == "split" else 2, 3)
    peak, peak_src = measured_peak()
    achieved = alg / (phase_ms[dom] / 1000.0) / 1e9
    step_bytes = step_algorithmic_bytes(B, T, V, _core.total_feats(sc.min_level, sc.max_level), sc.feat_dim, P_, 3)
    traffic = read_traffic(dom)

    # ---------------- the headline workload in the other precision -------------
    side = None
    if rank == 0 and args.side:
        other = "bf16" if args.precision == "split" else "split"
        ostep = TrainStep(T, V, hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim, sc.n_layers,
                          stochastic=True, seed=1234 + rank, device=dev, precision=other, target_u8=True)
        ostep.capacity = step.capacity
        ostep.cfg.frag_records = step.cfg.frag_records
        ostep.cfg.block_shape = step.cfg.block_shape
        ostep._alloc()
        og = [ostep.capture(**kw(s)) for s in dsets]
        for i in range(args.warmup):
            og[i % N_INPUT_SETS].replay()
        torch.cuda.synchronize()
        e0.record()
        for i in range(args.steps):
            og[i % N_INPUT_SETS].replay()
        e1.record()
        torch.cuda.synchronize()
        oms = e0.elapsed_time(e1)
        side = {f"config2_{other}": {"workload": WORKLOAD, "precision": PRECISION_TEXT[other],
                                      "value": B * args.steps / (oms / 1000.0), "unit": "views/s",
                                      "ms_per_step": oms / args.steps, "steps": args.steps, "warmup": args.warmup}}
        del og, ostep
        # the reference's own shading model and the other benchmark configurations
        side.update(run_side_entries(args, dev, peak))

    # ---------------- plain FP32 single-view path (denominator) ---------------
    plain = None
    if not args.no_plain and rank == 0:
        plain = run_plain(sc, mlp, sets[0], dev, n_views=16)

    # ---------------- inference render (the viewer's frame) -------------------
    render = None
    if rank == 0 and args.render:
        render = run_render(dev, cpu_sample=not args.no_cpu_baseline)

    # ---------------- soup subdivision (resampling step) -----------------------
    remesh_line = None
    if rank == 0 and args.render:
        remesh_line = run_remesh(dev, cpu_sample=not args.no_cpu_baseline)

    # ---------------- CPU baseline --------------------------------------------
    cpu_base = None
    if not args.no_cpu_baseline and rank == 0:
        cpu_base = run_cpu_baseline(sc, mlp, sets[0])

    line = {
        "metric": METRIC, "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "repeat_windows": {"ms_per_step": [round(w, 5) for w in windows],
                           "median_ms_per_step": round(statistics.median(windows), 5),
                           "steps_each": args.steps},
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16", "data": "synthetic (seeded; stands in for the reference datasets)",
        "precision": PRECISION_TEXT[args.precision],
        "config": bench_config(world, B),
        "graph": "one CUDA graph per step", "list_overflow": overflow,
        "autotuned": {"block": tuned["block"], "shade": tuned["shade"],
                      "frag_records_per_px": round(tuned["frag_records"], 3),
                      "list_capacity": tuned["list_capacity"],
                      "ms_per_step_by_layout": {k: round(v, 4) for k, v in tuned["ms_per_step"].items()}},
        "e2e": {"value": e2e, "unit": "views/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 4},
        "mfragments_per_s": nfrag * args.steps * world / (ms / 1000.0) / 1e6,
        "fragments_per_step": int(nfrag),
        "gpu_launches": KERNELS_PER_STEP * args.steps,
        "clocks": clocks,
        "phase_ms": {k: round(v, 4) for k, v in phase_ms.items()},
        "step_roofline": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_bytes / (ms / args.steps / 1000.0)
                          / 1e9, "frac": step_bytes / (ms / args.steps / 1000.0) / 1e9 / peak, "unit": "GB/s"},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                     "algorithmic_bytes": alg},
    }
    if side is not None:
        line["side"] = side
    if plain is not None:
        line["plain_fp32"] = plain
        line["speedup_vs_plain_fp32"] = value / plain["value"]
    if cpu_base is not None:
        line["cpu_baseline"] = cpu_base
    if render is not None:
        line["render"] = render
    if remesh_line is not None:
        line["remesh"] = remesh_line
    if rank == 0:
        print(json.dumps(line), flush=True)
    del graphs, egraphs
    replicas.shutdown(rep)


def count_fragments(hw, pos, tri) -> int:
    """Covered fragments (every (pixel, triangle) pair passing the coverage test, before the depth test)
    of every view, counted by the library's fragment operators one view at a time."""
    import diffsoup_b200 as ds

    n = 0
    for b, (H, W) in enumerate(hw):
        fp, _ = ds.rasterize._compute_fragments((H, W), pos[b:b + 1].contiguous(), tri)
        n += int(fp.shape[0])
        del fp
    return n


# Side workloads: (entry, benchmark configuration, shading model, precision, fragment records per pixel;
# None = the autotuner sizes the record store, 0 = tile-wise recomputation of the fragments)
SIDE_WORKLOADS = [
    ("config2_reference_model_split", 2, "reference", "split", None),
    ("config2_reference_model_bf16", 2, "reference", "bf16", None),
    ("config1", 1, "config", "split", None),
    ("config3", 3, "config", "split", None),
    ("config4_bf16", 4, "config", "bf16", None),
    ("config4_split", 4, "config", "split", None),
    ("config5_records", 5, "config", "bf16", None),
    ("config5_recompute", 5, "config", "bf16", 0.0),
]
SIDE_TEXT = {
    1: "config1: 5K-tri soup in U[-1,1]^3, 1 view 256x256, levels 0..2 x 8 ch, MLP 11-16-3",
    2: "config2: 15K-tri sphere-shell soup, 8 views 800x800, levels 0..2",
    3: "config3: 50K tris in 20 clusters + 10K on a shell of radius 10, 64 views of uneven size (widths 400..1200, "
       "aspects 4:3/16:9/1:1), levels 0..2 x 8 ch, MLP 11-16-3, one CUDA graph",
    4: "config4: 5K-tri soup, 1 view 256x256, levels 0..3 x 16 ch, MLP 19-64-64-3",
    5: "config5: 200K tris (shell + clusters), 16 views 1920x1080, levels 0..3 x 16 ch, MLP 19-64-64-3",
}


def measure_workload(dev, sc, mlp, precision: str, steps: int, warmup: int, peak: float,
                     frag_records=None, cpu_sample: bool = True) -> dict:
    """One side workload: autotuned, captured in one CUDA graph, `warmup` untimed replays, then `steps`
    replays each timed with CUDA events and each preceded by an L2 flush (a 256 MB write, outside the
    timed pair).  Also the per-phase kernel times (the step's profiling events over eager steps), the
    dominant kernel's roofline fraction, covered fragments per second, the device memory the step holds
    and a CPU sample (view 0 through the FP32 oracle port)."""
    from diffsoup_b200 import _core
    from diffsoup_b200.step import TrainStep

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    hw = [(v.height, v.width) for v in sc.views]
    B, T, V = len(hw), sc.T, sc.verts.shape[0]
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats(dev)
    base_mem = torch.cuda.memory_allocated(dev)
    kw = dict(verts=t(sc.verts), tri=t(sc.tri), mvp=t(sc.mvps()), inv_mvp=t(sc.inv_mvps()), feat_src=t(sc.feat_src),
              alpha_src=t(sc.alpha_src[..., 0]), mlp_params=t(mlp_flat(mlp)),
              target=t(np.concatenate([x.reshape(-1, 3) for x in sc.targets])))
    step = TrainStep(T, V, hw, sc.feat_dim, sc.min_level, sc.max_level, sc.hidden_dim, sc.n_layers, stochastic=True,
                     seed=99, device=dev, precision=precision, view_enc=sc.view_enc,
                     frag_records=2.0 if frag_records is None else frag_records)
    tuned = step.autotune(**kw, steps=3)
    g = step.capture(**kw)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(warmup):
        g.replay()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in ev:
        flush.zero_()
        a.record()
        g.replay()
        b.record()
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    mem = torch.cuda.max_memory_allocated(dev) - base_mem - flush.numel()
    overflow = step.overflowed()
    del g, flush
    # per-phase kernel time
    names = ["prep", "bin", "raster", "shade", "aux", "edge", "finish"]
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(8)]
    for e in evs:
        e.record()
    torch.cuda.synchronize()
    _core.check(_core.lib.ds_train_step_set_events(ctypes_void_p_array(evs), 8))
    M = 5

    def phases():
        acc = {n: 0.0 for n in names}
        for _ in range(M):
            step.run(**kw)
            torch.cuda.synchronize()
            for k, n in enumerate(names):
                acc[n] += evs[k].elapsed_time(evs[k + 1])
        return {n: acc[n] / M for n in names}

    phase_ms = phases()
    # both shading kernels of the wide BF16 MLP, phase by phase (the autotuned one is kept)
    shade_ab = None
    if step.tcgen05_shading():
        chosen = step.cfg.shade_mode
        shade_ab = {}
        for mode in (0, 1):
            step.cfg.shade_mode = mode
            shade_ab[step.SHADE_MODES[mode]] = round(phases()["shade"], 4)
        step.cfg.shade_mode = chosen
    _core.check(_core.lib.ds_train_step_set_events(None, 0))
    dom = max(["raster", "shade", "aux", "edge"], key=lambda n: phase_ms[n])
    ST = _core.feats_at_level(sc.max_level)
    alg = algorithmic_bytes(dom, step.num_pixels, B, T, V, ST, sc.feat_dim, 4 if precision == "split" else 2)
    achieved = alg / (phase_ms[dom] / 1000.0) / 1e9
    try:
        nfrag = count_fragments(hw, step.intermediate("pos").clone(), kw["tri"])
    except RuntimeError:
        nfrag = None
    out = {"precision": PRECISION_TEXT[precision], "views_per_step": B, "triangles": T, "pixels_per_step": step.num_pixels,
           "value": B / (ms / 1000.0), "unit": "views/s", "ms_per_step": ms, "steps": steps, "warmup": warmup,
           "l2": "flushed (256 MB write) before every timed step",
           "mfragments_per_s": None if nfrag is None else nfrag / (ms / 1000.0) / 1e6, "fragments_per_step": nfrag,
           "phase_ms": {k: round(v, 4) for k, v in phase_ms.items()},
           "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "algorithmic_bytes": alg},
           "device_memory_bytes": int(mem), "workspace_bytes": int(step.workspace.numel()),
           "fragment_records": "tile-wise recomputation" if step.record_capacity == 0 else
                               f"stored ({step.cfg.frag_records:.3f} per pixel)",
           "autotuned": {"block": tuned["block"], "shade": tuned["shade"], "list_capacity": tuned["list_capacity"],
                         "ms_per_step_by_layout": {k: round(v, 4) for k, v in tuned["ms_per_step"].items()}},
           "list_overflow": overflow}
    if shade_ab is not None:
        out["shade_phase_ms_by_kernel"] = shade_ab
    del step, kw
    if cpu_sample:
        from oracle import cpu, pipeline as P

        v0 = sc.views[0]
        inp = P.StepInputs(verts=sc.verts, tri=sc.tri, mvps=sc.mvps()[:1], inv_mvps=sc.inv_mvps()[:1],
                           hw=[(v0.height, v0.width)], feat_src=sc.feat_src, alpha_src=sc.alpha_src[..., 0], mlp=mlp,
                           targets=sc.targets[:1], min_level=sc.min_level, max_level=sc.max_level, stochastic=True,
                           seed=99, iteration=0, view_enc=sc.view_enc)
        t0 = time.perf_counter()
        P.train_step(inp, "f32")
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "views/s", "cores": cpu.omp_threads(), "kind": "port",
                               "sample": f"view 0 ({v0.width}x{v0.height}) through the FP32 oracle port"}
    return out


def run_side_entries(args, dev, peak: float) -> dict:
    """The reference's own shading model on the benchmark soup and the other benchmark configurations
    (seeded synthetic scenes of their shapes), with the same --steps / --warmup."""
    from diffsoup_b200 import scenes

    out = {}
    for name, config, shading, precision, records in SIDE_WORKLOADS:
        sc = scenes.make_scene(config, seed=0, shading=shading)
        mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=0)
        r = measure_workload(dev, sc, mlp, precision, args.steps, args.warmup, peak, records,
                             cpu_sample=not args.no_cpu_baseline and not name.endswith(("_bf16", "_recompute")))
        text = SIDE_TEXT[config]
        if shading == "reference":
            text += ", the reference's own shading model: 7 features + SH2 -> 16 -> 16 -> 3"
        r["workload"] = text
        out[name] = r
        del sc
    return out


def ctypes_void_p_array(events):
    import ctypes as C

    arr = (C.c_void_p * len(events))()
    for i, e in enumerate(events):
        arr[i] = C.c_void_p(e.cuda_event)
    return arr


def read_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for l in open(path):
            f = l.split()
            if len(f) >= 2 and f[0] == kernel and not l.startswith("#"):
                return float(f[1])
    except Exception:
        pass
    return None


def run_plain(sc, mlp, s, dev, n_views: int):
    """The drop-in API, one view per call, FP32, eager (no graph): the
    reference's own training-step structure (examples/02_synthetic.py:354-385)."""
    import diffsoup_b200 as ds

    mvp, inv, tgt = s
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    verts = t(sc.verts).requires_grad_(True)
    tri = t(sc.tri)
    feat_src = t(sc.feat_src).requires_grad_(True)
    alpha_src = t(sc.alpha_src).requires_grad_(True)
    net = ds.ColorMLP(sc.mlp_input_dim, 3, hidden_dim=sc.hidden_dim, n_layers=sc.n_layers).to(dev)
    with torch.no_grad():
        lins = [m for m in net.mlp if isinstance(m, torch.nn.Linear)]
        for lin, (W, b) in zip(lins, mlp):
            lin.weight.copy_(t(W))
            lin.bias.copy_(t(b))
    mvps, invs = t(mvp), t(inv)
    tg = t(target_f32(tgt).reshape(-1, 800, 800, 3))
    lo, hi = sc.min_level, sc.max_level

    def one(b):
        vh = torch.cat([verts, torch.ones_like(verts[:, :1])], dim=-1)
        clip = torch.einsum("bij,nj->bni", mvps[b:b + 1], vh).contiguous()
        alpha_acc = ds.accumulate_to_level(lo, hi, alpha_src).sigmoid()
        feat_acc = ds.accumulate_to_level(lo, hi, feat_src).sigmoid()
        rast = ds.rasterize_multires_triangle_alpha((800, 800), clip, tri, hi, alpha_acc)
        feat = ds.multires_triangle_color(rast, hi, feat_acc)
        x = torch.cat([feat, ds.encode_view_dir(rast, invs[b:b + 1])], dim=-1)
        color = net(x, mask=rast[..., -1] > 0)
        m = (rast.detach()[..., -1:] > 0).float()
        color = m * color + (1.0 - m)
        target = tg[b:b + 1]
        aux = ds.opacity_aux_loss(color.detach(), target, rast, clip, tri, hi, alpha_acc)
        color = ds.edge_grad(color, rast, clip, tri)
        loss = aux + ((color - target) ** 2).mean()
        for p in (verts, feat_src, alpha_src, *net.parameters()):
            p.grad = None
        loss.backward()
        return loss

    nb = mvps.shape[0]
    for i in range(4):
        one(i % nb)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(n_views):
        one(i % nb)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": n_views / (ms / 1000.0), "unit": "views/s", "views": n_views,
            "path": "diffsoup_b200 drop-in API, one 800x800 view per call, FP32, eager autograd, torch ColorMLP"}


def run_render(dev, cpu_sample: bool = True, frames: int = 200):
    """The viewer's frame (examples/05_benchmark_fps.py, Viewer::launch_benchmark)
    on the soup of the training workload: 15K triangles, LUT at level 5, MLP
    16-16-16-3, 800x800.  Single-view frames as the viewer draws them (one CUDA
    graph replay each, mean over the 8 cameras), 8 views per call, and the
    deferred-shading kernel alone on the same G-buffer."""
    from diffsoup_b200 import _core, scenes, viewer

    vi = scenes.make_viewer_inputs(2, seed=0, level=5)
    (W1, b1), (W2, b2), (W3, b3) = vi.mlp
    r = viewer.Renderer(vi.verts, vi.faces, vi.lut0, vi.lut1, W1, b1, W2, b2, W3, b3, level=vi.level, device=dev)
    H, W, B = vi.height, vi.width, vi.mvps.shape[0]
    for _ in range(2):
        r.render(vi.mvps, H, W)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # one view per frame, as the viewer renders
    for b in range(B):  # a bin-list capacity that fits every single view
        f1 = r.frame(vi.mvps[b:b + 1], H, W)
    g1 = f1.capture()
    per_view = []
    for b in range(B):
        f1.set_views(torch.from_numpy(vi.mvps[b:b + 1]))
        for _ in range(3):
            g1.replay()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(frames // B):
            g1.replay()
        e1.record()
        e1.synchronize()
        per_view.append(e0.elapsed_time(e1) / (frames // B))
    ms1 = sum(per_view) / len(per_view)
    # all 8 views in one call
    f8 = r.frame(vi.mvps, H, W)
    g8 = f8.capture()
    for _ in range(3):
        g8.replay()
    torch.cuda.synchronize()
    n8 = max(5, frames // B)
    e0.record()
    for _ in range(n8):
        g8.replay()
    e1.record()
    e1.synchronize()
    ms8 = e0.elapsed_time(e1) / n8
    # the post pass alone on the 8-view G-buffer (inputs: 8 x 640K x 16 B > L2)
    covered = int((f8.gbuf[:, 3] > 0).sum().item())
    P = f8.num_pixels

    def post():
        _core.check(_core.lib.ds_render_deferred(
            B, _core.ptr(f8.views), P, _core.ptr(f8.gbuf), r.level, _core.ptr(r.lut0), _core.ptr(r.lut1),
            r.lut0.shape[0], _core.ptr(f8.inv_mvp), _core.ptr(r.mlp), 1.0, 1.0, 1.0, _core.ptr(None),
            _core.ptr(f8.rgba8), _core.stream()))

    for _ in range(3):
        post()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(50):
        post()
    e1.record()
    e1.synchronize()
    post_ms = e0.elapsed_time(e1) / 50
    alg = 20.0 * P + 24.0 * covered  # G-buffer read + RGBA8 write + 6 texels of 4 B per covered pixel
    flops = 2.0 * (256 + 256 + 48) * covered
    out = {"workload": "viewer frame: 15,000 triangles, LUT level 5 (561 texels/face, RGBA8 x 2), "
                       "MLP 16-16-16-3 with SH2, 800x800, background white",
           "ms_per_frame": ms1, "fps": 1000.0 / ms1, "ms_per_frame_by_view": [round(t, 4) for t in per_view],
           "views_per_s_batched": B * 1000.0 / ms8, "views_per_call": B,
           "post_pass": {"ms_per_8_views": post_ms, "covered_fraction": covered / P,
                         "achieved_gbs": alg / (post_ms / 1000.0) / 1e9, "fp32_tflops": flops / (post_ms / 1000.0) / 1e12,
                         "algorithmic_bytes": alg},
           "gpu_launches_per_frame": RENDER_KERNELS_PER_FRAME}
    del g1, g8
    if cpu_sample:
        from oracle import cpu, viewer as ov
        t0 = time.perf_counter()
        pos = cpu.project(vi.verts, vi.mvps[:1])
        S = r.S
        alpha = (vi.lut1.reshape(-1, 4)[:, 3].astype(np.float32) / np.float32(255))[:r.T * S].reshape(r.T, S)
        g, _ = cpu.rasterize_alpha(H, W, pos, vi.faces, vi.level, alpha, False)
        inv = np.linalg.inv(vi.mvps[:1].astype(np.float64)).astype(np.float32)
        ov.to_rgba8(ov.post_pass(g, inv, vi.level, vi.lut0, vi.lut1, [a for wb in vi.mlp for a in wb]))
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"fps": 1.0 / dt, "cores": cpu.omp_threads(), "kind": "port",
                               "sample": "1 frame of view 0: oracle rasterizer (OpenMP) + numpy FP64 post pass"}
    return out


def run_remesh(dev, cpu_sample: bool = True, reps: int = 5):
    """The resampling step's subdivision on the benchmark soup: 15,000 faces
    split in screen space under one 800x800 view until every edge is below
    0.004 image heights (split_triangle_soup_clip_until), timed end to end
    through the public call with device tensors (two kernels, one scan and the
    count read back), beside the reference's own CPU remesher."""
    from diffsoup_b200 import remesh, scenes

    sc = scenes.make_scene(2, seed=0, num_views=1, with_targets=False)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    args = ((800, 800), t(sc.mvps()[0]), t(sc.verts), t(sc.tri), t(np.ones(sc.T, np.int32)), 0.004)
    out = remesh.split_triangle_soup_clip_until(*args)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        out = remesh.split_triangle_soup_clip_until(*args)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1000.0 / reps
    res = {"workload": "split_triangle_soup_clip_until, 15,000 faces, 800x800 view, tau_ratio 0.004",
           "faces_out": int(out[1].shape[0]), "splits": int(out[1].shape[0]) - sc.T, "ms": ms,
           "msplits_per_s": (int(out[1].shape[0]) - sc.T) / ms / 1e3}
    if cpu_sample:
        from oracle import remesh as R
        if R.reference_available():
            t0 = time.perf_counter()
            R.reference_split(sc.verts, sc.tri, -1, 0.004, mvp=sc.mvps()[0], valid=np.ones(sc.T, np.int32),
                              aspect_wh=1.0)
            res["cpu_baseline"] = {"ms": (time.perf_counter() - t0) * 1000.0, "cores": 1, "kind": "reference",
                                   "sample": "the same call through the reference's own remesher (src/remesh_clip.cpp,"
                                             " one host thread, as the reference runs it)"}
    return res


def run_cpu_baseline(sc, mlp, s):
    from oracle import cpu, pipeline as P

    mvp, inv, tgt = s
    cores = cpu.omp_threads()
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    t0 = time.perf_counter()
    n = 0
    while n < 8 and (n < 2 or time.perf_counter() - t0 < 15.0):
        b = n % 8
        inp = P.StepInputs(verts=sc.verts, tri=sc.tri, mvps=mvp[b:b + 1], inv_mvps=inv[b:b + 1], hw=[(800, 800)],
                           feat_src=sc.feat_src, alpha_src=sc.alpha_src[..., 0], mlp=mlp,
                           targets=[target_f32(tgt).reshape(-1, 800, 800, 3)[b]], min_level=sc.min_level, max_level=sc.max_level,
                           stochastic=True, seed=7, iteration=n)
        P.train_step(inp, "f32")
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "views/s", "cores": cores, "kind": "port",
            "sample": f"{n} views of config 2 (800x800, 15K tris) through the FP32 oracle port, {cores} threads"}


def measured_peak():
    """HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json, else the pool's earlier measurement."""
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    return float(peaks.get("hbm_gbs", 6650.0)), ("measured" if "hbm_gbs" in peaks else "fallback")


def run_side_case(args):
    """One side workload alone (a small profiling case with --side-views)."""
    from diffsoup_b200 import scenes

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    name, config, shading, precision, records = next(w for w in SIDE_WORKLOADS if w[0] == args.side_case)
    sc = scenes.make_scene(config, seed=0, shading=shading, num_views=args.side_views)
    mlp = scenes.mlp_weights(sc.mlp_input_dim, 3, sc.hidden_dim, sc.n_layers, seed=0)
    r = measure_workload(dev, sc, mlp, precision, args.steps, args.warmup, measured_peak()[0], records,
                         cpu_sample=False)
    print(json.dumps({"side_case": name, "views": len(sc.views), **r}), flush=True)


def main():
    args = parse()
    if args.side_case:
        run_side_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark: forward + adjoint + Adam iterations of the plain method on a
Kuhn 64^3 grid (1,572,864 tets, 274,625 vertices) at 1024x1024, one camera per
step, fitting RGBA and positions to target images of a different-seed mesh
of the same topology (seeded synthetic inputs; no dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is device-timed iterations/s with all
inputs resident in HBM; `e2e` is the same loop through the public Python API
(DifferentiableRenderer + l2_loss + optim.Adam) with each step's target image
copied from pinned host memory (on a copy stream, while the previous step
computes) and the loss read back (to pinned memory; the host reads it once the
next step is queued).  Under torchrun each
rank runs an independent replica (the path has no data-path collective).
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adj iter/s at 1.57M tets 1024²"
# Kernels of this library per timed step of the plain method: project 1,
# count 2 (32- and 64-bit faces) + row prefix 1, scan 3, fill order 3 (band
# count, scan, scatter) + fill 2, sort 8 (classify, five register /
# distribution classes, shared-memory and block classes), composite 1;
# adjoint 1 + scatter 1; l2 loss 1; Adam 2 (colours, positions).
LIST_STEP_LAUNCHES = 1 + 3 + 3 + 3 + 2 + 8 + 1 + 2 + 1 + 2
LR_COL, LR_POS = 1e-2, 1e-4


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=64, help="Kuhn grid cubes per axis")
    ap.add_argument("--res", type=int, default=1024)
    ap.add_argument("--views", type=int, default=16)
    ap.add_argument("--cpu-steps", type=int, default=2, help="whole CPU-port steps timed for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel configuration")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-raytet", action="store_true")
    ap.add_argument("--profile", choices=["ppll", "intersection", "cells"], default=None,
                    help="profiling case: Kuhn --n^3 at --res^2, one warm-up and one render + adjoint, no timing "
                         "(cells: one RGBA per tet, the cell mean of the vertex colours)")
    ap.add_argument("--no-scale", action="store_true")
    ap.add_argument("--no-next", action="store_true", help="skip the per-cell and regularizer sections")
    ap.add_argument("--scale-n", type=int, default=128)
    ap.add_argument("--scale-res", type=int, default=2048)
    ap.add_argument("--scale-steps", type=int, default=5)
    ap.add_argument("--scale-warmup", type=int, default=3)
    ap.add_argument("--scale-cap-gb", type=float, default=40.0)
    ap.add_argument("--scale-recompute-gb", type=float, default=4.0)
    ap.add_argument("--batched-res", type=str, default="512,1024")
    ap.add_argument("--batched-steps", type=int, default=20)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-rates", type=str, default="50,200,500,1000,2000")
    ap.add_argument("--serving-requests", type=int, default=150,
                    help="requests per rate (at least one second of arrivals is used, up to 1000)")
    ap.add_argument("--serving-slots", type=int, default=4)
    ap.add_argument("--serving-batch-mfrags", type=float, default=16.0,
                    help="estimated fragments (millions) a serving batch is filled to")
    ap.add_argument("--serving-priority-slots", type=int, default=0,
                    help="slots on a high-priority stream taking the largest queued request alone")
    ap.add_argument("--serving-policy", choices=["fifo", "sjf"], default="sjf")
    ap.add_argument("--serving-isolated", type=int, default=500, help="requests timed alone for the isolated p99")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic_per_unit():
    """Per-launch DRAM traffic of the dominant kernels per fragment, from one ncu
    capture summarised in profiles/roofline_traffic.json (None if absent)."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


RED_PROBE_SRC = r"""
extern "C" __global__ void red_probe(float4* rows, unsigned nrows, unsigned iters, unsigned seed) {
    unsigned h = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + seed;
    for (unsigned i = 0; i < iters; ++i) {
        h = h * 1664525u + 1013904223u;
        const unsigned r = (h >> 8) % nrows;
        atomicAdd(rows + 2 * r, make_float4(1.f, 1.f, 1.f, 0.f));
        atomicAdd(rows + 2 * r + 1, make_float4(1.f, 1.f, 1.f, 1.f));
    }
}
"""


def l2_red_peak(num_rows: int):
    """Float4 atomic adds per second that the L2 reduction units take when
    every lane adds two float4 (one 32-byte row) into random rows of a table of
    num_rows rows: the pattern of the adjoint's vertex-row atomics with no
    other work.  Compiled at run time (NVRTC, sm_100a), launched on torch's
    current stream, timed with CUDA events (best of 3)."""
    import ctypes
    import torch
    from cuda.bindings import driver, nvrtc

    err, prog = nvrtc.nvrtcCreateProgram(RED_PROBE_SRC.encode(), b"red_probe.cu", 0, [], [])
    opts = [b"--gpu-architecture=sm_100a", b"-std=c++17"]
    (err,) = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
    if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
        raise RuntimeError(f"NVRTC: {err}")
    err, size = nvrtc.nvrtcGetCUBINSize(prog)
    cubin = b" " * size
    (err,) = nvrtc.nvrtcGetCUBIN(prog, cubin)
    torch.cuda.init()
    err, mod = driver.cuModuleLoadData(cubin)
    if err != driver.CUresult.CUDA_SUCCESS:
        raise RuntimeError(f"cuModuleLoadData: {err}")
    err, fn = driver.cuModuleGetFunction(mod, b"red_probe")
    rows = torch.zeros(2 * num_rows, 4, device="cuda")
    blocks, threads, iters = 148 * 8, 256, 128
    stream = torch.cuda.current_stream().cuda_stream
    args = ((rows.data_ptr(), num_rows, iters, 7), (ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint))
    best = None
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        (err,) = driver.cuLaunchKernel(fn, blocks, 1, 1, threads, 1, 1, 0, stream, args, 0)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    driver.cuModuleUnload(mod)
    return 2.0 * blocks * threads * iters / (best / 1e3)


# ---------------------------------------------------------------------------
def build_scene(args, device, renderer_type=None):
    import numpy as np
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S

    cells, pos = S.kuhn_mesh(args.n, seed=0)
    col = S.gaussian_colors(pos, seed=0)
    _, pos_t = S.kuhn_mesh(args.n, seed=1)
    col_t = S.gaussian_colors(pos_t, seed=1)
    views = [S.sphere_camera(100 + i) for i in range(args.views)]

    def make(cells, pos, col):
        mesh = d.TetMesh()
        mesh.set_use_gradients(True)
        mesh.set_tet_mesh_data(cells, pos, col)
        r = d.Renderer(d.RendererType.PPLL if renderer_type is None else renderer_type)
        r.set_tet_mesh(mesh)
        r.set_viewport_size(args.res, args.res)
        r.set_camera_fovy(S.FOVY_45)
        r.set_attenuation(1.0)
        r.set_clear_color(d.vec4(0, 0, 0, 0))
        return mesh, r

    mesh_t, r_t = make(cells, pos_t, col_t)
    targets = []
    with torch.no_grad():
        for v in views:
            r_t.set_view_matrix(v)
            targets.append(r_t.render().clone())
    del r_t, mesh_t
    mesh, r = make(cells, pos, col)
    return {"cells": cells, "pos": pos, "col": col, "views": views, "targets": targets, "mesh": mesh,
            "renderer": r, "np": np}


def max_over_ranks(ms: float, world: int, device=None) -> float:
    """The slowest rank's device-timed duration (every rank calls this with its
    own CUDA-event time; all ranks get the maximum)."""
    if world <= 1:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, ms: float) -> float:
    """Iterations/s of the whole job: every rank (replica) ran `steps` views."""
    return world * steps / (ms / 1e3)


def run_ours(args, rank, world):
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import _lib
    from difftetvr_b200.optim import CLAMP_NONNEGATIVE, Adam, l2_loss

    device = torch.device("cuda", torch.cuda.current_device())
    sc = build_scene(args, device)
    mesh, r, views, targets = sc["mesh"], sc["renderer"], sc["views"], sc["targets"]
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    opt = Adam([{"params": [col], "lr": LR_COL, "clamp": CLAMP_NONNEGATIVE},
                {"params": [pos], "lr": LR_POS}], betas=(0.9, 0.999), eps=1e-8)
    n_img = targets[0].numel()
    adj = torch.empty_like(targets[0])
    loss_acc = torch.zeros(1, device=device)
    stream = torch.cuda.current_stream(device)
    # Kernel configuration from the library's autotuner on the first view
    # (pixel tiles of composite / adjoint, sort method per list-length class).
    from difftetvr_b200.autotune import autotune_renderer
    r.set_view_matrix(views[0])
    tuned = r.get_tuning() if args.no_autotune else autotune_renderer(r)["tuning"]

    def step(i):
        # Device-resident step: render, fused loss + image adjoint, adjoint, Adam.
        pos.grad.zero_()
        col.grad.zero_()
        r.set_view_matrix(views[i % len(views)])
        image = r.render()
        _lib.call("dtv_loss_l2", image.data_ptr(), targets[i % len(views)].data_ptr(), n_img,
                  1.0 / n_img, adj.data_ptr(), loss_acc.data_ptr(), stream.cuda_stream)
        r.render_adjoint(adj)
        opt.step()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for i in range(args.warmup):
        step(i)
    nf_sum = 0
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else torch.cuda.current_device())
    barrier()
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
        nf_sum += r.get_num_fragments()  # known since the render's scan read-back
    t1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(t0.elapsed_time(t1), world, device)
    value = whole_job_rate(world, args.steps, ms)

    # Stage breakdown (CUDA events on the launching stream) over a second pass
    # of the same number of steps: reading each step's events makes the host
    # wait, so this pass is not the timed one.
    r.set_stage_timing(True)
    stage_sum = {k: 0.0 for k in r.STAGES}
    for i in range(args.steps):
        step(args.warmup + args.steps + i)
        for k, v in r.get_stage_times().items():
            stage_sum[k] += v
    r.set_stage_timing(False)

    # End-to-end through the public API, host buffers in the timed region.
    e2e = None
    if not args.no_e2e:
        diff = d.DifferentiableRenderer(r)
        opt2 = Adam([{"params": [col], "lr": LR_COL, "clamp": CLAMP_NONNEGATIVE},
                     {"params": [pos], "lr": LR_POS}])
        host_targets = [t.cpu().pin_memory() for t in targets]
        h2d = host_targets[0].numel() * 4
        # Each step's target is copied from pinned host memory on a copy stream
        # into one of two device buffers while the previous step computes.
        dev_targets = [torch.empty_like(targets[0]) for _ in range(2)]
        copy_stream = torch.cuda.Stream()
        copied = [torch.cuda.Event(), torch.cuda.Event()]
        consumed = [torch.cuda.Event(), torch.cuda.Event()]

        def issue_copy(i):
            k = i % 2
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(consumed[k])  # the step that read this buffer is done with it
                dev_targets[k].copy_(host_targets[i % len(views)], non_blocking=True)
                copied[k].record(copy_stream)

        # Each step's loss is copied to pinned host memory right after the loss
        # kernel and read on the host once the next step is queued, so the
        # host never waits with the GPU idle.
        loss_host = torch.zeros(2, dtype=torch.float32).pin_memory()
        loss_read = [torch.cuda.Event(), torch.cuda.Event()]
        losses = []
        pending = [None]  # buffer holding a loss not read yet

        def read_pending():
            if pending[0] is not None:
                loss_read[pending[0]].synchronize()
                losses.append(float(loss_host[pending[0]]))
                pending[0] = None

        def e2e_step(i):
            k = i % 2
            opt2.zero_grad(set_to_none=False)
            r.set_view_matrix(views[i % len(views)])
            image = diff()
            stream.wait_event(copied[k])
            loss = l2_loss(image, dev_targets[k])
            consumed[k].record(stream)
            loss_host[k:k + 1].copy_(loss.detach(), non_blocking=True)
            loss_read[k].record(stream)
            issue_copy(i + 1)
            loss.backward()
            opt2.step()
            read_pending()  # the previous step's loss
            pending[0] = k

        issue_copy(0)
        for i in range(args.warmup):
            e2e_step(i)
        read_pending()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.warmup, args.warmup + args.steps):
            e2e_step(i)
        read_pending()
        e1.record(stream)
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1), world, device)
        e2e = {"value": whole_job_rate(world, args.steps, ems), "unit": "iter/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": 4, "ms_per_step": ems / args.steps,
               "api": "DifferentiableRenderer + optim.l2_loss + optim.Adam",
               "h2d_overlap": "each step's target copied on a copy stream while the previous step computes",
               "d2h": "each step's loss copied to pinned memory and read once the next step is queued"}

    # Roofline of the dominant kernel (algorithmic bytes per launch / its event time).
    K = args.steps
    avg = {k: v / K for k, v in stage_sum.items()}
    nf = nf_sum / K
    P = args.res * args.res
    V = mesh.get_num_vertices()
    F = mesh.get_num_faces()
    algo = {
        "composite": 8 * nf + 16 * P + 4 * P + 4 * P + 28 * V + 16 * F,
        "adjoint": 8 * nf + 36 * P + 16 * F + 28 * V + 28 * V,
        "fill": 8 * nf + 16 * F + 24 * V + 16 * P,
        "sort": 16 * nf + 16 * P,
        "count": 4 * P + 16 * F + 24 * V,
    }
    dominant = max(algo, key=lambda k: avg.get(k, 0.0))
    peak, peak_kind = measured_peaks()
    achieved = algo[dominant] / (avg[dominant] / 1e3) / 1e9
    tr = ncu_traffic_per_unit().get(dominant)
    traffic = None if tr is None else float(tr["bytes_per_fragment"]) * nf + float(tr.get("bytes_per_pixel", 0)) * P
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic, "algorithmic_bytes": algo[dominant], "kernel_ms": avg[dominant]}
    # The adjoint is bound by instruction issue and its vertex-row atomics, not
    # by HBM: its issue rate against 148 SMs x 4 schedulers x the sampled SM
    # clock, and its float4 atomic rate against the probe's, from the
    # per-fragment counts of one ncu capture (profiles/roofline_traffic.json).
    prof = ncu_traffic_per_unit().get("adjoint", {})
    t_adj = avg.get("adjoint", 0.0) / 1e3
    if t_adj > 0 and "warp_inst_per_fragment" in prof:
        sm_hz = (clk.get("sm_mhz") or 1965.0) * 1e6
        inst = float(prof["warp_inst_per_fragment"]) * nf / t_adj
        roofline["issue"] = {"kernel": "adjoint", "achieved_warp_inst_per_s": inst,
                             "peak_warp_inst_per_s": 148 * 4 * sm_hz, "frac": round(inst / (148 * 4 * sm_hz), 4),
                             "warp_inst_per_fragment": prof["warp_inst_per_fragment"]}
    if t_adj > 0 and "red_float4_per_fragment" in prof:
        try:
            red_peak = l2_red_peak(V)
        except Exception as exc:  # the probe is a report, not part of the step
            red_peak = None
            roofline["l2_red_error"] = str(exc)[:200]
        if red_peak:
            red = float(prof["red_float4_per_fragment"]) * nf / t_adj
            roofline["l2_red"] = {"kernel": "adjoint", "achieved_float4_per_s": red, "peak_float4_per_s": red_peak,
                                  "frac": round(red / red_peak, 4), "per_fragment": prof["red_float4_per_fragment"],
                                  "peak_source": "float4 atomicAdd probe over random 32-byte rows of a "
                                                 f"{V}-row table (bench.py l2_red_peak)"}

    result = {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Kuhn grid, Gaussian densities, sphere cameras)",
        "config": {"workload": f"plain method, Kuhn {args.n}^3 ({6 * args.n ** 3} tets, {V} verts), "
                               f"{args.res}x{args.res}, one camera per step, fwd+adj+Adam",
                   "tets": 6 * args.n ** 3, "vertices": V, "faces": F, "res": args.res,
                   "fragments_per_step": nf, "views": len(views), "parallelism": f"replicas x{world}",
                   "tuning": tuned,
                   "l2": "inputs larger than L2 (fragment records ~%.1f GB per step)" % (8 * nf / 1e9)},
        "e2e": e2e,
        "gpu_launches": LIST_STEP_LAUNCHES * K,
        "stage_ms": {k: round(v, 4) for k, v in avg.items()},
        "fragments_per_s": nf * value / world * world,
        "roofline": roofline,
        "clocks": clk,
    }
    return result, sc


def run_raytet(args):
    """Ray-tet traversal path (intersection renderer) on the plain workload:
    same mesh, views, targets and step (render, loss, adjoint, Adam)."""
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import _lib
    from difftetvr_b200.optim import CLAMP_NONNEGATIVE, Adam

    device = torch.device("cuda", torch.cuda.current_device())
    sc = build_scene(args, device, d.RendererType.INTERSECTION)
    mesh, r, views, targets = sc["mesh"], sc["renderer"], sc["views"], sc["targets"]
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    opt = Adam([{"params": [col], "lr": LR_COL, "clamp": CLAMP_NONNEGATIVE},
                {"params": [pos], "lr": LR_POS}], betas=(0.9, 0.999), eps=1e-8)
    n_img = targets[0].numel()
    adj = torch.empty_like(targets[0])
    loss_acc = torch.zeros(1, device=device)
    stream = torch.cuda.current_stream(device)

    def step(i):
        pos.grad.zero_()
        col.grad.zero_()
        r.set_view_matrix(views[i % len(views)])
        image = r.render()
        _lib.call("dtv_loss_l2", image.data_ptr(), targets[i % len(views)].data_ptr(), n_img,
                  1.0 / n_img, adj.data_ptr(), loss_acc.data_ptr(), stream.cuda_stream)
        r.render_adjoint(adj)
        opt.step()

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    # Stage breakdown on separate steps (stage events add host waits).
    r.set_stage_timing(True)
    stage_sum, segs = {k: 0.0 for k in r.STAGES}, 0
    n_st = min(args.steps, 5)
    for i in range(n_st):
        step(i)
        for k, v in r.get_stage_times().items():
            stage_sum[k] += v
        segs += int(r.get_pixel_state()[1].sum())
    r.set_stage_timing(False)
    out = {"iter_per_s": 1e3 / ms, "ms_per_step": ms, "segments_per_step": segs / n_st,
           "boundary_fragments_per_step": r.get_num_fragments(),
           "stage_ms": {k: round(v / n_st, 4) for k, v in stage_sum.items()},
           "note": "segments = (pixel, tet) pairs composited; stages count/fill/sort run on boundary faces only"}
    del sc
    torch.cuda.empty_cache()
    return out


def run_cells_and_regularizer(args):
    """The path's next rows on the plain workload: per-cell colours (the same
    Kuhn mesh with one RGBA per tet, the cell mean of the vertex colours; step
    = render, fused L2 loss, adjoint, Adam on positions and cell colours) and
    the tet-quality regularizer's gradient over all tets (lambda 0.1, softplus
    beta 100: the reference training script's defaults)."""
    import numpy as np
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import _lib
    from difftetvr_b200 import synthetic as S
    from difftetvr_b200.optim import CLAMP_NONNEGATIVE, Adam

    device = torch.device("cuda", torch.cuda.current_device())
    cells, pos = S.kuhn_mesh(args.n, seed=0)
    _, pos_t = S.kuhn_mesh(args.n, seed=1)
    views = [S.sphere_camera(100 + i) for i in range(args.views)]

    def cell_colors(p, seed):
        return S.gaussian_colors(p, seed=seed)[cells].mean(axis=1).astype(np.float32)

    def make(p, cc):
        m = d.TetMesh()
        m.set_use_gradients(True)
        m.set_tet_mesh_data_cell(cells, p, cc)
        r = d.Renderer(d.RendererType.PPLL)
        r.set_tet_mesh(m)
        r.set_viewport_size(args.res, args.res)
        r.set_camera_fovy(S.FOVY_45)
        r.set_attenuation(1.0)
        r.set_clear_color(d.vec4(0, 0, 0, 0))
        return m, r

    m_t, r_t = make(pos_t, cell_colors(pos_t, 1))
    targets = []
    with torch.no_grad():
        for v in views:
            r_t.set_view_matrix(v)
            targets.append(r_t.render().clone())
    del r_t, m_t
    mesh, r = make(pos, cell_colors(pos, 0))
    p, cc = mesh.get_vertex_positions(), mesh.get_cell_colors()
    opt = Adam([{"params": [cc], "lr": LR_COL, "clamp": CLAMP_NONNEGATIVE},
                {"params": [p], "lr": LR_POS}], betas=(0.9, 0.999), eps=1e-8)
    n_img = targets[0].numel()
    adj = torch.empty_like(targets[0])
    loss_acc = torch.zeros(1, device=device)
    stream = torch.cuda.current_stream(device)

    def step(i):
        p.grad.zero_()
        cc.grad.zero_()
        r.set_view_matrix(views[i % len(views)])
        image = r.render()
        _lib.call("dtv_loss_l2", image.data_ptr(), targets[i % len(views)].data_ptr(), n_img,
                  1.0 / n_img, adj.data_ptr(), loss_acc.data_ptr(), stream.cuda_stream)
        r.render_adjoint(adj)
        opt.step()

    def timed(fn, warmup, n):
        for i in range(warmup):
            fn(i)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i in range(n):
            fn(warmup + i)
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / n

    ms = timed(step, max(args.warmup, 3), args.steps)
    r.set_stage_timing(True)
    stage_sum = {k: 0.0 for k in r.STAGES}
    n_st = min(args.steps, 5)
    for i in range(n_st):
        step(i)
        for k, v in r.get_stage_times().items():
            stage_sum[k] += v
    r.set_stage_timing(False)
    cells_out = {"iter_per_s": 1e3 / ms, "ms_per_step": ms, "fragments_per_step": r.get_num_fragments(),
                 "stage_ms": {k: round(v / n_st, 4) for k, v in stage_sum.items()},
                 "workload": f"Kuhn {args.n}^3 with per-cell RGBA at {args.res}x{args.res}, one camera per step"}
    reg = d.TetRegularizer(mesh, 0.1, 100.0)
    reg_ms = timed(lambda i: reg.compute_grad(), 3, 20)
    T = int(cells.shape[0])
    reg_out = {"ms_per_call": reg_ms, "tets_per_s": T / (reg_ms / 1e3), "tets": T,
               "note": "gradient of the tet-quality penalty added into the position .grad (float atomics)"}
    del r, mesh
    torch.cuda.empty_cache()
    return cells_out, reg_out


def run_scale(args):
    """Differentiation at scale: Kuhn n^3 at res^2, forward + autograd backward
    (DifferentiableRenderer, L2 loss against a second-seed target) + Adam, with
    the fragment lists stored whole under a 40 GB cap vs rebuilt per row band in
    backward under a smaller budget."""
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    from difftetvr_b200.optim import CLAMP_NONNEGATIVE, Adam, l2_loss

    n, res = args.scale_n, args.scale_res
    t_setup = time.perf_counter()
    cells, pos = S.kuhn_mesh(n, seed=0)
    col = S.gaussian_colors(pos, seed=0)
    _, pos_t = S.kuhn_mesh(n, seed=1)
    col_t = S.gaussian_colors(pos_t, seed=1)
    view = S.sphere_camera(100)

    def make(p, c):
        m = d.TetMesh()
        m.set_use_gradients(True)
        m.set_tet_mesh_data(cells, p, c)
        r = d.Renderer(d.RendererType.PPLL)
        r.set_tet_mesh(m)
        r.set_viewport_size(res, res)
        r.set_camera_fovy(S.FOVY_45)
        r.set_attenuation(1.0)
        r.set_clear_color(d.vec4(0, 0, 0, 0))
        r.set_view_matrix(view)
        return m, r

    m_t, r_t = make(pos_t, col_t)
    with torch.no_grad():
        target = r_t.render().clone()
    del r_t, m_t
    mesh, r = make(pos, col)
    setup_s = time.perf_counter() - t_setup
    p, c = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    opt = Adam([{"params": [c], "lr": LR_COL, "clamp": CLAMP_NONNEGATIVE}, {"params": [p], "lr": LR_POS}])
    diff = d.DifferentiableRenderer(r)
    stream = torch.cuda.current_stream()

    def step():
        opt.zero_grad(set_to_none=False)
        img = diff()
        loss = l2_loss(img, target)
        loss.backward()
        opt.step()
        return img

    out = {"workload": f"Kuhn {n}^3 ({6 * n ** 3} tets, {mesh.get_num_vertices()} verts), {res}x{res}, "
                       f"fwd + autograd bwd + Adam", "setup_s": round(setup_s, 1), "modes": []}
    for name, budget in (("stored", int(args.scale_cap_gb * 1e9)), ("recompute", int(args.scale_recompute_gb * 1e9))):
        r.set_fragment_budget_bytes(budget)
        for _ in range(args.scale_warmup):
            img = step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.scale_steps):
            img = step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.scale_steps
        nf = r.get_num_fragments()
        bands = r.get_num_bands()
        covered = int((img[..., 3] > 0).sum())
        # Stage times from one more step with stage events (not in the timed loop).
        r.set_stage_timing(True)
        step()
        torch.cuda.synchronize()
        stage = {k: round(v, 3) for k, v in r.get_stage_times().items()}
        r.set_stage_timing(False)
        out["modes"].append({
            "mode": name, "budget_bytes": budget, "bands": bands, "ms_per_step": ms, "iter_per_s": 1e3 / ms,
            "fragments": nf, "record_bytes": 8 * nf,
            "record_bytes_held": 8 * nf if bands == 0 else min(8 * nf, budget),
            "mean_list_length_covered": nf / max(covered, 1), "fragments_per_s": nf / (ms / 1e3),
            "stage_ms": stage})
    del diff, r, mesh
    torch.cuda.empty_cache()
    return out


def run_batched(args, res: int, steps: int, warmup: int = 2):
    """Batching config: meshes Kuhn 64^3 / 24^3 / 40^3, 32 views per step on a
    Fibonacci sphere split 16 / 10 / 6, all at res x res; forward + adjoint +
    Adam per step.  Batched (one launch per stage, CUDA graph) vs the plain
    one-view-per-launch loop on the same GPU, both device-timed."""
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import _lib
    from difftetvr_b200 import synthetic as S
    from difftetvr_b200.batch import BatchRenderer, View
    from difftetvr_b200.optim import CLAMP_NONNEGATIVE, Adam

    sizes = [64, 24, 40]
    counts = [16, 10, 6]

    def mk(n, seed):
        cells, pos = S.kuhn_mesh(n, seed=seed)
        m = d.TetMesh()
        m.set_use_gradients(True)
        m.set_tet_mesh_data(cells, pos, S.gaussian_colors(pos, seed=seed))
        return m

    cams = S.fibonacci_cameras(sum(counts))
    views, k = [], 0
    for mi, c in enumerate(counts):
        for _ in range(c):
            views.append(View(mesh=mi, view_matrix=cams[k], width=res, height=res))
            k += 1
    # Targets from seed+1 meshes of the same topology.
    tgt_meshes = [mk(n, 11 + i) for i, n in enumerate(sizes)]
    tr = BatchRenderer(tgt_meshes, attenuation=1.0)
    for v, img in zip(views, tr.render(views)):
        v.target = img.clone()
        v.image = None
    del tr, tgt_meshes
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()

    def timed(fn, n):
        for i in range(warmup):
            fn(i)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(n):
            fn(warmup + i)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    from difftetvr_b200.autotune import autotune_batch, autotune_renderer

    meshes = [mk(n, 1 + i) for i, n in enumerate(sizes)]
    br = BatchRenderer(meshes, attenuation=1.0)
    tuned_batch = autotune_batch(br, views)["tuning"]
    br.set_graph(True)
    ms_batched = timed(lambda i: br.train_step(views, lr_positions=LR_POS, lr_colors=LR_COL, clamp_colors=1), steps)
    info = br.info()
    del br

    meshes_p = [mk(n, 1 + i) for i, n in enumerate(sizes)]
    rends = []
    for m in meshes_p:
        r = d.Renderer(d.RendererType.PPLL)
        r.set_tet_mesh(m)
        r.set_viewport_size(res, res)
        r.set_camera_fovy(S.FOVY_45)
        r.set_attenuation(1.0)
        rends.append(r)
    opts = [Adam([{"params": [m.get_vertex_colors()], "lr": LR_COL, "clamp": CLAMP_NONNEGATIVE},
                  {"params": [m.get_vertex_positions()], "lr": LR_POS}]) for m in meshes_p]
    adj = torch.empty((res, res, 4), device="cuda")
    loss = torch.zeros(1, device="cuda")
    n_img = res * res * 4

    def plain_step(i):
        for o in opts:
            o.zero_grad(set_to_none=False)
        for v in views:
            r = rends[v.mesh]
            r.set_view_matrix(v.view_matrix)
            img = r.render()
            _lib.call("dtv_loss_l2", img.data_ptr(), v.target.data_ptr(), n_img, 1.0 / n_img, adj.data_ptr(),
                      loss.data_ptr(), stream.cuda_stream)
            r.render_adjoint(adj)
        for o in opts:
            o.step()

    # Each plain renderer tuned on its own mesh's first view, as the batch is.
    for mi, r in enumerate(rends):
        r.set_view_matrix(next(v.view_matrix for v in views if v.mesh == mi))
        autotune_renderer(r)
    ms_plain = timed(plain_step, steps)
    # Where the plain loop's time goes: one more step with per-view stage
    # events.  busy = the sum of the stage times (device work); the rest of
    # the step is launch and host time between views, which is what one launch
    # per stage over all views can remove.  plain / busy bounds the speed-up
    # of batching that keeps per-fragment work as it is.
    for r in rends:
        r.set_stage_timing(True)
    busy = {f"{n}^3": 0.0 for n in sizes}
    stage_busy = {}
    for o in opts:
        o.zero_grad(set_to_none=False)
    for v in views:
        r = rends[v.mesh]
        r.set_view_matrix(v.view_matrix)
        img = r.render()
        _lib.call("dtv_loss_l2", img.data_ptr(), v.target.data_ptr(), n_img, 1.0 / n_img, adj.data_ptr(),
                  loss.data_ptr(), stream.cuda_stream)
        r.render_adjoint(adj)
        st = r.get_stage_times()
        busy[f"{sizes[v.mesh]}^3"] += sum(st.values())
        for k2, v2 in st.items():
            stage_busy[k2] = stage_busy.get(k2, 0.0) + v2
    for r in rends:
        r.set_stage_timing(False)
    busy_total = sum(busy.values())
    # Each mesh's views alone: a batch of that mesh only (tuned, CUDA graph)
    # against the plain loop over the same views, both device-timed.  The
    # small meshes show how much launch and host time one launch per stage
    # removes when per-view work is small.
    per_mesh = {}
    k_steps = max(5, steps // 2)
    for mi, n in enumerate(sizes):
        own = [v for v in views if v.mesh == mi]
        vm = [View(mesh=0, view_matrix=v.view_matrix, width=res, height=res, target=v.target) for v in own]
        bm = BatchRenderer([mk(n, 1 + mi)], attenuation=1.0)
        autotune_batch(bm, vm)
        bm.set_graph(True)
        ms_b = timed(lambda i: bm.train_step(vm, lr_positions=LR_POS, lr_colors=LR_COL, clamp_colors=1), k_steps)
        del bm

        def plain_mesh(i, mi=mi, own=own):
            opts[mi].zero_grad(set_to_none=False)
            r = rends[mi]
            for v in own:
                r.set_view_matrix(v.view_matrix)
                img = r.render()
                _lib.call("dtv_loss_l2", img.data_ptr(), v.target.data_ptr(), n_img, 1.0 / n_img, adj.data_ptr(),
                          loss.data_ptr(), stream.cuda_stream)
                r.render_adjoint(adj)
            opts[mi].step()

        ms_p = timed(plain_mesh, k_steps)
        per_mesh[f"{n}^3"] = {"views": len(own), "batched_views_per_s": round(len(own) / (ms_b / 1e3), 1),
                              "plain_views_per_s": round(len(own) / (ms_p / 1e3), 1),
                              "speedup": round(ms_p / ms_b, 3), "steps": k_steps}
    nv = len(views)
    return {"res": res, "views": nv, "views_per_mesh": counts, "meshes": [f"{n}^3" for n in sizes],
            "batched_views_per_s": nv / (ms_batched / 1e3), "plain_views_per_s": nv / (ms_plain / 1e3),
            "batched_ms_per_step": ms_batched, "plain_ms_per_step": ms_plain,
            "speedup": ms_plain / ms_batched, "fragments_per_step": info["fragments"],
            "plain_device_busy_ms": {k2: round(v2, 3) for k2, v2 in busy.items()},
            "plain_stage_busy_ms": {k2: round(v2, 3) for k2, v2 in stage_busy.items()},
            "plain_overhead_ms": round(ms_plain - busy_total, 3),
            "speedup_bound_same_kernels": round(ms_plain / busy_total, 3) if busy_total > 0 else None,
            "per_mesh": per_mesh,
            "tuning_batch": tuned_batch,
            "graph": info["graph"], "steps": steps, "warmup": warmup}


def run_serving(args):
    """Serving config: Kuhn 16^3 / 32^3 / 64^3 meshes resident; Poisson arrivals
    at each rate; resolution 256^2 / 512^2 / 1024^2 with weights 0.5 / 0.3 / 0.2;
    70 % forward-only, 30 % forward + adjoint against a supplied target image.
    Continuous batching over --serving-slots slots, admission by fragment
    storage (shortest estimate first with a 20 ms age bound, or arrival order);
    the first --serving-priority-slots slots run on a high-priority stream and
    take the largest queued request alone.
    Reports p50 / p99 latency and throughput per rate beside the latency of the
    same kind of requests served alone (serial plain solves, --serving-isolated
    of them)."""
    import numpy as np
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    from difftetvr_b200.serve import GpuBackend, Request, ServingEngine

    names = {"16^3": 16, "32^3": 32, "64^3": 64}
    meshes = {}
    for i, (k, n) in enumerate(names.items()):
        cells, pos = S.kuhn_mesh(n, seed=20 + i)
        m = d.TetMesh()
        m.set_use_gradients(True)
        m.set_tet_mesh_data(cells, pos, S.gaussian_colors(pos, seed=20 + i))
        meshes[k] = m
    be = GpuBackend(meshes, slots=args.serving_slots, priority_slots=args.serving_priority_slots)
    be.calibrate(S.sphere_camera(0), res=256)
    res_choices, res_w = [256, 512, 1024], [0.5, 0.3, 0.2]
    targets = {r: torch.rand(r, r, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(r))
               for r in res_choices}

    def make_requests(rng, n):
        out = []
        for i in range(n):
            res = int(rng.choice(res_choices, p=res_w))
            mode = "gradient" if rng.random() < 0.3 else "forward"
            out.append(Request(mesh=str(rng.choice(list(names))), view_matrix=S.sphere_camera(int(rng.integers(1 << 30))),
                               width=res, height=res, mode=mode, target=targets[res] if mode == "gradient" else None))
        return out

    # Isolated latency: each request alone through the plain path.
    rends = {}
    for k, m in meshes.items():
        r = d.Renderer(d.RendererType.PPLL)
        r.set_tet_mesh(m)
        r.set_camera_fovy(S.FOVY_45)
        r.set_attenuation(1.0)
        rends[k] = r
    def solve_alone(q):
        r = rends[q.mesh]
        r.set_viewport_size(q.width, q.height)
        r.set_view_matrix(q.view_matrix)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = r.render()
        if q.mode == "gradient":
            r.render_adjoint(((img - q.target) * (2.0 / img.numel())).contiguous())
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3

    # Warm every (mesh, resolution, mode) once (first-use allocations), largest
    # resolution first, then time a seeded sample of the request mix.
    for k in names:
        for res in sorted(res_choices, reverse=True):
            for mode in ("gradient", "forward"):
                solve_alone(Request(mesh=k, view_matrix=S.sphere_camera(1), width=res, height=res, mode=mode,
                                    target=targets[res] if mode == "gradient" else None))
    iso = np.array([solve_alone(q) for q in make_requests(np.random.default_rng(7), args.serving_isolated)])
    out = {"meshes": list(names), "resolutions": res_choices, "resolution_weights": res_w, "gradient_fraction": 0.3,
           "slots": be.slots, "priority_slots": be.priority_slots, "policy": args.serving_policy,
           "batch_fragments": int(args.serving_batch_mfrags * 1e6),
           "isolated": {"requests": int(iso.size), "p50_ms": float(np.percentile(iso, 50)),
                        "p99_ms": float(np.percentile(iso, 99))}, "rates": []}
    budget = int(max(be.fragments_per_pixel(k) for k in names) * 1024 * 1024 * 4)
    be.reserve(32, max(res_choices) ** 2, int(1.5 * budget))
    # Warm-up pass (first batches of each slot), not reported.
    batch_frags = int(args.serving_batch_mfrags * 1e6)
    eng = ServingEngine(be, budget_fragments=budget, max_batch=32, policy=args.serving_policy,
                        batch_fragments=batch_frags)
    eng.start()
    for f in [eng.submit(q) for q in make_requests(np.random.default_rng(3), 24)]:
        f.result(timeout=600)
    eng.stop()
    for rate in [float(x) for x in args.serving_rates.split(",") if x]:
        rng = np.random.default_rng(int(rate))
        reqs = make_requests(rng, max(args.serving_requests, min(int(rate), 1000)))
        gaps = rng.exponential(1.0 / rate, size=len(reqs))
        eng = ServingEngine(be, budget_fragments=budget, max_batch=32, policy=args.serving_policy,
                            batch_fragments=batch_frags)
        eng.start()
        t = time.perf_counter()
        # The client takes each result as it completes (so result tensors are
        # released as a real client would, back to the slots' memory pools).
        futs = collections.deque()
        for q, g in zip(reqs, gaps):
            while futs and futs[0].done():
                futs.popleft().result()
            t += g
            dt = t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)  # sleeping (not spinning) keeps the GIL free for the engine thread
            futs.append(eng.submit(q))
        while futs:
            futs.popleft().result(timeout=600)
        eng.stop()
        st = eng.latency_stats()
        st["rate_rps"] = rate
        st["p99_over_isolated_p99"] = round(st["p99_ms"] / out["isolated"]["p99_ms"], 3)
        out["rates"].append(st)
    return out


class CpuPortLoop:
    """The workload's iteration on the host cores: the oracle's FP32 port
    (all threads) renders the whole image, the L2 loss adjoint is taken
    against a target image of the seed-1 mesh, the port's adjoint gives the
    vertex position / colour gradients and a host Adam (lr 1e-2 colours
    clamped at zero, 1e-4 positions) updates them.  Inputs come from
    oracle/scene.py, so no product code is loaded.  One camera
    (sphere_camera(100), the first of the GPU loop's cameras) for every step;
    its target image is rendered once, untimed."""

    def __init__(self, n: int, res: int):
        import numpy as np
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        import scene as OS

        self.np, self.O, self.res = np, O, res
        cells, pos = OS.kuhn_mesh(n, seed=0)
        self.pos = pos.copy()
        self.col = OS.gaussian_colors(pos, seed=0)
        _, pos_t = OS.kuhn_mesh(n, seed=1)
        col_t = OS.gaussian_colors(pos_t, seed=1)
        self.faces = O.Faces(cells, pos.shape[0])
        self.cam = O.make_camera(OS.sphere_camera(100), OS.FOVY_45, res, res)
        self.prm = O.make_params(attenuation=1.0, use_ert=True, ert_thresh=1e-4)
        self.target = O.render(self.faces, pos_t, col_t, self.cam, self.prm, precision=32)[0]
        self.opt_col = OS.Adam(self.col, LR_COL, clamp_nonnegative=True)
        self.opt_pos = OS.Adam(self.pos, LR_POS)
        self.times = []

    def step(self) -> float:
        np, O = self.np, self.O
        t = time.perf_counter()
        img = O.render(self.faces, self.pos, self.col, self.cam, self.prm, precision=32)[0]
        gimg = (2.0 / img.size) * (img - self.target)
        gp, gc = O.adjoint(self.faces, self.pos, self.col, self.cam, self.prm, gimg, precision=32)
        self.opt_col.step(gc.astype(np.float32))
        self.opt_pos.step(gp.astype(np.float32))
        dt = time.perf_counter() - t
        self.times.append(dt)
        return dt

    def describe(self, n: int) -> str:
        return (f"{len(self.times)} whole steps (forward + L2 adjoint + adjoint + Adam) of one view "
                f"(Kuhn {n}^3 at {self.res}x{self.res}, sphere_camera(100)) on the oracle's FP32 port, "
                f"{self.O.num_threads()} threads, mean {sum(self.times) / len(self.times):.2f} s per step")


def run_reference(args, rank, world):
    """The CPU implementation of the path (the oracle's FP32 port: the
    reference's own Vulkan path is unavailable on this box and its build
    needs the un-vendored sgl framework) timed on the host cores: W untimed
    and K timed whole steps of the workload."""
    loop = CpuPortLoop(args.n, args.res)
    for _ in range(args.warmup):
        loop.step()
    loop.times.clear()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        loop.step()
    total = time.perf_counter() - t0
    value = args.steps / total
    cores = loop.O.num_threads()
    return {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"plain method, Kuhn {args.n}^3 ({6 * args.n ** 3} tets), {args.res}x{args.res}, "
                               "one camera per step, fwd+adj+Adam (CPU port)", "res": args.res},
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": cores, "kind": "port",
                         "sample": loop.describe(args.n)},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's Vulkan renderer (and lavapipe) is unavailable on this box; the timed CPU "
                "implementation is this repository's FP32 restatement of its algorithm (oracle/), fed by "
                "oracle/scene.py so that no product code is loaded",
    }


def run_profile_case(args):
    """A small fixed case for ncu: one warm-up and one render + adjoint of the
    Kuhn n^3 mesh (seed 0) from sphere camera 100 at res x res (per-cell
    colours for `cells`)."""
    import torch

    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    cells, pos = S.kuhn_mesh(args.n, seed=0)
    col = S.gaussian_colors(pos, seed=0)
    mesh = d.TetMesh()
    mesh.set_use_gradients(True)
    if args.profile == "cells":
        mesh.set_tet_mesh_data_cell(cells, pos, col[cells].mean(axis=1).astype(col.dtype))
    else:
        mesh.set_tet_mesh_data(cells, pos, col)
    rt = d.RendererType.INTERSECTION if args.profile == "intersection" else d.RendererType.PPLL
    r = d.Renderer(rt)
    r.set_tet_mesh(mesh)
    r.set_viewport_size(args.res, args.res)
    r.set_camera_fovy(S.FOVY_45)
    r.set_attenuation(1.0)
    r.set_clear_color(d.vec4(0, 0, 0, 0))
    r.set_view_matrix(S.sphere_camera(100))
    w = torch.randn(args.res, args.res, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
    w *= 1e-3
    for _ in range(2):
        r.render()
        r.render_adjoint(w)
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile, "n": args.n, "res": args.res, "fragments": r.get_num_fragments()}))
    return 0


def main():
    args = parse_args()
    if args.profile:
        return run_profile_case(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args, rank, world)))
        return 0
    import torch
    if world > 1:
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    from difftetvr_b200 import build as B
    if not B.up_to_date() and rank == 0:
        B.build()
    if world > 1:
        torch.distributed.barrier()
    result, sc = run_ours(args, rank, world)
    if not args.no_raytet:
        result["raytet"] = run_raytet(args)
    if not args.no_next:
        result["cells"], result["regularizer"] = run_cells_and_regularizer(args)
    if not args.no_scale:
        result["scale"] = run_scale(args)
    if not args.no_batched:
        import torch
        del sc["renderer"], sc["mesh"], sc["targets"]
        torch.cuda.empty_cache()
        result["batched"] = [run_batched(args, int(r), args.batched_steps) for r in args.batched_res.split(",") if r]
    if not args.no_serving:
        import torch
        torch.cuda.empty_cache()
        result["served"] = run_serving(args)
    if rank == 0 and not args.no_cpu_baseline:
        loop = CpuPortLoop(args.n, args.res)
        for _ in range(args.cpu_steps):
            loop.step()
        v = len(loop.times) / sum(loop.times)
        result["cpu_baseline"] = {"value": v, "unit": "iter/s", "cores": loop.O.num_threads(), "kind": "port",
                                  "sample": loop.describe(args.n), "seconds": sum(loop.times)}
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

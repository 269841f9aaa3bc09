"""Serving: a request loop over meshes kept resident on the device.

Requests (forward renders, or forward + adjoint against a supplied target
image) of mixed resolution arrive at any time.  The engine batches them with
continuous batching: it keeps a small number of execution slots (each a CUDA
stream with its own batch renderer and fragment storage); whenever a slot is
free it admits queued requests (in arrival order, or smallest estimate first
with an age bound) while their estimated fragment storage fits the slot's
budget, launches the batch asynchronously,
and goes back to admitting - so requests that arrive while other batches run
on the GPU start as soon as a slot and memory are free, and the batches of
different slots overlap on the device.  Results are delivered through
futures; each request records its arrival, start and finish times.

The fragment-storage estimate per request is (pixels) x (fragments per pixel
of its mesh), where the per-mesh figure is learned from the exact counts of
completed batches (seeded from one probe render per mesh).
"""
from __future__ import annotations

import itertools
import math
import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    mesh: str
    view_matrix: list
    width: int
    height: int
    mode: str = "forward"            # "forward" or "gradient"
    target: object = None            # gradient: target image [H, W, 4] (torch CUDA tensor)
    fovy: float = math.radians(45.0)
    id: int = -1
    t_arrival: float = 0.0
    t_start: float = 0.0
    t_finish: float = 0.0
    batch_id: int = -1
    batch_size: int = 0
    info: dict = field(default_factory=dict)   # backend's per-batch figures (enqueue / device time, rerun)
    future: Future = field(default_factory=Future, repr=False)

    @property
    def pixels(self) -> int:
        return self.width * self.height


@dataclass
class Result:
    request_id: int
    image: object                    # [H, W, 4]
    grad_positions: object = None    # gradient mode: [V, 3]
    grad_colors: object = None       # gradient mode: [V, 4]
    loss: float | None = None


class ServingEngine:
    """Continuous-batching request loop.

    backend: object with
      - slots (int): number of execution slots
      - priority_slots (int, optional): slots 0 .. priority_slots-1 run on
        high-priority streams; a free one takes the largest queued request
        alone (the requests that set the latency tail), so its kernels are
        scheduled ahead of the other slots' batches
      - launch(slot, requests) -> handle (asynchronous)
      - done(handle) -> bool
      - finish(handle) -> list[Result] (in request order)
      - fragments_per_pixel(mesh) -> float
      - observe(mesh, pixels, fragments) (optional; refines the estimate)
    """

    def __init__(self, backend, budget_fragments: int, max_batch: int = 32, poll_s: float = 5e-5,
                 policy: str = "fifo", age_ms: float = 20.0, batch_fragments: int | None = None):
        """policy "fifo": admit in arrival order.  "sjf": requests queued for
        at least age_ms first (in arrival order), then the rest by estimated
        fragments, smallest first, so small requests do not wait behind large
        ones and no request waits longer than about age_ms plus one batch.
        budget_fragments bounds a batch's fragment storage (a request over it
        is rejected); batch_fragments (default: the budget) is the size a
        batch is filled to: a batch's device time is about proportional to its
        fragments and every request in it waits for all of them, so a smaller
        batch keeps the latency of its requests near their own (a request
        larger than batch_fragments runs alone)."""
        if policy not in ("fifo", "sjf"):
            raise ValueError("policy must be 'fifo' or 'sjf'")
        self.backend = backend
        self.budget = int(budget_fragments)
        self.batch_fragments = self.budget if batch_fragments is None else min(int(batch_fragments), self.budget)
        self.max_batch = int(max_batch)
        self.poll_s = poll_s
        self.policy = policy
        self.age_s = age_ms / 1e3
        self.queue: deque[Request] = deque()
        self.lock = threading.Lock()
        self.cv = threading.Condition(self.lock)
        self.ids = itertools.count()
        self.busy: dict[int, tuple[object, list[Request]]] = {}
        self.completed: list[Request] = []
        self.rejected = 0
        self.batches = 0
        self.running = False
        self.thread: threading.Thread | None = None

    # -- client side -------------------------------------------------------
    def submit(self, req: Request) -> Future:
        req.id = next(self.ids)
        req.t_arrival = time.perf_counter()
        if self.estimate(req) > self.budget:
            self.rejected += 1
            req.future.set_exception(RuntimeError(
                f"request {req.id} needs about {self.estimate(req):.0f} fragments, over the slot budget "
                f"of {self.budget}"))
            return req.future
        with self.cv:
            self.queue.append(req)
            self.cv.notify()
        return req.future

    def cancel_pending(self) -> int:
        """Cancel every request still waiting in the queue."""
        with self.cv:
            n = 0
            while self.queue:
                r = self.queue.popleft()
                r.future.cancel()
                n += 1
        return n

    def estimate(self, req: Request) -> float:
        return req.pixels * self.backend.fragments_per_pixel(req.mesh)

    # -- engine ------------------------------------------------------------
    def admit(self) -> list[Request]:
        """Requests for the next batch within the budget, in the policy's order."""
        batch, frags = [], 0.0
        if self.policy == "fifo":
            while self.queue and len(batch) < self.max_batch:
                e = self.estimate(self.queue[0])
                if batch and frags + e > self.batch_fragments:
                    break
                batch.append(self.queue.popleft())
                frags += e
            return batch
        now = time.perf_counter()
        aged = [r for r in self.queue if now - r.t_arrival >= self.age_s]
        fresh = sorted((r for r in self.queue if now - r.t_arrival < self.age_s), key=self.estimate)
        taken = set()
        for r in aged + fresh:
            if len(batch) >= self.max_batch:
                break
            e = self.estimate(r)
            if batch and frags + e > self.batch_fragments:
                if r in aged:
                    break  # an aged request waits for the next batch, not behind younger ones
                continue
            batch.append(r)
            taken.add(id(r))
            frags += e
        if taken:
            self.queue = deque(r for r in self.queue if id(r) not in taken)
        return batch

    def admit_largest(self) -> list[Request]:
        """The largest queued request alone (for a high-priority slot)."""
        if not self.queue:
            return []
        r = max(self.queue, key=self.estimate)
        self.queue.remove(r)
        return [r]

    def step(self) -> bool:
        """One scheduling pass: finish completed batches, launch on free slots.
        Returns True if anything happened."""
        progressed = False
        for slot, (handle, reqs) in list(self.busy.items()):
            if self.backend.done(handle):
                results = self.backend.finish(handle)
                t = time.perf_counter()
                for r, res in zip(reqs, results):
                    r.t_finish = t
                    if not r.future.cancelled():
                        r.future.set_result(res)
                    self.completed.append(r)
                del self.busy[slot]
                progressed = True
        prio = int(getattr(self.backend, "priority_slots", 0))
        for slot in range(self.backend.slots):
            if slot in self.busy:
                continue
            with self.lock:
                batch = self.admit_largest() if slot < prio else self.admit()
            if not batch:
                break
            t = time.perf_counter()
            for r in batch:
                r.t_start = t
                r.batch_id = self.batches
                r.batch_size = len(batch)
            self.busy[slot] = (self.backend.launch(slot, batch), batch)
            self.batches += 1
            progressed = True
        return progressed

    def _loop(self):
        while self.running or self.busy or self.queue:
            if not self.step():
                with self.cv:
                    if not self.queue and self.running:
                        self.cv.wait(timeout=self.poll_s if self.busy else 0.01)
                if self.busy:
                    time.sleep(self.poll_s)

    def start(self):
        self.running = True
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()

    def stop(self, timeout: float = 60.0):
        self.running = False
        with self.cv:
            self.cv.notify_all()
        if self.thread:
            self.thread.join(timeout=timeout)

    # -- statistics ------------------------------------------------------------
    def latency_stats(self, slowest: int = 3) -> dict:
        """Latency percentiles (arrival to result), split into queueing
        (arrival to batch launch) and service (launch to result), plus the
        `slowest` requests with their batch."""
        done = self.completed
        if not done:
            return {"requests": 0}
        lat = np.array([(r.t_finish - r.t_arrival) * 1e3 for r in done])
        wait = np.array([(r.t_start - r.t_arrival) * 1e3 for r in done])
        svc = lat - wait
        span = max(r.t_finish for r in done) - min(r.t_arrival for r in done)
        worst = np.argsort(lat)[::-1][:slowest]
        return {"requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "queue_p50_ms": float(np.percentile(wait, 50)), "queue_p99_ms": float(np.percentile(wait, 99)),
                "service_p50_ms": float(np.percentile(svc, 50)), "service_p99_ms": float(np.percentile(svc, 99)),
                "throughput_rps": float(lat.size / span) if span > 0 else float("nan"),
                "batches": self.batches, "rejected": self.rejected,
                "slowest": [{"ms": round(float(lat[i]), 3), "queue_ms": round(float(wait[i]), 3),
                             "batch": done[i].batch_id, "batch_size": done[i].batch_size,
                             "mesh": done[i].mesh, "pixels": done[i].pixels, "mode": done[i].mode,
                             **done[i].info}
                            for i in worst]}


class GpuBackend:
    """Executes request batches with the batched CUDA path; one CUDA stream and
    one batch renderer (own fragment storage) per slot, meshes shared."""

    def __init__(self, meshes: dict, slots: int = 2, attenuation: float = 1.0, priority_slots: int = 0):
        """priority_slots: the first slots run on the device's highest stream
        priority (the engine gives each the largest queued request alone)."""
        import torch

        from .batch import BatchRenderer
        self.torch = torch
        self.names = list(meshes)
        self.meshes = [meshes[n] for n in self.names]
        self.index = {n: i for i, n in enumerate(self.names)}
        self.slots = int(slots)
        self.priority_slots = min(int(priority_slots), self.slots)
        high = torch.cuda.Stream.priority_range()[1] if hasattr(torch.cuda.Stream, "priority_range") else -1
        self.streams = [torch.cuda.Stream(priority=high if i < self.priority_slots else 0)
                        for i in range(self.slots)]
        self.renderers = [BatchRenderer(self.meshes, attenuation=attenuation, use_early_ray_termination=True)
                          for _ in range(self.slots)]
        self.fpp = {n: 64.0 for n in self.names}

    def _rerun(self, handle):
        torch = self.torch
        br, stream = self.renderers[handle["slot"]], self.streams[handle["slot"]]
        with torch.cuda.stream(stream):
            br.render(handle["views"])
            # Same slot order as launch(): views name their slot in grad_slot.
            slots = [(handle["views"][i].mesh, gp, gc) for i, gp, gc in handle["grads"]]
            for _, gp, gc in slots:
                gp.zero_()
                gc.zero_()
            for i, (r, v) in enumerate(zip(handle["reqs"], handle["views"])):
                if r.mode == "gradient":
                    n = float(v.width * v.height * 4)
                    v.image_adjoint = (v.image - r.target) * (2.0 / n)
            if slots:
                br.render_adjoint(slots)
        stream.synchronize()
        return handle

    def reserve(self, max_batch: int, max_pixels_per_request: int, budget_fragments: int,
                result_batches: int = 4) -> None:
        """Sizes every slot's scratch for the largest admissible batch, so no
        device allocation (an implicit synchronisation of the whole device,
        which would wait for the other slots' batches) happens while serving.
        The library's scratch is reserved directly; the per-request tensors
        (images, image adjoints, gradients) come from PyTorch's caching
        allocator, whose pool of each slot stream is grown here to hold
        `result_batches` full batches of them at once."""
        torch = self.torch
        maxV = max(m.get_num_vertices() for m in self.meshes)
        for br in self.renderers:
            br.reserve(max_batch, max_batch * maxV, max_batch * max_pixels_per_request, budget_fragments,
                       max_batch * maxV)
        per_batch = max_batch * (2 * 16 * max_pixels_per_request + 28 * maxV)
        dev = self.meshes[0].get_vertex_positions().device
        for st in self.streams:
            with torch.cuda.stream(st):
                block = torch.empty(result_batches * per_batch, dtype=torch.uint8, device=dev)
                # Tensors under 1 MiB (small meshes' gradients, losses) come
                # from the allocator's separate pool of 2 MiB segments.
                small = [torch.empty(1 << 19, dtype=torch.uint8, device=dev)
                         for _ in range(4 * result_batches * max_batch)]
                del block, small
        torch.cuda.synchronize()
        self._reserved = True

    def fragments_per_pixel(self, mesh: str) -> float:
        return self.fpp[mesh]

    def observe(self, mesh: str, pixels: int, fragments: int) -> None:
        self.fpp[mesh] = 0.7 * self.fpp[mesh] + 0.3 * max(fragments / max(pixels, 1), 1.0)

    def calibrate(self, view_matrix, res: int = 256) -> None:
        """One probe render per mesh to seed the fragments-per-pixel estimate."""
        from .batch import View
        for n in self.names:
            br = self.renderers[0]
            br.render([View(mesh=self.index[n], view_matrix=view_matrix, width=res, height=res)])
            self.fpp[n] = max(br.info()["fragments"] / float(res * res), 1.0)

    def launch(self, slot: int, reqs: list[Request]):
        torch = self.torch
        from .batch import View
        br = self.renderers[slot]
        stream = self.streams[slot]
        views = [View(mesh=self.index[r.mesh], view_matrix=r.view_matrix, width=r.width, height=r.height,
                      fovy=r.fovy) for r in reqs]
        grads = []
        reserved = getattr(self, "_reserved", False)
        t0, c0 = time.perf_counter(), time.thread_time()
        with torch.cuda.stream(stream):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            # With reserved scratch the batch is enqueued without a host
            # synchronisation; finish() checks that it fit.
            (br.render_async if reserved else br.render)(views)
            t1 = time.perf_counter()
            slots = []
            for i, (r, v) in enumerate(zip(reqs, views)):
                if r.mode == "gradient":
                    n = float(v.width * v.height * 4)
                    v.image_adjoint = (v.image - r.target) * (2.0 / n)
                    v.grad_slot = len(slots)
                    m = self.meshes[v.mesh]
                    gp = torch.zeros_like(m.get_vertex_positions(), memory_format=torch.contiguous_format)
                    gc = torch.zeros_like(m.get_vertex_colors(), memory_format=torch.contiguous_format)
                    slots.append((v.mesh, gp.detach(), gc.detach()))
                    grads.append((i, gp, gc))
            t2 = time.perf_counter()
            if slots:
                br.render_adjoint([(m, gp, gc) for (m, gp, gc) in slots])
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
        t3 = time.perf_counter()
        px = sum(r.pixels for r in reqs)
        # Host time of the enqueue: forward, adjoint inputs, adjoint; and the
        # engine thread's CPU time over it (wall >> CPU: the thread was blocked).
        parts = [round((b - a) * 1e3, 3) for a, b in ((t0, t1), (t1, t2), (t2, t3))]
        return {"event": ev, "start_event": ev0, "enqueue_ms": (t3 - t0) * 1e3, "enqueue_parts_ms": parts,
                "enqueue_cpu_ms": round((time.thread_time() - c0) * 1e3, 3), "views": views,
                "reqs": reqs, "grads": grads, "pixels": px, "slot": slot, "async": reserved}

    def done(self, handle) -> bool:
        return handle["event"].query()

    def finish(self, handle) -> list[Result]:
        tf = time.perf_counter()
        handle["event"].synchronize()
        reqs, views = handle["reqs"], handle["views"]
        br = self.renderers[handle["slot"]]
        info = {"enqueue_ms": round(handle["enqueue_ms"], 3), "enqueue_parts_ms": handle["enqueue_parts_ms"],
                "enqueue_cpu_ms": handle["enqueue_cpu_ms"],
                "device_ms": round(handle["start_event"].elapsed_time(handle["event"]), 3), "rerun": False}
        if handle["async"]:
            fits, nf = br.render_status()
            if not fits:
                # Over the reserved capacity: run the batch again with exact sizing.
                t0 = time.perf_counter()
                handle = self._rerun(handle)
                nf = br.info()["fragments"]
                info.update(rerun=True, rerun_ms=round((time.perf_counter() - t0) * 1e3, 3))
            handle["fragments"] = nf
        else:
            handle["fragments"] = br.info()["fragments"]
        info["fragments"] = int(handle["fragments"])
        for r in reqs:
            r.info = info
        # Per-mesh fragments-per-pixel estimate from the exact batch count.
        by_mesh = {}
        for r in reqs:
            by_mesh[r.mesh] = by_mesh.get(r.mesh, 0) + r.pixels
        if len(by_mesh) == 1:
            (m, px), = by_mesh.items()
            self.observe(m, px, handle["fragments"])
        g = {i: (gp, gc) for i, gp, gc in handle["grads"]}
        # Losses of the gradient requests on the slot's stream, read back at once.
        grad_idx = [i for i, r in enumerate(reqs) if r.mode == "gradient"]
        losses = {}
        if grad_idx:
            torch = self.torch
            with torch.cuda.stream(self.streams[handle["slot"]]):
                vals = torch.stack([((views[i].image - reqs[i].target) ** 2).mean() for i in grad_idx])
                losses = dict(zip(grad_idx, vals.tolist()))
        out = []
        for i, (r, v) in enumerate(zip(reqs, views)):
            gp, gc = g.get(i, (None, None))
            out.append(Result(r.id, v.image, gp, gc, losses.get(i)))
        info["finish_ms"] = round((time.perf_counter() - tf) * 1e3, 3)
        return out

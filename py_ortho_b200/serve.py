"""Continuous-batching depth-map server.

Requests (one reference view each: grey images, cameras, inverse-depth planes, window radius,
optional PatchMatch iterations) arrive over time. The server admits them FIFO while a slot and
the HBM budget allow, uploads their images once, and keeps every admitted job's images, winner
state and PatchMatch state resident on the device until it completes. Each scheduler step:

  1. admits arrived requests (H2D copies, window statistics, state initialisation);
  2. runs the next plane chunk of resident sweep jobs - oldest first, as many as a per-step work
     budget allows, all their tiles - in one persistent launch (mvs_server_step), merging each
     chunk into its job's state in hypothesis order;
  3. finalises jobs whose last chunk ran, and advances PatchMatch-phase jobs by one iteration;
     PatchMatch runs on a pool of its own streams (one per job, ordered after the job's finalize
     by an event), so it overlaps the next sweep steps and other jobs' PatchMatch;
  4. returns finished jobs' depth (and normal / score) to the host and frees their slot (a
     PatchMatch job's copies are queued on its stream and collected once its event completes,
     without blocking the step).

Precision "fp16" stores the sources in FP16 for the sweep (one converted copy per source tensor,
shared by the jobs that use it; FP32 window sums), as MVS_PREC_FP16; PatchMatch reads the float32
sources.

A job's arithmetic does not depend on which other jobs share its steps (fixed chunk boundaries,
ordered merge, same tile engine as the single-view path), so its result equals the plain
per-request path's bit for bit. `serve_plain` is that comparator: one request at a time with
mvs_sweep (+ PatchMatch), no batching.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import fast
from .dense import Hypotheses, new_state, stream_start, sweep_args


@dataclass
class DepthRequest:
    ref: np.ndarray                  # (H, W) float32 grey (host)
    srcs: list                       # (h, w) float32 grey (host) or device tensors (shared sources)
    ref_cam: object                  # R, C, f, k1..k3, cx, cy (pinhole)
    src_cams: list
    planes_inv: np.ndarray           # (n,) float32 inverse depths
    r: int = 2
    top_k: int = 2
    pm_iters: int = 0
    pm_radius: int = 3
    pm_step: int = 1
    depth_range: tuple = (1e-3, 1e9)
    seed: int = 0
    pm_precision: str = "fp32"       # PatchMatch cost arithmetic (mvs_pm_precision)
    arrival: float = 0.0             # seconds from the start of the trace
    rid: int = 0

    @property
    def evals(self) -> int:
        H, W = self.ref.shape
        n = len(self.srcs)
        return H * W * len(self.planes_inv) * n + H * W * self.pm_iters * 11 * n


@dataclass
class Result:
    rid: int
    depth: np.ndarray
    score: np.ndarray | None
    normal: np.ndarray | None
    arrival: float
    admitted: float
    finished: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def _geo(ref_cam, src_cams):
    rows = []
    for cs in src_cams:
        Rs = np.asarray(cs.R, np.float64)
        b = Rs @ (np.asarray(ref_cam.C, np.float64) - np.asarray(cs.C, np.float64))
        rows.append(np.r_[Rs.ravel(), b, [cs.f, cs.k1, cs.k2, cs.k3, cs.cx, cs.cy]])
    return np.array(rows, np.float64)


def footprint(req: DepthRequest, shared_sources: bool = False) -> int:
    """Device bytes a job holds while resident."""
    H, W = req.ref.shape
    px = H * W
    b = px * 4 * (1 + 2 + 5 + 6 + 1)                 # ref, mu/sd, state, chunk record, depth
    if not shared_sources:
        b += sum(int(np.prod(s.shape)) * 4 for s in req.srcs)
    if req.pm_iters:
        b += px * 4 * (3 + 3 + 1) + px            # ray, normal, score, active
        # mvs_pm_refine's scratch while a step runs it: per-pixel pass state and cost cache, and
        # the float32 mode's 2 x 2 footprints of every source
        b += px * (21 + 16) + sum(int(np.prod(s.shape)) * 16 for s in req.srcs)
    return b


def admissions(footprints, free_slots: int, used: float, budget: float):
    """FIFO admission policy over queued jobs with byte footprints `footprints` (in order).
    Returns (n, reject): the first n jobs start now; reject is True when job n can never fit the
    budget (it is rejected; the jobs behind it then get their turn). A job that does not fit yet
    waits and blocks the ones behind it."""
    n = 0
    for need in footprints:
        if need > budget:
            return n, True
        if n >= free_slots or used + need > budget:
            break
        used += need
        n += 1
    return n, False


class _Job:
    def __init__(self, req: DepthRequest, slot: int, dev, stream, plane_chunk: int, precision: int = L.PREC_FP32,
                 half=None):
        self.req, self.slot = req, slot
        H, W = req.ref.shape
        self.H, self.W = H, W
        with torch.cuda.stream(stream):
            self.ref = torch.from_numpy(np.ascontiguousarray(req.ref, np.float32)).to(dev, non_blocking=True)
            self.srcs = [s if isinstance(s, torch.Tensor) else
                         torch.from_numpy(np.ascontiguousarray(s, np.float32)).to(dev, non_blocking=True)
                         for s in req.srcs]
            self.mu = torch.empty_like(self.ref)
            self.sd = torch.empty_like(self.ref)
            L.check(L.load().mvs_ref_stats(H, W, self.ref.data_ptr(), int(req.r), self.mu.data_ptr(), self.sd.data_ptr(),
                                           stream.cuda_stream), "ref_stats")
            self.state = new_state(H, W, dev)
            self.rec = torch.empty((6, H, W), dtype=torch.float32, device=dev)
            self.depth = torch.empty((H, W), dtype=torch.float32, device=dev)
            # the sweep's sources: FP16 copies (shared per source tensor) in the FP16 form
            self.sweep_srcs = [half(s) for s in self.srcs] if precision == L.PREC_FP16 else self.srcs
        self.hyp = Hypotheses.planes_inv(req.planes_inv)
        self.args, self.keep = sweep_args(self.ref, self.mu, self.sd, None, self.sweep_srcs,
                                          _geo(req.ref_cam, req.src_cams), fast.cam_row(req.ref_cam), self.hyp, req.r,
                                          req.top_k, self.state, precision=precision)
        self.nchunks = -(-len(req.planes_inv) // plane_chunk)
        self.next_chunk = 0
        self.pm_done = 0
        self.phase = "sweep"
        self.admitted = 0.0


class DepthServer:
    """Continuous batching over resident jobs (see the module docstring)."""

    def __init__(self, hbm_budget: float = 120e9, max_slots: int = 64, plane_chunk: int = 32,
                 max_items: int = 1 << 20, max_radius: int = 3, shared_sources: bool = False,
                 step_evals: float = 2.5e10, precision: str = "fp32", pm_streams: int = 4):
        if precision not in ("fp32", "fp16"):
            raise ValueError("server: precision must be 'fp32' or 'fp16'")
        self.dev = L.require_cuda()
        self.stream = torch.cuda.Stream(self.dev)
        self.pm_streams = [torch.cuda.Stream(self.dev) for _ in range(max(1, pm_streams))]
        self._pm_next = 0
        self.precision = L.PREC_FP16 if precision == "fp16" else L.PREC_FP32
        self._half: dict = {}          # source tensor address -> (source, FP16 copy, jobs using it)
        self.budget = float(hbm_budget)
        self.max_slots = max_slots
        self.plane_chunk = plane_chunk
        self.shared_sources = shared_sources
        # work budget of one step (ZNCC evaluations): the oldest resident jobs advance first, and
        # younger ones join the same launch while the budget lasts (enough work to fill the GPU
        # without time-slicing every resident job)
        self.step_evals = float(step_evals)
        h = ctypes.c_void_p()
        L.check(L.load().mvs_server_create(max_slots, max_items, max_radius, self.precision, ctypes.byref(h)),
                "server_create")
        self._h = h
        self.free_slots = list(range(max_slots))[::-1]
        self.queue: list = []
        self.active: dict = {}
        self.used = 0.0
        self.results: list = []
        self.steps = 0
        self.launch_count = 0

    def close(self):
        if getattr(self, "_h", None):
            torch.cuda.synchronize(self.dev)
            L.load().mvs_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- admission
    def submit(self, req: DepthRequest):
        if req.r > 3:
            raise ValueError("server: window radius above 3")
        self.queue.append(req)

    def _half_of(self, src: torch.Tensor) -> torch.Tensor:
        """The FP16 copy of a source tensor (converted on the server's stream once, shared)."""
        key = src.data_ptr()
        ent = self._half.get(key)
        if ent is None:
            ent = [src, fast.to_fp16(src, stream=self.stream), 0]
            self._half[key] = ent
        ent[2] += 1
        return ent[1]

    def _release_half(self, job):
        if self.precision != L.PREC_FP16:
            return
        for s in job.srcs:
            ent = self._half.get(s.data_ptr())
            if ent is not None:
                ent[2] -= 1
                if ent[2] == 0:
                    del self._half[s.data_ptr()]

    def _admit(self, now: float):
        needs = [footprint(q, self.shared_sources) for q in self.queue]
        n, reject = admissions(needs, len(self.free_slots), self.used, self.budget)
        for _ in range(n):
            req = self.queue.pop(0)
            need = footprint(req, self.shared_sources)
            slot = self.free_slots.pop()
            job = _Job(req, slot, self.dev, self.stream, self.plane_chunk, self.precision, self._half_of)
            L.check(L.load().mvs_server_set_job(self._h, slot, ctypes.addressof(job.args),
                                                job.rec.data_ptr(), self.plane_chunk), "server_set_job")
            job.admitted = now
            job.bytes = need
            self.used += need
            self.active[slot] = job
        if reject:
            req = self.queue.pop(0)
            raise MemoryError(f"request {req.rid} needs {footprint(req, self.shared_sources) / 1e9:.2f} GB, "
                              f"above the HBM budget of {self.budget / 1e9:.2f} GB")

    # ---------------------------------------------------------------- one scheduler step
    def step(self, now: float) -> int:
        """Admit, run one chunk of every sweeping job in one launch, advance PatchMatch jobs,
        complete finished jobs. Returns the number of jobs completed."""
        self._admit(now)
        if not self.active:
            return 0
        lib = L.load()
        sh = self.stream.cuda_stream
        sweeping = []
        work = 0.0
        for j in sorted((j for j in self.active.values() if j.phase == "sweep"), key=lambda j: (j.req.arrival, j.req.rid)):
            if sweeping and work >= self.step_evals:
                break
            sweeping.append(j)
            work += j.H * j.W * len(j.req.srcs) * min(self.plane_chunk, len(j.req.planes_inv) - j.next_chunk * self.plane_chunk)
        if sweeping:
            slots = (ctypes.c_int32 * len(sweeping))(*[j.slot for j in sweeping])
            chunks = (ctypes.c_int32 * len(sweeping))(*[j.next_chunk for j in sweeping])
            L.check(lib.mvs_server_step(self._h, slots, chunks, len(sweeping), sh), "server_step")
            self.launch_count += 2
            for j in sweeping:
                j.next_chunk += 1
                if j.next_chunk == j.nchunks:
                    h = j.hyp.c()
                    L.check(lib.mvs_sweep_finalize(j.H, j.W, ctypes.addressof(h), j.state[0].data_ptr(),
                                                   j.state[2].data_ptr(), j.state[3].data_ptr(), j.state[4].data_ptr(),
                                                   j.depth.data_ptr(), sh), "finalize")
                    self.launch_count += 1
                    j.phase = "pm" if j.req.pm_iters > 0 else "done"
                    if j.phase == "pm":
                        self._start_pm(j)
        for j in [j for j in self.active.values() if j.phase == "pm" and j.pm_started]:
            j.pm.it0 = j.pm_done
            L.check(lib.mvs_pm_refine(ctypes.addressof(j.pm), j.pm_stream.cuda_stream), "pm_refine")
            self.launch_count += 1 + 10
            j.pm_done += 1
            if j.pm_done == j.req.pm_iters:
                # results queued on the job's stream; collected once its event has completed
                with torch.cuda.stream(j.pm_stream):
                    j.h_depth = torch.empty((j.H, j.W), dtype=torch.float32).pin_memory()
                    j.h_depth.copy_(j.pm_depth, non_blocking=True)
                    j.h_score = j.pm_score.to("cpu", non_blocking=True)
                    j.h_normal = j.pm_normal.to("cpu", non_blocking=True)
                    j.pm_done_event = torch.cuda.Event()
                    j.pm_done_event.record(j.pm_stream)
                j.phase = "pm_copy"
        for j in self.active.values():
            if j.phase == "pm" and not j.pm_started:
                j.pm_started = True          # PatchMatch starts on the step after the sweep ends
        done = [j for j in self.active.values() if j.phase == "done"]
        for j in done:
            j.h_depth = torch.empty((j.H, j.W), dtype=torch.float32).pin_memory()
            with torch.cuda.stream(self.stream):
                j.h_depth.copy_(j.depth, non_blocking=True)
        self.stream.synchronize()
        done += [j for j in self.active.values() if j.phase == "pm_copy" and j.pm_done_event.query()]
        t = time.perf_counter()
        for j in done:
            self.results.append(Result(j.req.rid, j.h_depth.numpy(), getattr(j, "h_score", None),
                                       getattr(j, "h_normal", None), j.req.arrival, j.admitted, t))
            self._release_half(j)
            del self.active[j.slot]
            self.free_slots.append(j.slot)
            self.used -= j.bytes
        if not done and self.active and all(j.phase == "pm_copy" for j in self.active.values()):
            time.sleep(2e-4)                 # only PatchMatch copies in flight: do not spin hot
        self.steps += 1
        return len(done)

    def _start_pm(self, j: _Job):
        req = j.req
        H, W = j.H, j.W
        j.pm_stream = self.pm_streams[self._pm_next % len(self.pm_streams)]
        self._pm_next += 1
        ready = torch.cuda.Event()
        ready.record(self.stream)              # after the job's finalize
        j.pm_stream.wait_event(ready)
        with torch.cuda.stream(j.pm_stream):
            j.pm_ray = fast.rays_world((H, W), req.ref_cam)
            j.pm_depth = j.depth.clone()
            rng = np.random.default_rng(req.seed)
            from .scene import tilted_normals
            j.pm_normal = torch.from_numpy(tilted_normals(H, W, int(rng.integers(1 << 30)))).to(self.dev, non_blocking=True)
            j.pm_score = torch.zeros((H, W), dtype=torch.float32, device=self.dev)
            j.pm_active = torch.ones((H, W), dtype=torch.uint8, device=self.dev)
            # the job's random stream stays on the device between its one-iteration steps
            j.pm_rng = stream_start(req.seed, self.dev)
        j.pm, j.pm_keep = pm_args(j.ref, j.pm_ray, req.ref_cam, j.srcs, req.src_cams, j.pm_depth, j.pm_normal,
                                  j.pm_score, j.pm_active, req, iters=1)
        j.pm.rng_state = j.pm_rng.data_ptr()
        j.pm_started = False


def pm_args(ref, ray, ref_cam, srcs, src_cams, depth, normal, score, active, req: DepthRequest, iters: int):
    """mvs_pm_args for device tensors (PatchMatch without neighbour depth maps)."""
    par = np.array([fast.cam_row(c) for c in src_cams], np.float64)
    Cr = np.ascontiguousarray(np.asarray(ref_cam.C, np.float64))
    a = L.PMArgs()
    H, W = int(ref.shape[0]), int(ref.shape[1])
    a.H, a.W, a.S = H, W, len(srcs)
    a.ref, a.ray, a.Cr = ref.data_ptr(), ray.data_ptr(), L.host_ptr(Cr)
    for k, s in enumerate(srcs):
        a.src[k] = s.data_ptr()
        a.src_depth[k] = 0
        a.src_h[k], a.src_w[k] = int(s.shape[0]), int(s.shape[1])
    a.par = L.host_ptr(par)
    a.depth, a.normal, a.score, a.active = depth.data_ptr(), normal.data_ptr(), score.data_ptr(), active.data_ptr()
    a.r, a.step, a.top_k, a.iters = req.pm_radius, req.pm_step, req.top_k, iters
    a.geo_w, a.geo_tol, a.dmin, a.dmax = 0.0, 0.02, float(req.depth_range[0]), float(req.depth_range[1])
    a.seed, a.it0, a.changed = req.seed, 0, 0
    a.precision = 1 if req.pm_precision == "fp32" else 0
    return a, (par, Cr)


def serve(requests, server: DepthServer, realtime: bool = True):
    """Runs an arrival trace through the server. Returns (results sorted by id, wall seconds)."""
    pending = sorted(requests, key=lambda q: q.arrival)
    t0 = time.perf_counter()
    k = 0
    while k < len(pending) or server.queue or server.active:
        now = time.perf_counter() - t0
        while k < len(pending) and (pending[k].arrival <= now or not realtime):
            pending[k].arrival = pending[k].arrival if realtime else now
            server.submit(pending[k])
            k += 1
        if not server.queue and not server.active:
            if k < len(pending):
                time.sleep(max(0.0, pending[k].arrival - (time.perf_counter() - t0)))
            continue
        server.step(time.perf_counter() - t0)
    for r in server.results:
        r.finished -= t0
        r.admitted = r.admitted
    return sorted(server.results, key=lambda r: r.rid), time.perf_counter() - t0


def serve_plain(requests, realtime: bool = True, precision: str = "fp32"):
    """The plain per-request comparator: FIFO, one request at a time, mvs_sweep + finalize
    (+ PatchMatch), results copied back. Same arrival trace semantics as serve(). precision
    "fp16": the sweep reads FP16 copies of the sources, as the FP16 server does."""
    from .dense import sweep, finalize
    dev = L.require_cuda()
    pending = sorted(requests, key=lambda q: q.arrival)
    t0 = time.perf_counter()
    out = []
    for req in pending:
        now = time.perf_counter() - t0
        if realtime and req.arrival > now:
            time.sleep(req.arrival - now)
        start = time.perf_counter() - t0
        ref = torch.from_numpy(np.ascontiguousarray(req.ref, np.float32)).to(dev)
        srcs = [s if isinstance(s, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(s, np.float32)).to(dev)
                for s in req.srcs]
        mu, sd = fast.ref_stats(ref, req.r)
        hyp = Hypotheses.planes_inv(req.planes_inv)
        half = precision == "fp16"
        st = sweep(ref, mu, sd, None, [fast.to_fp16(s) for s in srcs] if half else srcs,
                   _geo(req.ref_cam, req.src_cams), hyp, req.r, req.top_k, ref_cam=fast.cam_row(req.ref_cam),
                   precision=L.PREC_FP16 if half else L.PREC_FP32)
        depth = finalize(hyp, st)
        score = normal = None
        if req.pm_iters:
            H, W = ref.shape
            ray = fast.rays_world((H, W), req.ref_cam)
            rng = np.random.default_rng(req.seed)
            from .scene import tilted_normals
            nrm = torch.from_numpy(tilted_normals(H, W, int(rng.integers(1 << 30)))).to(dev)
            scr = torch.zeros((H, W), dtype=torch.float32, device=dev)
            act = torch.ones((H, W), dtype=torch.uint8, device=dev)
            a, keep = pm_args(ref, ray, req.ref_cam, srcs, req.src_cams, depth, nrm, scr, act, req, iters=req.pm_iters)
            L.check(L.load().mvs_pm_refine(ctypes.addressof(a), L.stream_handle()), "pm_refine")
            score, normal = scr.cpu().numpy(), nrm.cpu().numpy()
        d = depth.cpu().numpy()
        out.append(Result(req.rid, d, score, normal, req.arrival, start, time.perf_counter() - t0))
    return sorted(out, key=lambda r: r.rid), time.perf_counter() - t0


def latency_stats(results) -> dict:
    lat = np.array([r.latency for r in results]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "n": int(len(lat))}

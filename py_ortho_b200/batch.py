"""Batched depth maps: many reference views of uneven size, source count, plane count and window
radius in one persistent launch (mvs_batch_*), replayed as a CUDA graph, with a small
autotuner for the plane-chunk size, CTAs per SM and tile height.

A job is one view swept over constant inverse-depth planes (pinhole cameras). Its result does
not depend on the other jobs of the batch (per-pixel reduction order is fixed by plane index).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import fast
from .dense import Hypotheses, new_state, sweep_args


@dataclass
class ViewJob:
    """One depth-map job: device images (float32, or float16 for the FP16 precision), cameras
    (objects with R, C, f, k1..k3, cx, cy), inverse-depth planes, window radius and top_k."""
    ref: torch.Tensor
    srcs: list
    ref_cam: object
    src_cams: list
    planes_inv: np.ndarray
    r: int = 2
    top_k: int = 2
    # filled by prepare()
    mu: torch.Tensor = None
    sd: torch.Tensor = None
    state: tuple = None
    depth: torch.Tensor = None
    keep: list = field(default_factory=list)

    @property
    def evals(self) -> int:
        return int(self.ref.shape[0] * self.ref.shape[1] * len(self.planes_inv) * len(self.srcs))

    def prepare(self, stream=None):
        """Window statistics of the reference and output buffers (device, no host sync)."""
        H, W = int(self.ref.shape[0]), int(self.ref.shape[1])
        self.mu = torch.empty_like(self.ref)
        self.sd = torch.empty_like(self.ref)
        L.check(L.load().mvs_ref_stats(H, W, self.ref.data_ptr(), int(self.r), self.mu.data_ptr(), self.sd.data_ptr(),
                                       L.stream_handle(stream)), "ref_stats")
        self.state = new_state(H, W, self.ref.device)
        self.depth = torch.empty((H, W), dtype=torch.float32, device=self.ref.device)
        return self


def _geo(ref_cam, src_cams):
    rows = []
    for cs in src_cams:
        Rs = np.asarray(cs.R, np.float64)
        b = Rs @ (np.asarray(ref_cam.C, np.float64) - np.asarray(cs.C, np.float64))
        rows.append(np.r_[Rs.ravel(), b, [cs.f, cs.k1, cs.k2, cs.k3, cs.cx, cs.cy]])
    return np.array(rows, np.float64)


class Batch:
    """A persistent batched plan (mvs_batch_create); run() replays it (CUDA graph by default)."""

    def __init__(self, jobs, plane_chunk: int = 0, ctas_per_sm: int = 0, precision: int = L.PREC_FP32,
                 tile_h: int = 0):
        self.jobs = jobs
        self.precision = precision
        self.tile_h = int(tile_h) or 32
        arr = (L.BatchJob * len(jobs))()
        self._keep = []
        for j, job in enumerate(jobs):
            if job.mu is None:
                job.prepare()
            hyp = Hypotheses.planes_inv(job.planes_inv)
            a, keep = sweep_args(job.ref, job.mu, job.sd, None, job.srcs, _geo(job.ref_cam, job.src_cams),
                                 fast.cam_row(job.ref_cam), hyp, job.r, job.top_k, job.state, precision=precision)
            arr[j].sweep = a
            arr[j].depth = job.depth.data_ptr()
            self._keep.append(keep)
        tun = L.BatchTuning(int(plane_chunk), int(ctas_per_sm), int(tile_h))
        h = ctypes.c_void_p()
        L.check(L.load().mvs_batch_create(ctypes.addressof(arr), len(jobs), ctypes.addressof(tun), ctypes.byref(h)),
                "batch_create")
        self._h = h
        items, evals = ctypes.c_int64(), ctypes.c_int64()
        L.check(L.load().mvs_batch_stats(h, ctypes.byref(items), ctypes.byref(evals)), "batch_stats")
        self.work_items, self.evals = int(items.value), int(evals.value)

    def run(self, graph: bool = True, stream=None):
        L.check(L.load().mvs_batch_run(self._h, 1 if graph else 0, L.stream_handle(stream)), "batch_run")

    def close(self):
        if getattr(self, "_h", None):
            L.load().mvs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def time_plan(b: Batch, reps: int = 3, stream=None) -> float:
    """Milliseconds per run (CUDA events on the launching stream, after one warm-up)."""
    s = stream or torch.cuda.current_stream()
    b.run(stream=s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        b.run(stream=s)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


_TUNE_CACHE: dict = {}


def autotune(jobs, precision: int = L.PREC_FP32, chunks=(0, 16, 32, 64), ctas=(0, 1), tile_hs=(32,), reps: int = 2):
    """Picks (plane_chunk, ctas_per_sm, tile_h) by timing each candidate plan on the actual jobs
    (tile_h: rows of the 64-column output tiles, 16 / 32 / 64; 16 and 64 need top_k <= 2);
    results are cached per job-shape signature. Returns (best_batch, table of
    (chunk, ctas, tile_h, ms))."""
    key = (precision, tuple(tile_hs), tuple((int(j.ref.shape[0]), int(j.ref.shape[1]), len(j.srcs),
                                             len(j.planes_inv), j.r, j.top_k) for j in jobs))
    table = []
    if key in _TUNE_CACHE:
        pc, cps, th = _TUNE_CACHE[key]
        return Batch(jobs, pc, cps, precision, th), table
    best = None
    for th in tile_hs:
        for pc in chunks:
            for cps in ctas:
                b = Batch(jobs, pc, cps, precision, th)
                ms = time_plan(b, reps)
                table.append((pc, cps, th, ms))
                if best is None or ms < best[0]:
                    if best is not None:
                        best[1].close()
                    best = (ms, b, pc, cps, th)
                else:
                    b.close()
    _TUNE_CACHE[key] = (best[2], best[3], best[4])
    return best[1], table

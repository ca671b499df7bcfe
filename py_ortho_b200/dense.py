"""Drop-in replacements for the reference's depth-map kernels (``orthomosaic._dense``):
``sweep_hypothesis`` and ``pm_refine``, plus the multi-hypothesis ``sweep`` that replaces the
per-hypothesis loop of ``densify._sweep``.

Arrays may be NumPy (copied to the device once, results copied back in place, as the reference
updates its memoryviews in place) or torch CUDA tensors (used in place, no copies). Argument
order, meaning and error behaviour are the reference's (``_dense.pyx:566-569``,
``_dense.pyx:740-743``). Everything runs in libmvs_b200 (sm_100a); there is no CPU path.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from . import _lib as L


# ------------------------------------------------------------------ device staging
class _Dev:
    """Moves NumPy / torch inputs to the current CUDA device and writes results back."""

    def __init__(self):
        self.device = L.require_cuda()
        self.back = []              # (numpy array, device tensor) pairs written back at close()

    def t(self, a, dtype: torch.dtype, name: str, out: bool = False) -> torch.Tensor:
        if a is None:
            raise ValueError(f"{name} is required")
        if isinstance(a, torch.Tensor):
            if a.dtype != dtype:
                raise ValueError(f"{name}: expected {dtype}, got {a.dtype}")
            if not a.is_contiguous():
                raise ValueError(f"{name} must be C-contiguous")
            if a.device.type != "cuda":
                if out:
                    raise ValueError(f"{name}: output tensors must live on the CUDA device")
                return a.to(self.device)
            return a
        arr = np.asarray(a)
        npd = torch.empty((), dtype=dtype).numpy().dtype
        if arr.dtype != npd:
            if out:
                raise ValueError(f"{name}: expected {npd}, got {arr.dtype}")
            arr = arr.astype(npd)
        if out and not arr.flags.c_contiguous:
            raise ValueError(f"{name} must be C-contiguous")
        t = torch.from_numpy(np.ascontiguousarray(arr)).to(self.device, non_blocking=False)
        if out:
            self.back.append((a, t))
        return t

    def close(self):
        if self.back:
            torch.cuda.current_stream().synchronize()
            for a, t in self.back:
                np.copyto(a, t.cpu().numpy())
        self.back = []


def _shape2(t: torch.Tensor) -> tuple:
    return tuple(t.shape)


# ------------------------------------------------------------------ sweep_hypothesis
def sweep_hypothesis(ref, mu_i, sd_i, srcs: Sequence, ray, geo, inv, r: int, top_k: int, i: int, best, prev,
                     s_prev_best, s_next_best, idx) -> None:
    """One hypothesis of the plane sweep for all sources (reference: _dense.pyx:740-838).

    ray: (3, H, W) world rays; geo: (n, 18) Rs(9) b(3) f k1 k2 k3 cx cy; inv: (H, W) inverse depth;
    best / prev / s_prev_best / s_next_best: (H, W) float32 and idx: (H, W) int32, updated in place."""
    n = len(srcs)
    if n < 1 or n > L.MAX_SOURCES:
        raise ValueError("sweep_hypothesis needs 1..16 sources")
    g = L.host_f64(geo)
    if g.ndim != 2 or g.shape[0] != n or g.shape[1] != 18:
        raise ValueError("geo must be (n_sources, 18)")
    D = _Dev()
    try:
        ref_t = D.t(ref, torch.float32, "ref")
        H, W = _shape2(ref_t)
        ts = {nm: D.t(a, torch.float32, nm) for nm, a in (("mu_i", mu_i), ("sd_i", sd_i), ("inv", inv))}
        ray_t = D.t(ray, torch.float32, "ray")
        st = {nm: D.t(a, torch.float32, nm, out=True) for nm, a in (("best", best), ("prev", prev),
                                                                    ("s_prev_best", s_prev_best),
                                                                    ("s_next_best", s_next_best))}
        idx_t = D.t(idx, torch.int32, "idx", out=True)
        if (any(_shape2(t) != (H, W) for t in list(ts.values()) + list(st.values()) + [idx_t])
                or tuple(ray_t.shape) != (3, H, W)):
            raise ValueError("sweep_hypothesis: array shapes do not match the reference image")
        if r < 0:
            raise ValueError("sweep_hypothesis: negative window radius")
        if H == 0 or W == 0:
            return
        src_t = [D.t(s, torch.float32, f"srcs[{k}]") for k, s in enumerate(srcs)]
        ptrs = (L.vp * n)(*[t.data_ptr() for t in src_t])
        hs = (L.i32 * n)(*[t.shape[0] for t in src_t])
        ws = (L.i32 * n)(*[t.shape[1] for t in src_t])
        lib = L.load()
        L.check(lib.mvs_sweep_hypothesis(H, W, ref_t.data_ptr(), ts["mu_i"].data_ptr(), ts["sd_i"].data_ptr(), n,
                                         ptrs, hs, ws, ray_t.data_ptr(), L.host_ptr(g), ts["inv"].data_ptr(),
                                         int(r), int(top_k), int(i), st["best"].data_ptr(), st["prev"].data_ptr(),
                                         st["s_prev_best"].data_ptr(), st["s_next_best"].data_ptr(),
                                         idx_t.data_ptr(), L.stream_handle()), "sweep_hypothesis")
        D.close()
    finally:
        D.back = []


# ------------------------------------------------------------------ multi-hypothesis sweep
class Hypotheses:
    """Device-side hypothesis families of a sweep (see mvs_hyp in include/mvs_b200.h).

    Construct with one of the classmethods; ``n`` is the number of hypotheses."""

    def __init__(self, kind: int, n: int, maps=None, base=None, step=None, t0: int = 0, planes=None):
        self.kind, self.n, self.maps, self.base, self.step, self.t0 = kind, int(n), maps, base, step, int(t0)
        self.planes = None if planes is None else np.ascontiguousarray(planes, np.float32)

    @classmethod
    def planes_inv(cls, inv_depths) -> "Hypotheses":
        """Fronto-parallel planes at constant inverse depths (pinhole cameras): homography path."""
        p = np.ascontiguousarray(inv_depths, np.float32)
        return cls(L.HYP_PLANES, len(p), planes=p)

    @classmethod
    def linear(cls, base: torch.Tensor, step: torch.Tensor, n: int) -> "Hypotheses":
        """inv_i = base + (float)i * step (the reference's coarse band, _fast.hyp_linear)."""
        return cls(L.HYP_LINEAR, n, base=base, step=step)

    @classmethod
    def refine(cls, iu: torch.Tensor, ds: torch.Tensor, steps: int) -> "Hypotheses":
        """inv_q = max(iu + (q - steps) ds, 1e-6), q = 0..2 steps (densify.py:423-429)."""
        return cls(L.HYP_REFINE, 2 * steps + 1, base=iu, step=ds, t0=-steps)

    @classmethod
    def maps_(cls, maps: torch.Tensor) -> "Hypotheses":
        """Explicit (n, H, W) float32 maps on the device."""
        return cls(L.HYP_MAPS, maps.shape[0], maps=maps)

    def c(self) -> L.Hyp:
        h = L.Hyp()
        h.kind, h.n, h.t0 = self.kind, self.n, self.t0
        if self.maps is not None:
            h.maps = self.maps.data_ptr()
            h.map_stride = self.maps.shape[1] * self.maps.shape[2]
        if self.base is not None:
            h.base = self.base.data_ptr()
            h.step = self.step.data_ptr()
        if self.planes is not None:
            h.planes = self.planes.ctypes.data
        return h


def sweep_args(ref, mu, sd, ray, srcs, geo, ref_cam, hyp: Hypotheses, r, top_k, state, i0=0, i1=None,
               precision=L.PREC_FP32, plane_chunks=0, tile_h=0):
    """Fills an mvs_sweep_args for device tensors (no copies). Returns (args, keepalive)."""
    a = L.SweepArgs()
    a.H, a.W = int(ref.shape[0]), int(ref.shape[1])
    a.ref, a.mu, a.sd = ref.data_ptr(), mu.data_ptr(), sd.data_ptr()
    a.ray = 0 if ray is None else ray.data_ptr()
    n = len(srcs)
    if n < 1 or n > L.MAX_SOURCES:
        raise ValueError("sweep_hypothesis needs 1..16 sources")
    a.n_src = n
    a.precision = precision
    for k, s in enumerate(srcs):
        a.src[k] = s.data_ptr()
        a.src_h[k], a.src_w[k] = int(s.shape[0]), int(s.shape[1])
    g = L.host_f64(geo)
    if g.shape != (n, 18):
        raise ValueError("geo must be (n_sources, 18)")
    a.geo = L.host_ptr(g)
    rc = None
    if ref_cam is not None:
        rc = L.host_f64(ref_cam).reshape(-1)
        a.ref_cam = L.host_ptr(rc)
    a.hyp = hyp.c()
    a.i0 = int(i0)
    a.i1 = int(hyp.n if i1 is None else i1)
    a.r, a.top_k, a.plane_chunks, a.tile_h = int(r), int(top_k), int(plane_chunks), int(tile_h)
    best, prev, spb, snb, idx = state
    a.best, a.prev, a.s_prev_best, a.s_next_best, a.idx = (best.data_ptr(), prev.data_ptr(), spb.data_ptr(),
                                                          snb.data_ptr(), idx.data_ptr())
    return a, (g, rc, hyp)


def new_state(H: int, W: int, device=None):
    """Initial winner-take-all state (densify.py:331-335): best/prev/spb/snb = -2, idx = -1."""
    device = device or L.require_cuda()
    f = [torch.full((H, W), -2.0, dtype=torch.float32, device=device) for _ in range(4)]
    return (*f, torch.full((H, W), -1, dtype=torch.int32, device=device))


def sweep(ref, mu, sd, ray, srcs, geo, hyp: Hypotheses, r: int, top_k: int, state=None, ref_cam=None,
          precision=L.PREC_FP32, plane_chunks: int = 0, stream=None, tile_h: int = 0):
    """All hypotheses of ``hyp`` in one call on device tensors; returns the state tuple
    (best, prev, s_prev_best, s_next_best, idx), updated in place when given. tile_h: rows of the
    kernel's 64-column output tiles (0 = 32; 16 and 64 for FP32 / FP16 plane sweeps with
    top_k <= 2); it changes the float32 rounding of the plane maps, not the arithmetic."""
    H, W = int(ref.shape[0]), int(ref.shape[1])
    if state is None:
        state = new_state(H, W, ref.device)
    a, keep = sweep_args(ref, mu, sd, ray, srcs, geo, ref_cam, hyp, r, top_k, state, precision=precision,
                         plane_chunks=plane_chunks, tile_h=tile_h)
    L.check(L.load().mvs_sweep(C_addr(a), L.stream_handle(stream)), "sweep")
    del keep
    return state


def finalize(hyp: Hypotheses, state, out=None, stream=None) -> torch.Tensor:
    """Parabola + depth (densify.py:354-361) on the device."""
    best, _, spb, snb, idx = state
    H, W = best.shape
    out = torch.empty((H, W), dtype=torch.float32, device=best.device) if out is None else out
    h = hyp.c()
    L.check(L.load().mvs_sweep_finalize(H, W, C_addr(h), best.data_ptr(), spb.data_ptr(), snb.data_ptr(),
                                        idx.data_ptr(), out.data_ptr(), L.stream_handle(stream)), "finalize")
    return out


def C_addr(struct) -> int:
    import ctypes
    return ctypes.addressof(struct)


# ------------------------------------------------------------------ pm_refine
PM_PRECISIONS = {"fp64": 0, "fp32": 1}     # mvs_pm_precision

def pm_refine(ref, ray, Cr, srcs: Sequence, src_depths: Sequence, par, depth, normal, score, active, r: int,
              step: int, top_k: int, geo_w: float, geo_tol: float, iters: int, dmin: float, dmax: float,
              seed: int, it0: int = 0, precision: str = "fp64", rng_state=None) -> int:
    """Slanted-plane PatchMatch repair (reference: _dense.pyx:566-666); depth / normal / score are
    updated in place; returns the number of accepted hypothesis changes. The random trials draw
    from the reference's own xorshift32 stream (started at seed | 1), in its raster order.

    precision: "fp64" evaluates the reference's float64 cost operation for operation (bit-identical
    to the reference's pm_refine); "fp32" evaluates the windows in float32 from one
    float64-composed homography per candidate and source (costs within ~1e-6 of float64; near-ties
    may be decided differently).

    rng_state: None, or a 1-element int32 CUDA tensor holding the stream state (initialise it
    with stream_start(seed)); the call starts there and leaves the state after its draws, so a
    job split over calls (it0 = iterations done) matches one call."""
    if precision not in PM_PRECISIONS:
        raise ValueError(f"pm_refine: precision must be one of {sorted(PM_PRECISIONS)}")
    S = len(srcs)
    if S == 0 or S > L.MAX_SOURCES:
        return 0
    D = _Dev()
    try:
        ref_t = D.t(ref, torch.float32, "ref")
        H, W = _shape2(ref_t)
        ray_t = D.t(ray, torch.float32, "ray")
        d_t = D.t(depth, torch.float32, "depth", out=True)
        n_t = D.t(normal, torch.float32, "normal", out=True)
        s_t = D.t(score, torch.float32, "score", out=True)
        a_t = D.t(active, torch.uint8, "active")
        src_t = [D.t(s, torch.float32, f"srcs[{k}]") for k, s in enumerate(srcs)]
        dep_t = [None if d is None else D.t(d, torch.float32, f"src_depths[{k}]") for k, d in enumerate(src_depths)]
        if len(dep_t) != S:
            raise ValueError("pm_refine: src_depths must match srcs")
        par_h = L.host_f64(par)
        if par_h.shape != (S, 18):
            raise ValueError("pm_refine: par must be (n_sources, 18)")
        cr_h = L.host_f64(Cr).reshape(-1)
        if tuple(ray_t.shape) != (3, H, W) or tuple(n_t.shape) != (3, H, W) or any(
                _shape2(t) != (H, W) for t in (d_t, s_t, a_t)):
            raise ValueError("pm_refine: array shapes do not match the reference image")
        for k, (s, d) in enumerate(zip(src_t, dep_t)):
            if d is not None and tuple(d.shape) != tuple(s.shape):
                raise ValueError(f"pm_refine: src_depths[{k}] shape differs from its image")
        changed = torch.zeros(1, dtype=torch.int64, device=ref_t.device)
        a = L.PMArgs()
        a.H, a.W, a.S = H, W, S
        a.precision = PM_PRECISIONS[precision]
        a.ref, a.ray, a.Cr = ref_t.data_ptr(), ray_t.data_ptr(), L.host_ptr(cr_h)
        for k in range(S):
            a.src[k] = src_t[k].data_ptr()
            a.src_depth[k] = 0 if dep_t[k] is None else dep_t[k].data_ptr()
            a.src_h[k], a.src_w[k] = int(src_t[k].shape[0]), int(src_t[k].shape[1])
        a.par = L.host_ptr(par_h)
        a.depth, a.normal, a.score, a.active = d_t.data_ptr(), n_t.data_ptr(), s_t.data_ptr(), a_t.data_ptr()
        a.r, a.step, a.top_k, a.iters = int(r), int(step), int(top_k), int(iters)
        a.geo_w, a.geo_tol, a.dmin, a.dmax = float(geo_w), float(geo_tol), float(dmin), float(dmax)
        a.seed = int(seed) & 0xFFFFFFFF
        a.it0 = int(it0)
        a.changed = changed.data_ptr()
        if rng_state is not None:
            if not (isinstance(rng_state, torch.Tensor) and rng_state.is_cuda and rng_state.numel() == 1
                    and rng_state.dtype == torch.int32 and rng_state.device == ref_t.device):
                raise ValueError("pm_refine: rng_state must be a 1-element int32 tensor on the image's device")
            a.rng_state = rng_state.data_ptr()
        L.check(L.load().mvs_pm_refine(C_addr(a), L.stream_handle()), "pm_refine")
        out = int(changed.item())
        D.close()
        return out
    finally:
        D.back = []


def stream_start(seed: int, device=None) -> torch.Tensor:
    """A PatchMatch stream state for pm_refine(rng_state=...): seed | 1, as the reference starts."""
    v = (int(seed) | 1) & 0xFFFFFFFF
    return torch.tensor([v - (1 << 32) if v >= 1 << 31 else v], dtype=torch.int32,
                        device=device if device is not None else L.require_cuda())


def stream_advance(state: int, n: int) -> int:
    """The xorshift32 state after n steps of the PatchMatch stream (GF(2) jump-ahead, host)."""
    return int(L.load().mvs_pm_stream_advance(int(state) & 0xFFFFFFFF, int(n)))

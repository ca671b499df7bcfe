"""CPU oracle for the depth-map path - TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py (cpu_baseline and --impl reference
legs), always as the checker or the timed CPU baseline, never as part of the product path.

Two layers:
  * ``libmvs_oracle.so`` (oracle/mvs_oracle.c): plain-C restatement of the reference kernels with
    the reference's rounding points (see that file's header for the file:line each follows);
  * the NumPy parts of ``densify._sweep`` restated here (window statistics, the hypothesis loop,
    the parabola finalize), each citing the reference line it follows.
Optionally the reference itself: ``oracle/_ref`` holds the reference's own ``_dense`` / ``_fast``
Cython kernels compiled from its sources by ``make -C oracle ref`` (see oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmvs_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None
_ref = None

fp = C.POINTER(C.c_float)
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


def build() -> str:
    """Compiles libmvs_oracle.so (gcc) if missing or stale."""
    src = os.path.join(HERE, "mvs_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.oracle_sweep_hypothesis.restype = C.c_int
        L.oracle_sweep_hypothesis.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp,
                                              C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
        L.oracle_sweep_fp64.restype = C.c_int
        L.oracle_sweep_fp64.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int,
                                        C.c_int, C.c_int, vp, vp, vp]
        L.oracle_box_zero_mean.restype = C.c_int
        L.oracle_box_zero_mean.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp]
        L.oracle_pm_refine.restype = C.c_int64
        L.oracle_pm_refine.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp,
                                       vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                       C.c_double, C.c_double, C.c_uint32, vp, C.c_int]
        L.oracle_consistency.restype = None
        L.oracle_consistency.argtypes = [C.c_int, C.c_int, vp, vp, C.c_int, vp, vp, vp, vp, vp, C.c_double, vp, vp, vp,
                                         C.c_double, C.c_int, vp]
        L.oracle_sample_view.restype = None
        L.oracle_sample_view.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp] + [C.c_double] * 9 + \
            [C.c_int, C.c_int, vp, vp, vp]
        L.oracle_box_sat_mean.restype = C.c_int
        L.oracle_box_sat_mean.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp]
        L.oracle_sgm.restype = C.c_int
        L.oracle_sgm.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_float, C.c_float, vp]
        L.oracle_fuse_view.restype = None
        L.oracle_fuse_view.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, C.c_double,
                                       C.c_int, C.c_int, vp, vp, vp]
        L.oracle_init_normals.restype = None
        L.oracle_init_normals.argtypes = [C.c_int, C.c_int, vp, vp, vp]
        _lib = L
    return _lib


def reference():
    """The reference's own compiled kernels (module namespace with ``_dense`` and ``_fast``), or
    None when oracle/_ref has not been built from the reference sources."""
    global _ref
    if _ref is None:
        try:
            if REF_DIR not in sys.path:
                sys.path.insert(0, REF_DIR)
            import _dense  # noqa: F401
            import _fast  # noqa: F401

            class _NS:
                pass

            ns = _NS()
            ns._dense, ns._fast = _dense, _fast
            _ref = ns
        except ImportError:
            _ref = False
    return _ref or None


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _f64(a):
    return np.ascontiguousarray(a, np.float64)


# ------------------------------------------------------------------ NumPy parts of densify._sweep
def box(a: np.ndarray, r: int) -> np.ndarray:
    """densify._box (densify.py:94-103): zero-padded float32 window mean (via the C restatement
    of _fast.box_zero_mean, _fast.pyx:661-713)."""
    a = _f32(a)
    out = np.empty_like(a)
    if a.size:
        lib().oracle_box_zero_mean(a.shape[0], a.shape[1], _p(a), int(r), _p(out))
    return out


def ref_stats(ref: np.ndarray, r: int):
    """densify.py:327-328: mu = box(ref), sd = sqrt(max(box(ref*ref) - mu*mu, 1e-6)), float32."""
    ref = _f32(ref)
    mu = box(ref, r)
    sd = np.sqrt(np.maximum(box(ref * ref, r) - mu * mu, 1e-6)).astype(np.float32)
    return mu, sd


def init_state(H: int, W: int):
    """densify.py:331-335: best = prev = spb = snb = -2, idx = -1."""
    st = [np.full((H, W), -2.0, np.float32) for _ in range(4)]
    return st[0], st[1], st[2], st[3], np.full((H, W), -1, np.int32)


def finalize(best, spb, snb, idx, inv0, inv1, n):
    """densify.py:354-361 verbatim in NumPy semantics: float32 parabola offset, float64 depth."""
    inv0 = _f32(inv0)
    dinv = (_f32(inv1) - inv0) if n > 1 else np.zeros_like(inv0)
    den = spb - 2 * best + snb
    interior = (idx > 0) & (idx < n - 1) & (den < -1e-6)
    off = np.where(interior, 0.5 * (spb - snb) / np.where(interior, den, -1.0), 0.0)
    inv = inv0 + (idx + np.clip(off, -0.5, 0.5)) * dinv
    return (1.0 / np.maximum(inv, 1e-9)).astype(np.float32)


def geo_rows(cam_r, cams_s) -> np.ndarray:
    """densify.py:329-338: (n, 18) rows Rs(9) b(3) f k1 k2 k3 cx cy, b = Rs (C_ref - C_src)."""
    rows = []
    for cs in cams_s:
        Rs = np.asarray(cs.R, np.float64)
        b = Rs @ (np.asarray(cam_r.C, np.float64) - np.asarray(cs.C, np.float64))
        rows.append(np.r_[Rs.ravel(), b, [cs.f, cs.k1, cs.k2, cs.k3, cs.cx, cs.cy]])
    return np.array(rows, np.float64)


def rays_world(shape, cam) -> np.ndarray:
    """densify._rays_world (densify.py:288-297) with _Cam.rays (densify.py:144-152), float64
    NumPy arithmetic then float32."""
    H, W = shape
    vv, uu = np.mgrid[0:H, 0:W].astype(np.float64)
    nx, ny = (uu - cam.cx) / cam.f, (vv - cam.cy) / cam.f
    x, y = nx.copy(), ny.copy()
    for _ in range(8):
        r2 = x * x + y * y
        d = 1 + r2 * (cam.k1 + r2 * (cam.k2 + r2 * cam.k3))
        x, y = nx / d, ny / d
    ray_c = np.stack([x, y, np.ones_like(x)])
    return np.ascontiguousarray(np.einsum("ji,jhw->ihw", np.asarray(cam.R, np.float64), ray_c), np.float32)


# ------------------------------------------------------------------ sweep
def sweep_hypothesis(ref, mu, sd, srcs, ray, geo, inv, r, top_k, i, best, prev, spb, snb, idx, scores=None):
    """One hypothesis, in place on the state (the definitional ncc_warp + combine)."""
    H, W = ref.shape
    n = len(srcs)
    srcs = [_f32(s) for s in srcs]
    ptrs = (C.c_void_p * n)(*[s.ctypes.data for s in srcs])
    hs = np.array([s.shape[0] for s in srcs], np.int32)
    ws = np.array([s.shape[1] for s in srcs], np.int32)
    geo = _f64(geo)
    inv = _f32(inv)
    rc = lib().oracle_sweep_hypothesis(H, W, _p(ref), _p(mu), _p(sd), n, ptrs, _p(hs), _p(ws), _p(ray), _p(geo),
                                       _p(inv), int(r), int(top_k), int(i), _p(best), _p(prev), _p(spb), _p(snb),
                                       _p(idx), None if scores is None else _p(scores))
    if rc != 0:
        raise MemoryError("oracle sweep")


def sweep(ref, srcs, ray, geo, hyps, r, top_k, keep_scores=False):
    """densify._sweep's loop (densify.py:323-342) + finalize (:354-361) with explicit
    per-hypothesis inverse-depth maps `hyps` (list of (H, W) float32). Returns
    dict(depth, best, sd, mu, idx, prev, spb, snb[, scores (n_hyp, H, W) top-k scores])."""
    ref = _f32(ref)
    H, W = ref.shape
    ray = _f32(ray)
    mu, sd = ref_stats(ref, r)
    best, prev, spb, snb, idx = init_state(H, W)
    n = len(hyps)
    volume = np.empty((n, H, W), np.float32) if keep_scores else None
    for i, inv in enumerate(hyps):
        sweep_hypothesis(ref, mu, sd, srcs, ray, geo, inv, r, top_k, i, best, prev, spb, snb, idx)
        if keep_scores:
            volume[i] = prev          # prev holds hypothesis i's score (_sweep.h:212)
    depth = finalize(best, spb, snb, idx, hyps[0], hyps[1] if n > 1 else hyps[0], n)
    out = dict(depth=depth, best=best, sd=sd, mu=mu, idx=idx, prev=prev, spb=spb, snb=snb)
    if keep_scores:
        out["scores"] = volume
    return out


def sweep_fp64(ref, srcs, ray, geo, hyps, r, top_k):
    """All-float64 sweep (precision reference): returns (depth f64, best f64, idx)."""
    ref = _f32(ref)
    H, W = ref.shape
    r64 = ref.astype(np.float64)
    k = 2 * r + 1
    pad = np.pad(r64, r)
    m1 = np.zeros((H, W))
    m2 = np.zeros((H, W))
    for dy in range(k):
        for dx in range(k):
            m1 += pad[dy:dy + H, dx:dx + W]
            m2 += pad[dy:dy + H, dx:dx + W] ** 2
    mu = m1 / (k * k)
    sd = np.sqrt(np.maximum(m2 / (k * k) - mu * mu, 1e-6))
    n = len(srcs)
    srcs = [_f32(s) for s in srcs]
    ptrs = (C.c_void_p * n)(*[s.ctypes.data for s in srcs])
    hs = np.array([s.shape[0] for s in srcs], np.int32)
    ws = np.array([s.shape[1] for s in srcs], np.int32)
    inv = _f64(np.stack([np.asarray(h, np.float64) for h in hyps]))
    ray64 = _f64(ray)
    geo = _f64(geo)
    depth = np.empty((H, W), np.float64)
    best = np.empty((H, W), np.float64)
    idx = np.empty((H, W), np.int32)
    rc = lib().oracle_sweep_fp64(H, W, _p(ref), _p(_f64(mu)), _p(_f64(sd)), n, ptrs, _p(hs), _p(ws), _p(ray64),
                                 _p(geo), _p(inv), len(hyps), int(r), int(top_k), _p(depth), _p(best), _p(idx))
    if rc != 0:
        raise MemoryError("oracle fp64 sweep")
    return depth, best, idx


# ------------------------------------------------------------------ PatchMatch
def pm_refine(ref, ray, Cr, srcs, src_depths, par, depth, normal, score, active, r, step, top_k, geo_w, geo_tol,
              iters, dmin, dmax, seed, it0=0, state=None) -> int:
    """_dense.pm_refine (_dense.pyx:566-666) restated, in place, with the reference's xorshift32
    stream. state: None (start at seed | 1, as the reference) or a 1-element uint32 array carried
    from call to call (in: the stream state to start at; out: the state after the draws)."""
    H, W = ref.shape
    S = len(srcs)
    srcs = [_f32(s) for s in srcs]
    deps = [None if d is None else _f32(d) for d in src_depths]
    sp = (C.c_void_p * max(S, 1))(*[s.ctypes.data for s in srcs])
    dpp = (C.c_void_p * max(S, 1))(*[(None if d is None else d.ctypes.data) for d in deps])
    hs = np.array([s.shape[0] for s in srcs] or [0], np.int32)
    ws = np.array([s.shape[1] for s in srcs] or [0], np.int32)
    par = _f64(par)
    Cr = _f64(Cr)
    for a, t in ((depth, np.float32), (normal, np.float32), (score, np.float32)):
        assert a.dtype == t and a.flags.c_contiguous
    if state is not None:
        assert state.dtype == np.uint32 and state.size == 1 and state.flags.c_contiguous
    act = np.ascontiguousarray(active, np.uint8)
    return int(lib().oracle_pm_refine(H, W, _p(_f32(ref)), _p(_f32(ray)), _p(Cr), S, sp, dpp, _p(hs), _p(ws),
                                      _p(par), _p(depth), _p(normal), _p(score), _p(act), int(r), int(step),
                                      int(top_k), float(geo_w), float(geo_tol), int(iters), float(dmin), float(dmax),
                                      int(seed) & 0xFFFFFFFF, None if state is None else _p(state), int(it0)))


def xorshift_steps(state: int, n: int) -> int:
    """n sequential steps of the reference's xorshift32 (_dense.pyx:559-563): the checker of the
    device stream's jump-ahead."""
    s = int(state) & 0xFFFFFFFF
    for _ in range(int(n)):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
    return s


# ------------------------------------------------------------------ pass-2 geometry
def cam_row(cam) -> np.ndarray:
    """R (9), C (3), f, k1, k2, k3, cx, cy of a densify._Cam-like camera, float64."""
    return np.r_[np.asarray(cam.R, np.float64).ravel(), np.asarray(cam.C, np.float64), cam.f, cam.k1, cam.k2,
                 cam.k3, cam.cx, cam.cy].astype(np.float64)


def consistency(D, cam_r, nb_maps, nb_cams, px_tol, rel_tol, grey=None, score=None, min_ncc=0.0, min_views=0):
    """densify._consistency (densify.py:441-478) restated: int16 agreement count per pixel; with
    grey and score also pass 2's active mask (densify.py:621). Returns (count, active or None)."""
    D = _f32(D)
    H, W = D.shape
    n = len(nb_maps)
    maps = [_f32(m) for m in nb_maps]
    mp = (C.c_void_p * max(n, 1))(*[m.ctypes.data for m in maps])
    hs = np.array([m.shape[0] for m in maps] or [0], np.int32)
    ws = np.array([m.shape[1] for m in maps] or [0], np.int32)
    rows = _f64(np.array([cam_row(c) for c in nb_cams], np.float64).reshape(-1))
    tol = _f64(np.asarray(rel_tol, np.float64).reshape(-1))
    cnt = np.zeros((H, W), np.int16)
    act = None
    g = s = None
    if grey is not None:
        act = np.zeros((H, W), np.uint8)
        g, s = _f32(grey), _f32(score)
    lib().oracle_consistency(H, W, _p(D), _p(_f64(cam_row(cam_r))), n, mp, _p(hs), _p(ws), _p(rows), _p(tol),
                             float(px_tol), _p(cnt), None if g is None else _p(g), None if s is None else _p(s),
                             float(min_ncc), int(min_views), None if act is None else _p(act))
    return cnt, act


def init_normals(D, ray) -> np.ndarray:
    """densify._init_normals (densify.py:481-496) restated in float32."""
    D = _f32(D)
    H, W = D.shape
    out = np.empty((3, H, W), np.float32)
    lib().oracle_init_normals(H, W, _p(D), _p(_f32(ray)), _p(out))
    return out


def fuse(order, maps, cams, nbrs, rel_tols, px_tol, min_views, point_stride, rgbs):
    """densify._fuse (densify.py:676-762) restated: views in `order`, each fused against its
    neighbours (nbrs[k], rel_tols[k][j]) with the used masks of the views carried from one view to
    the next. maps[k]: float32 depth (NaN = none); rgbs[k]: (H, W, 3) uint8. Returns
    (xyz float64 (n, 3), cols uint8 (n, 3), nv uint8 (n,), owner int32 (n,), used {k: bool})."""
    used = {k: np.zeros(maps[k].shape, np.uint8) for k in maps}
    pts, cols, nv, owner = [], [], [], []
    for k in order:
        D = _f32(maps[k])
        H, W = D.shape
        nb = [j for j in nbrs[k] if j in maps]
        n = len(nb)
        nmaps = [_f32(maps[j]) for j in nb]
        mp = (C.c_void_p * max(n, 1))(*[m.ctypes.data for m in nmaps])
        up = (C.c_void_p * max(n, 1))(*[used[j].ctypes.data for j in nb])
        hs = np.array([m.shape[0] for m in nmaps] or [0], np.int32)
        ws = np.array([m.shape[1] for m in nmaps] or [0], np.int32)
        rows = _f64(np.array([cam_row(cams[j]) for j in nb], np.float64).reshape(-1))
        tol = _f64(np.array([rel_tols[k][j] for j in nb], np.float64).reshape(-1))
        keep = np.zeros((H, W), np.uint8)
        xyz = np.zeros((3, H, W), np.float64)
        cnt = np.zeros((H, W), np.int32)
        lib().oracle_fuse_view(H, W, _p(D), _p(used[k]), _p(_f64(cam_row(cams[k]))), n, mp, up, _p(hs), _p(ws),
                               _p(rows), _p(tol), float(px_tol), int(min_views), int(point_stride), _p(keep),
                               _p(xyz), _p(cnt))
        vv, uu = np.nonzero(keep)
        if len(vv) == 0:
            continue
        pts.append(xyz[:, vv, uu].T.copy())
        cols.append(rgbs[k][vv, uu])
        nv.append(np.minimum(cnt[vv, uu], 255).astype(np.uint8))
        owner.append(np.full(len(vv), k, np.int32))
    cat = lambda a, shape, dt: np.concatenate(a) if a else np.zeros(shape, dt)
    return (cat(pts, (0, 3), np.float64), cat(cols, (0, 3), np.uint8), cat(nv, (0,), np.uint8),
            cat(owner, (0,), np.int32), {k: u.astype(bool) for k, u in used.items()})


# ------------------------------------------------------------------ legacy height sweep (mvs.py)
def sample_view(img, cam, X0, Y0, gsd, Z):
    """CPUBackend.sample_view (backend.py:67-76) over _mvs.sample_view (_mvs.pyx:13-58) restated:
    img (h, w, ch) float32, cam = (R, C, f, k1, k2, k3, cx, cy), Z (H, W) or (D, H, W) heights.
    Returns (samples (..., H, W, ch) float32, zero where invalid; valid (..., H, W) uint8)."""
    img = np.ascontiguousarray(img, np.float32)
    R, Cc, f, k1, k2, k3, cx, cy = cam
    Z = np.ascontiguousarray(Z, np.float32)
    h, w, nch = img.shape
    out = np.zeros(Z.shape + (nch,), np.float32)
    valid = np.zeros(Z.shape, np.uint8)
    Zs = Z.reshape((-1,) + Z.shape[-2:])
    os_ = out.reshape((-1,) + out.shape[-3:])
    vs = valid.reshape((-1,) + Z.shape[-2:])
    Rm, Cv = _f64(np.asarray(R, np.float64).reshape(-1)), _f64(np.asarray(Cc, np.float64).reshape(-1))
    for d in range(Zs.shape[0]):
        lib().oracle_sample_view(h, w, nch, _p(img), _p(Rm), _p(Cv), float(f), float(k1), float(k2), float(k3),
                                 float(cx), float(cy), float(X0), float(Y0), float(gsd), Zs.shape[1], Zs.shape[2],
                                 _p(Zs[d]), _p(os_[d]), _p(vs[d]))
    return out, valid


def box_sat_mean(a, r: int):
    """_fast.box_sat_mean (_fast.pyx:897-942) restated: (..., H, W) float32 -> window mean."""
    a = np.ascontiguousarray(a, np.float32)
    shape = a.shape
    planes = a.reshape((-1,) + shape[-2:])
    out = np.empty_like(planes)
    if lib().oracle_box_sat_mean(planes.shape[0], shape[-2], shape[-1], _p(planes), int(r), _p(out)) != 0:
        raise ValueError("box_sat_mean: bad radius or out of memory")
    return out.reshape(shape)


def sgm(cost, P1: float, P2: float):
    """_mvs.sgm (_mvs.pyx:98-251) restated: (D, H, W) float32 cost -> aggregated (D, H, W)."""
    cost = np.ascontiguousarray(cost, np.float32)
    D, H, W = cost.shape
    agg = np.empty_like(cost)
    if D and H and W:
        if lib().oracle_sgm(D, H, W, _p(cost), float(P1), float(P2), _p(agg)) != 0:
            raise MemoryError("sgm")
    return agg

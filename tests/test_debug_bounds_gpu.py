"""The bounds-checked debug build (libmvs_b200_debug.so, MVS_DEBUG_BOUNDS): every shared-memory and
global index of the tile engine (single-view, batched and served kernels) and of PatchMatch is
checked on small, odd cases - the reference's own parity shapes (2 x 40, 40 x 3, 5 x 4, ...), NaN
sources, infinite and negative hypotheses, border tiles at every radius, PatchMatch with masked
pixels and 3-8 sources - and no index may fall outside its buffer. Runs in a child process that
loads the debug library (MVS_LIBRARY=debug-bounds)."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r'''
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, ROOT)
sys.path.insert(0, ROOT + "/tests")
from conftest import golden, sweep_case
from py_ortho_b200 import _lib as L, batch, dense, fast, scene as S
from oracle import oracle as O
lib = L.load()
assert L.LIB_PATH.endswith("libmvs_b200_debug.so")
n = ctypes.c_uint32(0)
L.check(lib.mvs_debug_bound_violations(ctypes.byref(n)))
z = golden("sweep_cases.npz")
for k in range(int(z["ncases"])):
    c = sweep_case(z, k)
    st = O.init_state(c["H"], c["W"])
    for i, inv in enumerate(c["hyps"]):
        dense.sweep_hypothesis(c["ref"], c["mu"], c["sd"], c["srcs"], c["ray"], c["geo"], inv, c["r"], c["top_k"], i, *st)
T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
for (w, h, r) in ((70, 40, 0), (97, 51, 3), (64, 32, 7), (131, 66, 2), (33, 17, 5)):
    sc = S.make_scene("c1", seed=r + 3, width=w, height=h)
    ref = T(sc.grey(sc.ref)); srcs = [T(sc.grey(s)) for s in sc.srcs]
    mu, sd = fast.ref_stats(ref, r)
    hyp = dense.Hypotheses.planes_inv(S.plane_list(35.0, 55.0, 9))
    geo = S.geo_rows(sc.ref_cam, sc.src_cams)
    for prec, ss in ((L.PREC_FP32, srcs), (L.PREC_FP16, [fast.to_fp16(s) for s in srcs]),
                     (L.PREC_FP64_SUMS, srcs), (L.PREC_FP32_COMP, srcs)):
        dense.sweep(ref, mu, sd, None, ss, geo, hyp, r, 2, ref_cam=sc.ref_cam.row(), precision=prec, plane_chunks=2)
    if r <= 3:
        job = batch.ViewJob(ref, srcs, sc.ref_cam, sc.src_cams, S.plane_list(35.0, 55.0, 9), r=r, top_k=2).prepare()
        b = batch.Batch([job]); b.run(); b.close()
pz = golden("pm_case.npz")
srcs3 = [pz[f"src{j}"] for j in range(3)]
for prec in ("fp64", "fp32"):
    st = [pz["depth0"].copy(), pz["normal0"].copy(), pz["score0"].copy()]
    dense.pm_refine(pz["ref"], pz["ray"], pz["Cr"], srcs3, [None, pz["sdep1"], None], pz["par"], *st, pz["active"],
                    2, 1, 2, 0.5, 0.02, 2, 35.0, 55.0, 7, precision=prec)
for (w, h, ns, rr, step) in ((41, 23, 8, 3, 1), (30, 19, 5, 2, 2)):
    sc = S.make_scene("c2", seed=ns, width=w, height=h)
    ref = sc.grey(sc.ref).astype(np.float32); ref[3, 4] = np.nan
    srcs = [sc.grey(s).astype(np.float32) for s in sc.srcs[:ns]]
    srcs[0][5, 6] = np.nan
    ray = O.rays_world((h, w), sc.ref_cam)
    par = np.array([cam.row() for cam in sc.src_cams[:ns]], np.float64)
    d = (sc.depth_true * 1.01).astype(np.float32); d[0, 0] = np.nan
    zr = float(sc.ref_cam.C[2])
    for prec in ("fp64", "fp32"):
        st = [d.copy(), S.tilted_normals(h, w, 1), np.zeros((h, w), np.float32)]
        dense.pm_refine(ref, ray, sc.ref_cam.C, srcs, [None] * ns, par, *st, np.ones((h, w), np.uint8), rr, step, 2,
                        0.0, 0.02, 2, zr - 40, zr + 5, 3, precision=prec)
torch.cuda.synchronize()
L.check(lib.mvs_debug_bound_violations(ctypes.byref(n)))
print("bound violations:", n.value)
sys.exit(0 if n.value == 0 else 3)
'''


def test_debug_build_finds_no_index_outside_its_buffer():
    lib = os.path.join(ROOT, "py_ortho_b200", "libmvs_b200_debug.so")
    if not os.path.exists(lib):
        pytest.skip("the bounds-checked build is not present (python -m py_ortho_b200.build --debug-bounds)")
    env = dict(os.environ, MVS_LIBRARY="debug-bounds")
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CHILD], env=env, capture_output=True, text=True,
                       timeout=900)
    print(r.stdout[-2000:], r.stderr[-4000:])
    assert r.returncode == 0, r.stdout[-500:] + r.stderr[-2000:]
    assert "bound violations: 0" in r.stdout

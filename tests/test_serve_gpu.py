"""Continuous-batching server: each job's result is the same alone and in the mix (bit for bit:
the server runs the single-view tile engine with fixed chunk boundaries and an ordered merge),
including PatchMatch jobs whose state stays resident across steps, and under a tight HBM budget
that forces queueing."""
import numpy as np
import pytest
import torch

from conftest import same_bits

pytestmark = pytest.mark.gpu


def _requests():
    from py_ortho_b200 import scene as S
    from py_ortho_b200.serve import DepthRequest
    specs = [(128, 96, 4, 24, 2, 0), (96, 72, 3, 17, 3, 2), (160, 120, 4, 40, 2, 0), (64, 48, 2, 9, 3, 0),
             (112, 84, 4, 33, 2, 2), (144, 108, 3, 28, 3, 0)]
    reqs = []
    for k, (w, h, ns, npl, r, pm) in enumerate(specs):
        sc = S.make_scene("c1", seed=40 + k, width=w, height=h)
        reqs.append(DepthRequest(sc.grey(sc.ref), [sc.grey(s) for s in sc.srcs[:ns]], sc.ref_cam, sc.src_cams[:ns],
                                 S.plane_list(35.0, 55.0, npl), r=r, top_k=2, pm_iters=pm, pm_radius=2,
                                 depth_range=(35.0, 55.0), seed=100 + k, arrival=0.002 * k, rid=k))
    return reqs


def _check(a, b):
    assert same_bits(a.depth, b.depth)
    if a.normal is not None or b.normal is not None:
        assert same_bits(a.normal, b.normal) and same_bits(a.score, b.score)


def test_each_result_is_the_same_alone_and_in_the_mix():
    from py_ortho_b200.serve import DepthServer, serve, serve_plain
    mix, _ = serve(_requests(), DepthServer(plane_chunk=8, max_slots=8), realtime=False)
    plain, _ = serve_plain(_requests(), realtime=False)
    assert [r.rid for r in mix] == list(range(6))
    for a, b in zip(mix, plain):
        _check(a, b)
    for req, b in zip(_requests(), plain):             # alone in the server
        alone, _ = serve([req], DepthServer(plane_chunk=8, max_slots=2), realtime=False)
        _check(alone[0], b)


def test_budget_forces_queueing_without_changing_results():
    from py_ortho_b200.serve import DepthServer, footprint, serve, serve_plain
    reqs = _requests()
    budget = max(footprint(q) for q in reqs) * 1.5      # about one job at a time
    srv = DepthServer(hbm_budget=budget, plane_chunk=16, max_slots=4)
    got, _ = serve(reqs, srv, realtime=False)
    plain, _ = serve_plain(_requests(), realtime=False)
    for a, b in zip(got, plain):
        _check(a, b)
    too_big = DepthServer(hbm_budget=1e5, plane_chunk=16, max_slots=4)
    too_big.submit(_requests()[0])
    with pytest.raises(MemoryError):
        too_big.step(0.0)


def test_fp16_server_matches_the_plain_fp16_path_with_patchmatch_overlapped():
    """The FP16-storage server (sources converted once and shared, FP32 sums) against the plain
    per-request path with the same FP16 sources: the same bits per job, PatchMatch jobs included
    (they run on the server's PatchMatch streams, overlapping the sweep steps)."""
    from py_ortho_b200.serve import DepthServer, serve, serve_plain
    srv = DepthServer(plane_chunk=8, max_slots=8, precision="fp16", pm_streams=2)
    mix, _ = serve(_requests(), srv, realtime=False)
    plain, _ = serve_plain(_requests(), realtime=False, precision="fp16")
    assert [r.rid for r in mix] == list(range(6))
    for a, b in zip(mix, plain):
        _check(a, b)
    assert not srv._half                         # every FP16 copy released with its last job

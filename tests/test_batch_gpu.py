"""Batched persistent launch: every job's result equals its single-view sweep at the same tile
height, alone or in a mix of uneven jobs (sizes, source counts, plane counts, radii), with and
without the CUDA graph."""
import numpy as np
import pytest
import torch

from conftest import same_bits

pytestmark = pytest.mark.gpu


def _jobs(seed=0):
    from py_ortho_b200 import batch, scene
    cfgs = [(96, 72, 4, 24, 2), (160, 120, 2, 40, 3), (64, 48, 4, 17, 2), (128, 96, 3, 33, 3)]
    jobs = []
    for k, (w, h, ns, npl, r) in enumerate(cfgs):
        sc = scene.make_scene("c1", seed=seed + k, width=w, height=h)
        grey = lambda u8: torch.from_numpy(sc.grey(u8)).cuda()
        jobs.append(batch.ViewJob(grey(sc.ref), [grey(s) for s in sc.srcs[:ns]], sc.ref_cam, sc.src_cams[:ns],
                                  scene.plane_list(35.0, 55.0, npl), r=r, top_k=2))
    return jobs


def _single(job, tile_h=0):
    from py_ortho_b200 import dense, fast
    hyp = dense.Hypotheses.planes_inv(job.planes_inv)
    from py_ortho_b200.batch import _geo
    st = dense.sweep(job.ref, job.mu, job.sd, None, job.srcs, _geo(job.ref_cam, job.src_cams), hyp, job.r, job.top_k,
                     ref_cam=fast.cam_row(job.ref_cam), tile_h=tile_h)
    return st, dense.finalize(hyp, st)


@pytest.mark.parametrize("plane_chunk,tile_h", [(0, 0), (8, 0), (0, 16), (8, 64)])
def test_batch_equals_single_view_and_is_isolated(plane_chunk, tile_h):
    from py_ortho_b200 import batch
    jobs = [j.prepare() for j in _jobs()]
    singles = [_single(j, tile_h) for j in jobs]
    b = batch.Batch(jobs, plane_chunk=plane_chunk, tile_h=tile_h)
    assert b.evals == sum(j.evals for j in jobs)
    for use_graph in (False, True, True):
        for j in jobs:
            j.depth.fill_(0)
            for t in j.state:
                t.fill_(0)
        b.run(graph=use_graph)
        torch.cuda.synchronize()
        for j, (st, d) in zip(jobs, singles):
            assert same_bits(j.depth.cpu().numpy(), d.cpu().numpy())
            for x, y in zip(j.state, st):
                assert same_bits(x.cpu().numpy(), y.cpu().numpy())
    b.close()
    # each job alone in its own batch gives the same bits as in the mix
    for j, (st, d) in zip(jobs, singles):
        b1 = batch.Batch([j], plane_chunk=plane_chunk, tile_h=tile_h)
        b1.run()
        torch.cuda.synchronize()
        assert same_bits(j.depth.cpu().numpy(), d.cpu().numpy())
        b1.close()


def test_autotuner_picks_a_plan():
    from py_ortho_b200 import batch
    jobs = [j.prepare() for j in _jobs(seed=10)]
    best, table = batch.autotune(jobs, chunks=(0, 8), ctas=(0,), tile_hs=(16, 32, 64), reps=1)
    assert len(table) == 6 and all(ms > 0 for *_, ms in table)
    assert sorted({th for _, _, th, _ in table}) == [16, 32, 64]
    best.run()
    torch.cuda.synchronize()
    assert all(np.isfinite(j.depth.cpu().numpy()).all() for j in jobs)
    best.close()

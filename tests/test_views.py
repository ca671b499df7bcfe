"""Multi-view passes 1 and 2 on the host side: the neighbour choice and pass-2 settings against
the reference's own values (views_case.npz), the oracle's consistency check / normals /
PatchMatch repair against the reference's recorded calls, and the sharded orchestration
(assignment, map exchange) on world_size-2 gloo process groups. CPU only."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import golden, same_bits
from oracle import oracle as O
from tests_support import views_fixture
from py_ortho_b200 import views as V
from py_ortho_b200.densify import DepthOptions


def test_neighbours_and_settings_match_reference():
    z, rec, cams, _ = views_fixture()
    opt = DepthOptions()
    nb = V.neighbours(rec, opt.neighbors)
    st = V.PassSettings(rec, dict(enumerate(cams)), nb, opt)
    assert st.px_tol == float(z["px_tol"]) and st.min_views == 3
    for k in z["have"]:
        assert nb[k] == list(z[f"nbrs{k}"]), k
        tol = st.rel_tols(k)
        assert np.array_equal(np.array([tol[j] for j in nb[k]]), z[f"tol{k}"]), k


def test_oracle_consistency_matches_reference():
    z, rec, cams, greys = views_fixture()
    mn = float(z["fopt"][0])
    for k in z["have"]:
        nb = list(z[f"nbrs{k}"])
        S = z[f"s{k}"].astype(np.float32)
        cnt, act = O.consistency(z[f"p{k}"], cams[k], [z[f"p{j}"] for j in nb], [cams[j] for j in nb],
                                 float(z["px_tol"]), z[f"tol{k}"], grey=greys[k], score=S, min_ncc=mn, min_views=3)
        assert np.array_equal(cnt, z[f"cnt{k}"]), k
        assert np.array_equal(act, z[f"pm{k}_active"]), k


def test_oracle_init_normals_and_pass2_patchmatch_match_reference():
    z, rec, cams, greys = views_fixture()
    k = int(z["norm_view"])
    H, W = greys[k].shape
    ray = O.rays_world((H, W), cams[k])
    N0 = O.init_normals(z[f"p{k}"], ray)
    assert same_bits(N0, z["norm_out"])
    # the reference's pass-2 PatchMatch (its sequential xorshift draws), geometric term on
    k = int(z["have"][0])
    nb = list(z[f"nbrs{k}"])
    r, step, top_k, iters, seed = (int(v) for v in z[f"pm{k}_args"])
    gw, gt, dmin, dmax = (float(v) for v in z[f"pm{k}_fargs"])
    ray = O.rays_world((H, W), cams[k])
    D = z[f"p{k}"].copy()
    N = O.init_normals(D, ray)
    S = z[f"s{k}"].astype(np.float32)
    par = np.array([O.cam_row(cams[j]) for j in nb])
    ch = O.pm_refine(greys[k], ray, np.asarray(cams[k].C, np.float64), [greys[j] for j in nb],
                     [z[f"p{j}"] for j in nb], par, D, N, S, z[f"pm{k}_active"], r, step, top_k, gw, gt, iters,
                     dmin, dmax, seed)
    assert ch == int(z[f"pm{k}_changed"])
    assert same_bits(D, z[f"pm{k}_depth_out"]) and same_bits(N, z[f"pm{k}_normal_out"])
    assert same_bits(S, z[f"pm{k}_score_out"])


def test_assign_views_is_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    costs = rng.integers(1, 100, 37).astype(float)
    for world in (1, 2, 3, 8):
        owner = V.assign_views(costs, world)
        assert owner == V.assign_views(list(costs), world)
        loads = np.bincount(owner, weights=costs, minlength=world)
        assert loads.max() - loads.min() <= costs.max()          # LPT bound
    assert V.assign_views([], 4) == []
    assert V.assign_views([5.0, 5.0, 5.0], 2) == [0, 1, 0]


def test_wanted_maps():
    owner = [0, 1, 0, 1]
    nbrs = [[1, 2], [0], [3], [2]]
    assert V.wanted_maps(owner, nbrs, have=[0, 1, 2, 3]) == [0, 1, 2, 3]
    assert V.wanted_maps(owner, nbrs, have=[0, 2, 3]) == [2, 3]
    assert V.wanted_maps([0, 0, 0, 0], nbrs, have=[0, 1, 2, 3]) == []
    # each map goes only to the ranks whose views read it
    assert V.map_destinations([0, 1, 2, 1], [[1], [0], [1], []], have=[0, 1, 2, 3]) == {0: [1], 1: [0, 2]}


# ------------------------------------------------------------------ sharded orchestration on gloo
N_VIEWS = 7
SHAPES = {k: (3 + k % 3, 4 + k % 2) for k in range(N_VIEWS)}
NBRS = [[(k + 1) % N_VIEWS, (k + 3) % N_VIEWS, (k + 5) % N_VIEWS] for k in range(N_VIEWS)]
COSTS = [float(h * w * 3) for (h, w) in SHAPES.values()]
NO_MAP = 4                                   # this view produces no depth map in pass 1


def _pass1(k):
    if k == NO_MAP:
        return None
    h, w = SHAPES[k]
    return torch.arange(h * w, dtype=torch.float32).reshape(h, w) * 0.25 + k


def _pass2(k, maps):
    # every neighbour that has a map must be readable, and bit-identical to what its owner made
    got = []
    for j in NBRS[k]:
        if j == NO_MAP:
            assert j not in maps
            continue
        assert torch.equal(maps[j], _pass1(j)), (k, j)
        got.append(float(maps[j].sum()))
    return (k, tuple(got), float(maps[k].mean()))


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = V.run_passes(N_VIEWS, NBRS, COSTS, SHAPES, _pass1, _pass2, device=torch.device("cpu"))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_run_passes_on_gloo_ranks_matches_one_rank(world):
    """Passes 1 and 2 sharded over 2 and 3 gloo ranks: every view's pass 2 sees exactly the maps a
    single process gives it (each map sent point to point to the ranks that read it)."""
    single = V.run_passes(N_VIEWS, NBRS, COSTS, SHAPES, _pass1, _pass2, device=torch.device("cpu"))
    assert sorted(single) == [k for k in range(N_VIEWS) if k != NO_MAP]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    owner = V.assign_views(COSTS, world)
    merged = {}
    for rank, out in res.items():
        assert all(owner[k] == rank for k in out)                   # each view on its owner only
        merged.update(out)
    assert merged == single


# ------------------------------------------------------------------ point fusion (densify._fuse)
def _fuse_inputs(z, fz, c):
    from tests_support import views_fixture
    _, rec, cams, greys = views_fixture()
    have = [int(k) for k in z["have"]]
    maps = {k: np.ascontiguousarray(z[f"final{k}"], np.float32) for k in have}
    nbrs = {k: [int(j) for j in z[f"nbrs{k}"]] for k in have}
    tols = {k: {j: float(t) for j, t in zip(nbrs[k], z[f"tol{k}"])} for k in have}
    rgbs = {k: np.ascontiguousarray(np.repeat(z[f"img{k}"][:, :, None], 3, axis=2)) for k in range(len(cams))}
    min_views, stride = (int(v) for v in fz[f"f{c}_args"])
    return sorted(have), maps, cams, nbrs, tols, float(fz["px_tol"]), min_views, stride, rgbs


@pytest.mark.parametrize("c", [0, 1])
def test_oracle_fuse_matches_the_reference(c):
    """The oracle's fusion reproduces the reference's densify._fuse bit for bit: every fused point,
    colour, view count and owner, in the reference's order, and the used masks it leaves."""
    z, fz = golden("views_case.npz"), golden("fuse_case.npz")
    order, maps, cams, nbrs, tols, px_tol, min_views, stride, rgbs = _fuse_inputs(z, fz, c)
    xyz, cols, nv, owner, used = O.fuse(order, maps, cams, nbrs, tols, px_tol, min_views, stride, rgbs)
    assert len(xyz) == len(fz[f"f{c}_xyz"]) > 0
    assert same_bits(xyz, fz[f"f{c}_xyz"])
    assert np.array_equal(cols, fz[f"f{c}_cols"])
    assert np.array_equal(nv, fz[f"f{c}_nv"])
    assert np.array_equal(owner, fz[f"f{c}_owner"])
    for k in order:
        assert np.array_equal(used[k], fz[f"f{c}_used{k}"])

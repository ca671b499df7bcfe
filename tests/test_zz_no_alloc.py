"""mvs_sweep_noalloc: the sweep for callers that cannot allocate device memory (a process whose
device memory belongs to another allocator with a fixed budget, or a latency-critical loop that
must not enter the driver's allocator, which can synchronise the device).

Called through the C ABI and checked against mvs_sweep on the same inputs, bit for bit (the
plane-chunk merge is exact, so any chunk count gives the same bits), on two calls in a row -
the static scratch array keeps the previous call's contents, which must not leak into the next.
This file is collected last; it runs the same alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import same_bits

pytestmark = pytest.mark.gpu

CAPACITY = 32 << 20          # bytes of the library's static scratch array


def _inputs():
    from py_ortho_b200 import dense, fast, scene as S
    sc = S.make_scene("c1", seed=21, width=320, height=240)
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ref = T(sc.grey(sc.ref))
    srcs = [T(sc.grey(s)) for s in sc.srcs]
    mu, sd = fast.ref_stats(ref, 2)
    planes = S.plane_list(35.0, 55.0, 48)
    return dense, ref, mu, sd, srcs, S.geo_rows(sc.ref_cam, sc.src_cams), sc.ref_cam.row(), planes


def _run(fn_name, plane_chunks=0):
    from py_ortho_b200 import _lib as L
    dense, ref, mu, sd, srcs, geo, ref_cam, planes = _inputs()
    hyp = dense.Hypotheses.planes_inv(planes)
    state = dense.new_state(ref.shape[0], ref.shape[1])
    a, keep = dense.sweep_args(ref, mu, sd, None, srcs, geo, ref_cam, hyp, 2, 2, state, plane_chunks=plane_chunks)
    L.check(getattr(L.load(), fn_name)(ctypes.addressof(a), L.stream_handle()), fn_name)
    depth = dense.finalize(hyp, state)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in state] + [depth.cpu().numpy()]


def test_noalloc_sweep_matches_mvs_sweep_on_two_calls_in_a_row():
    expect = _run("mvs_sweep")
    first = _run("mvs_sweep_noalloc")            # automatic chunking: several chunk records
    second = _run("mvs_sweep_noalloc")           # the array now holds the first call's records
    for got in (first, second):
        for x, y in zip(got, expect):
            assert same_bits(x, y)
    explicit = _run("mvs_sweep_noalloc", plane_chunks=6)
    for x, y in zip(explicit, expect):
        assert same_bits(x, y)


def _pool():
    """The device's current memory pool: the one stream-ordered allocations (cudaMallocAsync,
    as mvs_sweep uses for its chunk records) draw from."""
    from cuda.bindings import driver as d
    err, dev = d.cuCtxGetDevice()
    assert err == d.CUresult.CUDA_SUCCESS, err
    err, pool = d.cuDeviceGetMemPool(dev)
    assert err == d.CUresult.CUDA_SUCCESS, err
    return d, pool


def _pool_used_high(d, pool) -> int:
    err, v = d.cuMemPoolGetAttribute(pool, d.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH)
    assert err == d.CUresult.CUDA_SUCCESS, err
    return int(v)


def _pool_reset_high(d, pool):
    err, = d.cuMemPoolSetAttribute(pool, d.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH, d.cuuint64_t(0))
    assert err == d.CUresult.CUDA_SUCCESS, err


def test_noalloc_allocates_nothing_and_rejects_oversized_scratch():
    """No allocation, shown two ways: the pool's high-water mark of memory in use (reset to zero
    first) stays zero across noalloc calls while one mvs_sweep call with the same arguments raises
    it - so a pooled stream-ordered allocation, which returns its memory to the pool and leaves
    the free-memory figure unchanged, would be seen - and the device's free memory is unchanged."""
    from py_ortho_b200 import _lib as L
    dense, ref, mu, sd, srcs, geo, ref_cam, planes = _inputs()
    hyp = dense.Hypotheses.planes_inv(planes)
    state = dense.new_state(ref.shape[0], ref.shape[1])
    a, keep = dense.sweep_args(ref, mu, sd, None, srcs, geo, ref_cam, hyp, 2, 2, state, plane_chunks=8)
    lib = L.load()
    L.check(lib.mvs_sweep_noalloc(ctypes.addressof(a), L.stream_handle()))   # set-up call
    torch.cuda.synchronize()
    d, pool = _pool()
    free0 = torch.cuda.mem_get_info()[0]
    _pool_reset_high(d, pool)
    assert _pool_used_high(d, pool) == 0
    for _ in range(3):
        L.check(lib.mvs_sweep_noalloc(ctypes.addressof(a), L.stream_handle()))
    torch.cuda.synchronize()
    assert _pool_used_high(d, pool) == 0
    assert torch.cuda.mem_get_info()[0] == free0
    # the probe sees a pooled allocation: the allocating entry point, same arguments
    L.check(lib.mvs_sweep(ctypes.addressof(a), L.stream_handle()))
    torch.cuda.synchronize()
    assert _pool_used_high(d, pool) >= 6 * 8 * ref.shape[0] * ref.shape[1] * 4
    # 48 chunks x 6 records x 320 x 240 floats = 88 MB > 32 MiB: a clear error, nothing launched
    big = 6 * 48 * ref.shape[0] * ref.shape[1] * 4
    assert big > CAPACITY
    a.plane_chunks = 48
    with pytest.raises(ValueError, match="static buffer"):
        L.check(lib.mvs_sweep_noalloc(ctypes.addressof(a), L.stream_handle()))

"""The C ABI without a GPU: the library loads, exports every function include/mvs_b200.h
declares, the ctypes structs match the C layout (gcc probe), and argument validation returns the
reference's error classes before any device work."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "mvs_b200.h")


def _lib():
    from py_ortho_b200 import _lib as L
    return L


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mvs_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    L = _lib()
    lib = ctypes.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)
    assert L.load().mvs_version().startswith(b"libmvs_b200")


def test_ctypes_structs_match_the_c_layout(tmp_path):
    L = _lib()
    structs = {"mvs_hyp": L.Hyp, "mvs_sweep_args": L.SweepArgs, "mvs_pm_args": L.PMArgs,
               "mvs_batch_job": L.BatchJob, "mvs_batch_tuning": L.BatchTuning,
               "mvs_consistency_args": L.ConsArgs, "mvs_fuse_args": L.FuseArgs,
               "mvs_sample_view_args": L.SampleViewArgs, "mvs_height_score_args": L.HeightScoreArgs,
               "mvs_depth_band_args": L.DepthBandArgs}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    c = tmp_path / "probe.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(c)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.split("\n") if l)
    for cname, py in structs.items():
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_validation_errors_need_no_device():
    L = _lib()
    lib = L.load()
    a = L.SweepArgs()
    a.n_src = 0
    assert lib.mvs_sweep(ctypes.addressof(a), None) == L.ERR_VALUE
    assert "1..16 sources" in L.last_error()
    a.n_src = 17
    assert lib.mvs_sweep(ctypes.addressof(a), None) == L.ERR_VALUE
    a.n_src, a.r = 2, -1
    assert lib.mvs_sweep(ctypes.addressof(a), None) == L.ERR_VALUE
    assert "negative window radius" in L.last_error()
    a.r = 9
    geo = np.zeros((2, 18))
    a.geo = geo.ctypes.data
    a.top_k = 2
    assert lib.mvs_sweep(ctypes.addressof(a), None) == L.ERR_UNSUPPORTED
    with pytest.raises(NotImplementedError):
        L.check(L.ERR_UNSUPPORTED)
    with pytest.raises(ValueError):
        L.check(L.ERR_VALUE)
    with pytest.raises(MemoryError):
        L.check(L.ERR_MEMORY)
    with pytest.raises(TimeoutError):
        L.check(L.ERR_TIMEOUT)
    assert lib.mvs_box_zero_mean(4, 4, None, -1, 0, None, None) == L.ERR_VALUE
    assert lib.mvs_box_zero_mean(0, 4, None, 1, 0, None, None) == L.OK        # empty input: no work
    # PatchMatch with 0 or > 16 sources returns without work, as the reference does
    p = L.PMArgs()
    p.S = 0
    assert lib.mvs_pm_refine(ctypes.addressof(p), None) == L.OK
    p.S = 17
    assert lib.mvs_pm_refine(ctypes.addressof(p), None) == L.OK
    assert lib.mvs_batch_create(None, 0, None, ctypes.byref(ctypes.c_void_p())) == L.ERR_VALUE
    # precision modes: an unknown one is refused; float64 and compensated window sums are
    # single-view only, and the compensated ones need constant planes
    b = L.SweepArgs()
    b.n_src, b.r, b.top_k, b.geo, b.precision = 1, 1, 1, geo.ctypes.data, 5
    assert lib.mvs_sweep(ctypes.addressof(b), None) == L.ERR_VALUE
    assert "unknown precision" in L.last_error()
    h = ctypes.c_void_p()
    assert lib.mvs_server_create(4, 4, 3, L.PREC_FP64_SUMS, ctypes.byref(h)) == L.ERR_UNSUPPORTED
    assert lib.mvs_server_create(4, 4, 3, L.PREC_FP16_COMP, ctypes.byref(h)) == L.ERR_UNSUPPORTED
    assert "single-view" in L.last_error()
    jobs = (L.BatchJob * 1)()
    j = jobs[0].sweep
    j.n_src, j.r, j.top_k, j.geo, j.precision = 1, 1, 1, geo.ctypes.data, L.PREC_FP64_SUMS
    j.hyp.kind = L.HYP_PLANES
    assert lib.mvs_batch_create(ctypes.addressof(jobs), 1, None, ctypes.byref(h)) == L.ERR_UNSUPPORTED
    assert "single-view" in L.last_error()
    # tile heights: 0 (= 32), 16, 32, 64; 16 and 64 only for FP32 / FP16 plane sweeps, top_k <= 2
    c = L.SweepArgs()
    c.n_src, c.r, c.top_k, c.geo, c.tile_h = 1, 1, 1, geo.ctypes.data, 48
    assert lib.mvs_sweep(ctypes.addressof(c), None) == L.ERR_VALUE
    assert "tile height 48" in L.last_error()
    c.tile_h = 64                                  # per-pixel hypotheses: the default shape only
    assert lib.mvs_sweep(ctypes.addressof(c), None) == L.ERR_UNSUPPORTED
    c.hyp.kind, c.precision = L.HYP_PLANES, L.PREC_FP64_SUMS
    assert lib.mvs_sweep(ctypes.addressof(c), None) == L.ERR_UNSUPPORTED
    c.precision, c.tile_h = L.PREC_FP32, 16
    assert lib.mvs_sweep(ctypes.addressof(c), None) == L.OK     # valid (an empty image: no work)
    tun = L.BatchTuning(0, 0, 24)
    assert lib.mvs_batch_create(ctypes.addressof(jobs), 1, ctypes.addressof(tun), ctypes.byref(h)) == L.ERR_VALUE
    assert "tile height 24" in L.last_error()


def test_depth_map_keeps_only_the_float64_sums_mode_on_per_pixel_sweeps():
    from py_ortho_b200 import densify
    L = _lib()
    opt = densify.DepthOptions()
    assert densify._per_pixel_precision(opt) == L.PREC_FP32
    opt.precision = L.PREC_FP16              # FP16 storage needs constant planes
    assert densify._per_pixel_precision(opt) == L.PREC_FP32
    opt.precision = L.PREC_FP64_SUMS
    assert densify._per_pixel_precision(opt) == L.PREC_FP64_SUMS


def test_precision_values_match_the_header(tmp_path):
    L = _lib()
    names = {"MVS_PREC_FP32": L.PREC_FP32, "MVS_PREC_FP16": L.PREC_FP16, "MVS_PREC_FP64_SUMS": L.PREC_FP64_SUMS}
    src = ['#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    src += [f'printf("{n} %d\\n", (int){n});' for n in names] + ["return 0; }"]
    c = tmp_path / "enums.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "enums"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(c)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    assert {k: int(v) for k, v in out.items()} == names


def test_python_layer_validates_before_touching_the_device():
    from py_ortho_b200 import dense
    with pytest.raises(ValueError, match="1..16 sources"):
        dense.sweep_hypothesis(None, None, None, [], None, np.zeros((0, 18)), None, 1, 2, 0, None, None, None, None,
                               None)
    with pytest.raises(ValueError, match="geo must be"):
        dense.sweep_hypothesis(None, None, None, [np.zeros((2, 2), np.float32)], None, np.zeros((2, 18)), None, 1, 2,
                               0, None, None, None, None, None)
    assert dense.pm_refine(None, None, None, [], [], None, None, None, None, None, 1, 1, 2, 0.0, 1.0, 1, 0, 1, 0) == 0


def test_stream_jump_ahead_matches_sequential_steps():
    """mvs_pm_stream_advance (GF(2) matrix powers, the jumps mvs_pm_refine's trials take) against
    the reference's xorshift32 stepped one draw at a time."""
    from oracle import oracle as O
    lib = _lib().load()
    for state in (1, 12345 | 1, 0xDEADBEEF, 0xFFFFFFFF):
        for n in (0, 1, 2, 7, 8, 31, 64, 1000, 4099):
            assert lib.mvs_pm_stream_advance(state, n) == O.xorshift_steps(state, n)
    # composition over a large jump: (a + b) steps = b steps after a steps
    s = 0x2545F491
    for a, b in ((1 << 20, 12345), (3 << 27, 1 << 31), ((1 << 40) + 5, 777)):
        assert lib.mvs_pm_stream_advance(lib.mvs_pm_stream_advance(s, a), b) == lib.mvs_pm_stream_advance(s, a + b)
    # the period of a full-period xorshift32 is 2^32 - 1
    assert lib.mvs_pm_stream_advance(s, (1 << 32) - 1) == s

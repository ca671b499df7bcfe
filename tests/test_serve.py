"""Serving host logic on the CPU: the FIFO / HBM-budget admission policy and job footprints."""
import numpy as np

from py_ortho_b200.serve import DepthRequest, admissions, footprint


def test_admission_is_fifo_and_respects_slots_and_budget():
    gb = 1e9
    assert admissions([10 * gb, 20 * gb, 30 * gb], free_slots=8, used=0.0, budget=120 * gb) == (3, False)
    assert admissions([10 * gb, 20 * gb, 30 * gb], free_slots=2, used=0.0, budget=120 * gb) == (2, False)
    assert admissions([50 * gb, 80 * gb, 1 * gb], free_slots=8, used=0.0, budget=120 * gb) == (1, False)  # FIFO
    assert admissions([50 * gb], free_slots=8, used=90 * gb, budget=120 * gb) == (0, False)
    assert admissions([], free_slots=8, used=0.0, budget=120 * gb) == (0, False)
    # a job that can never fit is rejected after the ones ahead of it are admitted
    assert admissions([121 * gb], free_slots=8, used=0.0, budget=120 * gb) == (0, True)
    assert admissions([10 * gb, 121 * gb, 5 * gb], free_slots=8, used=0.0, budget=120 * gb) == (1, True)


def test_footprint_counts_resident_buffers():
    H, W = 300, 400
    req = DepthRequest(np.zeros((H, W), np.float32), [np.zeros((H, W), np.float32)] * 4, None, [None] * 4,
                       np.linspace(0.01, 0.02, 96).astype(np.float32))
    base = H * W * 4 * 15
    assert footprint(req, shared_sources=True) == base
    assert footprint(req) == base + 4 * H * W * 4
    req.pm_iters = 4
    # + ray, normal, score, active; + PatchMatch scratch (pass state, cost cache, the sources' footprints)
    assert footprint(req, shared_sources=True) == base + H * W * (4 * 7 + 1) + H * W * 37 + 4 * H * W * 16
    assert req.evals == H * W * 96 * 4 + H * W * 4 * 11 * 4

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); runs the product kernels")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


def same_bits(a, b) -> bool:
    """Raw-bit equality of every non-NaN value (signed zeros included) and identical NaN
    positions. NaN payloads are not compared: the GPU returns the canonical NaN where x86
    propagates the payload of the NaN input."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        if not np.array_equal(na, nb):
            return False
        u = f"u{a.itemsize}"
        return bool((a.view(u)[~na] == b.view(u)[~nb]).all())
    return bool((a == b).all())


def sweep_case(z, k):
    """Case k of sweep_cases.npz -> dict of inputs and reference outputs."""
    p = f"c{k}_"
    H, W, n, r, top_k, nh = (int(v) for v in z[p + "meta"])
    c = dict(H=H, W=W, n=n, r=r, top_k=top_k, nh=nh)
    for key in ("ref", "ray", "geo", "hyps", "mu", "sd", "best", "prev", "spb", "snb", "idx", "scores"):
        c[key] = z[p + key]
    c["srcs"] = [z[p + f"src{j}"] for j in range(n)]
    return c


@pytest.fixture(scope="session")
def sweep_cases():
    z = golden("sweep_cases.npz")
    return [sweep_case(z, k) for k in range(int(z["ncases"]))]

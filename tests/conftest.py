"""Shared fixtures. Tests marked `gpu` need a CUDA device; the rest run on the CPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


def _ensure_built():
    lib = os.path.join(ROOT, "vite_b200", "libvite_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "vite_b200", "csrc"), "-j8"], check=True,
                       stdout=subprocess.DEVNULL)
    orc = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restate"], check=True,
                       stdout=subprocess.DEVNULL)


_ensure_built()


def multi_hub_csr(n, hubs, leaves, seed, real_weights):
    """Symmetric CSR (rowptr, tail, weight) with `hubs` hub vertices 0..hubs-1, each
    joined to `leaves` distinct random non-hub vertices, over a ring through all n
    vertices; weights U(0,1) per undirected edge, or 1.0."""
    import numpy as np

    rng = np.random.default_rng(seed)
    a, b = [], []
    for h in range(hubs):
        t = rng.choice(np.arange(hubs, n), size=leaves, replace=False)
        a.append(np.full(leaves, h))
        b.append(t)
    ring = np.arange(n)
    a.append(ring)
    b.append((ring + 1) % n)
    a = np.concatenate(a)
    b = np.concatenate(b)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(lo.astype(np.int64) * n + hi)
    lo, hi = key // n, key % n
    w = rng.random(len(key)) if real_weights else np.ones(len(key))
    src = np.concatenate([lo, hi])
    dst = np.concatenate([hi, lo])
    ww = np.concatenate([w, w])
    o = np.lexsort((dst, src))
    src, dst, ww = src[o], dst[o], ww[o]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, src + 1, 1)
    return np.cumsum(rp), dst.astype(np.int64), ww


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session")
def ctx():
    import vite_b200
    c = vite_b200.Context(0)
    yield c
    c.close()

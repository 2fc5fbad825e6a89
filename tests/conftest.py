import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def ctx():
    from ldsc_b200.build import build
    build()
    from ldsc_b200.api import Context
    c = Context(0)
    yield c
    c.close()


def brute_force_l2(body, n_indiv, chr_, cm, bp, left, annot=None, iid=None, pq=None):
    """Direct definition on a small panel: l2[j] = a_j + sum over in-band pairs
    of r2u_jk a_k, with r2u computed from standardised columns in f64."""
    from ldsc_b200.plink import decode_genotypes
    G = decode_genotypes(body, n_indiv)             # M x N, NaN missing
    if iid is not None:
        G = G[:, iid]
    N = G.shape[1]
    present = ~np.isnan(G)
    n = present.sum(1)
    s = np.where(present, G, 0).sum(1)
    q = np.where(present, G * G, 0).sum(1)
    mean = np.where(n > 0, s / np.maximum(n, 1), 0.0)
    css = q - n * mean * mean
    var = css / N
    sd = np.sqrt(np.maximum(var, 0))
    inv = np.where(sd > 0, 1.0 / np.where(sd > 0, sd, 1), 0.0)
    X = np.where(present, (G - mean[:, None]) * inv[:, None], 0.0)
    R = X @ X.T
    denom = N - 2.0 if N > 2 else float(N)
    r2u = R * R / (N * N) * (1 + 1 / denom) - 1 / denom
    m = len(chr_)
    a = np.ones((m, 1)) if annot is None else np.asarray(annot, dtype=np.float64).reshape(m, -1)
    if pq is not None:
        a = a * pq[:, None]
    l2 = a.copy()
    for j in range(m):
        for k in range(left[j], j):
            l2[j] += r2u[j, k] * a[k]
            l2[k] += r2u[j, k] * a[j]
    freq = np.clip(mean / 2.0, 0, 1)
    maf = np.minimum(freq, 1 - freq)
    return l2, maf

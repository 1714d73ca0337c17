import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.join(ROOT, "tests")
GOLDEN = os.path.join(TESTS, "golden")
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def geometry():
    from cuda_hlt_b200 import events
    return events.load_geometry()


@pytest.fixture(scope="session")
def minbias():
    from cuda_hlt_b200 import events
    return events.read_bank_folder(os.path.join(GOLDEN, "minbias", "VP"), os.path.join(GOLDEN, "minbias", "MC_tracks"))


def golden_batch(name):
    """Inputs of the committed reference-GPU golden files (see tests/golden/make_golden.py)."""
    from cuda_hlt_b200 import events
    if name == "minbias":
        return events.read_bank_folder(os.path.join(GOLDEN, "minbias", "VP"))
    if name == "plain":
        return events.generate_config("plain_1k", n_events=64)
    if name == "batched":
        return events.generate_config("batched_500k", n_events=32)
    if name == "pruned1m":
        return events.generate_config("pruned_1m", n_events=64)
    raise KeyError(name)


def load_golden(name):
    path = os.path.join(GOLDEN, f"ref_gpu_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} missing")
    return dict(np.load(path))


def golden_event_clusters(g, e):
    """Per-module cluster dicts of event e from a golden file."""
    nm = g["module_num"]
    starts = np.concatenate([[0], np.cumsum(nm.astype(np.int64))])
    out = []
    for m in range(52):
        a, b = starts[e * 52 + m], starts[e * 52 + m + 1]
        out.append({k: g["cl_" + k][a:b] for k in ("x", "y", "z", "phi", "id")})
    return out


def golden_event_tracks(g, e):
    N = (len(g["atomics"]) - 1) // 2
    t0, t1 = int(g["atomics"][N + e]), int(g["atomics"][N + e + 1])
    thn, ids = g["track_hit_number"], g["hit_id"]
    return [tuple(int(v) for v in ids[thn[t]:thn[t + 1]]) for t in range(t0, t1)]


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False

"""The CPU oracle, pinned against the reference itself:
  * cluster sets against the reference's own x86 restatement of the masked clustering
    (cuda_clustering_cpu_optimized, x86/velo/clustering/src/CudaClusteringCpuOptimized.cpp:4),
    run from the reference build on real and synthetic events;
  * clusters, tracks and states against the golden outputs of the reference's CUDA
    kernels (tests/golden/ref_gpu_*.npz, written by tests/golden/make_golden.py on a B200).
The oracle computes in IEEE fp32 without FMA contraction while the reference runs with
--use_fast_math on the GPU, so float fields are compared with a tolerance and discrete
decisions may flip on near-boundary cases (bounded below)."""
import os

import numpy as np
import pytest

import oracle
import parity_utils as pu
from conftest import golden_batch, golden_event_clusters, golden_event_tracks, load_golden
from cuda_hlt_b200 import events

needs_ref_x86 = pytest.mark.skipif(not os.path.exists(oracle.REF_X86_LIB), reason="reference x86 build missing")


@needs_ref_x86
@pytest.mark.parametrize("which", ["minbias", "plain", "batched", "pruned1m"])
def test_oracle_clusters_equal_reference_x86(geometry, which):
    b = golden_batch(which)
    r = oracle.run(b, geometry, stages=1)
    counts, ids, io = oracle.ref_x86_clustering(b, geometry, algo=1, threads=4)
    for e in range(b.n_events):
        mine = np.sort(r.event_clusters(e)["id"])
        ref = np.sort(ids[io[e]:io[e + 1]])
        assert np.array_equal(mine, ref), f"event {e}"


def _oracle_modules(r, e):
    oc = r.event_clusters(e)
    out, a = [], 0
    for m in range(52):
        n = int(oc["module_num"][m])
        out.append({k: oc[k][a:a + n] for k in ("x", "y", "z", "phi", "id")})
        a += n
    return out


@pytest.mark.parametrize("which", ["minbias", "plain", "batched", "pruned1m"])
def test_oracle_vs_reference_gpu_golden(geometry, which):
    g = load_golden(which)
    b = golden_batch(which)
    r = oracle.run(b, geometry)
    n_tracks = n_diff = 0
    for e in range(b.n_events):
        if r.flags[e] & oracle.UNDEFINED_IN_REFERENCE:
            continue
        cm = pu.compare_event_clusters(_oracle_modules(r, e), golden_event_clusters(g, e), exact=False, tol=2e-5)
        assert cm["count"] == 0 and cm["id"] == 0 and cm["xyz"] == 0 and cm["phi"] == 0, (e, cm)
        gt = golden_event_tracks(g, e)
        a, bb = pu.compare_event_tracks(r.event_tracks(e), gt)
        n_tracks += len(gt)
        n_diff += a + bb
    # ulp-level float differences flip at most a few near-boundary decisions
    assert n_diff <= max(3, 0.005 * n_tracks), (n_diff, n_tracks)


# 99th-percentile bounds of |oracle - reference| per state field. The oracle rounds in
# IEEE order without FMA, the reference with --use_fast_math and contraction; the fp32
# beamline fit stays within these, while the fp32 simplified Kalman amplifies rounding
# (chi2 and covariances move by O(1) relative), so only its position and slopes are
# bounded here. The CUDA chain reproduces every field bit for bit (tests/test_gpu_chain.py).
ORACLE_STATE_Q99 = {
    ("states", "x"): ("abs", 2e-4), ("states", "y"): ("abs", 2e-4), ("states", "tx"): ("abs", 5e-6),
    ("states", "ty"): ("abs", 5e-6), ("states", "z"): ("abs", 3e-2), ("states", "c00"): ("rel", 1e-4),
    ("states", "c20"): ("rel", 1e-4), ("states", "c22"): ("rel", 1e-4), ("kalman", "x"): ("abs", 3e-2),
    ("kalman", "y"): ("abs", 3e-2), ("kalman", "tx"): ("abs", 1e-3), ("kalman", "ty"): ("abs", 1e-3),
}


@pytest.mark.parametrize("which", ["minbias", "plain", "pruned1m"])
def test_oracle_states_vs_reference_gpu_golden(geometry, which):
    g = load_golden(which)
    b = golden_batch(which)
    r = oracle.run(b, geometry)
    N = b.n_events
    diffs = {k: [] for k in ORACLE_STATE_Q99}
    backward_mismatch = checked = 0
    for e in range(N):
        gt = golden_event_tracks(g, e)
        gi = pu.track_index(gt)
        t0g = int(g["atomics"][N + e])
        t0o = int(r.event_track_offsets[e])
        for i, t in enumerate(r.event_tracks(e)):
            j = gi.get(t)
            if j is None:
                continue
            for (name, key), (kind, _) in ORACLE_STATE_Q99.items():
                mine = (r.lsq if name == "states" else r.kal)[t0o + i, pu.STATE_KEYS.index(key)]
                ref = g[f"{name}_{key}"][t0g + j]
                d = abs(float(mine) - float(ref))
                diffs[(name, key)].append(d if kind == "abs" else d / max(abs(float(ref)), 1e-30))
            backward_mismatch += bool(r.lsq[t0o + i, 12]) != bool(g["states_backward"][t0g + j])
            checked += 1
    assert checked > 100
    assert backward_mismatch <= 0.001 * checked
    for k, (_, bound) in ORACLE_STATE_Q99.items():
        assert np.quantile(diffs[k], 0.99) < bound, (k, np.quantile(diffs[k], 0.99))


# 99th-percentile absolute residual of the fp32 fit against its fp64 twin, per field
# (x, y, z in mm; tx, ty dimensionless). The fp32 normal equations of the reference's
# means_square_fit and the fp32 simplified Kalman set these; the chain reproduces the fp32
# values bit for bit, so these are the accuracy of the reference algorithm itself.
FIT_RESIDUAL_Q99 = {
    "lsq": {"x": 1e-4, "y": 1e-4, "tx": 2e-6, "ty": 2e-6, "z": 1e-2},
    "kalman": {"x": 1e-2, "y": 1e-2, "tx": 3e-4, "ty": 3e-4},
}


def test_fp32_fit_residuals_against_fp64_twin(geometry):
    b = events.generate_config("plain_1k", n_events=100)
    r = oracle.run(b, geometry)
    for name, a32, a64 in (("lsq", r.lsq, r.lsq64), ("kalman", r.kal, r.kal64)):
        for key, bound in FIT_RESIDUAL_Q99[name].items():
            q = oracle.STATE_FIELDS.index(key)
            d = np.abs(a32[:, q].astype(np.float64) - a64[:, q])
            assert np.quantile(d, 0.99) < bound, (name, key, np.quantile(d, 0.99))


def test_oracle_empty_and_bad_events(geometry):
    nb = 208
    payload, offs = [], [0]
    for k in range(nb):
        payload += [k, 0]
        offs.append(4 * len(payload))
    empty = np.array([nb] + offs + payload, np.uint32).view(np.uint8)
    bad = empty.copy().view(np.uint32)
    bad[0] = 3
    bad = bad.view(np.uint8)
    raw = np.concatenate([empty, bad, empty])
    o = np.array([0, empty.size, empty.size + bad.size, raw.size], np.uint64)
    r = oracle.run(events.EventBatch(raw, o), geometry)
    assert r.module_num.sum() == 0
    assert list(np.diff(r.event_track_offsets)) == [0, 0, 0]
    assert r.flags[1] & oracle.F_BAD_RAW and not r.flags[0] and not r.flags[2]

"""The phi windows of fill_candidates (FillCandidates.cu:8-70, searches of
VeloTools.cuh:6-42) that the decode kernel's windows pass writes (hit_windows), against the
probe-for-probe oracle (oracle/window_oracle.py), exactly, on events of the bench workload
(nu ~ U(2,20)) and of the high-occupancy workload (nu = 15 with noise), whose largest events
search their windows in the cluster records instead of shared memory.
"""
import numpy as np
import pytest

from oracle import window_oracle
from cuda_hlt_b200 import chain, events

pytestmark = pytest.mark.gpu

PHI_STAGE_CAP = 9216  # events above this many clusters read the records (kPhiStageCap)


def windows_of(vc, res, n_events):
    ms = res["module_start"].reshape(-1, 52).astype(np.int64)
    mn = res["module_num"].reshape(-1, 52).astype(np.int64)
    span = int((ms + mn).max())
    win = vc._down(vc.out.hit_windows, np.uint32, 2 * span).reshape(-1, 2)
    phi = res["cluster_phi"]
    records = 0
    for e in range(n_events):
        base = int(ms[e, 0])
        nh = int(ms[e, 51] + mn[e, 51] - base)
        if nh == 0 or res["status"][e] & chain.STATUS["hit_overflow"]:
            continue
        records += nh > PHI_STAGE_CAP
        h1, f0, l0, f2, l2 = window_oracle.event_windows(phi[base:base + nh], ms[e] - base, mn[e])
        w = win[base + h1]
        w = w.astype(np.int64)
        got = [np.where((w[:, k] & 0xFFFF) == 0xFFFF, -1, w[:, k] & 0xFFFF) for k in (0, 1)]
        got_l = [np.where((w[:, k] & 0xFFFF) == 0xFFFF, -1, w[:, k] >> 16) for k in (0, 1)]
        assert np.array_equal(got[0], f0) and np.array_equal(got_l[0], l0), (e, "h0 window")
        assert np.array_equal(got[1], f2) and np.array_equal(got_l[1], l2), (e, "h2 window")
    return records


@pytest.mark.parametrize("config, n, first", [("pruned_1m", 300, 20_000), ("high_occupancy_200k", 120, 0)])
def test_chain_windows_equal_oracle(config, n, first):
    b = events.generate_config(config, n_events=n, first_event=first, threads=8, with_mc=False)
    vc = chain.VeloChain(max_events=n, max_raw_bytes=int(b.raw.size) + 4096)
    vc.run_host(b)
    vc.sync()
    res = vc.results()
    records = windows_of(vc, res, n)
    vc.close()
    if config == "high_occupancy_200k":
        assert records > 0, "no event took the records path"

"""velo_search_static, the search entry point that allocates nothing (for callers that
cannot allocate device memory, such as a host framework that reserves the device up front
and hands out fixed slices), against the chain's own search on the same clusters: track
hit lists identical after a canonical sort, on two calls in a row. Collected last so that
a run stopping at the first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from cuda_hlt_b200 import _lib, chain, events

pytestmark = pytest.mark.gpu

MAX_TRACKS, MAX_TRACK_SIZE = 1200, 26


def _static_tracks(cluster_id, module_start, track_n, track_hits, event_tracks, e):
    base = int(module_start[e * 52])
    out = []
    for t in range(int(event_tracks[e])):
        n = int(track_n[e * MAX_TRACKS + t])
        idx = track_hits[(e * MAX_TRACKS + t) * MAX_TRACK_SIZE:(e * MAX_TRACKS + t) * MAX_TRACK_SIZE + n]
        out.append(tuple(int(cluster_id[base + int(i)]) for i in idx))
    return out


def test_static_search_matches_chain():
    import torch
    b = events.generate_config("batched_500k", n_events=300, first_event=12345)
    vc = chain.VeloChain(max_events=300, max_raw_bytes=int(b.raw.size) + 4096)
    vc.run_host(b)
    vc.sync()
    res = vc.results()
    N = b.n_events
    lib = _lib.gpu_lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        track_n = torch.zeros(N * MAX_TRACKS, dtype=torch.int16, device="cuda")
        track_hits = torch.zeros(N * MAX_TRACKS * MAX_TRACK_SIZE, dtype=torch.int16, device="cuda")
        event_tracks = torch.zeros(N, dtype=torch.int32, device="cuda")
        status = torch.zeros(N, dtype=torch.int32, device="cuda")
        o = vc.out
        rc = lib.velo_search_static(C.c_void_p(o.hit_xyzp), C.c_void_p(o.module_hit_start),
                                    C.c_void_p(o.module_hit_num), C.c_void_p(o.status), N,
                                    C.c_void_p(track_n.data_ptr()), C.c_void_p(track_hits.data_ptr()),
                                    C.c_void_p(event_tracks.data_ptr()), C.c_void_p(status.data_ptr()),
                                    C.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        tn = track_n.cpu().numpy().view(np.uint16)
        th = track_hits.cpu().numpy().view(np.uint16)
        et = event_tracks.cpu().numpy().view(np.uint32)
        st = status.cpu().numpy().view(np.uint32)
        assert np.array_equal(et, res["n_tracks"]), call
        assert np.array_equal(st, res["status"]), call
        for e in range(N):
            mine = _static_tracks(res["cluster_id"], res["module_start"], tn, th, et, e)
            assert sorted(mine) == sorted(chain.event_tracks(res, e)), (call, e)
    vc.close()


def test_static_search_rejects_oversized_batch():
    lib = _lib.gpu_lib()
    dummy = C.c_void_p(16)
    assert lib.velo_search_static(dummy, dummy, dummy, dummy, 513, dummy, dummy, dummy, dummy, None) == -3

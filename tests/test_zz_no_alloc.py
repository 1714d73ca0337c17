"""velo_search_static, the search entry point that allocates nothing, against the chain's
own warp-per-event search on the same clusters.

Some callers cannot allocate device memory: a host framework that reserves the whole device
at start-up and hands its plugins fixed slices of that reservation (as the stage this
library replaces is run: one arena per stream, every buffer a slice of it) gives them no
allocator to call. The entry point keeps its scratch in a fixed array inside the library;
this test checks that its tracks and status flags equal the chain's, call after call.

The status given to the entry point keeps only the decode stage's bits, so every search
flag in its output (exact ties, ring and track overflows, weak-tracklet overflow, reads of
empty modules) is set by the entry point itself; the high-occupancy batch holds events that
overflow the reference's 500 weak tracklets. Collected last, so that a run that stops at the
first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from cuda_hlt_b200 import _lib, chain, events

pytestmark = pytest.mark.gpu

MAX_TRACKS, MAX_TRACK_SIZE = 1200, 26
# status bits written before the search (decode); the search adds the others
DECODE_BITS = sum(chain.STATUS[k] for k in ("bad_raw", "module_overflow", "hit_overflow", "candidate_overflow",
                                            "big_sp_index", "not_selected"))


def _static_tracks(cluster_id, module_start, track_n, track_hits, event_tracks, e):
    base = int(module_start[e * 52])
    out = []
    for t in range(int(event_tracks[e])):
        n = int(track_n[e * MAX_TRACKS + t])
        idx = track_hits[(e * MAX_TRACKS + t) * MAX_TRACK_SIZE:(e * MAX_TRACKS + t) * MAX_TRACK_SIZE + n]
        out.append(tuple(int(cluster_id[base + int(i)]) for i in idx))
    return out


@pytest.mark.parametrize("config,n,first", [("batched_500k", 300, 12345), ("high_occupancy_200k", 200, 4000)])
def test_static_search_matches_chain(config, n, first):
    import torch
    b = events.generate_config(config, n_events=n, first_event=first)
    # the chain's warp-per-event search is the one the entry point shares its code with
    vc = chain.VeloChain(max_events=n, max_raw_bytes=int(b.raw.size) + 4096, mapping=chain.MAP_WARP)
    vc.run_host(b)
    vc.sync()
    res = vc.results()
    N = b.n_events
    lib = _lib.gpu_lib()
    stream = torch.cuda.current_stream().cuda_stream
    o = vc.out
    status_in = torch.from_numpy((res["status"] & DECODE_BITS).astype(np.int32)).cuda()
    search_flags = res["status"] & ~np.uint32(DECODE_BITS)
    if config == "high_occupancy_200k":
        assert (res["status"] & chain.STATUS["weak_overflow"]).sum() > 0
    for call in range(2):
        track_n = torch.zeros(N * MAX_TRACKS, dtype=torch.int16, device="cuda")
        track_hits = torch.zeros(N * MAX_TRACKS * MAX_TRACK_SIZE, dtype=torch.int16, device="cuda")
        event_tracks = torch.zeros(N, dtype=torch.int32, device="cuda")
        status = torch.zeros(N, dtype=torch.int32, device="cuda")
        rc = lib.velo_search_static(C.c_void_p(o.hit_xyzp), C.c_void_p(o.module_hit_start),
                                    C.c_void_p(o.module_hit_num), C.c_void_p(status_in.data_ptr()), N,
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
        assert np.array_equal(st, res["status"]), (call, np.flatnonzero(st != res["status"])[:8])
        assert np.array_equal(st & ~np.uint32(DECODE_BITS), search_flags), call
        for e in range(N):
            mine = _static_tracks(res["cluster_id"], res["module_start"], tn, th, et, e)
            assert sorted(mine) == sorted(chain.event_tracks(res, e)), (call, e)
    vc.close()


def test_static_search_rejects_oversized_batch():
    lib = _lib.gpu_lib()
    dummy = C.c_void_p(16)
    assert lib.velo_search_static(dummy, dummy, dummy, dummy, 513, dummy, dummy, dummy, dummy, None) == -3

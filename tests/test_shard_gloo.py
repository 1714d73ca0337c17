"""The multi-GPU path on CPU: two ranks over gloo (127.0.0.1), one process each, as
bench.py --gpus 2 runs them under torchrun.

* each rank takes its own event range (cuda_hlt_b200.shard.event_range); together the ranks
  hold exactly the events a single process generates, byte for byte, with no overlap;
* each rank reconstructs its events on its own (the CPU oracle stands in for the GPU chain):
  the per-event track counts equal those of the single process;
* the elapsed time is the maximum over the ranks (shard.max_over_ranks).
"""
import hashlib
import os
import socket

import numpy as np
import pytest

N_PER_RANK = 6
WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _digest(a):
    return hashlib.blake2b(a.tobytes(), digest_size=8).hexdigest()


def _rank(rank, port, out_dir):
    import datetime
    import json

    import torch.distributed as dist

    from cuda_hlt_b200 import events, shard
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        first, n = shard.event_range(rank, N_PER_RANK)
        b = events.generate_config("pruned_1m", n_events=n, first_event=first, threads=2, with_mc=False)
        r = oracle.run(b, events.load_geometry(), threads=2)
        mine = {"first": first, "digests": [_digest(b.event(i)) for i in range(n)],
                "tracks": [int(r.event_track_offsets[i + 1] - r.event_track_offsets[i]) for i in range(n)]}
        everyone = [None] * WORLD
        dist.all_gather_object(everyone, mine)
        elapsed = shard.max_over_ranks(10.0 + rank, dist, "cpu")
        dist.barrier()
        if rank == 0:
            with open(os.path.join(out_dir, "result.json"), "w") as f:
                json.dump({"ranks": everyone, "elapsed": elapsed}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo(tmp_path):
    import json

    import torch.multiprocessing as mp

    from cuda_hlt_b200 import events
    import oracle
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = json.load(open(tmp_path / "result.json"))
    ranks = sorted(res["ranks"], key=lambda d: d["first"])
    assert [d["first"] for d in ranks] == [0, N_PER_RANK]
    # the single-process run over the same events
    b = events.generate_config("pruned_1m", n_events=WORLD * N_PER_RANK, first_event=0, threads=2, with_mc=False)
    r = oracle.run(b, events.load_geometry(), threads=2)
    want_digests = [_digest(b.event(i)) for i in range(b.n_events)]
    want_tracks = [int(r.event_track_offsets[i + 1] - r.event_track_offsets[i]) for i in range(b.n_events)]
    got_digests = [d for x in ranks for d in x["digests"]]
    got_tracks = [t for x in ranks for t in x["tracks"]]
    assert got_digests == want_digests
    assert len(set(got_digests)) == len(got_digests)
    assert got_tracks == want_tracks
    assert res["elapsed"] == 10.0 + (WORLD - 1)
    assert np.sum(want_tracks) > 0

"""Autotuner of the launch shapes, by timing stages on a sample batch:

* the search mapping: the cluster count above which an event runs the block-per-event search
  instead of the warp-per-event one (hit-count buckets);
* the decode block size: 4 or 8 warps per event (the tile of SuperPixels one block sorts and
  clusters at a time)."""
import numpy as np

from . import chain

THRESHOLDS = (0, 1024, 1536, 2048, 2560, 3072, 4096, 16384)


def tune_block_threshold(vc, raw_ptr, offsets_ptr, n_events, stream, reps=3, thresholds=THRESHOLDS):
    """Returns (best threshold, {threshold: search ms}) and leaves vc set to the best."""
    import torch
    timings = {}
    vc.set_timing(True)  # before any capture, so that every graph records its stage events
    for t in thresholds:
        vc.set_block_threshold(t)
        vc.run_device(raw_ptr, offsets_ptr, n_events, stream)  # warm-up (and graph capture)
        torch.cuda.synchronize()
        vc.set_timing(True)
        for _ in range(reps):
            vc.run_device(raw_ptr, offsets_ptr, n_events, stream)
        torch.cuda.synchronize()
        st = vc.stage_times()
        runs = max(1, st["runs"])
        timings[t] = st["search_by_triplet"] / runs
    best = min(timings, key=timings.get)
    vc.set_block_threshold(best)
    return best, timings


DECODE_WARPS = (8, 4)


def _stage_ms(vc, stage, raw_ptr, offsets_ptr, n_events, stream, reps):
    import torch
    vc.run_device(raw_ptr, offsets_ptr, n_events, stream)  # warm-up (and graph capture)
    torch.cuda.synchronize()
    vc.set_timing(True)
    for _ in range(reps):
        vc.run_device(raw_ptr, offsets_ptr, n_events, stream)
    torch.cuda.synchronize()
    st = vc.stage_times()
    return st[stage] / max(1, st["runs"])


def tune_decode_warps(vc, raw_ptr, offsets_ptr, n_events, stream, reps=3, choices=DECODE_WARPS):
    """Returns (best warps per decode block, {warps: decode ms}) and leaves vc set to the best."""
    timings = {}
    vc.set_timing(True)
    for w in choices:
        vc.set_decode_warps(w)
        timings[w] = _stage_ms(vc, "decode_cluster_sort", raw_ptr, offsets_ptr, n_events, stream, reps)
    best = min(timings, key=timings.get)
    vc.set_decode_warps(best)
    return best, timings

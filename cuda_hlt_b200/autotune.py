"""Autotuner of the search mapping: picks the cluster count above which an event runs the
block-per-event search instead of the warp-per-event one, by timing the search stage on a
sample batch for a set of thresholds (hit-count buckets)."""
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

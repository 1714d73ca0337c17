"""ORACLE — test infrastructure only (imported by tests/, __graft_entry__.smoke() and the
bench's baseline legs; never by the product path).

CPU restatement of the reference's global event cut, global_event_cut
(cuda/global_event_cut/src/GlobalEventCut.cu:3-55, maxSciFiUTClusters = 9750 from
cuda/global_event_cut/include/GlobalEventCut.cuh:9), one event at a time:

  * SciFi (GlobalEventCut.cu:14-32): over the FTCluster banks, sum (offset[i+1] - offset[i]
    - 4) in 32-bit unsigned arithmetic, then estimate = sum / 2 - 2 (unsigned: an event
    with no bank bytes wraps to a huge value and fails); the event fails when estimate >= max.
  * UT (GlobalEventCut.cu:34-47): sum over the UT banks of the low 16 bits of the second
    word of each bank (UTRawBank::number_of_hits, UTRaw.cuh:9-19).
  * The event passes when UT + SciFi < max (GlobalEventCut.cu:49-54).

Raw layout of both detectors (SciFiRaw.cuh:22-41, UTRaw.cuh:21-43): u32 number of banks,
u32 bank byte offsets [banks + 1], then the banks. The reference reads these tables without
bounds checks; an event whose table, or a UT bank's first two words, lie outside the event's
bytes is "malformed" here and fails the cut, as in the CUDA kernel of this package.

Parity is pinned by tests/golden/ref_gec.npz: the selection of the reference's own kernel
(oracle/_ref/libvelo_ref_gpu.so, run on a B200 by tests/golden/make_golden.py --ref-gec) on
the ten minbias events and on seeded synthetic events.
"""
import numpy as np

MAX_CLUSTERS = 9750
PASS, MALFORMED = 1, 2
U32 = 0xFFFFFFFF


def _table(raw_event, aligned=True):
    """(u32 words, number of banks) or None when the event does not start on a 4-byte
    boundary or its bank table does not fit."""
    if not aligned or raw_event.size < 8:
        return None
    w = raw_event[:raw_event.size // 4 * 4].view(np.uint32)
    nb = int(w[0])
    if (nb + 2) * 4 > raw_event.size:
        return None
    return w, nb


def event_counts(ut_event, scifi_event, ut_aligned=True, scifi_aligned=True):
    """(SciFi estimate, UT hits, malformed) of one event, as global_event_cut computes them;
    counts are 0xFFFFFFFF where the detector's tables are malformed."""
    t = _table(np.ascontiguousarray(scifi_event), scifi_aligned)
    bad = t is None
    n_scifi = U32
    if not bad:
        w, nb = t
        off = w[1:nb + 2].astype(np.int64)
        s = int(np.sum((off[1:] - off[:-1] - 4) & U32)) & U32
        n_scifi = ((s // 2) - 2) & U32
    t = _table(np.ascontiguousarray(ut_event), ut_aligned)
    ut_bad = t is None
    n_ut = U32
    if not ut_bad:
        w, nb = t
        payload_words = w.size - (nb + 2)
        off = w[1:nb + 1].astype(np.int64)
        if np.any(off & 3) or np.any(off + 8 > 4 * payload_words):
            ut_bad = True
        else:
            hits = int(np.sum(w[nb + 2 + off // 4 + 1] & 0xFFFF, dtype=np.int64))
            n_ut = min(hits, U32 - 1)
    return n_scifi, n_ut, bad or ut_bad


def run(ut_batch, scifi_batch, max_clusters=MAX_CLUSTERS):
    """Per event (counts [N, 2] u32, flags [N] u8), and the passing events in ascending order."""
    n = ut_batch.n_events
    counts = np.zeros((n, 2), np.uint32)
    flags = np.zeros(n, np.uint8)
    ut_aligned = (ut_batch.offsets[:-1] - ut_batch.offsets[0]) % 4 == 0
    scifi_aligned = (scifi_batch.offsets[:-1] - scifi_batch.offsets[0]) % 4 == 0
    for e in range(n):
        n_scifi, n_ut, bad = event_counts(ut_batch.event(e), scifi_batch.event(e), ut_aligned[e], scifi_aligned[e])
        counts[e] = (n_scifi, n_ut)
        ok = not bad and n_scifi < max_clusters and n_ut + n_scifi < max_clusters
        flags[e] = (PASS if ok else 0) | (MALFORMED if bad else 0)
    return counts, flags, np.flatnonzero(flags & PASS).astype(np.uint32)

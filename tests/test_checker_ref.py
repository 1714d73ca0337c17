"""The MC-truth checker of this library (velo_check_tracks) against the reference's own
TrackCheckerVelo (checker/tracking, built from the reference tree without ROOT into
oracle/_ref/libvelo_ref_checker.so) on the same tracks: reconstructible, found and clone
counts of "Not electron long eta25" and "Not electron Velo", tracks and ghosts, equal.

Tracks: the reference kernels' own tracks of the 10 real minbias events (committed golden
file, real MC truth with hits shared by several particles), and the CPU oracle's tracks of
200 synthetic events with clones, ghosts and truncated tracks added."""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, load_golden
from cuda_hlt_b200 import chain, events

pytestmark = pytest.mark.skipif(not os.path.exists(oracle.REF_CHECKER_LIB),
                                reason="reference checker build missing (oracle/build.py)")

LONG, VELO = "Not electron long eta25", "Not electron Velo"


def compare(batch, evt, tho, ids):
    ref = oracle.ref_check_velo_tracks(batch, evt, tho, ids)
    mine = chain.check_tracks(batch, dict(track_offsets=evt, track_hit_number=tho, hit_id=ids))
    assert ref["categories"][LONG] == (mine.long_reconstructible, mine.long_found, mine.long_clones)
    assert ref["categories"][VELO] == (mine.velo_reconstructible, mine.velo_found, mine.velo_clones)
    assert (ref["tracks"], ref["ghosts"]) == (mine.tracks, mine.ghosts)
    assert abs(ref["ghost_per_event"] - mine.ghost_rate_per_event) < 1e-5
    return ref, mine


def test_minbias_reference_tracks():
    mb = events.read_bank_folder(os.path.join(GOLDEN, "minbias", "VP"), os.path.join(GOLDEN, "minbias", "MC_tracks"))
    g = load_golden("minbias")
    N = mb.n_events
    ref, mine = compare(mb, g["atomics"][N:2 * N + 1], g["track_hit_number"], g["hit_id"])
    assert mine.long_found > 0 and mine.ghosts > 0 and mine.long_clones > 0


def _perturbed_tracks(r, n_events, rng):
    """The oracle's tracks of each event plus, per event, a clone of a few tracks, a few
    tracks whose hits come from two tracks (ghosts or not, by the 0.7 weight) and a few
    tracks cut to their first three hits."""
    out_evt, out_tho, out_ids = [0], [0], []
    for e in range(n_events):
        tracks = r.event_tracks(e)
        extra = []
        if tracks:
            pick = rng.integers(0, len(tracks), size=min(4, len(tracks)))
            extra += [tracks[i] for i in pick]                                   # clones
            for i in pick[:2]:
                j = rng.integers(0, len(tracks))
                a, b = list(tracks[i]), list(tracks[j])
                extra.append(tuple(a[:len(a) // 2] + b[len(b) // 2:]))          # mixed
                extra.append(tuple(a[:3]))                                       # truncated
        for t in list(tracks) + extra:
            out_ids += list(t)
            out_tho.append(len(out_ids))
        out_evt.append(len(out_tho) - 1)
    return (np.array(out_evt, np.uint32), np.array(out_tho, np.uint32), np.array(out_ids, np.uint32))


def test_synthetic_oracle_tracks_with_clones_and_ghosts(geometry):
    b = events.generate_config("pruned_1m", n_events=200, first_event=700)
    r = oracle.run(b, geometry)
    evt, tho, ids = _perturbed_tracks(r, b.n_events, np.random.default_rng(5))
    ref, mine = compare(b, evt, tho, ids)
    assert mine.long_clones > 100 and mine.ghosts > 100 and mine.long_reconstructible > 10000


def test_empty_tracks():
    mb = events.read_bank_folder(os.path.join(GOLDEN, "minbias", "VP"), os.path.join(GOLDEN, "minbias", "MC_tracks"))
    N = mb.n_events
    ref, mine = compare(mb, np.zeros(N + 1, np.uint32), np.zeros(1, np.uint32), np.zeros(0, np.uint32))
    assert mine.long_found == 0 and mine.tracks == 0

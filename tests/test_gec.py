"""Global event cut on the CPU: the oracle against the reference kernel's selections
(tests/golden/ref_gec.npz), its edge cases, the UT / SciFi readers and the synthetic
generator."""
import os
import sys

import numpy as np
import pytest

from cuda_hlt_b200 import events
from oracle import gec_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402


def raw_event(n_banks, bank_words, second_words=None):
    """u32 raw event: n_banks, offsets, banks of bank_words[i] words each (second word from
    second_words when given)."""
    offs = np.concatenate([[0], np.cumsum(bank_words)]) * 4
    banks = []
    for i, w in enumerate(bank_words):
        b = np.zeros(w, np.uint32)
        if w:
            b[0] = i
        if second_words is not None and w > 1:
            b[1] = second_words[i]
        banks.append(b)
    words = np.concatenate([[n_banks], offs.astype(np.uint32)] + banks).astype(np.uint32)
    return words.view(np.uint8)


def batch_of(raws):
    off = np.zeros(len(raws) + 1, np.uint64)
    off[1:] = np.cumsum([r.size for r in raws])
    return events.EventBatch(np.concatenate(raws), off)


def ut_with_hits(hits, n_banks=3):
    per = [hits // n_banks + (1 if i < hits % n_banks else 0) for i in range(n_banks)]
    return raw_event(n_banks, [2 + h for h in per], second_words=[0xABCD0000 | h for h in per])


def test_oracle_matches_reference_selection_on_minbias():
    g = np.load(os.path.join(GOLDEN, "ref_gec.npz"))
    ut, sf = make_golden.minbias_gec_batches()
    counts, flags, selected = gec_oracle.run(ut, sf)
    assert np.array_equal(selected, g["minbias_selected"])
    # the first event is above the cut: SciFi 7,776 + UT 2,108 >= 9,750
    assert counts[0].tolist() == [7776, 2108] and not flags[0] & gec_oracle.PASS
    assert selected.size == 9


def test_oracle_matches_reference_selection_on_synthetic():
    g = np.load(os.path.join(GOLDEN, "ref_gec.npz"))
    ut, sf, keep = make_golden.gec_synthetic_batches()
    assert np.array_equal(keep, g["synthetic_events"])
    _, _, selected = gec_oracle.run(ut, sf)
    assert np.array_equal(selected, g["synthetic_selected"])
    assert 0 < selected.size < ut.n_events


def test_oracle_edge_cases():
    M = gec_oracle.MAX_CLUSTERS
    def est(ev):  # SciFi estimate: (sum of bank bytes - 4 per bank) / 2 - 2
        return gec_oracle.event_counts(ut_with_hits(0), ev)[0]
    ev = raw_event(2, [1 + 10, 1 + 20])
    assert est(ev) == (4 * 30) // 2 - 2
    # no SciFi bank bytes: 0 / 2 - 2 wraps and fails
    empty = raw_event(0, [])
    n_scifi, _, bad = gec_oracle.event_counts(ut_with_hits(5), empty)
    assert n_scifi == 0xFFFFFFFE and not bad
    # boundary: UT + SciFi = M - 1 passes, = M fails
    sf = raw_event(1, [1 + 2000])            # estimate 4 * 2000 / 2 - 2 = 3998
    assert est(sf) == 3998
    ut_ok, ut_cut = ut_with_hits(M - 1 - 3998), ut_with_hits(M - 3998)
    b = gec_oracle.run(batch_of([ut_ok, ut_cut]), batch_of([sf, sf]))
    assert b[1].tolist() == [gec_oracle.PASS, 0]
    # malformed: table larger than the event, UT bank header outside the event
    short = np.array([50, 0, 4], np.uint32).view(np.uint8)
    assert gec_oracle.event_counts(ut_with_hits(3), short)[2]
    bad_ut = raw_event(1, [2], second_words=[7])
    w = bad_ut.view(np.uint32).copy()
    w[1] = 4000  # first bank offset far outside
    assert gec_oracle.event_counts(w.view(np.uint8), sf)[2]
    # unaligned event start
    c, f, _ = gec_oracle.run(batch_of([np.zeros(2, np.uint8), ut_with_hits(1)]), batch_of([sf[:8], sf]))
    assert f[0] & gec_oracle.MALFORMED and f[1] & gec_oracle.MALFORMED


def test_ut_and_scifi_from_mdf_match_bank_folders():
    mdf = os.path.join(GOLDEN, "minbias", "mdf")
    for bank in ("UT", "FTCluster"):
        folder = events.read_bank_folder(os.path.join(GOLDEN, "minbias", bank))
        m = events.read_mdf(mdf, bank=bank)
        assert m.n_events == folder.n_events == 10
        assert m.names == [n[:-len(".bin")] for n in folder.names]
        assert np.array_equal(m.offsets, folder.offsets) and np.array_equal(m.raw, folder.raw)
    with pytest.raises(KeyError):
        events.read_mdf(mdf, bank="Calo")


def test_synthetic_ut_scifi_are_seeded_and_well_formed():
    vp = events.generate_config("pruned_1m", n_events=64, with_mc=False)
    a = events.generate_ut_scifi(vp, seed=3)
    b = events.generate_ut_scifi(vp, seed=3)
    for x, y in zip(a, b):
        assert np.array_equal(x.raw, y.raw) and np.array_equal(x.offsets, y.offsets)
    counts, flags, _ = gec_oracle.run(*a)
    assert not np.any(flags & gec_oracle.MALFORMED)
    # occupancy follows the VELO event's size
    vp_words = np.diff(vp.offsets) / 4
    assert np.corrcoef(vp_words, counts[:, 0].astype(np.float64))[0, 1] > 0.9
    assert np.corrcoef(vp_words, counts[:, 1].astype(np.float64))[0, 1] > 0.9

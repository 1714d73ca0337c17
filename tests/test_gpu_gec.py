"""Global event cut on the GPU (velo_run_gec / velo_run_gec_host): per-event counts, flags
and the selected list against the oracle, the selection against the reference's own kernel
run live, and the chain on the selected events against the chain on the same events
passed without the cut."""
import os
import sys

import numpy as np
import pytest

from cuda_hlt_b200 import chain, events
from oracle import gec_oracle

import test_gec

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402


def run_gec(vp, ut, sf, max_clusters=chain.GEC_MAX_CLUSTERS, **kw):
    vc = chain.VeloChain(max_events=max(1, vp.n_events), max_raw_bytes=int(vp.raw.size) + 4096, **kw)
    try:
        vc.run_gec_host(vp, ut, sf, max_clusters=max_clusters)
        vc.sync()
        return vc.results()
    finally:
        vc.close()


def run_plain(vp, **kw):
    vc = chain.VeloChain(max_events=max(1, vp.n_events), max_raw_bytes=int(vp.raw.size) + 4096, **kw)
    try:
        vc.run_host(vp)
        vc.sync()
        return vc.results()
    finally:
        vc.close()


def assert_gec_equal(res, ut, sf, max_clusters=chain.GEC_MAX_CLUSTERS):
    counts, flags, selected = gec_oracle.run(ut, sf, max_clusters)
    assert np.array_equal(res["gec_counts"], counts)
    assert np.array_equal(res["gec_flags"], flags)
    assert res["n_selected"] == selected.size
    assert np.array_equal(res["event_list"], selected)
    return selected


def assert_positions_match(res_gec, res_sub, n_sel, n_events):
    """Positions 0 .. n_sel - 1 of the cut run equal the run over the selected events alone;
    later positions are empty."""
    for e in range(n_sel):
        assert chain.event_tracks(res_gec, e) == chain.event_tracks(res_sub, e), e
        assert res_gec["status"][e] == res_sub["status"][e], e
        assert np.array_equal(res_gec["module_num"][e * 52:(e + 1) * 52], res_sub["module_num"][e * 52:(e + 1) * 52])
    for e in range(n_sel, n_events):
        assert res_gec["status"][e] == chain.STATUS["not_selected"]
        assert res_gec["n_tracks"][e] == 0
        assert res_gec["module_num"][e * 52:(e + 1) * 52].sum() == 0


def test_minbias_against_oracle_and_chain():
    ut, sf = make_golden.minbias_gec_batches()
    vp = events.read_bank_folder(os.path.join(HERE, "golden", "minbias", "VP"))
    res = run_gec(vp, ut, sf)
    selected = assert_gec_equal(res, ut, sf)
    assert selected.tolist() == list(range(1, 10))
    sub = run_plain(make_golden.pick(vp, selected))
    assert_positions_match(res, sub, selected.size, vp.n_events)


def test_selection_matches_reference_kernel_live():
    import oracle
    ut, sf = make_golden.minbias_gec_batches()
    vp = events.read_bank_folder(os.path.join(HERE, "golden", "minbias", "VP"))
    res = run_gec(vp, ut, sf)
    assert np.array_equal(np.sort(oracle.ref_gec_run(ut, sf)), res["event_list"])
    sut, ssf, keep = make_golden.gec_synthetic_batches()
    svp = make_golden.pick(events.generate_config("pruned_1m", n_events=make_golden.GEC_SYNTH_EVENTS,
                                                  with_mc=False), keep)
    res = run_gec(svp, sut, ssf)
    assert_gec_equal(res, sut, ssf)
    assert np.array_equal(np.sort(oracle.ref_gec_run(sut, ssf)), res["event_list"])


@pytest.mark.parametrize("mode", ["plain", "pruned_graphs"])
def test_synthetic_batch_chain_on_selected(mode):
    vp = events.generate_config("pruned_1m", n_events=3000, first_event=7000, with_mc=False)
    ut, sf = events.generate_ut_scifi(vp, seed=11)
    kw = {}
    if mode == "pruned_graphs":
        from cuda_hlt_b200 import mlp, train_scorer
        kw = dict(mode=chain.MODE_PRUNED, use_graphs=True)
    vc = chain.VeloChain(max_events=vp.n_events, max_raw_bytes=int(vp.raw.size) + 4096, **kw)
    if mode == "pruned_graphs":
        vc.set_mlp(mlp.load_weights(train_scorer.DEFAULT_WEIGHTS))
    try:
        for _ in range(2):  # the second run replays the captured graph
            vc.run_gec_host(vp, ut, sf)
            vc.sync()
        res = vc.results()
        selected = assert_gec_equal(res, ut, sf)
        assert 0 < selected.size < vp.n_events
        vc.run_host(make_golden.pick(vp, selected))
        vc.sync()
        sub = vc.results()
    finally:
        vc.close()
    assert_positions_match(res, sub, selected.size, vp.n_events)


def test_edge_cases_threshold_and_malformed():
    M = 9750
    sf = test_gec.raw_event(1, [1 + 2000])  # estimate 3998
    ut_events = [test_gec.ut_with_hits(M - 1 - 3998), test_gec.ut_with_hits(M - 3998), test_gec.ut_with_hits(0)]
    sf_events = [sf, sf, test_gec.raw_event(0, [])]  # the last: no SciFi bytes, the estimate wraps
    short = np.array([50, 0, 4], np.uint32).view(np.uint8)
    bad_ut = test_gec.raw_event(1, [2], second_words=[7]).view(np.uint32).copy()
    bad_ut[1] = 4000
    ut_events += [test_gec.ut_with_hits(3), bad_ut.view(np.uint8)]
    sf_events += [short, sf]
    ut, sfb = test_gec.batch_of(ut_events), test_gec.batch_of(sf_events)
    vp = events.read_bank_folder(os.path.join(HERE, "golden", "minbias", "VP"), limit=len(ut_events))
    res = run_gec(vp, ut, sfb)
    selected = assert_gec_equal(res, ut, sfb)
    assert selected.tolist() == [0]
    assert res["gec_flags"].tolist() == [1, 0, 0, 2, 2]
    # a lower cut selects nothing; an empty batch is fine
    res = run_gec(vp, ut, sfb, max_clusters=100)
    assert res["n_selected"] == 0 and np.all(res["status"] == chain.STATUS["not_selected"])
    empty = events.EventBatch(np.zeros(0, np.uint8), np.zeros(1, np.uint64))
    res = run_gec(empty, empty, empty)
    assert res["n_selected"] == 0

"""Host-side arithmetic of bench.py: the batch plan, the algorithmic bytes per stage, the
roofline of the dominant stage and the host-link bound of the end-to-end leg."""
import types

import pytest

import bench


def test_batch_plan_covers_every_event_once():
    chunks = [types.SimpleNamespace(n_events=n) for n in (bench.BUCKET * 2 + 5, 7, bench.BUCKET)]
    plan = bench.batch_plan(chunks)
    for ci, c in enumerate(chunks):
        spans = [(a, b) for k, a, b in plan if k == ci]
        assert spans[0][0] == 0 and spans[-1][1] == c.n_events
        assert all(b - a <= bench.BUCKET and b > a for a, b in spans)
        assert all(spans[i][1] == spans[i + 1][0] for i in range(len(spans) - 1))


def test_link_bound():
    link = {"h2d_GBps": 50.0, "d2h_GBps": 60.0, "both_GBps_each_direction": 40.0}
    # 4 GB up and 10 GB down: 4 GB each way at 40 GB/s, then 6 GB down alone at 60 GB/s
    assert bench.link_bound(1_000_000, 4e9, 10e9, link) == pytest.approx(1_000_000 / (0.1 + 0.1))
    # the larger direction up: its own rate for the rest
    assert bench.link_bound(1_000, 10e9, 4e9, link) == pytest.approx(1_000 / (0.1 + 6e9 / 50e9))
    # equal bytes: all at the concurrent rate
    assert bench.link_bound(1, 8e9, 8e9, link) == pytest.approx(1 / 0.2)


def test_roofline_of_the_dominant_serial_stage():
    census = dict(clusters=3_000, tracks=150, track_hits=1_200, raw_bytes=20_000)
    per = bench.stage_bytes(census, 1)
    assert per["decode_cluster_sort"] == 20_000 + 24 * 3_000
    assert per["search_by_triplet"] == 24 * 3_000 + 2 * 1_200 + 2 * 150
    stages = {k: 0.0 for k in bench.chain.STAGES}
    stages.update(decode_cluster_sort=8.0, search_by_triplet=10.0, consolidate_fit=2.0, runs=2)
    shares = {"decode_cluster_sort": 0.5, "search_by_triplet": 0.4, "consolidate_fit": 0.1}
    serial = {"decode_cluster_sort": 3.0, "search_by_triplet": 2.5}
    roof, _ = bench.roofline(stages, census, 1, 1, 1000.0, "measured", None, shares, serial)
    # the serial shares pick decode even though the search's timed-region brackets are longer
    assert roof["kernel"] == "decode_cluster_sort"
    assert roof["avg_launch_ms"] == pytest.approx(4.0)
    assert roof["achieved"] == pytest.approx(per["decode_cluster_sort"] / 4e-3 / 1e9)
    assert roof["frac"] == pytest.approx(roof["achieved"] / 1000.0)
    assert roof["serial_single_stream"]["avg_launch_ms"] == 3.0
    assert roof["serial_single_stream"]["achieved"] == pytest.approx(per["decode_cluster_sort"] / 3e-3 / 1e9)


def test_every_candidate_opens_only_the_gates():
    from cuda_hlt_b200 import mlp, train_scorer
    w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
    wa = bench.every_candidate(w)
    a, b = mlp.weights_to_dict(w), mlp.weights_to_dict(wa)
    assert b["min_pairs"] == 0 and b["min_event_clusters"] == 0
    assert a["min_pairs"] > 0 and a["min_event_clusters"] > 0  # the committed gates are untouched
    for k in ("mean", "inv_std", "w1", "w2", "w3"):
        assert (a[k] == b[k]).all()
    for k in ("seed_threshold", "ext_threshold", "max_event_clusters"):
        assert a[k] == b[k]


def test_operating_points_table():
    serial = {"decode_cluster_sort": 1.0}
    forms = {"plain": {"value": 100.0, "ms_per_step": 10.0, "stages_ms_per_batch_serial": serial},
             "pruned": {"value": 99.0, "ms_per_step": 10.1, "stages_ms_per_batch_serial": serial},
             "pruned_every_candidate": {"value": 86.0, "ms_per_step": 11.6, "stages_ms_per_batch_serial": serial}}
    quality = {"plain": {"long_efficiency": 0.9868, "ghost_rate": 0.0648},
               "pruned": {"long_efficiency": 0.9867, "ghost_rate": 0.0576},
               "pruned_every_candidate": {"long_efficiency": 0.9861, "ghost_rate": 0.0142}}
    op = bench.operating_points(forms, quality)
    assert op["committed_gates"]["vs_plain"] == pytest.approx(0.99)
    assert op["every_candidate"]["vs_plain"] == pytest.approx(0.86)
    assert op["every_candidate"]["long_efficiency_loss"] == pytest.approx(0.0007)
    assert op["every_candidate"]["ghost_rate"] == 0.0142 and op["every_candidate"]["plain_ghost_rate"] == 0.0648
    # without the every-candidate form (--no-operating-points) and without a quality leg
    del forms["pruned_every_candidate"]
    op = bench.operating_points(forms, None)
    assert list(op) == ["committed_gates"] and "ghost_rate" not in op["committed_gates"]

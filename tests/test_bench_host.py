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

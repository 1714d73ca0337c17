"""Parity of the CUDA chain (through the C ABI) with the reference.

Bit-exact bar (integer work and the float values the reference computes):
  * clusters: count per module, LHCb ids and per-module order, x/y/z/phi bit for bit;
    within a module the reference's order for exactly equal phi follows its atomics, so
    only permutations of equal-phi entries are tolerated;
  * tracks: per-event hit-id lists identical after a canonical sort;
  * beamline (LSQ) and Kalman states: all 12 floats bit for bit (the required bound is
    1e-5 relative), `backward` of the beamline state equal.
Events the reference leaves undefined (buffer spills, reads outside a module, exact
scatter ties resolved by atomics) are flagged by both sides and excluded.
"""
import os

import numpy as np
import pytest

import oracle
import parity_utils as pu
from conftest import golden_batch, golden_event_clusters, golden_event_tracks, load_golden
from cuda_hlt_b200 import chain, events

pytestmark = pytest.mark.gpu


def run_chain(b, **kw):
    vc = chain.VeloChain(max_events=max(1, b.n_events), max_raw_bytes=int(b.raw.size) + 4096, **kw)
    vc.run_host(b)
    vc.sync()
    res = vc.results()
    vc.close()
    return res


def assert_clusters_equal(mine_mods, ref_mods, ctx):
    for m, (a, r) in enumerate(zip(mine_mods, ref_mods)):
        assert len(a["id"]) == len(r["id"]), (ctx, m)
        same_phi = np.array_equal(pu.bits(a["phi"]), pu.bits(r["phi"]))
        assert same_phi, (ctx, m, "phi")
        if np.array_equal(a["id"], r["id"]):
            for k in ("x", "y", "z"):
                assert np.array_equal(pu.bits(a[k]), pu.bits(r[k])), (ctx, m, k)
        else:
            # only permutations inside runs of equal phi
            phis = pu.bits(a["phi"])
            for v in np.unique(phis):
                sel = phis == v
                key_a = sorted(zip(a["id"][sel], pu.bits(a["x"][sel]), pu.bits(a["y"][sel]), pu.bits(a["z"][sel])))
                key_r = sorted(zip(r["id"][sel], pu.bits(r["x"][sel]), pu.bits(r["y"][sel]), pu.bits(r["z"][sel])))
                assert key_a == key_r, (ctx, m)


def assert_states_equal(mine, e, mt, g_states, g_tracks, t0g, ctx):
    gi = pu.track_index(g_tracks)
    t0m = int(mine["track_offsets"][e])
    for i, t in enumerate(mt):
        j = gi[t]
        for which in ("states", "kalman"):
            for key in pu.STATE_KEYS:
                got = np.float32(mine[which][key][t0m + i])
                ref = np.float32(g_states[f"{which}_{key}"][t0g + j])
                assert got.view(np.uint32) == ref.view(np.uint32), (ctx, which, key, got, ref)
        assert bool(mine["states"]["backward"][t0m + i]) == bool(g_states["states_backward"][t0g + j])


@pytest.mark.parametrize("which", ["minbias", "plain", "batched", "pruned1m"])
def test_bit_exact_against_reference_golden(which):
    g = load_golden(which)
    b = golden_batch(which)
    res = run_chain(b)
    N = b.n_events
    compared = 0
    for e in range(N):
        if res["status"][e] & chain.REFERENCE_UNDEFINED:
            continue
        assert_clusters_equal(chain.event_clusters(res, e), golden_event_clusters(g, e), (which, e))
        mt, gt = chain.event_tracks(res, e), golden_event_tracks(g, e)
        assert pu.canonical_tracks(mt) == pu.canonical_tracks(gt), (which, e)
        assert_states_equal(res, e, mt, g, gt, int(g["atomics"][N + e]), (which, e))
        compared += 1
    assert compared >= N - 2


@pytest.mark.skipif(not os.path.exists(oracle.REF_GPU_LIB), reason="reference GPU build missing")
@pytest.mark.parametrize("config,n", [("plain_1k", 300), ("batched_500k", 300), ("high_occupancy_200k", 300),
                                      ("pruned_1m", 400)])
def test_bit_exact_against_reference_kernels_live(geometry, config, n):
    """The reference's own kernels run on the same events in the same process. On the
    nu ~ U(2,20) workload the chain also runs in the pruned mode with the committed scorer:
    its events above the trained occupancy (VELO_STATUS_MLP_FALLBACK) run the plain search
    and must equal the reference too."""
    b = events.generate_config(config, n_events=n, first_event=1000)
    # Events whose reference run spills past its per-event buffers would also corrupt the
    # following events of the reference's batch: they are left out of the batch.
    orc = oracle.run(b, geometry)
    undefined = [e for e in range(n) if orc.flags[e] & oracle.UNDEFINED_IN_REFERENCE]
    big_module = [e for e in range(n) if e not in undefined and orc.module_num[e * 52:(e + 1) * 52].max() >= 500]
    keep = [e for e in range(n) if e not in undefined and e not in big_module]
    why = (f"{config}: {n} events, {len(undefined)} left out as undefined in the reference (buffer spills, "
           f"reads outside a module, exact ties), {len(big_module)} with a module of >= 500 clusters")
    sub = events.EventBatch(np.concatenate([b.event(e) for e in keep]),
                            np.concatenate([[0], np.cumsum([b.event(e).size for e in keep])]).astype(np.uint64))
    ref, _ = oracle.ref_gpu_run(sub, geometry)
    res = run_chain(sub)
    N = sub.n_events
    rs = {k: oracle.ref_decode_states(ref, k) for k in ("states", "kalman")}
    flat = {f"{w}_{k}": v for w in rs for k, v in rs[w].items()}
    compared = flagged = 0
    for e in range(N):
        if res["status"][e] & chain.REFERENCE_UNDEFINED:
            flagged += 1
            continue
        assert_clusters_equal(chain.event_clusters(res, e), oracle.ref_event_clusters(ref, e), (config, e))
        mt, rt = chain.event_tracks(res, e), chain.event_tracks(ref, e)
        assert pu.canonical_tracks(mt) == pu.canonical_tracks(rt), (config, e)
        assert_states_equal(res, e, mt, flat, rt, int(ref["track_offsets"][e]), (config, e))
        compared += 1
    why += f"; of the {N} run, {flagged} flagged by the chain, {compared} compared bit for bit"
    print(why)
    assert len(keep) >= 0.8 * n, why
    assert compared >= 0.95 * N, why
    if config != "pruned_1m":
        return
    # nu > 15 events are in the sample: the largest ones exceed the trained occupancy
    from cuda_hlt_b200 import mlp, train_scorer
    hits = np.array([int(orc.module_num[e * 52:(e + 1) * 52].sum()) for e in keep])
    w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
    assert (hits > w.max_event_clusters).sum() >= 3, hits.max()
    vc = chain.VeloChain(max_events=N, max_raw_bytes=int(sub.raw.size) + 4096)
    vc.set_mlp(w)
    vc.set_mode(chain.MODE_PRUNED)
    vc.run_host(sub)
    vc.sync()
    pr = vc.results()
    vc.close()
    fallback = 0
    for e in range(N):
        fb = bool(pr["status"][e] & chain.STATUS["mlp_fallback"])
        assert fb == (hits[e] > w.max_event_clusters), e
        if not fb or pr["status"][e] & chain.REFERENCE_UNDEFINED:
            continue
        mt, rt = chain.event_tracks(pr, e), chain.event_tracks(ref, e)
        assert pu.canonical_tracks(mt) == pu.canonical_tracks(rt), ("pruned fallback", e)
        assert_states_equal(pr, e, mt, flat, rt, int(ref["track_offsets"][e]), ("pruned fallback", e))
        fallback += 1
    print(f"pruned mode: {fallback} fallback events equal to the reference")
    assert fallback >= 3


def test_against_cpu_oracle(geometry):
    b = events.generate_config("plain_1k", n_events=200, first_event=500)
    res = run_chain(b)
    r = oracle.run(b, geometry)
    diff = total = 0
    for e in range(b.n_events):
        oc = r.event_clusters(e)
        got = np.concatenate([m["id"] for m in chain.event_clusters(res, e)])
        assert np.array_equal(np.sort(got), np.sort(oc["id"])), e
        a, bb = pu.compare_event_tracks(chain.event_tracks(res, e), r.event_tracks(e))
        diff += a + bb
        total += len(r.event_tracks(e))
    assert diff <= 0.005 * total, (diff, total)


def test_deterministic_and_graph_equal():
    b = events.generate_config("batched_500k", n_events=257, first_event=77)
    r1 = run_chain(b)
    r2 = run_chain(b)
    r3 = run_chain(b, use_graphs=True)
    for k in ("atomics", "track_hit_number", "hit_id", "hit_x", "status", "module_num", "cluster_id", "cluster_phi"):
        assert np.array_equal(r1[k], r2[k]), k
        assert np.array_equal(r1[k], r3[k]), k
    for k in pu.STATE_KEYS:
        assert np.array_equal(pu.bits(r1["kalman"][k]), pu.bits(r3["kalman"][k])), k


def test_host_and_device_input_paths_agree():
    import torch
    b = events.generate_config("plain_1k", n_events=50)
    ref = run_chain(b)
    raw = torch.from_numpy(b.raw).cuda()
    off = torch.from_numpy(b.offsets.view(np.int64)).cuda()
    vc = chain.VeloChain(max_events=50, max_raw_bytes=int(b.raw.size))
    vc.run_device(raw.data_ptr(), off.data_ptr(), 50, torch.cuda.current_stream().cuda_stream)
    vc.sync()
    res = vc.results()
    vc.close()
    for k in ("atomics", "track_hit_number", "hit_id", "module_num"):
        assert np.array_equal(ref[k], res[k]), k


@pytest.mark.parametrize("shift", [4, 8, 12])
def test_batch_at_unaligned_address(shift):
    """A batch may start anywhere (4-byte aligned) inside the caller's buffer."""
    import torch
    b = events.generate_config("plain_1k", n_events=40, first_event=7)
    ref = run_chain(b)
    buf = torch.zeros(b.raw.size + 64, dtype=torch.uint8, device="cuda")
    buf[shift:shift + b.raw.size] = torch.from_numpy(b.raw).cuda()
    off = torch.from_numpy(b.offsets.view(np.int64)).cuda()
    vc = chain.VeloChain(max_events=40, max_raw_bytes=int(b.raw.size) + 64, use_graphs=True)
    vc.run_device(buf.data_ptr() + shift, off.data_ptr(), 40, torch.cuda.current_stream().cuda_stream)
    vc.sync()
    res = vc.results()
    vc.close()
    for k in ("atomics", "track_hit_number", "hit_id", "module_num", "cluster_id", "status"):
        assert np.array_equal(ref[k], res[k]), k


def _empty_event():
    nb = 208
    payload, offs = [], [0]
    for k in range(nb):
        payload += [k, 0]
        offs.append(4 * len(payload))
    return np.array([nb] + offs + payload, np.uint32).view(np.uint8)


def test_edge_cases_empty_corrupt_and_ragged(geometry):
    good = events.generate_config("plain_1k", n_events=5)
    empty = _empty_event()
    corrupt = good.event(2).copy().view(np.uint32)
    corrupt[3] = 0xFFFFFF00  # bank offset far outside the event
    truncated = good.event(3)[:500]
    parts = [good.event(0), empty, corrupt.view(np.uint8), good.event(1), truncated, good.event(4)]
    raw = np.concatenate(parts)
    offs = np.concatenate([[0], np.cumsum([p.size for p in parts])]).astype(np.uint64)
    res = run_chain(events.EventBatch(raw, offs))
    st = res["status"]
    assert st[0] == 0 and st[1] == 0 and st[3] == 0 and st[5] == 0
    assert st[2] & chain.STATUS["bad_raw"] and st[4] & chain.STATUS["bad_raw"]
    assert res["n_tracks"][1] == res["n_tracks"][2] == res["n_tracks"][4] == 0
    clean = run_chain(good)
    for mine_e, clean_e in ((0, 0), (3, 1), (5, 4)):
        assert pu.canonical_tracks(chain.event_tracks(res, mine_e)) == \
            pu.canonical_tracks(chain.event_tracks(clean, clean_e))
    # an empty batch
    vc = chain.VeloChain(max_events=4, max_raw_bytes=1 << 16)
    vc.run_host(events.EventBatch(np.zeros(0, np.uint8), np.zeros(1, np.uint64)))
    t, h, c = vc.sync()
    assert (t, h, c) == (0, 0, 0)
    vc.close()


def test_capacity_errors():
    b = events.generate_config("plain_1k", n_events=8)
    vc = chain.VeloChain(max_events=4, max_raw_bytes=int(b.raw.size))
    with pytest.raises(chain.VeloError):
        vc.run_host(b)
    vc.close()


def test_full_size_batch_properties():
    """16,384 events of the nu ~ U(2,15) workload: consistent offsets and layouts."""
    b = events.generate_config("batched_500k", n_events=16384, first_event=100000, with_mc=False)
    res = run_chain(b)
    N = b.n_events
    at = res["atomics"]
    assert np.array_equal(np.cumsum(np.concatenate([[0], at[:N]])), at[N:2 * N + 1])
    thn = res["track_hit_number"]
    n_hits = np.diff(thn)
    assert np.all(n_hits >= 3) and np.all(n_hits <= 26)
    # consolidated hit ids are clusters of the event and hits of a track are in distinct modules
    for e in range(0, N, 997):
        ids = set(np.concatenate([m["id"] for m in chain.event_clusters(res, e)]).tolist())
        for t in chain.event_tracks(res, e):
            assert set(t) <= ids
            mods = [(i >> 20) & 0x3F for i in t]  # sensor >> 2
            assert len(set(mods)) == len(mods)
    for k in pu.STATE_KEYS:
        assert np.all(np.isfinite(res["states"][k]))
    assert (res["status"] & chain.STATUS["bad_raw"]).sum() == 0


@pytest.mark.parametrize("mapping", [chain.MAP_WARP, chain.MAP_BLOCK])
def test_search_mappings_bit_exact(mapping):
    """Warp-per-event and block-per-event searches give the reference's result each."""
    g = load_golden("batched")
    b = golden_batch("batched")
    res = run_chain(b, mapping=mapping)
    N = b.n_events
    for e in range(N):
        if res["status"][e] & chain.REFERENCE_UNDEFINED:
            continue
        mt, gt = chain.event_tracks(res, e), golden_event_tracks(g, e)
        assert pu.canonical_tracks(mt) == pu.canonical_tracks(gt), (mapping, e)
        assert_states_equal(res, e, mt, g, gt, int(g["atomics"][N + e]), (mapping, e))


@pytest.mark.parametrize("which", ["minbias", "batched"])
def test_decode_block_sizes_bit_exact(which):
    """Both decode block sizes the autotuner chooses between (4 and 8 warps per event) give the
    reference's clusters and tracks."""
    g = load_golden(which)
    b = golden_batch(which)
    res = run_chain(b, decode_warps=4)
    N = b.n_events
    for e in range(N):
        if res["status"][e] & chain.REFERENCE_UNDEFINED:
            continue
        assert_clusters_equal(chain.event_clusters(res, e), golden_event_clusters(g, e), (which, e))
        mt, gt = chain.event_tracks(res, e), golden_event_tracks(g, e)
        assert pu.canonical_tracks(mt) == pu.canonical_tracks(gt), (which, e)
    with pytest.raises(RuntimeError):
        run_chain(b, decode_warps=6)


def test_mappings_identical_on_uneven_batch():
    b = events.generate_config("batched_500k", n_events=400, first_event=3000)
    outs = [run_chain(b, mapping=m) for m in (chain.MAP_WARP, chain.MAP_BLOCK, chain.MAP_AUTO)]
    for r in outs[1:]:
        for e in range(b.n_events):
            assert pu.canonical_tracks(chain.event_tracks(outs[0], e)) == pu.canonical_tracks(chain.event_tracks(r, e))


def test_bounded_wait_timeout_reported():
    """A bounded device wait that runs out (a barrier nothing completes, waited for with the
    scorer's wait function) is reported by velo_sync as VELO_ERR_DEVICE_TIMEOUT; the context
    stays usable and the next run clears the error."""
    b = events.generate_config("plain_1k", n_events=8)
    vc = chain.VeloChain(max_events=8, max_raw_bytes=int(b.raw.size) + 4096)
    assert vc.lib.velo_check_wait_timeout(vc.ctx, 0, None) == -1
    assert vc.lib.velo_check_wait_timeout(vc.ctx, 4096, None) == 0
    with pytest.raises(chain.VeloError, match="code -9"):
        vc.sync()
    vc.run_host(b)
    t, _, c = vc.sync()
    assert t > 0 and c > 0
    vc.close()


def _same_results(a, b, n_events, what):
    """Equal outputs of two runs: dense outputs whole, clusters event by event (the cluster
    buffers have unused gaps between events whose contents are not outputs)."""
    for k in ("atomics", "track_hit_number", "hit_id", "hit_x", "status", "module_num"):
        assert np.array_equal(a[k], b[k]), (what, k)
    for e in range(n_events):
        for ma, mb in zip(chain.event_clusters(a, e), chain.event_clusters(b, e)):
            assert np.array_equal(ma["id"], mb["id"]) and np.array_equal(ma["phi"], mb["phi"]), (what, e)


def test_u32_offsets_equal_u64():
    """velo_run_host_u32 / velo_run_u32 take the reference's u32 offsets directly; results
    equal the u64 entry points', also for a batch that starts inside the caller's buffer."""
    import torch
    b = events.generate_config("batched_500k", n_events=120, first_event=55)
    ref = run_chain(b)
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
    vc.run_host_u32(b.raw, b.offsets.astype(np.uint32))
    vc.sync()
    _same_results(ref, vc.results(), b.n_events, "host u32")
    # events 20..119 of the same buffer: offsets rebased from a nonzero start
    sub = b.subset(20, 120)
    ref_sub = run_chain(sub)
    vc.run_host_u32(b.raw, b.offsets[20:].astype(np.uint32))
    vc.sync()
    _same_results(ref_sub, vc.results(), sub.n_events, "host u32, rebased")
    # device-resident input with u32 offsets
    raw = torch.from_numpy(b.raw).cuda()
    off = torch.from_numpy(b.offsets.astype(np.uint32).view(np.int32)).cuda()
    vc.run_device_u32(raw.data_ptr(), off.data_ptr(), b.n_events, torch.cuda.current_stream().cuda_stream)
    vc.sync()
    _same_results(ref, vc.results(), b.n_events, "device u32")
    vc.close()


def test_host_offsets_staging():
    """velo_run_host stages the caller's offsets through pinned memory of the context,
    rebased to the batch's first byte: a batch that starts inside the caller's buffer equals
    the same events run alone, also when it follows another host run on the same stream
    without a wait in between (the staging is reused only once the previous copy is done),
    and the totals velo_sync reports are the last run's."""
    b = events.generate_config("batched_500k", n_events=120, first_event=700)
    sub = b.subset(20, 120)
    ref_sub = run_chain(sub)
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
    rebased = events.EventBatch(b.raw, np.ascontiguousarray(b.offsets[20:]))
    vc.run_host(rebased)
    t, h, _ = vc.sync(clusters=False)
    _same_results(ref_sub, vc.results(), sub.n_events, "host u64, rebased")
    assert t == int(ref_sub["atomics"][2 * sub.n_events]) and h == len(ref_sub["hit_id"])
    for _ in range(2):
        vc.run_host(b)
        vc.run_host(rebased)
    t, h, _ = vc.sync(clusters=False)
    _same_results(ref_sub, vc.results(), sub.n_events, "host u64, rebased, after another run")
    assert t == int(ref_sub["atomics"][2 * sub.n_events]) and h == len(ref_sub["hit_id"])
    vc.close()


def test_context_memory_released():
    """velo_destroy returns what velo_create and the runs took (device buffers, the pruned
    mode's buffers allocated on first use, CUDA graphs per batch-size bucket): free device
    memory after five create / run / destroy cycles equals free memory before them, to within
    what the CUDA runtime itself keeps."""
    import torch
    from cuda_hlt_b200 import mlp, train_scorer
    w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
    b = events.generate_config("pruned_1m", n_events=1500, first_event=40_000)
    torch.cuda.synchronize()

    def cycle():
        vc = chain.VeloChain(max_events=4096, max_raw_bytes=int(b.raw.size) + 4096, use_graphs=True)
        vc.set_mlp(w)
        for mode in (chain.MODE_PLAIN, chain.MODE_PRUNED):
            vc.set_mode(mode)
            vc.run_host(b)
            vc.run_host(b.subset(0, 1000))
            vc.sync()
        assert vc.graph_count() >= 1
        vc.close()

    cycle()  # first use: the runtime's own lazy allocations happen here
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        cycle()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < 64 << 20, (free0, free1)


def test_contexts_on_threads():
    """Separate contexts run concurrently: two host threads, each with its own context and
    stream (as Allen runs one Stream per thread), repeat their own batch (one in the plain
    mode, one pruned) while the other runs; every result equals the same batch run alone."""
    import threading

    import torch
    from cuda_hlt_b200 import mlp, train_scorer
    w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
    jobs = [(events.generate_config("batched_500k", n_events=200, first_event=900), chain.MODE_PLAIN),
            (events.generate_config("pruned_1m", n_events=200, first_event=30_000), chain.MODE_PRUNED)]
    alone = []
    for b, mode in jobs:
        vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
        vc.set_mlp(w)
        vc.set_mode(mode)
        vc.run_host(b)
        vc.sync()
        alone.append(vc.results())
        vc.close()
    got = [[] for _ in jobs]
    errors = []

    def worker(i):
        try:
            b, mode = jobs[i]
            stream = torch.cuda.Stream()
            vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096, use_graphs=True)
            vc.set_mlp(w)
            vc.set_mode(mode)
            for _ in range(4):
                vc.run_host(b, stream.cuda_stream)
                vc.sync()
                got[i].append(vc.results())
            vc.close()
        except Exception as ex:  # reported by the main thread
            errors.append((i, ex))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i, (b, _) in enumerate(jobs):
        assert len(got[i]) == 4
        for k, res in enumerate(got[i]):
            _same_results(alone[i], res, b.n_events, f"thread {i}, run {k}")


def test_selected_events_u32():
    """velo_run_selected_u32 decodes the caller's selection (Allen's dev_event_list after
    global_event_cut_t): position i holds raw event list[i], equal to a run over those events
    alone; a list entry beyond the batch leaves its position empty and flagged."""
    import torch
    b = events.generate_config("batched_500k", n_events=64, first_event=300)
    sel = np.array([3, 7, 8, 20, 41, 63, 0], np.uint32)
    alone = events.EventBatch(np.concatenate([b.event(int(i)) for i in sel]),
                              np.concatenate([[0], np.cumsum([b.event(int(i)).size for i in sel])]).astype(np.uint64))
    ref = run_chain(alone)
    raw = torch.from_numpy(b.raw).cuda()
    off = torch.from_numpy(b.offsets.astype(np.uint32).view(np.int32)).cuda()
    lst = torch.from_numpy(np.append(sel, 64).astype(np.uint32).view(np.int32)).cuda()
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
    vc.n_events = len(sel) + 1
    rc = vc.lib.velo_run_selected_u32(vc.ctx, chain.C.c_void_p(raw.data_ptr()), chain.C.c_void_p(off.data_ptr()),
                                      b.n_events, chain.C.c_void_p(lst.data_ptr()), len(sel) + 1,
                                      chain.C.c_void_p(torch.cuda.current_stream().cuda_stream), chain.C.byref(vc.out))
    assert rc == 0
    vc.sync()
    got = vc.results()
    vc.close()
    n = len(sel)
    assert got["status"][n] & chain.STATUS["bad_raw"] and got["n_tracks"][n] == 0
    assert np.array_equal(got["status"][:n], ref["status"])
    for e in range(n):
        assert pu.canonical_tracks(chain.event_tracks(got, e)) == pu.canonical_tracks(chain.event_tracks(ref, e)), e
        ids_a = np.concatenate([m["id"] for m in chain.event_clusters(got, e)])
        ids_b = np.concatenate([m["id"] for m in chain.event_clusters(ref, e)])
        assert np.array_equal(ids_a, ids_b), e


def test_graph_per_bucket_serves_any_batch():
    """With graphs, one graph per batch-size bucket (1,024 x 4^k events) serves batches of any
    size in the bucket and in any buffers (the kernels read each run's inputs from a
    device-side parameter block): results equal graph-free runs, the graph count is the
    number of buckets used, every launch's stage times are recorded, and at most 16 graphs are
    kept (least recently launched evicted)."""
    import torch
    sizes = (300, 1000, 1024, 1500, 700)
    batches = [events.generate_config("batched_500k", n_events=n, first_event=1000 * i) for i, n in enumerate(sizes)]
    refs = [run_chain(b) for b in batches]
    cap = max(int(b.raw.size) for b in batches) + 4096
    vc = chain.VeloChain(max_events=4096, max_raw_bytes=cap, use_graphs=True)
    vc.set_timing(True)
    s = torch.cuda.current_stream().cuda_stream
    keep = []
    for rep in range(2):
        for b, ref in zip(batches, refs):
            raw = torch.from_numpy(b.raw).cuda()  # a new buffer for every run
            off = torch.from_numpy(b.offsets.view(np.int64)).cuda()
            keep.append((raw, off))
            vc.run_device(raw.data_ptr(), off.data_ptr(), b.n_events, s)
            vc.sync()
            _same_results(ref, vc.results(), b.n_events, (rep, b.n_events))
    assert vc.graph_count() == 2  # buckets of 1,024 and 4,096 events
    st = vc.stage_times()
    assert st["runs"] == 2 * len(sizes) and st["search_by_triplet"] > 0
    # one graph per stream: at most 16 kept
    b = batches[0]
    raw = torch.from_numpy(b.raw).cuda()
    off = torch.from_numpy(b.offsets.view(np.int64)).cuda()
    streams = [torch.cuda.Stream() for _ in range(20)]
    for st_ in streams:
        vc.run_device(raw.data_ptr(), off.data_ptr(), b.n_events, st_.cuda_stream)
        st_.synchronize()
    assert vc.graph_count() == 16
    vc.sync()
    _same_results(refs[0], vc.results(), batches[0].n_events, "after eviction")
    vc.close()


def test_events_beyond_the_search_capacity():
    """Events above the search's 16,384 clusters (pileup nu = 60: 17,300-18,300 clusters) are
    flagged VELO_STATUS_HIT_OVERFLOW and keep no tracks; the events around them in the batch
    are reconstructed as in a batch of their own."""
    big = events.generate(seed=31, nu_min=60.0, nu_max=60.0, n_events=3, with_mc=False)
    small = events.generate_config("batched_500k", n_events=4, first_event=600, with_mc=False)
    parts = [small.event(0), big.event(0), small.event(1), big.event(1), small.event(2), big.event(2), small.event(3)]
    raw = np.concatenate(parts)
    offs = np.concatenate([[0], np.cumsum([p.size for p in parts])]).astype(np.uint64)
    res = run_chain(events.EventBatch(raw, offs))
    alone = run_chain(small)
    n_hits = res["module_num"].reshape(-1, 52).sum(axis=1)
    for pos in (1, 3, 5):
        st = int(res["status"][pos])
        assert n_hits[pos] > 16384, (pos, n_hits[pos])
        assert st & chain.STATUS["hit_overflow"] and res["n_tracks"][pos] == 0, (pos, st)
    for pos, e in ((0, 0), (2, 1), (4, 2), (6, 3)):
        assert pu.canonical_tracks(chain.event_tracks(res, pos)) == pu.canonical_tracks(chain.event_tracks(alone, e))
        assert res["status"][pos] == alone["status"][e]

"""The learned seed/extension scorer on the GPU, against its CPU oracle (oracle/mlp_oracle.py)
and against the plain search it prunes.

* inference and training gradients of the tensor-core kernels equal the oracle's bf16
  restatement up to the order of fp32 sums (bound: 1e-2 of the logit / gradient scale);
  the deviation of the bf16 gradient from exact float64 maths is stated and bounded;
* collected samples: features equal the oracle's restatement computed from the chain's own
  clusters, labels equal the plain search's tracks;
* the pruned mode with nothing pruned (every event past the occupancy limit, a scorer
  that keeps everything, or a scoring gate no candidate reaches) reproduces the plain chain
  exactly, and seeds below the gate are kept unscored;
* a trained scorer keeps long-track efficiency within 0.2% absolute of the plain search,
  does not raise the ghost rate, and makes the search explore fewer seeds and run faster.
"""
import numpy as np
import pytest

from cuda_hlt_b200 import chain, events, mlp
from oracle import mlp_oracle

pytestmark = pytest.mark.gpu


def random_weights(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    return dict(mean=rng.normal(0, 1, 12).astype(np.float32), inv_std=rng.uniform(0.5, 2, 12).astype(np.float32),
                w1=(rng.normal(0, 0.4, (64, 13)) * scale).astype(np.float32),
                w2=(rng.normal(0, 0.15, (64, 65)) * scale).astype(np.float32),
                w3=(rng.normal(0, 0.2, (2, 65)) * scale).astype(np.float32), seed_threshold=0.5, ext_threshold=0.0,
                max_event_clusters=0xFFFFFFFF)


def random_samples(seed, n):
    rng = np.random.default_rng(seed)
    f = rng.normal(0, 1.5, (n, 12)).astype(np.float32)
    lab = rng.integers(0, 4, n).astype(np.uint8)
    return f, lab


def test_inference_matches_oracle():
    d = random_weights(1)
    t = mlp.MlpTrainer(1024, seed=1)
    t.set_weights(mlp.dict_to_weights(d))
    f, _ = random_samples(2, 1000)  # not a multiple of the 128-row tile
    z = t.infer(f)
    zo, _ = mlp_oracle.forward_bf16(f, d)
    scale = 1.0 + np.abs(zo).max()
    assert np.abs(z - zo).max() < 1e-2 * scale
    # most rows agree to fp32 summation-order noise
    assert np.quantile(np.abs(z - zo), 0.9) < 1e-3 * scale
    t.close()


def test_gradient_matches_oracle():
    d = random_weights(3)
    t = mlp.MlpTrainer(1024, seed=3)
    t.set_weights(mlp.dict_to_weights(d))
    f, lab = random_samples(4, 700)
    g, loss = t.gradient(f, lab)
    lo, go = mlp_oracle.loss_and_gradient_bf16(f, lab, d)
    g64 = mlp_oracle.gradient_f64(f, lab, d)
    assert abs(loss - lo) < 1e-3 * max(1.0, abs(lo))
    for k in ("w1", "w2", "w3"):
        ref = np.linalg.norm(go[k])
        assert np.linalg.norm(g[k] - go[k]) < 1e-2 * ref, k
        # bf16 operands against exact maths: a few per cent of the gradient norm
        assert np.linalg.norm(g[k] - g64[k]) < 0.1 * np.linalg.norm(g64[k]), k
    t.close()


@pytest.fixture(scope="module")
def small_run():
    b = events.generate(seed=1, nu_min=2.0, nu_max=15.0, n_events=48, with_mc=False)
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
    vc.run_host(b)
    vc.sync()
    res = vc.results()
    t = mlp.MlpTrainer(1 << 20, seed=5)
    n = t.collect(vc)
    f, lab = t.samples(0, n)
    vc.close()
    t.close()
    return b, res, f, lab


def test_collected_samples_match_oracle(small_run):
    b, res, f, lab = small_run
    o = 0
    for e in range(16):
        mods = chain.event_clusters(res, e)
        cat = {k: np.concatenate([m[k] for m in mods]) for k in ("x", "y", "z", "phi", "id", "size")}
        idx, wins, fo = mlp_oracle.event_features(cat["x"], cat["y"], cat["z"], cat["phi"], cat["size"],
                                                  [len(m["id"]) for m in mods])
        n = len(idx)
        got = f[o:o + n]
        assert got.shape == fo.shape, e
        # module, window sizes and the size of h1 exactly; the proxy-pair features to
        # fast-math division / log accuracy (a near-tie between two pairs may pick the
        # other pair under different rounding: a few rows in a thousand at most)
        for k in (5, 6, 7, 9):
            assert np.array_equal(got[:, k], fo[:, k]), (e, k)
        rows_ok = np.all(np.isclose(got, fo, rtol=1e-4, atol=1e-5), axis=1)
        assert rows_ok.mean() > 0.995, e
        # labels from the event's tracks: on a track / fourth or later hit
        ids_on = {}
        for trk in chain.event_tracks(res, e):
            for k, hid in enumerate(trk):
                ids_on[hid] = 3 if k >= 3 else 1
        exp = np.array([ids_on.get(int(cat["id"][h]), 0) for h in idx], np.uint8)
        assert np.array_equal(lab[o:o + n], exp), e
        o += n


def test_training_reduces_loss(small_run):
    _, _, f, lab = small_run
    t = mlp.MlpTrainer(200_000, seed=7)
    # train on the kernels, through the library's own collection path
    b = events.generate(seed=1, nu_min=2.0, nu_max=15.0, n_events=256, first_event=1000, with_mc=False)
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
    vc.run_host(b)
    vc.sync()
    n = t.collect(vc)
    vc.close()
    t.normalize()
    w0 = mlp.weights_to_dict(t.weights())
    tf, tl = t.samples(0, min(n, 20000))
    l0, _ = mlp_oracle.loss_and_gradient_bf16(tf, tl, w0)
    last = t.train(epochs=3, batch=4096, lr=3e-3)
    w1 = mlp.weights_to_dict(t.weights())
    l1, _ = mlp_oracle.loss_and_gradient_bf16(tf, tl, w1)
    assert last < 0.8 * l0 and l1 < 0.8 * l0
    # held-out samples (the small_run batch): output 0 separates on-track candidates
    z, _ = mlp_oracle.forward_bf16(f, w1)
    pos, neg = z[(lab & 1) == 1, 0], z[(lab & 1) == 0, 0]
    auc = (pos[:, None] > neg[None, :2000]).mean()
    assert auc > 0.9
    t.close()


def keep_all_weights():
    d = random_weights(9, scale=0.0)
    d["w3"][:, 64] = 30.0  # logits +30 for every candidate
    d["seed_threshold"] = 0.5
    return d


def run_mode(b, mode, weights=None, timing=False):
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096, mode=chain.MODE_PLAIN)
    if weights is not None:
        vc.set_mlp(weights)
    vc.set_mode(mode)
    st = None
    if timing:
        vc.set_timing(True)
        for _ in range(3):
            vc.run_host(b)
        vc.sync()
        st = vc.stage_times()
    vc.run_host(b)
    vc.sync()
    res = vc.results()
    vc.close()
    return (res, st) if timing else res


def canonical(res, n):
    return [sorted(tuple(sorted(t)) for t in chain.event_tracks(res, e)) for e in range(n)]


def test_pruned_without_pruning_is_plain():
    b = events.generate(seed=11, nu_min=2.0, nu_max=15.0, n_events=64, with_mc=False)
    plain = run_mode(b, chain.MODE_PLAIN)
    ref = canonical(plain, b.n_events)
    # a scorer that keeps every candidate
    kept = run_mode(b, chain.MODE_PRUNED, mlp.dict_to_weights(keep_all_weights()))
    assert canonical(kept, b.n_events) == ref
    assert np.all((kept["status"] & chain.STATUS["mlp_fallback"]) == 0)
    # every event above the occupancy limit: per-event fallback to the plain search
    d = random_weights(10)
    d["max_event_clusters"] = 0
    fb = run_mode(b, chain.MODE_PRUNED, mlp.dict_to_weights(d))
    assert canonical(fb, b.n_events) == ref
    assert np.all((fb["status"] & chain.STATUS["mlp_fallback"]) != 0)
    for k in ("x", "y", "tx", "ty"):
        assert np.array_equal(fb["states"][k], plain["states"][k])


def test_score_kernel_verdicts_match_oracle():
    """The verdicts of score_candidates (bit 0 of the keep bits of every scored seed: kept or
    pruned) equal the oracle's forward pass on the oracle's features of the same clusters,
    wherever the logit clears the threshold by more than fp32 summation-order noise. Every
    event and every candidate is scored (no gates), over many 256-row tile pairs, the last
    of them partial; the threshold sits at the median logit, so half the seeds go."""
    b = events.generate(seed=14, nu_min=2.0, nu_max=15.0, n_events=48, with_mc=False)
    d = random_weights(15)
    d["min_pairs"] = 0
    d["min_event_clusters"] = 0
    plain = run_mode(b, chain.MODE_PLAIN)  # the clusters are the same in both modes
    per_event = []
    for e in range(b.n_events):
        mods = chain.event_clusters(plain, e)
        cat = {k: np.concatenate([m[k] for m in mods]) for k in ("x", "y", "z", "phi", "size")}
        idx, _, fo = mlp_oracle.event_features(cat["x"], cat["y"], cat["z"], cat["phi"], cat["size"],
                                               [len(m["x"]) for m in mods])
        per_event.append((idx, mlp_oracle.forward_bf16(fo, d)[0][:, 0] if len(idx) else np.zeros(0, np.float32)))
    z_all = np.concatenate([z for _, z in per_event])
    cut = float(np.median(z_all))
    d["seed_threshold"] = float(np.float32(1.0 / (1.0 + np.exp(-cut))))
    res = run_mode(b, chain.MODE_PRUNED, mlp.dict_to_weights(d))
    ms = res["module_start"].reshape(-1, 52)
    scale = 1.0 + np.abs(z_all).max()
    total = clear = mismatched = kept = 0
    for e, (idx, z) in enumerate(per_event):
        if len(idx) == 0:
            continue
        verdict = (res["cluster_keep"][int(ms[e, 0]) + idx] & 1).astype(bool)
        far = np.abs(z - cut) > 1e-2 * scale
        total += len(idx)
        clear += int(far.sum())
        mismatched += int((verdict[far] != (z[far] >= cut)).sum())
        kept += int(verdict.sum())
    assert total > 20_000 and clear > 0.8 * total, (total, clear)
    assert 0.3 * total < kept < 0.7 * total, (kept, total)
    # they agree except where the device picked the other proxy pair of a near-tie
    # (fast-math division: a few rows in a thousand)
    assert mismatched <= 0.005 * clear, (mismatched, clear)


def test_scoring_gate():
    b = events.generate(seed=12, nu_min=2.0, nu_max=15.0, n_events=64, with_mc=False)
    ref = canonical(run_mode(b, chain.MODE_PLAIN), b.n_events)
    # a scorer that prunes every candidate it scores
    d = random_weights(13, scale=0.0)
    d["w3"][:, 64] = -30.0
    d["seed_threshold"] = 0.5
    # gate above every pair count: nothing is scored, every seed kept
    d["min_pairs"] = 1 << 30
    gated = run_mode(b, chain.MODE_PRUNED, mlp.dict_to_weights(d))
    assert canonical(gated, b.n_events) == ref
    # gate of 8 pairs: seeds kept exactly when their windows give fewer than 8 pairs
    d["min_pairs"] = 8
    res = run_mode(b, chain.MODE_PRUNED, mlp.dict_to_weights(d))
    ms, mn = res["module_start"].reshape(-1, 52), res["module_num"].reshape(-1, 52)
    n_small = n_large = 0
    for e in range(b.n_events):
        mods = chain.event_clusters(res, e)
        cat = {k: np.concatenate([m[k] for m in mods]) for k in ("x", "y", "z", "phi", "size")}
        idx, _, fo = mlp_oracle.event_features(cat["x"], cat["y"], cat["z"], cat["phi"], cat["size"],
                                               [len(m["phi"]) for m in mods])
        keep = res["cluster_keep"][ms[e, 0]:ms[e, 51] + mn[e, 51]]
        pairs = fo[:, 6] * fo[:, 7]
        small = pairs < 8
        assert np.all(keep[idx[small]] & 1), e
        assert not np.any(keep[idx[~small]] & 1), e
        n_small += int(small.sum())
        n_large += int((~small).sum())
    assert n_small > 0 and n_large > 0
    # event gate: events below min_event_clusters keep every seed (the plain result), the
    # others lose every seed to the scorer (no tracks)
    n_hits = res["module_num"].reshape(-1, 52).sum(axis=1)
    cut = int(np.median(n_hits))
    d["min_pairs"] = 0
    d["min_event_clusters"] = cut
    ev = run_mode(b, chain.MODE_PRUNED, mlp.dict_to_weights(d))
    plain = run_mode(b, chain.MODE_PLAIN)
    below = above = 0
    for e in range(b.n_events):
        if n_hits[e] < cut:
            assert sorted(chain.event_tracks(ev, e)) == sorted(chain.event_tracks(plain, e)), e
            below += 1
        else:
            assert len(chain.event_tracks(ev, e)) == 0, e
            above += 1
    assert below > 0 and above > 0


def test_trained_scorer_prunes_at_no_efficiency_cost():
    # train on seed-1 events, evaluate on held-out seed-8 events with MC truth
    tr = events.generate(seed=1, nu_min=2.0, nu_max=15.0, n_events=1024, with_mc=False)
    vc = chain.VeloChain(max_events=tr.n_events, max_raw_bytes=int(tr.raw.size) + 4096)
    vc.run_host(tr)
    vc.sync()
    t = mlp.MlpTrainer(1 << 22, seed=2)
    t.collect(vc)
    vc.close()
    t.normalize()
    t.train(epochs=4, batch=8192, lr=3e-3)
    w = t.weights()
    w.seed_threshold = 0.1
    w.ext_threshold = 0.0
    w.max_event_clusters = 0xFFFFFFFF
    t.close()
    ev = events.generate(seed=8, nu_min=2.0, nu_max=15.0, n_events=1024, with_mc=True)
    plain = run_mode(ev, chain.MODE_PLAIN)
    pruned = run_mode(ev, chain.MODE_PRUNED, w)
    cp, cq = chain.check_tracks(ev, plain), chain.check_tracks(ev, pruned)
    assert cq.long_efficiency >= cp.long_efficiency - 0.002
    assert cq.ghost_rate <= cp.ghost_rate + 1e-4
    # fewer h1 kept as seeding candidates, and a faster search
    ms, mn = pruned["module_start"].reshape(-1, 52), pruned["module_num"].reshape(-1, 52)
    keep = np.concatenate([pruned["cluster_keep"][ms[e, 2]:ms[e, 49] + mn[e, 49]] for e in range(ev.n_events)])
    assert (keep & 1).mean() < 0.6
    # the search explores fewer combinations: faster on a full 16,384-event batch (at 1,024
    # events the search time is the latency of the slowest events, not the work)
    big = events.generate(seed=8, nu_min=2.0, nu_max=15.0, n_events=16384, first_event=2000, with_mc=False)
    _, st_plain = run_mode(big, chain.MODE_PLAIN, timing=True)
    _, st_pruned = run_mode(big, chain.MODE_PRUNED, w, timing=True)
    assert st_pruned["search_by_triplet"] < 0.95 * st_plain["search_by_triplet"]


def test_committed_scorer_with_every_candidate_scored():
    """The committed scorer with its gates open (every event and every seeding candidate
    scored: the quality operating point the bench reports) on events of the bench workload
    (nu ~ U(2,20)) with MC truth: long-track efficiency within 0.2% absolute of the plain
    search, and most ghosts gone."""
    from cuda_hlt_b200 import train_scorer
    w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
    w.min_pairs = 0
    w.min_event_clusters = 0
    ev = events.generate_config("pruned_1m", n_events=4096, first_event=100_000, threads=8, with_mc=True)
    plain = run_mode(ev, chain.MODE_PLAIN)
    pruned = run_mode(ev, chain.MODE_PRUNED, w)
    cp, cq = chain.check_tracks(ev, plain), chain.check_tracks(ev, pruned)
    assert cq.long_efficiency >= cp.long_efficiency - 0.002, (cp.long_efficiency, cq.long_efficiency)
    assert cq.ghost_rate < 0.5 * cp.ghost_rate, (cp.ghost_rate, cq.ghost_rate)


def test_label_mode_is_the_pruning_ceiling():
    """VELO_MODE_LABELS prunes with the plain search's own labels of the same batch (a perfect
    scorer at no cost). Every final track of the plain search - ghosts included - is made of
    labelled hits, and a seed without the label only ever forms a tracklet that ends as a
    rejected weak tracklet; the chosen extension of every final track is labelled. So label
    pruning of seeds, and of extensions too, gives the plain tracks exactly, with less work:
    the ceiling of what a scorer trained on these labels can save. With every event above the
    occupancy limit nothing is pruned."""
    b = events.generate(seed=14, nu_min=2.0, nu_max=20.0, n_events=512, with_mc=False)
    vc = chain.VeloChain(max_events=b.n_events, max_raw_bytes=int(b.raw.size) + 4096)
    with pytest.raises(chain.VeloError):  # no labels yet
        vc.set_mode(chain.MODE_LABELS)
        vc.run_host(b)
    vc.set_mode(chain.MODE_PLAIN)
    vc.run_host(b)
    vc.sync()
    plain = vc.results()
    ref = canonical(plain, b.n_events)
    defined = (plain["status"] & chain.REFERENCE_UNDEFINED) == 0
    vc.capture_labels(ext=True, max_event_clusters=0)  # every event falls back
    vc.set_mode(chain.MODE_LABELS)
    vc.run_host(b)
    vc.sync()
    fb = vc.results()
    assert canonical(fb, b.n_events) == ref
    assert np.all((fb["status"] & chain.STATUS["mlp_fallback"]) != 0)
    for ext in (False, True):
        vc.set_mode(chain.MODE_PLAIN)
        vc.run_host(b)
        vc.sync()
        vc.capture_labels(ext=ext)
        vc.set_mode(chain.MODE_LABELS)
        vc.run_host(b)
        vc.sync()
        lab = vc.results()
        got = canonical(lab, b.n_events)
        same = [got[e] == ref[e] for e in range(b.n_events)]
        assert all(s for s, d in zip(same, defined) if d), (ext, [e for e in range(b.n_events) if not same[e]][:8])
        assert defined.sum() >= 0.95 * b.n_events
        assert not np.any(lab["status"] & chain.STATUS["mlp_fallback"])
        # the labels as outputs: bit 0 exactly on the hits of the plain search's tracks, and
        # seeds without it have no h0 window
        ms, mn = lab["module_start"].reshape(-1, 52), lab["module_num"].reshape(-1, 52)
        span = int((lab["module_start"] + lab["module_num"]).max())
        win = vc._down(vc.out.hit_windows, np.uint32, 2 * span).reshape(-1, 2)
        for e in range(0, b.n_events, 7):
            a, z = int(ms[e, 0]), int(ms[e, 51] + mn[e, 51])
            on_track = np.isin(lab["cluster_id"][a:z], [i for t in chain.event_tracks(plain, e) for i in t])
            assert np.array_equal((lab["cluster_keep"][a:z] & 1).astype(bool), on_track), (ext, e)
            lo, hi = int(ms[e, 2]), int(ms[e, 50])
            assert np.all(win[lo:hi, 0][~on_track[lo - a:hi - a]] & 0xFFFF == 0xFFFF), (ext, e)
    vc.close()

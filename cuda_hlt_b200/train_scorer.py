"""Trains the learned seed/extension scorer on the GPU and evaluates the pruned search.

python -m cuda_hlt_b200.train_scorer [--samples 2000000] [--epochs 6] [--out PATH] [--report PATH]

1. Training set: seeding candidates of `mlp_train` events (seed 1, pileup nu ~ U(2,15)),
   run through the plain chain and labelled by its tracks, until --samples triplets.
   The largest cluster count of those events is the scorer's occupancy range: events
   above it fall back to the plain search.
2. Minibatch Adam on the tensor-core training kernels.
3. Operating point: on validation events (seed 1, after the training events), over seed
   thresholds x scoring gates (min_pairs: seeds with fewer (h0, h2) pairs stay unscored),
   the fastest pruned chain whose long-track efficiency loss against the plain search stays
   within --eff-budget (absolute) and whose ghost rate does not rise.
4. Evaluation on held-out events (seed 3, nu ~ U(2,15)): plain vs pruned against generator
   truth (efficiency, ghost rate), seeds explored and search time.
Writes the weights (VeloMlpWeights, binary) and prints a JSON report.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

from . import chain, events, mlp

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "velo_mlp_weights.bin")
BATCH = 16384
THRESHOLDS = (0.1, 0.3, 0.5, 0.7, 0.85)
MIN_PAIRS = (0, 8, 16, 24, 32, 48, 64, 96)
# Events scored on the nu ~ U(2,20) bench workload: only those with at least this many clusters
# (measured: pruned / plain 0.959 with every event scored, 0.972 from 4,500, 0.980 from 5,600,
# with the long-track efficiency loss 0.028% -> 0.010% and the ghost-rate gain 1.5 -> 0.7
# points). The search time of small events is hidden behind the large ones; scoring them costs
# more than their pruning saves.
BENCH_EVENT_GATE = 5600


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def quality(batch, res):
    c = chain.check_tracks(batch, res)
    return dict(long_efficiency=c.long_efficiency, velo_efficiency=c.velo_efficiency, ghost_rate=c.ghost_rate,
                long_reconstructible=int(c.long_reconstructible), long_found=int(c.long_found),
                tracks=int(c.tracks), ghosts=int(c.ghosts), long_clones=int(c.long_clones))


def seed_fraction(res, n):
    """Fraction of the h1 of modules 2..49 kept as seeding candidates (pruned mode)."""
    if "cluster_keep" not in res:
        return 1.0
    ms, mn = res["module_start"].reshape(-1, 52), res["module_num"].reshape(-1, 52)
    keep = np.concatenate([res["cluster_keep"][ms[e, 2]:ms[e, 49] + mn[e, 49]] for e in range(n)])
    return float((keep & 1).mean())


def collect_training(trainer, n_samples, threads):
    """Plain runs over mlp_train events until n_samples candidates are held; returns
    (samples, largest cluster count of an event, events run, next event index)."""
    first, held, max_clusters, n_events = 0, 0, 0, 0
    while held < n_samples:
        b = events.generate_config("mlp_train", n_events=BATCH, first_event=first, threads=threads, with_mc=False)
        vc = chain.VeloChain(max_events=BATCH, max_raw_bytes=int(b.raw.size) + 4096)
        vc.run_host(b)
        vc.sync()
        st = vc.results(clusters=True)
        held = trainer.collect(vc)
        vc.close()
        max_clusters = max(max_clusters, int(st["module_num"].reshape(-1, 52).sum(1).max()))
        n_events += b.n_events
        first += b.n_events
    return held, max_clusters, n_events, first


def evaluate(weights, batch, timing_reps=3):
    """Plain vs pruned on one MC-carrying batch."""
    out = {}
    for name, mode in (("plain", chain.MODE_PLAIN), ("pruned", chain.MODE_PRUNED)):
        vc = chain.VeloChain(max_events=batch.n_events, max_raw_bytes=int(batch.raw.size) + 4096,
                             mapping=chain.MAP_WARP)  # the mapping the bench's autotuner keeps
        vc.set_mlp(weights)
        vc.set_mode(mode)
        vc.run_host(batch)  # warm-up
        vc.sync()
        vc.set_timing(True)
        for _ in range(timing_reps):
            vc.run_host(batch)
        vc.sync()
        st = vc.stage_times()
        vc.run_host(batch)
        vc.sync()
        res = vc.results()
        vc.close()
        q = quality(batch, res)
        q["search_ms"] = st["search_by_triplet"] / max(1, st["runs"])
        q["fill_ms"] = st["fill_candidates"] / max(1, st["runs"])
        q["chain_ms"] = sum(v for k, v in st.items() if k != "runs") / max(1, st["runs"])
        q["seed_candidates_kept"] = seed_fraction(res, batch.n_events)
        q["fallback_events"] = int(((res["status"] & chain.STATUS["mlp_fallback"]) != 0).sum())
        out[name] = q
    return out


def choose_operating_point(weights, batch, eff_budget):
    """(seed threshold, min_pairs) of the fastest feasible pruned chain; the plain chain's
    figures; the scan. Falls back to the most conservative point when none is feasible."""
    w = mlp.dict_to_weights(mlp.weights_to_dict(weights))
    plain = None
    best, best_ms = (THRESHOLDS[0], MIN_PAIRS[-1]), None
    scan = {}
    for mp in MIN_PAIRS:
        for thr in THRESHOLDS:
            w.seed_threshold, w.min_pairs = thr, mp
            r = evaluate(w, batch, timing_reps=3)
            if plain is None:
                plain = r["plain"]
            scan[f"{thr}/{mp}"] = r["pruned"]
            loss = plain["long_efficiency"] - r["pruned"]["long_efficiency"]
            if loss <= eff_budget and r["pruned"]["ghost_rate"] <= plain["ghost_rate"]:
                if best_ms is None or r["pruned"]["chain_ms"] < best_ms:
                    best, best_ms = (thr, mp), r["pruned"]["chain_ms"]
    return best, plain, scan


def aggregate(rows):
    """Sums counts over batches and recomputes the rates from them; times summed."""
    out = {}
    for k in rows[0].keys():
        if k in ("long_efficiency", "velo_efficiency", "ghost_rate", "seed_candidates_kept"):
            continue
        out[k] = sum(r[k] for r in rows)
    out["long_efficiency"] = out["long_found"] / max(1, out["long_reconstructible"])
    out["ghost_rate"] = out["ghosts"] / max(1, out["tracks"])
    out["seed_candidates_kept"] = float(np.mean([r["seed_candidates_kept"] for r in rows]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--eff-budget", type=float, default=0.001)
    ap.add_argument("--validation-events", type=int, default=16384)
    ap.add_argument("--eval-events", type=int, default=200_000)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--min-event-clusters", type=int, default=0,
                    help="score only events with at least this many clusters (a deployment choice: "
                         "the committed file uses BENCH_EVENT_GATE)")
    args = ap.parse_args()
    threads = os.cpu_count() or 1
    t0 = time.time()
    trainer = mlp.MlpTrainer(args.samples, seed=args.seed)
    held, max_clusters, n_train_events, next_event = collect_training(trainer, args.samples, threads)
    log(f"collected {held} samples from {n_train_events} events in {time.time() - t0:.1f}s; max clusters "
        f"{max_clusters}")
    trainer.normalize()
    t1 = time.time()
    losses = []
    for ep in range(args.epochs):
        losses.append(trainer.train(1, args.batch, args.lr))
        log(f"epoch {ep}: loss {losses[-1]:.5f}")
    train_s = time.time() - t1
    w = trainer.weights()
    w.max_event_clusters = max_clusters
    w.ext_threshold = 0.0
    trainer.close()
    val = events.generate_config("mlp_train", n_events=args.validation_events, first_event=next_event,
                                 threads=threads, with_mc=True)
    (thr, min_pairs), val_plain, scan = choose_operating_point(w, val, args.eff_budget)
    w.seed_threshold = thr
    w.min_pairs = min_pairs
    w.min_event_clusters = args.min_event_clusters
    log(f"seed threshold {thr}, min_pairs {min_pairs}")
    mlp.save_weights(w, args.out)
    # held-out evaluation in batches of BATCH events
    ev = {"plain": [], "pruned": []}
    for a in range(0, args.eval_events, BATCH):
        n = min(BATCH, args.eval_events - a)
        b = events.generate(seed=3, nu_min=2.0, nu_max=15.0, n_events=n, first_event=a, threads=threads,
                            with_mc=True)
        r = evaluate(w, b)
        for k in ev:
            ev[k].append(r[k])
    evaluation = {k: aggregate(v) for k, v in ev.items()}
    report = {
        "training": {"samples": held, "events": n_train_events, "workload": "mlp_train: seed 1, nu ~ U(2,15)",
                     "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "loss_per_epoch": losses,
                     "train_seconds": train_s, "max_event_clusters": max_clusters},
        "threshold": {"chosen": thr, "min_pairs": min_pairs, "eff_budget": args.eff_budget,
                      "validation_events": val.n_events,
                      "plain": val_plain, "scan": {str(k): v for k, v in scan.items()}},
        "evaluation": {"events": args.eval_events, "workload": "seed 3, nu ~ U(2,15), held out", **evaluation,
                       "long_efficiency_loss": evaluation["plain"]["long_efficiency"]
                       - evaluation["pruned"]["long_efficiency"],
                       "search_speedup": evaluation["plain"]["search_ms"] / max(1e-9, evaluation["pruned"]["search_ms"]),
                       "chain_speedup": evaluation["plain"]["chain_ms"] / max(1e-9, evaluation["pruned"]["chain_ms"])},
        "weights": os.path.relpath(args.out, os.path.dirname(HERE)),
    }
    text = json.dumps(report, indent=1)
    if args.report:
        with open(args.report, "w") as f:
            f.write(text)
    print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())

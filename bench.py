#!/usr/bin/env python
"""Throughput of the B200 VELO chain, MLP-pruned vs plain, on the 1,000,000-event
nu ~ U(2,20) workload.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one pass of the chain over the rank's 1,000,000 synthetic events (seed 4,
events rank*1000000 ...), in batches of 65,536 events (one CUDA graph per batch). Both
forms run on the same device-resident input: the plain chain (reference semantics) and
the pruned chain (learned seed scorer; events above the scorer's trained occupancy fall
back to the plain search). Events are independent, so ranks process disjoint event
ranges with no data-path collective (weak scaling); NCCL is used only for the barrier and
the max over ranks of the elapsed device time. Prints one JSON line (rank 0):
  value     events/s of the pruned chain, raw banks resident in HBM (CUDA events around
            K steps); plain.value the same for the plain chain; pruned_vs_plain their ratio
  quality   long-track efficiency and ghost rate of both forms against generator truth on
            the head of the workload
  e2e       events/s of the pruned chain through velo_run_host from pinned host memory,
            each batch's consolidated tracks and Kalman states read back to pinned memory
  roofline  the stage with the largest serial share (first batches, one stream), its
            algorithmic bytes per launch over its live CUDA-event time in the timed region,
            against the measured HBM copy bandwidth; traffic from the committed ncu summary
  cpu_baseline  the CPU oracle (full chain) on the host cores, and the reference's x86
            clustering; clocks: nvidia-smi samples during the timed region; gpu_launches:
            this library's kernel launches in the timed region
--impl reference times the CPU implementation of the chain (the CPU oracle restating the
reference kernels; the reference has no CPU tracking) on the host cores, on a bounded
sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cuda_hlt_b200 import chain, events, shard  # noqa: E402

METRIC = "VELO events/s on 1 B200, MLP-pruned vs plain at ≤0.2% eff loss; % HBM peak"
UNIT = "events/s"
WORKLOAD = "pruned_1m"
N_EVENTS = 1_000_000
BUCKET = 65536   # events per batch (one CUDA graph); --batch
CHUNK = 4 * BUCKET
SIDE_BATCH = 16384  # batches of the MC-quality and reference-kernel legs
E2E_CONTEXTS = 4    # contexts (and streams) in rotation in the end-to-end leg


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def generate_workload(first_event, n_events, threads):
    """Returns a list of EventBatch chunks (CHUNK events each, last one shorter)."""
    chunks = []
    for a in range(0, n_events, CHUNK):
        n = min(CHUNK, n_events - a)
        chunks.append(events.generate_config(WORKLOAD, n_events=n, first_event=first_event + a, threads=threads,
                                             with_mc=False))
    return chunks


def batch_plan(chunks):
    """Batches of at most BUCKET events inside each chunk: (chunk index, first, last)."""
    plan = []
    for ci, c in enumerate(chunks):
        for a in range(0, c.n_events, BUCKET):
            plan.append((ci, a, min(c.n_events, a + BUCKET)))
    return plan


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


TRAFFIC_SUMMARIES = ["velo_chain_pruned_1m_16384_ncu.md"]


def load_traffic():
    """DRAM bytes per event of each kernel from the first committed ncu summary that
    holds them (the ```json block of the summary), if present."""
    merged = {}
    for name in TRAFFIC_SUMMARIES:
        try:
            with open(os.path.join(ROOT, "profiles", name)) as f:
                text = f.read()
            block = text.split("```json", 1)[1].split("```", 1)[0]
            for k, v in json.loads(block).get("bytes_per_event", {}).items():
                merged.setdefault(k, v)
        except (OSError, IndexError, ValueError):
            continue
    return {"bytes_per_event": merged} if merged else None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def load_scorer(args):
    """The committed scorer weights (trained on the GPU by cuda_hlt_b200.train_scorer), or a
    scorer trained here with --retrain / when the file is missing."""
    from cuda_hlt_b200 import mlp, train_scorer
    path = args.weights or train_scorer.DEFAULT_WEIGHTS
    if not args.retrain and os.path.exists(path):
        w = mlp.load_weights(path)
        return w, {"weights": os.path.relpath(path, ROOT), "trained": "committed", "seed_threshold": w.seed_threshold,
                   "min_pairs": w.min_pairs, "max_event_clusters": w.max_event_clusters,
                   "min_event_clusters": w.min_event_clusters}
    log("training the scorer (train_scorer pipeline, 1M samples, 4 epochs)")
    t0 = time.time()
    trainer = mlp.MlpTrainer(1_000_000, seed=1)
    threads = os.cpu_count() or 1
    held, max_clusters, _, next_event = train_scorer.collect_training(trainer, 1_000_000, threads)
    trainer.normalize()
    trainer.train(4, 16384, 2e-3)
    w = trainer.weights()
    trainer.close()
    w.max_event_clusters = max_clusters
    w.ext_threshold = 0.0
    val = events.generate_config("mlp_train", n_events=8192, first_event=next_event, threads=threads, with_mc=True)
    (w.seed_threshold, w.min_pairs), _, _ = train_scorer.choose_operating_point(w, val, 0.001)
    w.min_event_clusters = train_scorer.BENCH_EVENT_GATE
    return w, {"trained": f"in bench: {held} samples, {time.time() - t0:.1f}s", "seed_threshold": w.seed_threshold,
               "min_pairs": w.min_pairs, "max_event_clusters": max_clusters,
               "min_event_clusters": w.min_event_clusters}


def time_form(vcs, streams, batch_ptrs, args, world, dist, torch, local_rank):
    """Warm-up, then K timed steps of one form: (elapsed ms, max over ranks; stage times of
    each context; clocks during the timed region). Batches alternate between the contexts,
    each on its own stream, so that one batch's kernels fill the SMs that the other's leave
    idle (kernel tails, latency-bound phases)."""
    cur = torch.cuda.current_stream()

    def step():
        for k, (raw_p, off_p, n) in enumerate(batch_ptrs):
            j = k % len(vcs)
            vcs[j].run_device(raw_p, off_p, n, streams[j].cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for vc in vcs:
        vc.set_timing(True)  # keep only the timed region's event records
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record(cur)
        for s in streams:
            s.wait_event(start)
        for _ in range(args.steps):
            step()
        for s in streams:
            cur.wait_stream(s)
        end.record(cur)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    elapsed_ms = start.elapsed_time(end)
    if world > 1:
        elapsed_ms = shard.max_over_ranks(elapsed_ms, dist, torch.device("cuda", local_rank))
    # every timed launch records its stage events (the contexts keep the last 64): per-launch
    # means of each context times its launches per step give the stage times of one step
    stages = {}
    for j, vc in enumerate(vcs):
        st = vc.stage_times()
        runs = max(1, st.pop("runs"))
        per_step = sum(1 for k in range(len(batch_ptrs)) if k % len(vcs) == j)
        for k, v in st.items():
            stages[k] = stages.get(k, 0) + v / runs * per_step
    stages["runs"] = len(batch_ptrs)  # launches per step
    return elapsed_ms, stages, clocks.summary()


def single_stream_shares(vc, batch_ptrs, stream, torch, n_batches=2):
    """Share of each stage in the device time of the first batches run one after another on
    one stream (outside the timed region). The timed region overlaps two streams, which
    stretches each stage's event-to-event time by whatever the other stream runs meanwhile;
    the dominant kernel is picked from these serial shares, as ncu's serialised launch list
    would, and its live timed-region time then gives `achieved`."""
    vc.set_timing(True)
    for raw_p, off_p, n in batch_ptrs[:n_batches]:
        vc.run_device(raw_p, off_p, n, stream)
    torch.cuda.synchronize()
    st = vc.stage_times()
    runs = st.pop("runs")
    total = sum(st.values()) or 1.0
    return {k: v / total for k, v in st.items() if v > 0}, {k: v / max(1, runs) for k, v in st.items() if v > 0}


def roofline(stages, census, n_events, n_batches, peak, peak_kind, traffic_table, shares=None, serial_ms=None):
    """HBM roofline of the dominant kernel of one form (per launch = one batch): the stage
    with the largest serial share (`shares`), timed live over the timed region. With two
    streams a launch's event-to-event time includes what the other stream runs meanwhile, so
    the same figures from the serial single-stream pass (`serial_ms`, ms per batch) are added."""
    clusters, tracks, track_hits, raw_bytes = (census[k] for k in ("clusters", "tracks", "track_hits", "raw_bytes"))
    per = stage_bytes(census, n_events)  # algorithmic bytes of one step, per stage
    per["pv_beamline"] = 49 * tracks  # the Kalman states read once (the stage is off in both timed forms)
    stage_ms = {k: stages[k] for k in chain.STAGES}
    ranked = shares if shares else stage_ms
    dominant = max((k for k in ranked if k in per), key=ranked.get)
    avg_launch_ms = stage_ms[dominant] / max(1, stages["runs"])
    alg_bytes_launch = per[dominant] / n_batches
    achieved = alg_bytes_launch / (avg_launch_ms / 1e3) / 1e9
    traffic = None
    if traffic_table and dominant in traffic_table.get("bytes_per_event", {}):
        traffic = traffic_table["bytes_per_event"][dominant] * n_events / n_batches
    serial = None
    if serial_ms and dominant in serial_ms:
        # the serial pass runs the first batches: their bytes from the same per-event figure
        serial_achieved = alg_bytes_launch / (serial_ms[dominant] / 1e3) / 1e9
        serial = {"avg_launch_ms": serial_ms[dominant], "achieved": serial_achieved, "frac": serial_achieved / peak,
                  "what": "the same kernel timed alone on one stream (first batches, outside the timed region)"}
    return {"bound": "hbm", "kernel": dominant, "serial_stage_shares": shares, "achieved": achieved, "peak": peak,
            "peak_source": peak_kind,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": alg_bytes_launch, "avg_launch_ms": avg_launch_ms,
            "serial_single_stream": serial,
            "chain_alg_bytes_per_event": (raw_bytes + 16 * track_hits + 98 * tracks + 4 * (tracks + n_batches)
                                          + 8 * n_batches) / n_events}, stage_ms


# Label-pruned forms (VELO_MODE_LABELS: the plain search's own labels of the batch, a perfect
# scorer at no cost): (name, prune extensions too, events above the scorer's trained
# occupancy fall back to the plain search as in the pruned form)
LABEL_FORMS = (("labels_seed", False, True), ("labels_seed_ext", True, True),
               ("labels_seed_ext_all_events", True, False))


def every_candidate(weights):
    """The same scorer with its gates open: every event and every seeding candidate scored
    (the quality operating point: most ghosts pruned, at a throughput cost)."""
    from cuda_hlt_b200 import mlp
    return mlp.dict_to_weights({**mlp.weights_to_dict(weights), "min_pairs": 0, "min_event_clusters": 0})


def run_quality(weights, n, threads, label_events=2 * SIDE_BATCH):
    """Long-track efficiency and ghost rate of both forms against generator truth on the
    first n events of the workload (with MC truth), and of the label-pruned forms on the first
    label_events of them (their tracks equal the plain ones by construction; the GPU tests
    check it event by event). Events above the scorer's trained occupancy run the plain search
    in the pruned form; their number in the sample is reported."""
    rows = {"plain": [], "pruned": [], "pruned_every_candidate": []}
    rows.update({name: [] for name, _, _ in LABEL_FORMS})
    weights_all = every_candidate(weights)
    fallback = 0

    def add(name, b, res):
        c = chain.check_tracks(b, res)
        rows[name].append((c.long_reconstructible, c.long_found, c.tracks, c.ghosts, c.velo_reconstructible,
                           c.velo_found))

    for a in range(0, n, SIDE_BATCH):
        m = min(SIDE_BATCH, n - a)
        b = events.generate_config(WORKLOAD, n_events=m, first_event=a, threads=threads, with_mc=True)
        vc = chain.VeloChain(max_events=m, max_raw_bytes=int(b.raw.size) + 4096)
        vc.set_mlp(weights)
        for name, mode in (("plain", chain.MODE_PLAIN), ("pruned", chain.MODE_PRUNED)):
            vc.set_mode(mode)
            vc.run_host(b)
            vc.sync()
            res = vc.results(clusters=False)
            add(name, b, res)
            if mode == chain.MODE_PRUNED:
                fallback += int(((res["status"] & chain.STATUS["mlp_fallback"]) != 0).sum())
        vc.set_mlp(weights_all)
        vc.run_host(b)
        vc.sync()
        add("pruned_every_candidate", b, vc.results(clusters=False))
        vc.set_mlp(weights)
        if a < label_events:
            for name, ext, fb in LABEL_FORMS:
                vc.set_mode(chain.MODE_PLAIN)
                vc.run_host(b)
                vc.sync()
                vc.capture_labels(ext=ext, max_event_clusters=weights.max_event_clusters if fb else 0xFFFFFFFF)
                vc.set_mode(chain.MODE_LABELS)
                vc.run_host(b)
                vc.sync()
                add(name, b, vc.results(clusters=False))
        vc.close()
    out = {}
    for name, r in rows.items():
        lr, lf, t, g, vr, vf = (sum(x[i] for x in r) for i in range(6))
        out[name] = {"long_efficiency": lf / max(1, lr), "ghost_rate": g / max(1, t), "velo_efficiency": vf / max(1, vr),
                     "tracks": t, "long_reconstructible": lr}
        if name.startswith("labels"):
            out[name]["events"] = min(n, label_events)
    out["events"] = n
    out["fallback_events"] = fallback
    out["long_efficiency_loss"] = out["plain"]["long_efficiency"] - out["pruned"]["long_efficiency"]
    out["ghost_rate_change"] = out["pruned"]["ghost_rate"] - out["plain"]["ghost_rate"]
    out["every_candidate_long_efficiency_loss"] = (out["plain"]["long_efficiency"]
                                                   - out["pruned_every_candidate"]["long_efficiency"])
    return out


def pruning_ceiling(weights, batch_ptrs, max_batch_bytes, threshold, decode_warps, stream, torch, n_batches=2):
    """Device time per stage of the plain chain, the scorer-pruned chain and the label-pruned
    chains (the plain search's own labels: what a perfect scorer at no cost would save), on
    the first batches of the workload, one after another on one stream (CUDA events per
    stage, mean of 3 runs per batch after one untimed run)."""
    vc = chain.VeloChain(max_events=BUCKET, max_raw_bytes=max_batch_bytes + 4096)
    vc.set_mlp(weights)
    vc.set_block_threshold(threshold)
    vc.set_decode_warps(decode_warps)
    forms = ["plain", "pruned"] + [name for name, _, _ in LABEL_FORMS]
    acc = {f: {} for f in forms}
    n_events = 0

    def timed(name, raw_p, off_p, n):
        vc.run_device(raw_p, off_p, n, stream)
        torch.cuda.synchronize()
        vc.set_timing(True)
        for _ in range(3):
            vc.run_device(raw_p, off_p, n, stream)
        vc.sync(clusters=False)
        st = vc.stage_times()
        runs = max(1, st.pop("runs"))
        for k, v in st.items():
            acc[name][k] = acc[name].get(k, 0.0) + v / runs
        vc.set_timing(False)

    for raw_p, off_p, n in batch_ptrs[:n_batches]:
        n_events += n
        for name, mode in (("plain", chain.MODE_PLAIN), ("pruned", chain.MODE_PRUNED)):
            vc.set_mode(mode)
            timed(name, raw_p, off_p, n)
        for name, ext, fallback in LABEL_FORMS:
            vc.set_mode(chain.MODE_PLAIN)
            vc.run_device(raw_p, off_p, n, stream)
            vc.sync(clusters=False)
            vc.capture_labels(ext=ext, max_event_clusters=weights.max_event_clusters if fallback else 0xFFFFFFFF)
            vc.set_mode(chain.MODE_LABELS)
            timed(name, raw_p, off_p, n)
    vc.close()
    stage_keys = ("decode_cluster_sort", "fill_candidates", "search_by_triplet", "event_scan", "consolidate_fit")
    stages = {f: {k: acc[f].get(k, 0.0) for k in stage_keys} for f in forms}
    chain_ms = {f: sum(stages[f].values()) for f in forms}
    return {"events": n_events, "batches": n_batches,
            "timing": "one stream, stages bracketed by CUDA events, mean of 3 runs per batch, summed over batches",
            "forms": {"plain": "reference semantics", "pruned": "committed scorer",
                      "labels_seed": "seeds kept only where the plain search found a track (perfect seed scorer); "
                                     "events above the trained occupancy run the plain search",
                      "labels_seed_ext": "and extension candidates only where the plain search extended a track",
                      "labels_seed_ext_all_events": "both, on every event (no occupancy fallback)"},
            "stages_ms": stages, "chain_ms": chain_ms,
            "speedup_vs_plain": {f: chain_ms["plain"] / chain_ms[f] for f in forms},
            "search_speedup_vs_plain": {f: stages["plain"]["search_by_triplet"] / stages[f]["search_by_triplet"]
                                        for f in forms}}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    threads = max(1, (os.cpu_count() or 1) // max(1, world))
    weights, scorer_info = load_scorer(args)
    t0 = time.time()
    n_events = args.events
    first_event, n_events = shard.event_range(rank, n_events)
    chunks = generate_workload(first_event, n_events, threads)
    log(f"[rank {rank}] generated {n_events} events in {time.time() - t0:.1f}s, "
        f"{sum(c.raw.size for c in chunks) / 1e9:.2f} GB raw")
    plan = batch_plan(chunks)
    n_batches = len(plan)
    max_batch_bytes = max(int(chunks[ci].offsets[b] - chunks[ci].offsets[a]) for ci, a, b in plan)

    # device-resident copy of the raw banks and per-batch offset arrays
    d_raw = [torch.from_numpy(c.raw).to(dev) for c in chunks]
    offs_host = []
    for ci, a, b in plan:
        o = chunks[ci].offsets[a:b + 1]
        offs_host.append((o - o[0]).astype(np.uint64))
    d_offs = [torch.from_numpy(o.view(np.int64)).to(dev) for o in offs_host]
    batch_ptrs = [(d_raw[ci].data_ptr() + int(chunks[ci].offsets[a]), d_offs[k].data_ptr(), b - a)
                  for k, (ci, a, b) in enumerate(plan)]
    stream = torch.cuda.current_stream(dev).cuda_stream
    raw_bytes = sum(int(c.raw.size) for c in chunks)
    peak, peak_kind = load_peaks()
    traffic_table = load_traffic()
    from cuda_hlt_b200 import autotune

    forms = {}
    streams = [torch.cuda.Stream(device=dev) for _ in range(args.streams)]
    form_list = (("plain", chain.MODE_PLAIN, weights), ("pruned", chain.MODE_PRUNED, weights),
                 ("pruned_every_candidate", chain.MODE_PRUNED, every_candidate(weights)))
    for name, mode, form_weights in form_list:
        if name == "pruned_every_candidate" and args.no_operating_points:
            continue
        vcs = [chain.VeloChain(max_events=BUCKET, max_raw_bytes=max_batch_bytes + 4096, device=local_rank,
                               use_graphs=True) for _ in range(args.streams)]
        for vc in vcs:
            vc.set_mlp(form_weights)
            vc.set_mode(mode)
            vc.set_timing(True)  # before any graph capture: every graph then records its stage events
        vc = vcs[0]
        # search mapping per hit-count bucket, tuned on the first batch (outside the timed region)
        threshold, tune_ms = autotune.tune_block_threshold(vc, *batch_ptrs[0], stream)
        decode_warps, decode_ms = autotune.tune_decode_warps(vc, *batch_ptrs[0], stream)
        for other in vcs[1:]:
            other.set_block_threshold(threshold)
            other.set_decode_warps(decode_warps)
        # census: per-batch totals for the algorithmic-byte accounting and the fallback share
        census = dict(clusters=0, tracks=0, track_hits=0, raw_bytes=raw_bytes, fallback_events=0)
        for raw_p, off_p, n in batch_ptrs:
            vc.run_device(raw_p, off_p, n, stream)
            t, h, c = vc.sync()
            census["tracks"] += t
            census["track_hits"] += h
            census["clusters"] += c
            st = np.empty(n, np.uint32)
            chain._check(vc.lib.velo_download(vc.ctx, st.ctypes.data, chain.C.c_void_p(vc.out.status), 4 * n),
                         "velo_download")
            census["fallback_events"] += int(((st & chain.STATUS["mlp_fallback"]) != 0).sum())
        launches = vc.launch_count()
        shares, serial_ms = single_stream_shares(vc, batch_ptrs, stream, torch)
        elapsed_ms, stages, clocks = time_form(vcs, streams, batch_ptrs, args, world, dist, torch, local_rank)
        roof, stage_ms = roofline(stages, census, n_events, n_batches, peak, peak_kind, traffic_table, shares,
                                  serial_ms)
        forms[name] = {"value": n_events * world * args.steps / (elapsed_ms / 1e3),
                       "ms_per_step": elapsed_ms / args.steps,
                       # per-launch means times launches per step (stages of the two streams
                       # overlap in time)
                       "stages_ms_per_step": stage_ms,
                       "stages_ms_per_batch_serial": serial_ms,
                       "graphs": sum(v.graph_count() for v in vcs),
                       "roofline": roof, "census_per_step": census,
                       "search_mapping": {"block_above_clusters": threshold,
                                          "search_ms_per_threshold": {str(k): v for k, v in tune_ms.items()}},
                       "decode_block": {"warps": decode_warps,
                                        "decode_ms_per_warps": {str(k): v for k, v in decode_ms.items()}},
                       "gpu_launches": launches * n_batches * args.steps, "clocks": clocks, "threshold": threshold,
                       "decode_warps": decode_warps}
        for v in vcs:
            v.close()
        log(f"[rank {rank}] {name}: {forms[name]['value']:.0f} events/s")

    # ---- track quality of both forms on the MC-carrying head of the workload ----
    quality = run_quality(weights, args.quality_events, threads) if rank == 0 and args.quality_events > 0 else None

    # ---- per-stage times of every form, and the ceiling of pruning (label-pruned forms) ----
    ceiling = None
    if rank == 0 and not args.no_ceiling:
        ceiling = pruning_ceiling(weights, batch_ptrs, max_batch_bytes, forms["plain"]["threshold"],
                                  forms["plain"]["decode_warps"], stream, torch)

    # the device-resident copy of the workload is done with: the end-to-end leg reads host
    # buffers, and its contexts need the room
    del batch_ptrs, d_offs, d_raw
    torch.cuda.empty_cache()

    # ---- end to end through velo_run_host with host buffers (pruned form) ----
    e2e = run_e2e(args, chunks, plan, local_rank, torch, world, dist, forms["pruned"]["threshold"], weights,
                   forms["pruned"]["decode_warps"])
    # the same leg for the plain chain and for the scorer with every candidate scored: through
    # host buffers the link bounds the rate, and pruned ghosts are bytes not read back
    if not args.no_operating_points:
        e2e["by_form"] = {"committed_gates": {"value": e2e["value"], "d2h_bytes_per_step": e2e["d2h_bytes_per_step"]}}
        for name, mode, w in (("plain", chain.MODE_PLAIN, weights),
                              ("every_candidate", chain.MODE_PRUNED, every_candidate(weights))):
            r = run_e2e(args, chunks, plan, local_rank, torch, world, dist, forms["pruned"]["threshold"], w,
                        forms["pruned"]["decode_warps"], mode=mode)
            e2e["by_form"][name] = {"value": r["value"], "d2h_bytes_per_step": r["d2h_bytes_per_step"]}
        for row in e2e["by_form"].values():
            row["vs_plain"] = row["value"] / e2e["by_form"]["plain"]["value"]

    p, q = forms["pruned"], forms["plain"]
    result = {
        "metric": METRIC, "value": p["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": p["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32 (scorer: bf16 operands, fp32 accumulation)", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD}: {n_events} events per GPU, pileup nu ~ U(2,20), seed 4, events "
                               f"rank*{n_events}..., MLP-pruned search; events above the scorer's trained "
                               f"occupancy fall back to the plain search", "events_per_gpu": n_events,
                   "batch_events": BUCKET, "batches_per_step": n_batches, "mode": "pruned",
                   "graphs": f"{p['graphs']} CUDA graphs (one per batch-size bucket and stream), each serving every "
                             f"batch of its bucket",
                   "streams": args.streams,
                   "scorer": scorer_info, "search_mapping": p["search_mapping"],
                   "decode_block": p["decode_block"],
                   "l2": f"inputs larger than L2 ({raw_bytes / 1e9:.2f} GB raw banks per step)",
                   "parallelism": f"event shards x{world}"},
        "roofline": p["roofline"],
        "stages_ms_per_step": p["stages_ms_per_step"],
        "stages_note": "stages_ms_per_step: each stage's event-to-event time on its stream in the timed region, "
                       "two streams overlapping (a bracket includes the other stream's kernels, so the stages sum "
                       "to more than ms_per_step); stages_ms_per_batch_serial: the same stages on one stream, "
                       "first batches, nothing else running",
        "stages_ms_per_batch_serial": p["stages_ms_per_batch_serial"],
        "totals_per_step": p["census_per_step"],
        "fallback_fraction": p["census_per_step"]["fallback_events"] / n_events,
        "plain": {"value": q["value"], "ms_per_step": q["ms_per_step"], "stages_ms_per_step": q["stages_ms_per_step"],
                  "stages_ms_per_batch_serial": q["stages_ms_per_batch_serial"],
                  "roofline": q["roofline"], "totals_per_step": q["census_per_step"], "clocks": q["clocks"],
                  "search_mapping": q["search_mapping"], "decode_block": q["decode_block"],
                  "gpu_launches": q["gpu_launches"]},
        "pruned_vs_plain": p["value"] / q["value"],
        "operating_points": operating_points(forms, quality),
        "quality": quality,
        "pruning_ceiling": ceiling,
        "e2e": e2e,
        "gpu_launches": p["gpu_launches"],
        "clocks": p["clocks"],
    }
    return result, chunks


def host_link(torch, local_rank, nbytes=2 << 30, chunk=64 << 20, reps=5):
    """Copy rates of this GPU's host link in GB/s: pinned host to device and device to host,
    each alone and both at once (one stream per direction, 64 MB copies); the best of `reps`
    passes of `nbytes` each (a single pass can land on a slow moment of a shared host)."""
    dev = torch.device("cuda", local_rank)
    h_up = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_down = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_up = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d_down = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    s_up, s_down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

    def copies(dst, src, stream):
        with torch.cuda.stream(stream):
            for o in range(0, nbytes, chunk):
                dst[o:o + chunk].copy_(src[o:o + chunk], non_blocking=True)

    def rate(*jobs):
        for job in jobs:
            copies(*job)
        torch.cuda.synchronize(dev)
        best = 0.0
        for _ in range(reps):
            t0 = time.perf_counter()
            for job in jobs:
                copies(*job)
            torch.cuda.synchronize(dev)
            best = max(best, nbytes / (time.perf_counter() - t0) / 1e9)
        return best

    up, down = (d_up, h_up, s_up), (h_down, d_down, s_down)
    out = {"h2d_GBps": rate(up), "d2h_GBps": rate(down), "both_GBps_each_direction": rate(up, down)}
    del h_up, h_down, d_up, d_down
    return {k: round(v, 2) for k, v in out.items()}


def link_bound(n_events, h2d_bytes, d2h_bytes, link):
    """Events/s the host link allows for these bytes per step: both directions at the
    concurrent rate while both have bytes to move, then the larger one alone."""
    both = min(h2d_bytes, d2h_bytes) / (link["both_GBps_each_direction"] * 1e9)
    rest_rate = link["h2d_GBps"] if h2d_bytes > d2h_bytes else link["d2h_GBps"]
    rest = abs(h2d_bytes - d2h_bytes) / (rest_rate * 1e9)
    return n_events / (both + rest)


def operating_points(forms, quality):
    """The scorer at its committed gates (the bench's `value`) and with every candidate scored,
    side by side: events/s against the plain chain, and the track quality of each."""
    out = {}
    for name, form in (("committed_gates", "pruned"), ("every_candidate", "pruned_every_candidate")):
        if form not in forms:
            continue
        f = forms[form]
        row = {"value": f["value"], "ms_per_step": f["ms_per_step"], "vs_plain": f["value"] / forms["plain"]["value"],
               "stages_ms_per_batch_serial": f["stages_ms_per_batch_serial"]}
        if quality:
            qf = quality["pruned" if form == "pruned" else "pruned_every_candidate"]
            row.update(long_efficiency_loss=quality["plain"]["long_efficiency"] - qf["long_efficiency"],
                       ghost_rate=qf["ghost_rate"], plain_ghost_rate=quality["plain"]["ghost_rate"])
        out[name] = row
    return out


def run_e2e(args, chunks, plan, local_rank, torch, world, dist, threshold, weights, decode_warps=8,
            mode=None):
    """velo_run_host from pinned memory, E2E_CONTEXTS contexts in rotation, each on its own
    stream, so that the upload of one batch, the kernels of the next and the read-back of a
    third overlap (uploads and read-backs use the host link in opposite directions); outputs
    read back to pinned host buffers every batch."""
    import ctypes as C
    cudart = torch.cuda.cudart()
    for c in chunks:
        cudart.cudaHostRegister(c.raw.ctypes.data, c.raw.nbytes, 0)
    offs = []
    for ci, a, b in plan:
        o = chunks[ci].offsets[a:b + 1]
        offs.append(np.ascontiguousarray(o - o[0], dtype=np.uint64))
    max_batch_bytes = max(int(chunks[ci].offsets[b] - chunks[ci].offsets[a]) for ci, a, b in plan)
    # as many contexts as asked for and the device holds (at least two)
    ctxs = []
    for _ in range(args.e2e_contexts):
        vc = None
        try:
            vc = chain.VeloChain(max_events=BUCKET, max_raw_bytes=max_batch_bytes + 4096, device=local_rank)
            vc.set_block_threshold(threshold)
            vc.set_decode_warps(decode_warps)
            vc.set_mlp(weights)
            vc.set_mode(chain.MODE_PRUNED if mode is None else mode)
            ctxs.append(vc)
        except chain.VeloError:
            if vc is not None:
                vc.close()
            if len(ctxs) < 2:
                raise
            break
    nctx = len(ctxs)
    streams = [torch.cuda.Stream(device=local_rank) for _ in range(nctx)]
    # pinned result buffers per context: atomics, hit numbers, hits SoA, Kalman states
    # (the workload averages 166 tracks and 1,340 track hits per event; a batch beyond these
    # capacities raises before any copy)
    cap_t = 250 * BUCKET
    cap_h = 10 * cap_t
    outs = [dict(atomics=torch.empty(2 * BUCKET + 1, dtype=torch.int32, pin_memory=True),
                 thn=torch.empty(cap_t + 1, dtype=torch.int32, pin_memory=True),
                 hits=torch.empty(16 * cap_h, dtype=torch.uint8, pin_memory=True),
                 kal=torch.empty(52 * cap_t, dtype=torch.uint8, pin_memory=True)) for _ in range(nctx)]
    lib = ctxs[0].lib

    d2h = [0]
    h2d = [0]
    depth = max(1, min(args.e2e_depth, nctx - 1))  # batches in flight before the oldest is read back
    # The batches of consecutive steps form one pipeline: a step's last read-backs overlap the
    # next step's first uploads, and the pipeline drains once, at the end of the timed region
    # (every step's uploads and read-backs still happen inside it).
    pending = []  # (sequence number, batch) uploaded and launched, not yet read back
    seq = [0]

    def fetch(item):
        q, k = item
        vc, o, s = ctxs[q % nctx], outs[q % nctx], streams[q % nctx]
        t, h, _ = vc.sync(clusters=False)
        n = plan[k][2] - plan[k][1]
        for buf, src, nbytes in ((o["atomics"], vc.out.atomics, 4 * (2 * n + 1)),
                                 (o["thn"], vc.out.track_hit_number, 4 * (t + 1)),
                                 (o["hits"], vc.out.track_hits, 16 * h),
                                 (o["kal"], vc.out.kalman_states, 49 * t)):
            if nbytes > buf.numel() * buf.element_size():
                raise RuntimeError(f"e2e: batch {k} needs {nbytes} bytes, pinned buffer holds "
                                   f"{buf.numel() * buf.element_size()}")
            if nbytes:
                chain._check(lib.velo_download_async(vc.ctx, C.c_void_p(buf.data_ptr()), C.c_void_p(src), nbytes,
                                                     C.c_void_p(s.cuda_stream)), "velo_download_async")
                d2h[0] += nbytes

    def step():
        for k, (ci, a, b) in enumerate(plan):
            q = seq[0]
            seq[0] += 1
            vc, s = ctxs[q % nctx], streams[q % nctx]
            base = int(chunks[ci].offsets[a])
            nbytes = int(chunks[ci].offsets[b]) - base
            sub = events.EventBatch(chunks[ci].raw[base:base + nbytes], offs[k])
            vc.run_host(sub, s.cuda_stream)
            h2d[0] += nbytes + offs[k].nbytes
            pending.append((q, k))
            if len(pending) > depth:
                fetch(pending.pop(0))

    def drain():
        while pending:
            fetch(pending.pop(0))
        for s in streams:
            s.synchronize()

    for _ in range(max(1, args.warmup)):
        step()
    drain()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    d2h[0] = h2d[0] = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    drain()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    if world > 1:
        el = shard.max_over_ranks(el, dist, torch.device("cuda", local_rank))
    for vc in ctxs:
        vc.close()
    for c in chunks:
        cudart.cudaHostUnregister(c.raw.ctypes.data)
    n_events = sum(b - a for _, a, b in plan)
    value = n_events * world * args.steps / el
    link = host_link(torch, local_rank)
    bound = world * link_bound(n_events, h2d[0] / args.steps, d2h[0] / args.steps, link)
    return {"value": value, "unit": UNIT,
            "h2d_bytes_per_step": h2d[0] // args.steps, "d2h_bytes_per_step": d2h[0] // args.steps,
            "timing": "host wall clock around K steps, synchronised; the batches of consecutive steps "
                      "pipelined, drained at the end", "contexts": nctx, "depth": depth,
            "host_link": {**link, "bound": bound, "frac": value / bound,
                          "what": "events/s the measured host link allows for these bytes per step, "
                                  "and the e2e value's fraction of it"}}


# ---------------------------------------------------------------------------
# CPU baselines
# ---------------------------------------------------------------------------
def cpu_baseline(sample_events, threads):
    """The CPU oracle (restatement of the reference chain; the reference has no CPU
    tracking) on a bounded sample, plus the reference's own x86 clustering when built."""
    import oracle
    geo = events.load_geometry()
    b = events.generate_config(WORKLOAD, n_events=sample_events, threads=threads, with_mc=False)
    t0 = time.perf_counter()
    oracle.run(b, geo, threads=threads)
    dt = time.perf_counter() - t0
    out = {"value": sample_events / dt, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"first {sample_events} events of the workload, full chain, {threads} threads"}
    if os.path.exists(oracle.REF_X86_LIB):
        try:
            t0 = time.perf_counter()
            oracle.ref_x86_clustering(b, geo, algo=0, threads=threads)
            out["reference_x86_clustering_only"] = {
                "value": sample_events / (time.perf_counter() - t0), "unit": UNIT, "kind": "reference",
                "what": "x86/velo/clustering clustering() only (the reference's only CPU VELO code)"}
        except Exception as ex:  # pragma: no cover
            out["reference_x86_clustering_only"] = {"error": str(ex)}
    return out, b


def reference_gpu(batch):
    """The reference's own CUDA kernels (oracle/_ref) on one batch, visitor launch shapes
    and host synchronisations included; events above its 500-cluster module buffer are
    left out (they would overrun its shared memory)."""
    import oracle
    geo = events.load_geometry()
    if not os.path.exists(oracle.REF_GPU_LIB):
        return None
    r = oracle.run(batch, geo)
    # events that overrun the reference's fixed per-event buffers would spill into their
    # neighbours; they are left out so that the reference run stays well defined
    keep = [e for e in range(batch.n_events) if r.module_num[e * 52:(e + 1) * 52].max() < 500
            and not (int(r.flags[e]) & (oracle.UNDEFINED_IN_REFERENCE & ~oracle.F_SEED_TIE))]
    sub = events.EventBatch(np.concatenate([batch.event(e) for e in keep]),
                            np.concatenate([[0], np.cumsum([batch.event(e).size for e in keep])]).astype(np.uint64))
    _, ms = oracle.ref_gpu_run(sub, geo, reps=4)
    return {"value": len(keep) / (ms / 1e3), "unit": UNIT, "events": len(keep),
            "what": "reference cuda/velo kernels compiled for sm_100a, one batch per launch sequence"}


def pv_leg(batch, threshold):
    """The beamline PV stage appended to the plain chain on one batch (device-resident
    input, graphs, CUDA events per stage), next to the reference's own PV kernels
    (oracle/_ref) on the same consolidated tracks."""
    import torch
    raw = torch.from_numpy(batch.raw).cuda()
    off = torch.from_numpy(batch.offsets.view(np.int64)).cuda()
    s = torch.cuda.current_stream().cuda_stream
    vc = chain.VeloChain(max_events=batch.n_events, max_raw_bytes=int(batch.raw.size) + 4096, use_graphs=True)
    vc.set_block_threshold(threshold)
    vc.set_pv(True)
    vc.set_timing(True)
    for _ in range(2):
        vc.run_device(raw.data_ptr(), off.data_ptr(), batch.n_events, s)
    torch.cuda.synchronize()
    vc.set_timing(True)
    for _ in range(5):
        vc.run_device(raw.data_ptr(), off.data_ptr(), batch.n_events, s)
    vc.sync()
    st = vc.stage_times()
    res = vc.results(clusters=False)
    vc.close()
    runs = max(1, st.pop("runs"))
    pv_ms = st["pv_beamline"] / runs
    chain_ms = sum(st.values()) / runs
    n = batch.n_events
    out = {"events": n, "pv_stage_ms": pv_ms, "pv_events_per_s": n / (pv_ms / 1e3),
           "chain_with_pv_ms": chain_ms, "chain_with_pv_events_per_s": n / (chain_ms / 1e3),
           "peaks_per_event": float(res["pv_npeaks"].mean()), "vertices_per_event": float(res["pv_count"].mean()),
           "timing": "CUDA events around the stage, single stream, mean of 5 runs"}
    try:
        import oracle
        if os.path.exists(oracle.REF_GPU_LIB):
            r = oracle.ref_pv_run(res["atomics"], res["track_hit_number"], res["kalman_raw"], n, reps=4)
            out["reference_kernels_ms"] = r["ms"]
            out["reference_kernels_events_per_s"] = n / (r["ms"] / 1e3)
            out["reference_vertices_per_event"] = float(r["n_vertices"].mean())
    except Exception as ex:
        out["reference_error"] = str(ex)
    return out


def stage_bytes(census, n_events):
    """Algorithmic bytes of each stage for a pass with these totals (raw bytes, clusters,
    tracks, track hits): what the stage must read and write at least."""
    clusters, tracks, track_hits, raw_bytes = (census[k] for k in ("clusters", "tracks", "track_hits", "raw_bytes"))
    return {
        "decode_cluster_sort": raw_bytes + 16 * clusters + 8 * clusters,  # raw in, hits and windows out
        "search_by_triplet": 16 * clusters + 8 * clusters + 2 * track_hits + 2 * tracks,
        "event_scan": 16 * n_events,
        "consolidate_fit": 34 * track_hits + 98 * tracks + 8 * tracks,
    }


def workload_leg(config, n_events, batch_sizes, threshold, decode_warps, threads, torch, first_event=0):
    """The plain chain on another workload of the reference configuration list, device-resident,
    in consecutive batches whose sizes cycle through `batch_sizes` (one CUDA graph per batch-size
    bucket serves them all): events/s over one pass (CUDA events, one stream, after one untimed
    pass), the graphs used, and each stage's time and algorithmic GB/s."""
    chunks = [events.generate_config(config, n_events=min(CHUNK, n_events - a), first_event=first_event + a,
                                     threads=threads, with_mc=False) for a in range(0, n_events, CHUNK)]
    dev = torch.device("cuda")
    d_raw = [torch.from_numpy(c.raw).to(dev) for c in chunks]
    plan, keep = [], []
    for ci, c in enumerate(chunks):
        a, k = 0, 0
        while a < c.n_events:
            b = min(c.n_events, a + batch_sizes[k % len(batch_sizes)])
            o = (c.offsets[a:b + 1] - c.offsets[a]).astype(np.uint64)
            t = torch.from_numpy(o.view(np.int64)).to(dev)
            keep.append(t)
            plan.append((d_raw[ci].data_ptr() + int(c.offsets[a]), t.data_ptr(), b - a, int(o[-1])))
            a, k = b, k + 1
    vc = chain.VeloChain(max_events=max(batch_sizes), max_raw_bytes=max(p[3] for p in plan) + 4096, use_graphs=True)
    vc.set_block_threshold(threshold)
    vc.set_decode_warps(decode_warps)
    s = torch.cuda.current_stream()
    census = dict(clusters=0, tracks=0, track_hits=0, raw_bytes=sum(int(c.raw.size) for c in chunks))
    for raw_p, off_p, n, _ in plan:  # untimed pass: graphs, census
        vc.run_device(raw_p, off_p, n, s.cuda_stream)
        t, h, c = vc.sync()
        census["tracks"] += t
        census["track_hits"] += h
        census["clusters"] += c
    vc.set_timing(True)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(s)
    for raw_p, off_p, n, _ in plan:
        vc.run_device(raw_p, off_p, n, s.cuda_stream)
    end.record(s)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    st = vc.stage_times()
    runs = max(1, st.pop("runs"))
    out = {"workload": config, "events": n_events, "batches": len(plan), "batch_sizes": list(batch_sizes),
           "events_per_s": n_events / (ms / 1e3), "ms": ms, "graphs": vc.graph_count(),
           "timing": "CUDA events around one pass after an untimed one, one stream",
           "totals": census}
    if runs >= len(plan):  # every launch's stage events kept: per-stage times and GB/s
        alg = stage_bytes(census, n_events)
        out["stage_ms"] = {k: v for k, v in st.items() if v > 0}
        out["stage_gbs"] = {k: alg[k] / (st[k] / 1e3) / 1e9 for k in alg if st.get(k, 0) > 0}
    vc.close()
    return out


# Algorithmic bytes of the global event cut per event: the SciFi and UT bank offset tables,
# the hit-count word of each UT bank, and the outputs (two counts, a flag, a list entry).
def gec_bytes(ut, sf):
    nu = ut.raw[ut.offsets[:-1].astype(np.int64)[:, None] + np.arange(4)].copy().view(np.uint32).ravel()
    ns = sf.raw[sf.offsets[:-1].astype(np.int64)[:, None] + np.arange(4)].copy().view(np.uint32).ravel()
    return int(np.sum(4 * (ns.astype(np.int64) + 2) + 4 * (nu.astype(np.int64) + 2) + 4 * nu.astype(np.int64) + 13))


def gec_leg(batch, threshold, decode_warps):
    """The global event cut in front of the plain chain on one batch (synthetic UT and SciFi
    events of the same events, device-resident, graphs, CUDA events per stage), next to the
    chain without the cut and to the reference's own kernel (oracle/_ref) on the same input."""
    import torch
    ut, sf = events.generate_ut_scifi(batch, seed=0)
    dev = [torch.from_numpy(a).cuda() for a in (batch.raw, batch.offsets.view(np.int64), ut.raw,
                                                 ut.offsets.view(np.int64), sf.raw, sf.offsets.view(np.int64))]
    p = [t.data_ptr() for t in dev]
    s = torch.cuda.current_stream().cuda_stream
    n = batch.n_events
    out = {"events": n, "ut_bytes_per_event": ut.raw.size / n, "scifi_bytes_per_event": sf.raw.size / n,
           "timing": "CUDA events around the stage, single stream, mean of 5 runs"}
    for name in ("with_cut", "without_cut"):
        vc = chain.VeloChain(max_events=n, max_raw_bytes=int(batch.raw.size) + 4096, use_graphs=True)
        vc.set_block_threshold(threshold)
        vc.set_decode_warps(decode_warps)
        vc.set_timing(True)

        def once():
            if name == "with_cut":
                vc.run_gec_device(p[0], p[1], p[2], p[3], p[4], p[5], n, stream=s)
            else:
                vc.run_device(p[0], p[1], n, s)
        for _ in range(2):
            once()
        torch.cuda.synchronize()
        vc.set_timing(True)
        for _ in range(5):
            once()
        t, _, _ = vc.sync(clusters=False)
        st = vc.stage_times()
        res = vc.results(clusters=False) if name == "with_cut" else None
        vc.close()
        runs = max(1, st.pop("runs"))
        chain_ms = sum(st.values()) / runs
        out[name] = {"chain_ms": chain_ms, "events_per_s": n / (chain_ms / 1e3), "tracks": t}
        if res is not None:
            gec_ms = st["global_event_cut"] / runs
            b = gec_bytes(ut, sf)
            out["selected"] = res["n_selected"]
            out["gec_stage_ms"] = gec_ms
            out["gec_events_per_s"] = n / (gec_ms / 1e3)
            out["gec_algorithmic_bytes_per_event"] = b / n
            out["gec_achieved_gbs"] = b / (gec_ms / 1e3) / 1e9
    try:
        import oracle
        from oracle import gec_oracle
        if os.path.exists(oracle.REF_GPU_LIB):
            counts, _, _ = gec_oracle.run(ut, sf)
            if np.all(counts[:, 1] < gec_oracle.MAX_CLUSTERS):  # see ref_harness.cu
                sel, ms = oracle.ref_gec_run(ut, sf, reps=5, timed=True)
                out["reference_kernel_ms"] = ms
                out["reference_kernel_events_per_s"] = n / (ms / 1e3)
                out["reference_selected"] = int(sel.size)
    except Exception as ex:
        out["reference_error"] = str(ex)
    return out


# ---------------------------------------------------------------------------
# reference arm: the CPU implementation on the host cores
# ---------------------------------------------------------------------------
def run_reference(args):
    import oracle
    threads = os.cpu_count() or 1
    geo = events.load_geometry()
    sample = args.reference_sample
    b = events.generate_config(WORKLOAD, n_events=sample, threads=threads, with_mc=False)
    for _ in range(args.warmup):
        oracle.run(b, geo, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.run(b, geo, threads=threads)
        times.append(time.perf_counter() - t0)
    value = sample * args.steps / sum(times)
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD}: bounded sample of {sample} events per step (first events of the "
                               f"1,000,000-event nu ~ U(2,20) workload)",
                   "mode": "plain (the reference has no learned pruning)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample} events per step, full chain"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    global BUCKET, CHUNK
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--events", type=int, default=N_EVENTS, help="events per GPU (default: the 1,000,000 workload)")
    ap.add_argument("--cpu-sample", type=int, default=16384)
    ap.add_argument("--reference-sample", type=int, default=8192)
    ap.add_argument("--quality-events", type=int, default=131072, help="MC-checked events of the workload head")
    ap.add_argument("--streams", type=int, default=2, help="contexts / streams that batches alternate between")
    ap.add_argument("--batch", type=int, default=BUCKET, help="events per batch (one CUDA graph per batch)")
    ap.add_argument("--weights", default=None, help="scorer weights (default: the committed file)")
    ap.add_argument("--retrain", action="store_true", help="train the scorer here instead of loading it")
    ap.add_argument("--no-extras", action="store_true", help="skip the CPU baseline and reference-GPU legs")
    ap.add_argument("--no-ceiling", action="store_true", help="skip the per-stage / pruning-ceiling leg")
    ap.add_argument("--e2e-contexts", type=int, default=E2E_CONTEXTS,
                    help="contexts (and streams) in rotation in the end-to-end leg")
    ap.add_argument("--no-operating-points", action="store_true",
                    help="skip the timed form that scores every candidate")
    ap.add_argument("--e2e-depth", type=int, default=1,
                    help="end-to-end leg: batches launched before the oldest is read back (< contexts)")
    ap.add_argument("--batched-events", type=int, default=500_000,
                    help="events of the nu ~ U(2,15) leg in 1k/4k/16k-event batches (0: skip)")
    ap.add_argument("--high-occ-events", type=int, default=200_000,
                    help="events of the nu = 15, 10%% noisy leg (0: skip)")
    args = ap.parse_args()
    BUCKET, CHUNK = args.batch, 4 * args.batch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    result, chunks = run_ours(args, rank, world, local_rank)
    if rank == 0 and not args.no_extras:
        threads = os.cpu_count() or 1
        try:
            result["cpu_baseline"], sample = cpu_baseline(min(args.cpu_sample, args.events), threads)
        except Exception as ex:
            result["cpu_baseline"] = {"error": str(ex)}
            sample = None
        if world == 1:
            try:
                b0 = chunks[0].subset(0, min(SIDE_BATCH, chunks[0].n_events))
                result["reference_gpu_b200"] = reference_gpu(b0)
            except Exception as ex:
                result["reference_gpu_b200"] = {"error": str(ex)}
            try:
                result["pv"] = pv_leg(chunks[0].subset(0, min(SIDE_BATCH, chunks[0].n_events)),
                                      result["config"]["search_mapping"]["block_above_clusters"])
            except Exception as ex:
                result["pv"] = {"error": str(ex)}
            for key, cfg_name, n_ev, sizes in (("batched_500k", "batched_500k", args.batched_events,
                                                 (1000, 4000, 16000)),
                                                ("high_occupancy_200k", "high_occupancy_200k", args.high_occ_events,
                                                 (BUCKET,))):
                if n_ev <= 0:
                    continue
                try:
                    import torch
                    result[key] = workload_leg(cfg_name, n_ev, sizes, result["config"]["search_mapping"]["block_above_clusters"],
                                               result["config"]["decode_block"]["warps"], threads, torch)
                except Exception as ex:
                    result[key] = {"error": str(ex)}
            try:
                result["global_event_cut"] = gec_leg(chunks[0].subset(0, min(SIDE_BATCH, chunks[0].n_events)),
                                                     result["config"]["search_mapping"]["block_above_clusters"],
                                                     result["config"]["decode_block"]["warps"])
            except Exception as ex:
                result["global_event_cut"] = {"error": str(ex)}
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Small fixed workload for profiler captures: one batch of events of a synthetic workload
(default nu ~ U(2,15)), run `--runs` times through the chain (device-resident input, no
graphs, default output capacities: 400 tracks per event).

python -m cuda_hlt_b200.profile_case [--events 8192] [--runs 2] [--block-threshold N] [--mode plain|pruned] [--pv]
                                     [--gec] [--every-candidate]

--block-threshold: events with more clusters than N use the block-per-event search, the
others the warp-per-event one (1536 is the context default; 16384 sends every event to
the warp search).
--every-candidate: in the pruned mode, the committed scorer with its gates open (every event
and every seeding candidate scored).
"""
import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--events", type=int, default=8192)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--config", default="batched_500k")
    ap.add_argument("--block-threshold", type=int, default=1536)
    ap.add_argument("--mode", default="plain", choices=["plain", "pruned"])
    ap.add_argument("--pv", action="store_true", help="append the beamline PV stage")
    ap.add_argument("--every-candidate", action="store_true",
                    help="pruned mode: score every event and every seeding candidate")
    ap.add_argument("--gec", action="store_true",
                    help="global event cut in front of the chain, on synthetic UT / SciFi events (seed 0)")
    args = ap.parse_args()
    import torch
    from cuda_hlt_b200 import chain, events
    b = events.generate_config(args.config, n_events=args.events, with_mc=False)
    raw = torch.from_numpy(b.raw).cuda()
    off = torch.from_numpy(b.offsets.view(np.int64)).cuda()
    gec = None
    if args.gec:
        ut, sf = events.generate_ut_scifi(b, seed=0)
        gec = [torch.from_numpy(a).cuda() for a in (ut.raw, ut.offsets.view(np.int64), sf.raw,
                                                     sf.offsets.view(np.int64))]
    vc = chain.VeloChain(max_events=args.events, max_raw_bytes=int(b.raw.size) + 4096)
    vc.set_block_threshold(args.block_threshold)
    vc.set_pv(args.pv)
    if args.mode == "pruned":
        from cuda_hlt_b200 import mlp, train_scorer
        w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
        if args.every_candidate:
            w.min_pairs = 0
            w.min_event_clusters = 0
        vc.set_mlp(w)
        vc.set_mode(chain.MODE_PRUNED)
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(args.runs):
        if gec is None:
            vc.run_device(raw.data_ptr(), off.data_ptr(), args.events, s)
        else:
            vc.run_gec_device(raw.data_ptr(), off.data_ptr(), *[g.data_ptr() for g in gec], args.events, stream=s)
    t, h, c = vc.sync()
    vc.close()
    print(f"profile_case ({args.mode}): {args.events} events, {c} clusters, {t} tracks, {h} track hits, {b.raw.size} raw bytes")


if __name__ == "__main__":
    main()

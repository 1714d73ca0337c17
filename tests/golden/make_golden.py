"""Generates the committed fixtures under tests/golden/.

  minbias/VP/*.bin, minbias/UT/*.bin, minbias/FTCluster/*.bin, minbias/MC_tracks/*.bin,
  minbias/mdf/*.mdf
      the 10 real minbias events shipped with the reference (input/minbias/banks/{VP,UT,
      FTCluster}, input/minbias/MC_info/tracks and input/minbias/banks/mdf), copied as data:
      raw banks, their MC truth, and the same events as an MDF file (all banks, compressed).
  ref_gpu_*.npz
      outputs of the reference's own CUDA kernels (oracle/_ref/libvelo_ref_gpu.so) on the
      minbias events and on seeded synthetic events; written by `--ref-gpu` on a GPU box
      (the reference tree is not needed there: the library is prebuilt).
  ref_gec.npz
      the events the reference's global_event_cut kernel selects on the minbias events and on
      GEC_SYNTH_EVENTS seeded synthetic events (gec_synthetic_batches); written by
      `--ref-gec OUTDIR` on a GPU box.

Usage: python tests/golden/make_golden.py [--minbias] [--ref-gpu OUTDIR [--only NAME,...]] [--ref-gec OUTDIR]
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
# the reference tree (read only by --minbias): VELO_REFERENCE_TREE, else a checkout named
# "reference" beside this repository
REF = os.environ.get("VELO_REFERENCE_TREE", os.path.normpath(os.path.join(ROOT, os.pardir, "reference")))


def copy_minbias():
    for sub, dst in (("banks/VP", "VP"), ("banks/UT", "UT"), ("banks/FTCluster", "FTCluster"),
                     ("MC_info/tracks", "MC_tracks"), ("banks/mdf", "mdf")):
        src = os.path.join(REF, "input/minbias", sub)
        out = os.path.join(HERE, "minbias", dst)
        os.makedirs(out, exist_ok=True)
        for f in sorted(os.listdir(src)):
            shutil.copyfile(os.path.join(src, f), os.path.join(out, f))


def synthetic_batches():
    from cuda_hlt_b200 import events
    # 64 events of the 1,000-event nu=7.6 workload (seed 0), 32 events of the
    # nu ~ U(2,15) workload and 64 of the nu ~ U(2,20) workload (seed 4, about a quarter of
    # them above nu = 15), first events of each stream.
    return {"plain": events.generate_config("plain_1k", n_events=64),
            "batched": events.generate_config("batched_500k", n_events=32),
            "pruned1m": events.generate_config("pruned_1m", n_events=64)}


def compact_reference(res, n_events):
    """Compact form of the reference outputs: valid clusters per module in order, tracks and
    both state sets."""
    import numpy as np
    import oracle
    NM = 52
    sel = []
    for e in range(n_events):
        for m in range(NM):
            s, n = int(res["module_start"][e * NM + m]), int(res["module_num"][e * NM + m])
            sel.append(np.arange(s, s + n))
    sel = np.concatenate(sel) if sel else np.zeros(0, np.int64)
    out = dict(module_num=res["module_num"], cl_x=res["x"][sel], cl_y=res["y"][sel], cl_z=res["z"][sel],
               cl_phi=res["phi"][sel], cl_id=res["id"][sel], atomics=res["atomics"],
               track_hit_number=res["track_hit_number"], hit_x=res["hit_x"], hit_y=res["hit_y"],
               hit_z=res["hit_z"], hit_id=res["hit_id"], candidate_num=res["candidate_num"],
               weak_num=res["weak_num"])
    for key in ("states", "kalman"):
        st = oracle.ref_decode_states(res, key)
        for f, v in st.items():
            out[f"{key}_{f}"] = v
    return out


def ref_gpu(outdir, only=None):
    import numpy as np
    import oracle
    from cuda_hlt_b200 import events
    geo = events.load_geometry()
    batches = {"minbias": events.read_bank_folder(os.path.join(HERE, "minbias", "VP"))}
    batches.update(synthetic_batches())
    if only:
        batches = {k: v for k, v in batches.items() if k in only}
    os.makedirs(outdir, exist_ok=True)
    for name, b in batches.items():
        res, _ = oracle.ref_gpu_run(b, geo)
        np.savez_compressed(os.path.join(outdir, f"ref_gpu_{name}.npz"), **compact_reference(res, b.n_events))
        print(name, b.n_events, "events", res["T"], "tracks")


GEC_SYNTH_EVENTS = 2048


def gec_synthetic_batches():
    """(UT, SciFi) batches of the first GEC_SYNTH_EVENTS events of the nu ~ U(2,20) workload
    (generate_ut_scifi, seed 5) without the events whose UT hit total reaches the cut (the
    reference kernel is run only on events where every thread reaches every barrier)."""
    import numpy as np
    from cuda_hlt_b200 import events
    from oracle import gec_oracle
    vp = events.generate_config("pruned_1m", n_events=GEC_SYNTH_EVENTS, with_mc=False)
    ut, sf = events.generate_ut_scifi(vp, seed=5)
    counts, _, _ = gec_oracle.run(ut, sf)
    keep = np.flatnonzero(counts[:, 1] < gec_oracle.MAX_CLUSTERS)
    return pick(ut, keep), pick(sf, keep), keep


def pick(batch, idx):
    """A batch of the events `idx` of `batch`, in that order."""
    import numpy as np
    from cuda_hlt_b200 import events
    raws = [batch.event(int(i)) for i in idx]
    off = np.zeros(len(raws) + 1, np.uint64)
    off[1:] = np.cumsum([r.size for r in raws])
    return events.EventBatch(np.concatenate(raws) if raws else np.zeros(0, np.uint8), off)


def minbias_gec_batches():
    from cuda_hlt_b200 import events
    return (events.read_bank_folder(os.path.join(HERE, "minbias", "UT")),
            events.read_bank_folder(os.path.join(HERE, "minbias", "FTCluster")))


def ref_gec(outdir):
    import numpy as np
    import oracle
    ut, sf = minbias_gec_batches()
    sut, ssf, keep = gec_synthetic_batches()
    out = dict(minbias_selected=np.sort(oracle.ref_gec_run(ut, sf)),
               synthetic_events=keep.astype(np.uint32),
               synthetic_selected=np.sort(oracle.ref_gec_run(sut, ssf)))
    os.makedirs(outdir, exist_ok=True)
    np.savez_compressed(os.path.join(outdir, "ref_gec.npz"), **out)
    print("gec", {k: v.size for k, v in out.items()})


if __name__ == "__main__":
    if "--minbias" in sys.argv:
        copy_minbias()
    if "--ref-gpu" in sys.argv:
        only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else None
        ref_gpu(sys.argv[sys.argv.index("--ref-gpu") + 1], only)
    if "--ref-gec" in sys.argv:
        ref_gec(sys.argv[sys.argv.index("--ref-gec") + 1])

"""Generates the committed fixtures under tests/golden/.

  minbias/VP/*.bin, minbias/MC_tracks/*.bin, minbias/mdf/*.mdf
      the 10 real minbias events shipped with the reference (input/minbias/banks/VP,
      input/minbias/MC_info/tracks and input/minbias/banks/mdf), copied as data: raw VP
      banks, their MC truth, and the same events as an MDF file (all banks, compressed).
  ref_gpu_*.npz
      outputs of the reference's own CUDA kernels (oracle/_ref/libvelo_ref_gpu.so) on the
      minbias events and on seeded synthetic events; written by `--ref-gpu` on a GPU box
      (the reference tree is not needed there: the library is prebuilt).

Usage: python tests/golden/make_golden.py [--minbias] [--ref-gpu OUTDIR]
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = "/root/reference"


def copy_minbias():
    for sub, dst in (("banks/VP", "VP"), ("MC_info/tracks", "MC_tracks"), ("banks/mdf", "mdf")):
        src = os.path.join(REF, "input/minbias", sub)
        out = os.path.join(HERE, "minbias", dst)
        os.makedirs(out, exist_ok=True)
        for f in sorted(os.listdir(src)):
            shutil.copyfile(os.path.join(src, f), os.path.join(out, f))


def synthetic_batches():
    from cuda_hlt_b200 import events
    # 64 events of the 1,000-event nu=7.6 workload (seed 0) and 32 events of the
    # nu ~ U(2,15) workload, first events of each stream.
    return {"plain": events.generate_config("plain_1k", n_events=64),
            "batched": events.generate_config("batched_500k", n_events=32)}


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


def ref_gpu(outdir):
    import numpy as np
    import oracle
    from cuda_hlt_b200 import events
    geo = events.load_geometry()
    batches = {"minbias": events.read_bank_folder(os.path.join(HERE, "minbias", "VP"))}
    batches.update(synthetic_batches())
    os.makedirs(outdir, exist_ok=True)
    for name, b in batches.items():
        res, _ = oracle.ref_gpu_run(b, geo)
        np.savez_compressed(os.path.join(outdir, f"ref_gpu_{name}.npz"), **compact_reference(res, b.n_events))
        print(name, b.n_events, "events", res["T"], "tracks")


if __name__ == "__main__":
    if "--minbias" in sys.argv:
        copy_minbias()
    if "--ref-gpu" in sys.argv:
        ref_gpu(sys.argv[sys.argv.index("--ref-gpu") + 1])

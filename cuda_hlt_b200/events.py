"""Event batches: seeded synthetic VELO events and the raw-bank folder reader.

A batch is raw VP banks concatenated with u64 byte offsets (the reference concatenates
events with u32 offsets, main/src/InputReader.cpp:28-57; u64 lets a batch exceed 4 GiB),
plus the MC truth of each event in the MC_info layout (checker/tracking/src/MCEvent.cpp:16-92).
"""
import ctypes as C
import glob
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class EventBatch:
    raw: np.ndarray            # uint8, concatenated raw events
    offsets: np.ndarray        # uint64, n_events + 1
    mc: np.ndarray = None      # uint8, concatenated MC truth blobs
    mc_offsets: np.ndarray = None
    truth_clusters: np.ndarray = None
    names: list = field(default_factory=list)

    @property
    def n_events(self):
        return len(self.offsets) - 1

    def event(self, i):
        return self.raw[self.offsets[i]:self.offsets[i + 1]]

    def subset(self, start, stop):
        o = self.offsets[start:stop + 1]
        raw = self.raw[o[0]:o[-1]]
        mc = mco = tc = None
        if self.mc is not None:
            m = self.mc_offsets[start:stop + 1]
            mc, mco = self.mc[m[0]:m[-1]], m - m[0]
        if self.truth_clusters is not None:
            tc = self.truth_clusters[start:stop]
        return EventBatch(raw, o - o[0], mc, mco, tc, self.names[start:stop] if self.names else [])


# Generator settings of the synthetic workloads. Pileup nu sets the number of visible
# primary vertices ~ Poisson(0.7 nu), each with ~Poisson(20) straight tracks.
CONFIGS = {
    # 1,000 events, seed 0, nu = 7.6 (~2,400 clusters/event)
    "plain_1k": dict(seed=0, nu_min=7.6, nu_max=7.6, n_events=1000),
    # 500,000 events, nu ~ U(2,15) per event (500-6,000 clusters/event)
    "batched_500k": dict(seed=0, nu_min=2.0, nu_max=15.0, n_events=500_000),
    # 200,000 events at nu = 15, 10% of events with 3x the noise-pixel rate
    "high_occupancy_200k": dict(seed=2, nu_min=15.0, nu_max=15.0, noisy_event_fraction=0.1, noisy_factor=3.0,
                                n_events=200_000),
    # learned-scorer training sample, nu ~ U(2,15), seed 1
    "mlp_train": dict(seed=1, nu_min=2.0, nu_max=15.0, n_events=200_000),
    # pruned vs plain, 1,000,000 events at nu ~ U(2,20)
    "pruned_1m": dict(seed=4, nu_min=2.0, nu_max=20.0, n_events=1_000_000),
}


def gen_config(**overrides):
    lib = _lib.host_lib()
    cfg = _lib.VeloGenConfig()
    lib.velo_gen_default_config(C.byref(cfg))
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


def load_geometry(path=None):
    data = np.fromfile(path or _lib.GEOMETRY_PATH, dtype=np.uint8)
    if data.size != 19456:
        raise ValueError(f"geometry has {data.size} bytes, expected 19456")
    return data


def generate(n_events, first_event=0, threads=0, geometry=None, with_mc=True, **cfg_overrides):
    """Generates n_events synthetic events (event i depends only on seed and first_event+i)."""
    lib = _lib.host_lib()
    geometry = load_geometry() if geometry is None else geometry
    cfg = gen_config(**cfg_overrides)
    handle = C.c_void_p()
    rc = lib.velo_gen_create(C.byref(cfg), geometry.ctypes.data, first_event, n_events, threads, C.byref(handle))
    if rc != 0:
        raise RuntimeError(f"velo_gen_create failed: {rc}")
    try:
        raw = np.empty(lib.velo_gen_raw_bytes(handle), dtype=np.uint8)
        offsets = np.empty(n_events + 1, dtype=np.uint64)
        mc = np.empty(lib.velo_gen_mc_bytes(handle), dtype=np.uint8) if with_mc else None
        mco = np.empty(n_events + 1, dtype=np.uint64) if with_mc else None
        tc = np.empty(n_events, dtype=np.uint32)
        lib.velo_gen_copy(handle, raw.ctypes.data, offsets.ctypes.data,
                          mc.ctypes.data if with_mc else None, mco.ctypes.data if with_mc else None, tc.ctypes.data)
    finally:
        lib.velo_gen_destroy(handle)
    return EventBatch(raw, offsets, mc, mco, tc)


def generate_config(name, n_events=None, first_event=0, threads=0, with_mc=True):
    c = dict(CONFIGS[name])
    n = c.pop("n_events") if n_events is None else n_events
    c.pop("n_events", None)
    return generate(n, first_event=first_event, threads=threads, with_mc=with_mc, **c)


def read_bank_folder(vp_folder, mc_folder=None, limit=None):
    """Reads a folder of per-event raw VP bank files (and optional MC_info/tracks files
    with the same names), as main/src/InputReader.cpp:28-57 does."""
    files = sorted(glob.glob(os.path.join(vp_folder, "*.bin")))[:limit]
    raws = [np.fromfile(f, dtype=np.uint8) for f in files]
    offsets = np.zeros(len(raws) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([r.size for r in raws])
    batch = EventBatch(np.concatenate(raws) if raws else np.zeros(0, np.uint8), offsets,
                       names=[os.path.basename(f) for f in files])
    if mc_folder:
        mcs = [np.fromfile(os.path.join(mc_folder, os.path.basename(f)), dtype=np.uint8) for f in files]
        mo = np.zeros(len(mcs) + 1, dtype=np.uint64)
        mo[1:] = np.cumsum([m.size for m in mcs])
        batch.mc, batch.mc_offsets = np.concatenate(mcs), mo
    return batch


# LHCb raw bank type numbers (mdf/include/raw_bank.hpp) of the detectors the readers take
BANK_TYPES = {"VP": 63, "FTCluster": 64, "UT": 66, "Muon": 13}


def read_mdf(path, first_event=0, max_events=None, bank="VP"):
    """Raw banks of one type (VP by default; "UT", "FTCluster", "Muon") of the events of an
    MDF file (velo_mdf_read_banks, the counterpart of MDF::read_events) or of every *.mdf
    file of a folder in name order; event names are "run_event" from the ODIN bank."""
    import ctypes as C
    lib = _lib.host_lib()
    bank_type = BANK_TYPES[bank]
    files = sorted(glob.glob(os.path.join(path, "*.mdf"))) if os.path.isdir(path) else [path]
    raws, names, skip = [], [], first_event
    left = (1 << 62) if max_events is None else max_events
    for f in files:
        h = C.c_void_p()
        rc = lib.velo_mdf_read_banks(f.encode(), skip, left, bank_type, C.byref(h))
        if rc != 0:
            raise ValueError(f"velo_mdf_read_banks({f}, {bank}) failed with code {rc}")
        try:
            n = lib.velo_mdf_count(h)
            raw = np.zeros(lib.velo_mdf_raw_bytes(h), np.uint8)
            off = np.zeros(n + 1, np.uint64)
            run = np.zeros(n, np.uint32)
            evn = np.zeros(n, np.uint64)
            lib.velo_mdf_copy(h, raw.ctypes.data, off.ctypes.data, run.ctypes.data, evn.ctypes.data)
        finally:
            lib.velo_mdf_free(h)
        raws += [raw[off[i]:off[i + 1]] for i in range(n)]
        names += [f"{run[i]}_{evn[i]}" for i in range(n)]
        left -= n
        skip = 0  # counted in the first file only
        if left <= 0:
            break
    offsets = np.zeros(len(raws) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([r.size for r in raws])
    return EventBatch(np.concatenate(raws) if raws else np.zeros(0, np.uint8), offsets, names=names)


# Synthetic UT and SciFi (FTCluster) raw events for the global event cut. Occupancy follows
# the VELO event's: hits ~ Poisson(rate x VP raw words), with the rates of the ten minbias
# events shipped with the reference (UT hits / VP words = 0.38, SciFi cluster estimate /
# VP words = 1.41 over the ten). Bank counts are those of the same events: 180 UT banks,
# 240 SciFi banks. UT bank: source id, a word whose low 16 bits hold the hit count, one
# 32-bit word per hit (UTRaw.cuh; the minbias banks hold about 4 bytes per hit); SciFi bank:
# source id, then 16-bit clusters padded to 4 bytes (SciFiRaw.cuh). Hit and cluster words are
# random: the cut reads counts and sizes only.
UT_BANKS, SCIFI_BANKS = 180, 240
UT_PER_VP_WORD, SCIFI_PER_VP_WORD = 0.38, 1.41


def _banks_to_raw(counts, header_words, items_per_word, rng):
    """Raw events (u32 layout: number of banks, bank byte offsets [B + 1], banks) from a
    [N, B] array of items per bank, `items_per_word` items to a 32-bit word; each bank starts
    with `header_words` words, the source id and, with two header words, the item count."""
    n, nb = counts.shape
    words = header_words + (counts + items_per_word - 1) // items_per_word  # [N, B]
    ev_words = 1 + (nb + 1) + words.sum(axis=1)                  # [N]
    ev_start = np.zeros(n + 1, np.int64)
    ev_start[1:] = np.cumsum(ev_words)
    raw = rng.integers(0, 1 << 32, size=int(ev_start[-1]), dtype=np.uint64).astype(np.uint32)
    bank_off = np.zeros((n, nb + 1), np.int64)                   # word offsets inside the payload
    bank_off[:, 1:] = np.cumsum(words, axis=1)
    raw[ev_start[:-1]] = nb
    cols = np.arange(nb + 1)
    raw[(ev_start[:-1, None] + 1 + cols[None, :]).ravel()] = (4 * bank_off).astype(np.uint32).ravel()
    bank_at = ev_start[:-1, None] + 1 + (nb + 1) + bank_off[:, :-1]   # first word of each bank
    raw[bank_at.ravel()] = np.tile(np.arange(nb, dtype=np.uint32), n)
    if header_words == 2:
        raw[(bank_at + 1).ravel()] = counts.astype(np.uint32).ravel()
    offsets = (4 * ev_start).astype(np.uint64)
    return EventBatch(raw.view(np.uint8), offsets)


def generate_ut_scifi(vp_batch, seed=0):
    """(UT batch, SciFi batch) for the events of `vp_batch`, seeded."""
    rng = np.random.default_rng(seed)
    vp_words = np.diff(vp_batch.offsets).astype(np.float64) / 4.0
    ut = rng.poisson((UT_PER_VP_WORD * vp_words / UT_BANKS)[:, None], size=(vp_batch.n_events, UT_BANKS))
    sf = rng.poisson((SCIFI_PER_VP_WORD * vp_words / SCIFI_BANKS)[:, None], size=(vp_batch.n_events, SCIFI_BANKS))
    return _banks_to_raw(ut, 2, 1, rng), _banks_to_raw(sf, 1, 2, rng)


def validate(batch):
    """Per-event raw-format check; returns a bool array (True = well formed)."""
    lib = _lib.host_lib()
    ok = np.zeros(batch.n_events, dtype=bool)
    for i in range(batch.n_events):
        ev = batch.event(i)
        ok[i] = lib.velo_validate_raw_event(ev.ctypes.data, ev.size) == 0
    return ok


def sp_luts():
    lib = _lib.host_lib()
    pat = np.zeros(256, np.uint8)
    siz = np.zeros(256, np.uint8)
    fx = np.zeros(512, np.float32)
    fy = np.zeros(512, np.float32)
    lib.velo_build_sp_luts(pat.ctypes.data, siz.ctypes.data, fx.ctypes.data, fy.ctypes.data)
    return pat, siz, fx, fy

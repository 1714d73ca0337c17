"""Python mirror of the VELO stage, over the C ABI of libvelo_b200.so.

The reference drives this stage as a compile-time sequence of algorithms
(configuration/sequences/Velo.h:5-18): velo_estimate_input_size_t, prefix_sum_velo_clusters_t,
velo_masked_clustering_t, velo_calculate_phi_and_sort_t, velo_fill_candidates_t,
velo_search_by_triplet_t, velo_weak_tracks_adder_t, copy_and_prefix_sum_single_block_velo_t,
copy_velo_track_hit_number_t, prefix_sum_velo_track_hit_number_t, consolidate_velo_tracks_t,
velo_kalman_fit_t. Here the whole sequence is one call, VeloChain.run(), producing the
sequence's output arguments (stream/setup/include/OutputArguments.cuh:16-34) in the
reference layouts. Errors raise VeloError (the reference throws std::invalid_argument from
cudaCheck, main/include/CudaCommon.h:10-18).
"""
import ctypes as C

import numpy as np

from . import _lib

SEQUENCE = (
    "velo_estimate_input_size_t",
    "prefix_sum_velo_clusters_t",
    "velo_masked_clustering_t",
    "velo_calculate_phi_and_sort_t",
    "velo_fill_candidates_t",
    "velo_search_by_triplet_t",
    "velo_weak_tracks_adder_t",
    "copy_and_prefix_sum_single_block_velo_t",
    "copy_velo_track_hit_number_t",
    "prefix_sum_velo_track_hit_number_t",
    "consolidate_velo_tracks_t",
    "velo_kalman_fit_t",
)

STAGES = ("decode_cluster_sort", "fill_candidates", "search_by_triplet", "event_scan", "consolidate_fit", "pv_beamline",
          "global_event_cut")
PV_MAX_VERTICES = 32
# VeloPvVertex (PV::Vertex layout)
PV_VERTEX = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("chi2", "<f4"), ("ndof", "<i4"), ("n_tracks", "<u4"),
                      ("cov00", "<f4"), ("cov10", "<f4"), ("cov11", "<f4"), ("cov20", "<f4"), ("cov21", "<f4"),
                      ("cov22", "<f4"), ("n_tracks_unused", "<i4")])
MODE_PLAIN, MODE_PRUNED, MODE_LABELS = 0, 1, 2
MAP_AUTO, MAP_BLOCK, MAP_WARP = 0, 1, 2
N_MODULES = 52
STATE_FIELDS = ("x", "y", "tx", "ty", "c00", "c20", "c22", "c11", "c31", "c33", "chi2", "z")

STATUS = {
    "bad_raw": 1 << 0, "module_overflow": 1 << 1, "hit_overflow": 1 << 2, "candidate_overflow": 1 << 3,
    "track_overflow": 1 << 4, "ttf_overflow": 1 << 5, "weak_overflow": 1 << 6, "h1_overflow": 1 << 7,
    "big_sp_index": 1 << 8, "mlp_fallback": 1 << 9, "empty_module_read": 1 << 10, "seed_tie": 1 << 11,
    "block_stage_timeout": 1 << 12, "pv_overflow": 1 << 13, "not_selected": 1 << 14,
}
GEC_MAX_CLUSTERS = 9750  # maxSciFiUTClusters (cuda/global_event_cut/include/GlobalEventCut.cuh:9)
GEC_PASS, GEC_MALFORMED = 1, 2
# Flags of events whose reference result depends on unchecked buffer spills, reads outside
# a module or the order of atomics (exact float ties).
REFERENCE_UNDEFINED = sum(STATUS[k] for k in ("module_overflow", "candidate_overflow", "track_overflow",
                                              "ttf_overflow", "weak_overflow", "h1_overflow", "empty_module_read",
                                              "seed_tie", "hit_overflow"))


class VeloError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise VeloError(f"{what} failed with code {rc}")


def decode_states(blob, T):
    """Velo::Consolidated::States SoA (VeloConsolidated.cuh:68-144) -> dict of arrays."""
    f = np.frombuffer(blob, dtype=np.float32, count=12 * T).reshape(12, T) if T else np.zeros((12, 0), np.float32)
    out = {k: f[i].copy() for i, k in enumerate(STATE_FIELDS)}
    out["backward"] = np.frombuffer(blob, dtype=np.uint8, count=T, offset=48 * T).astype(bool) if T else \
        np.zeros(0, bool)
    return out


class VeloChain:
    def __init__(self, max_events, max_raw_bytes, device=0, mode=MODE_PLAIN, mapping=MAP_AUTO, use_graphs=False,
                 geometry=None, max_tracks=0, max_track_hits=0, decode_warps=None):
        from . import events
        self.lib = _lib.gpu_lib()
        geometry = events.load_geometry() if geometry is None else geometry
        cfg = _lib.VeloConfig(max_events=max_events, max_raw_bytes=max_raw_bytes, max_tracks=max_tracks,
                              max_track_hits=max_track_hits, device=device, mode=mode, mapping=mapping,
                              use_graphs=int(use_graphs))
        self.ctx = C.c_void_p()
        _check(self.lib.velo_create(C.byref(cfg), geometry.ctypes.data, geometry.size, C.byref(self.ctx)),
               "velo_create")
        self.out = _lib.VeloOutputs()
        self.n_events = 0
        if decode_warps is not None:
            self.set_decode_warps(decode_warps)

    def close(self):
        if self.ctx:
            self.lib.velo_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- running ----
    def run_host(self, batch, stream=0):
        """Copies the batch from host memory and runs the chain (asynchronous)."""
        self.n_events = batch.n_events
        _check(self.lib.velo_run_host(self.ctx, batch.raw.ctypes.data, batch.offsets.ctypes.data, batch.n_events,
                                      C.c_void_p(stream), C.byref(self.out)), "velo_run_host")

    def run_host_u32(self, raw, offsets32, stream=0):
        """Host batch with u32 byte offsets (the reference's input format): raw uint8 array,
        offsets32 uint32 array of n_events + 1 entries."""
        offsets32 = np.ascontiguousarray(offsets32, np.uint32)
        self.n_events = len(offsets32) - 1
        _check(self.lib.velo_run_host_u32(self.ctx, raw.ctypes.data, offsets32.ctypes.data, self.n_events,
                                          C.c_void_p(stream), C.byref(self.out)), "velo_run_host_u32")

    def run_device_u32(self, raw_ptr, offsets32_ptr, n_events, stream=0):
        """Device-resident input with u32 offsets[n+1]."""
        self.n_events = n_events
        _check(self.lib.velo_run_u32(self.ctx, C.c_void_p(raw_ptr), C.c_void_p(offsets32_ptr), n_events,
                                     C.c_void_p(stream), C.byref(self.out)), "velo_run_u32")

    def graph_count(self):
        n = C.c_uint32()
        _check(self.lib.velo_graph_count(self.ctx, C.byref(n)), "velo_graph_count")
        return n.value

    def run_device(self, raw_ptr, offsets_ptr, n_events, stream=0):
        """Runs on device-resident input (raw bytes, u64 offsets[n+1])."""
        self.n_events = n_events
        _check(self.lib.velo_run(self.ctx, C.c_void_p(raw_ptr), C.c_void_p(offsets_ptr), n_events,
                                 C.c_void_p(stream), C.byref(self.out)), "velo_run")

    def run_gec_host(self, batch, ut, scifi, max_clusters=GEC_MAX_CLUSTERS, stream=0):
        """Global event cut on the UT and SciFi batches (EventBatch of the same events), then
        the chain on the selected events: positions 0 .. n_selected - 1 hold raw events
        event_list[0 ..] (results() adds both)."""
        if not (batch.n_events == ut.n_events == scifi.n_events):
            raise VeloError("VP, UT and SciFi batches must hold the same events")
        self.n_events = batch.n_events
        g = _lib.VeloGecInput(ut.raw.ctypes.data, ut.offsets.ctypes.data, scifi.raw.ctypes.data,
                              scifi.offsets.ctypes.data, int(max_clusters))
        _check(self.lib.velo_run_gec_host(self.ctx, batch.raw.ctypes.data, batch.offsets.ctypes.data, C.byref(g),
                                          batch.n_events, C.c_void_p(stream), C.byref(self.out)), "velo_run_gec_host")

    def run_gec_device(self, raw_ptr, offsets_ptr, ut_ptr, ut_offsets_ptr, scifi_ptr, scifi_offsets_ptr, n_events,
                       max_clusters=GEC_MAX_CLUSTERS, stream=0):
        """Same on device-resident inputs (u64 offsets[n+1] for each detector)."""
        self.n_events = n_events
        g = _lib.VeloGecInput(ut_ptr, ut_offsets_ptr, scifi_ptr, scifi_offsets_ptr, int(max_clusters))
        _check(self.lib.velo_run_gec(self.ctx, C.c_void_p(raw_ptr), C.c_void_p(offsets_ptr), C.byref(g), n_events,
                                     C.c_void_p(stream), C.byref(self.out)), "velo_run_gec")

    def sync(self, clusters=True):
        """Waits for the last run; returns (tracks, track hits, clusters or None)."""
        t, h, c = C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(self.lib.velo_sync(self.ctx, C.byref(t), C.byref(h), C.byref(c) if clusters else None), "velo_sync")
        return t.value, h.value, (c.value if clusters else None)

    def set_timing(self, on):
        _check(self.lib.velo_set_timing(self.ctx, int(on)), "velo_set_timing")

    def stage_times(self):
        """Device milliseconds per stage, summed over the launch sequences recorded since
        set_timing(True); 'runs' is the number of sequences summed."""
        n = len(STAGES)
        ms = (C.c_float * (n + 1))()
        _check(self.lib.velo_stage_times(self.ctx, ms, n + 1), "velo_stage_times")
        out = dict(zip(STAGES, list(ms)[:n]))
        out["runs"] = int(ms[n])
        return out

    def set_pv(self, enabled=True):
        """Appends the beamline primary-vertex finder to every run (velo_set_pv)."""
        _check(self.lib.velo_set_pv(self.ctx, int(bool(enabled))), "velo_set_pv")

    def set_mode(self, mode):
        """MODE_PLAIN (reference semantics), MODE_PRUNED (learned scorer, set_mlp first) or
        MODE_LABELS (the plain search's own labels, capture_labels first)."""
        _check(self.lib.velo_set_mode(self.ctx, int(mode)), "velo_set_mode")

    def capture_labels(self, ext=False, max_event_clusters=0xFFFFFFFF):
        """After a plain run (and sync): keeps the plain search's labels of every hit for
        runs in MODE_LABELS on the same batch (a perfect scorer; velo_capture_labels)."""
        _check(self.lib.velo_capture_labels(self.ctx, int(bool(ext)), int(max_event_clusters)), "velo_capture_labels")

    def set_mlp(self, weights):
        """Loads a VeloMlpWeights (see cuda_hlt_b200.mlp) for the pruned mode."""
        _check(self.lib.velo_set_mlp(self.ctx, C.byref(weights), C.sizeof(weights)), "velo_set_mlp")

    def set_block_threshold(self, clusters):
        """Events above `clusters` clusters use the block-per-event search, others the warp one."""
        _check(self.lib.velo_set_block_threshold(self.ctx, int(clusters)), "velo_set_block_threshold")

    def set_decode_warps(self, warps):
        """Decode block size: 4 or 8 warps per event."""
        _check(self.lib.velo_set_decode_warps(self.ctx, int(warps)), "velo_set_decode_warps")

    def launch_count(self):
        n = C.c_uint32()
        _check(self.lib.velo_last_launch_count(self.ctx, C.byref(n)), "velo_last_launch_count")
        return n.value

    # ---- reading results back ----
    def _down(self, ptr, dtype, count, offset_bytes=0):
        arr = np.empty(count, dtype=dtype)
        if count:
            _check(self.lib.velo_download(self.ctx, arr.ctypes.data, C.c_void_p(ptr + offset_bytes), arr.nbytes),
                   "velo_download")
        return arr

    def results(self, clusters=True):
        """Downloads the outputs of the last run (after sync) into numpy arrays."""
        N = self.n_events
        o = self.out
        atomics = self._down(o.atomics, np.uint32, 2 * N + 1)
        T = int(atomics[2 * N])
        thn = self._down(o.track_hit_number, np.uint32, T + 1)
        H = int(thn[T]) if T else 0
        hits = self._down(o.track_hits, np.uint8, 16 * H)
        kalman_raw = self._down(o.kalman_states, np.uint8, 52 * T)
        hv = hits.view(np.float32).reshape(4, H) if H else np.zeros((4, 0), np.float32)
        res = dict(
            atomics=atomics, n_tracks=atomics[:N], track_offsets=atomics[N:2 * N + 1], track_hit_number=thn,
            hit_x=hv[0], hit_y=hv[1], hit_z=hv[2], hit_id=hv[3].view(np.uint32),
            states=decode_states(self._down(o.states, np.uint8, 52 * T).tobytes(), T),
            kalman=decode_states(kalman_raw.tobytes(), T), kalman_raw=kalman_raw,
            status=self._down(o.status, np.uint32, N))
        if o.pv_vertices:
            M = PV_MAX_VERTICES
            res["pv_vertices"] = self._down(o.pv_vertices, np.uint8, N * M * PV_VERTEX.itemsize).view(PV_VERTEX).reshape(N, M)
            res["pv_count"] = self._down(o.pv_count, np.uint32, N)
            res["pv_zpeaks"] = self._down(o.pv_zpeaks, np.float32, N * M).reshape(N, M)
            res["pv_npeaks"] = self._down(o.pv_npeaks, np.uint32, N)
        if o.event_list:
            res["n_selected"] = int(self._down(o.n_selected, np.uint32, 1)[0])
            res["event_list"] = self._down(o.event_list, np.uint32, N)[:res["n_selected"]]
            res["gec_counts"] = self._down(o.gec_counts, np.uint32, 2 * N).reshape(N, 2)
            res["gec_flags"] = self._down(o.gec_flags, np.uint8, N)
        if clusters:
            res["module_start"] = self._down(o.module_hit_start, np.uint32, N * N_MODULES)
            res["module_num"] = self._down(o.module_hit_num, np.uint32, N * N_MODULES)
            span = int((res["module_start"] + res["module_num"]).max()) if N else 0
            xyzp = self._down(o.hit_xyzp, np.float32, 4 * span).reshape(span, 4)
            for i, k in enumerate(("x", "y", "z", "phi")):
                res["cluster_" + k] = np.ascontiguousarray(xyzp[:, i])
            res["cluster_id"] = self._down(o.hit_id, np.uint32, span)
            res["cluster_size"] = self._down(o.hit_size, np.uint8, span)
            if o.hit_keep:
                res["cluster_keep"] = self._down(o.hit_keep, np.uint8, span)
        return res


def event_clusters(res, e):
    """Per-module cluster arrays of event e from VeloChain.results()."""
    out = []
    for m in range(N_MODULES):
        s, n = int(res["module_start"][e * N_MODULES + m]), int(res["module_num"][e * N_MODULES + m])
        out.append({k: res["cluster_" + k][s:s + n] for k in ("x", "y", "z", "phi", "id", "size")})
    return out


def event_tracks(res, e):
    """Tracks of event e as tuples of LHCb ids (track hit order)."""
    t0, t1 = int(res["track_offsets"][e]), int(res["track_offsets"][e + 1])
    thn, ids = res["track_hit_number"], res["hit_id"]
    return [tuple(int(v) for v in ids[thn[t]:thn[t + 1]]) for t in range(t0, t1)]


def check_tracks(batch, res):
    """MC-truth efficiency and ghost rate of the tracks in `res` (VeloChain.results()) against
    the batch's MC_info blobs, with the reference's VELO checker categories
    (checker/tracking/src/TrackChecker.cpp:349-405): VeloCheckResult."""
    lib = _lib.host_lib()
    if batch.mc is None:
        raise VeloError("batch has no MC truth")
    evt = np.ascontiguousarray(res["track_offsets"], np.uint32)
    tho = np.ascontiguousarray(res["track_hit_number"], np.uint32)
    ids = np.ascontiguousarray(res["hit_id"], np.uint32)
    out = _lib.VeloCheckResult()
    _check(lib.velo_check_tracks(batch.mc.ctypes.data, batch.mc_offsets.ctypes.data, batch.n_events, evt.ctypes.data,
                                 tho.ctypes.data, ids.ctypes.data, C.byref(out)), "velo_check_tracks")
    return out

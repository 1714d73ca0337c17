"""ORACLE — test infrastructure only (imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py; never by the product package).

Bindings of:
  liboracle.so            CPU restatement of the reference VELO chain (velo_oracle.cpp)
  _ref/libvelo_ref_gpu.so the reference's own CUDA kernels (cuda/velo, cuda/utils/prefix_sum)
                          compiled from the reference tree for sm_100a, driven by ref_harness.cu
  _ref/libvelo_ref_x86.so the reference's x86 clustering (x86/velo/clustering)
All three are built by oracle/build.py.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libvelo_ref_gpu.so")
REF_X86_LIB = os.path.join(HERE, "_ref", "libvelo_ref_x86.so")
REF_CHECKER_LIB = os.path.join(HERE, "_ref", "libvelo_ref_checker.so")

NM = 52
F_BAD_RAW = 1 << 0
F_MODULE_OVF = 1 << 1
F_HIT_OVF = 1 << 2
F_CAND_OVF = 1 << 3
F_TRACK_OVF = 1 << 4
F_TTF_OVF = 1 << 5
F_WEAK_OVF = 1 << 6
F_H1_OVF = 1 << 7
F_BIG_SP = 1 << 8
F_SEED_TIE = 1 << 16
F_EMPTY_MODULE_READ = 1 << 17
# Events whose reference result is undefined (buffer spills into neighbouring events,
# reads outside a module, or exact float ties resolved by atomic order).
UNDEFINED_IN_REFERENCE = (F_MODULE_OVF | F_HIT_OVF | F_CAND_OVF | F_TRACK_OVF | F_TTF_OVF | F_WEAK_OVF | F_H1_OVF
                          | F_SEED_TIE | F_EMPTY_MODULE_READ)

STATE_FIELDS = ["x", "y", "tx", "ty", "c00", "c20", "c22", "c11", "c31", "c33", "chi2", "z", "backward"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"{ORACLE_LIB} missing: run oracle/build.py")
        L = C.CDLL(ORACLE_LIB)
        P = C.c_void_p
        L.oracle_run.argtypes = [P, P, C.c_uint32, P, C.c_int, C.c_int, C.POINTER(P)]
        L.oracle_run.restype = C.c_int
        L.oracle_destroy.argtypes = [P]
        L.oracle_sizes.argtypes = [P, P, P, P]
        L.oracle_copy_clusters.argtypes = [P] * 10
        L.oracle_copy_tracks.argtypes = [P] * 9
        L.oracle_sp_luts.argtypes = [P, P, P]
        _lib = L
    return _lib


class OracleResult:
    """Per-batch oracle output in numpy arrays."""

    def __init__(self, batch, geometry, threads=0, stages=2):
        L = lib()
        h = C.c_void_p()
        rc = L.oracle_run(batch.raw.ctypes.data, batch.offsets.ctypes.data, batch.n_events, geometry.ctypes.data,
                          threads, stages, C.byref(h))
        if rc != 0:
            raise RuntimeError("oracle_run failed")
        try:
            nh, nt, nth = C.c_uint64(), C.c_uint64(), C.c_uint64()
            L.oracle_sizes(h, C.byref(nh), C.byref(nt), C.byref(nth))
            N = batch.n_events
            self.n_events = N
            self.event_hit_offsets = np.zeros(N + 1, np.uint64)
            self.module_num = np.zeros(N * NM, np.uint32)
            self.x, self.y, self.z, self.phi = (np.zeros(nh.value, np.float32) for _ in range(4))
            self.id = np.zeros(nh.value, np.uint32)
            self.flags = np.zeros(N, np.uint32)
            self.extras = np.zeros(3 * N, np.uint32)
            L.oracle_copy_clusters(h, self.event_hit_offsets.ctypes.data, self.module_num.ctypes.data,
                                   self.x.ctypes.data, self.y.ctypes.data, self.z.ctypes.data, self.phi.ctypes.data,
                                   self.id.ctypes.data, self.flags.ctypes.data, self.extras.ctypes.data)
            self.event_track_offsets = np.zeros(N + 1, np.uint64)
            self.track_hit_offsets = np.zeros(nt.value + 1, np.uint64)
            self.hit_index = np.zeros(nth.value, np.uint32)
            self.hit_id = np.zeros(nth.value, np.uint32)
            self.lsq = np.zeros((nt.value, 13), np.float32)
            self.kal = np.zeros((nt.value, 13), np.float32)
            self.lsq64 = np.zeros((nt.value, 13), np.float64)
            self.kal64 = np.zeros((nt.value, 13), np.float64)
            L.oracle_copy_tracks(h, self.event_track_offsets.ctypes.data, self.track_hit_offsets.ctypes.data,
                                 self.hit_index.ctypes.data, self.hit_id.ctypes.data, self.lsq.ctypes.data,
                                 self.kal.ctypes.data, self.lsq64.ctypes.data, self.kal64.ctypes.data)
        finally:
            L.oracle_destroy(h)

    def event_clusters(self, e):
        a, b = int(self.event_hit_offsets[e]), int(self.event_hit_offsets[e + 1])
        return dict(x=self.x[a:b], y=self.y[a:b], z=self.z[a:b], phi=self.phi[a:b], id=self.id[a:b],
                    module_num=self.module_num[e * NM:(e + 1) * NM])

    def event_tracks(self, e):
        """List of tuples of LHCb ids (track hit order) of event e."""
        t0, t1 = int(self.event_track_offsets[e]), int(self.event_track_offsets[e + 1])
        out = []
        for t in range(t0, t1):
            a, b = int(self.track_hit_offsets[t]), int(self.track_hit_offsets[t + 1])
            out.append(tuple(int(v) for v in self.hit_id[a:b]))
        return out


def run(batch, geometry, threads=0, stages=2):
    return OracleResult(batch, geometry, threads, stages)


def sp_luts():
    L = lib()
    pat = np.zeros(256, np.uint8)
    fx = np.zeros(512, np.float32)
    fy = np.zeros(512, np.float32)
    L.oracle_sp_luts(pat.ctypes.data, fx.ctypes.data, fy.ctypes.data)
    return pat, fx, fy


# ---------------------------------------------------------------------------
# The reference's own CUDA kernels (oracle/_ref/libvelo_ref_gpu.so)
# ---------------------------------------------------------------------------
class RefOutputs(C.Structure):
    _fields_ = [("n_events", C.c_uint32), ("total_estimated", C.c_uint32), ("total_tracks", C.c_uint32),
                ("total_track_hits", C.c_uint32), ("module_start", C.POINTER(C.c_uint32)),
                ("module_num", C.POINTER(C.c_uint32)), ("container", C.POINTER(C.c_uint32)),
                ("candidate_num", C.POINTER(C.c_uint32)), ("weak_num", C.POINTER(C.c_uint32)),
                ("atomics", C.POINTER(C.c_uint32)), ("track_hit_number", C.POINTER(C.c_uint32)),
                ("track_hits", C.POINTER(C.c_uint8)), ("states", C.POINTER(C.c_uint8)),
                ("kalman", C.POINTER(C.c_uint8))]


_ref_gpu = None


def ref_gpu_lib():
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(REF_GPU_LIB):
            raise RuntimeError(f"{REF_GPU_LIB} missing: run oracle/build.py where the reference tree exists")
        L = C.CDLL(REF_GPU_LIB)
        P = C.c_void_p
        L.ref_velo_run.argtypes = [P, P, C.c_uint32, P, C.c_int, C.POINTER(C.c_float), C.POINTER(RefOutputs)]
        L.ref_velo_run.restype = C.c_int
        L.ref_free.argtypes = [C.POINTER(RefOutputs)]
        L.ref_state_size.restype = C.c_int
        L.ref_pv_vertex_size.restype = C.c_int
        L.ref_pv_run.argtypes = [P, P, P, C.c_uint32, P, P, P, P, P, C.c_int, C.POINTER(C.c_float)]
        L.ref_pv_run.restype = C.c_int
        L.ref_gec_run.argtypes = [P, P, P, P, C.c_uint32, P, P, C.c_int, C.POINTER(C.c_float)]
        L.ref_gec_run.restype = C.c_int
        _ref_gpu = L
    return _ref_gpu


def _np(ptr, dtype, count):
    if count == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), shape=(count,)).copy()


def ref_gpu_run(batch, geometry, reps=1):
    """Runs the reference's VELO kernels on the GPU. Returns (dict of numpy arrays, ms per rep).
    Only events that fit the reference's fixed buffers may be passed (see ref_harness.cu)."""
    L = ref_gpu_lib()
    off32 = batch.offsets.astype(np.uint32)
    out = RefOutputs()
    ms = C.c_float()
    rc = L.ref_velo_run(batch.raw.ctypes.data, off32.ctypes.data, batch.n_events, geometry.ctypes.data, reps,
                        C.byref(ms), C.byref(out))
    if rc != 0:
        raise RuntimeError(f"ref_velo_run failed: {rc}")
    try:
        N, S, T, H = out.n_events, out.total_estimated, out.total_tracks, out.total_track_hits
        ss = L.ref_state_size()
        cont = _np(out.container, np.uint32, 6 * S)
        res = dict(module_start=_np(out.module_start, np.uint32, N * NM + 1),
                   module_num=_np(out.module_num, np.uint32, N * NM),
                   y=cont[0:S].view(np.float32), z=cont[S:2 * S].view(np.float32), id=cont[2 * S:3 * S],
                   phi=cont[4 * S:5 * S].view(np.float32), x=cont[5 * S:6 * S].view(np.float32),
                   candidate_num=_np(out.candidate_num, np.uint32, N), weak_num=_np(out.weak_num, np.uint32, N),
                   atomics=_np(out.atomics, np.uint32, 2 * N + 1),
                   track_hit_number=_np(out.track_hit_number, np.uint32, T + 1),
                   track_hits=_np(out.track_hits, np.uint8, 16 * H), states=_np(out.states, np.uint8, ss * T),
                   kalman=_np(out.kalman, np.uint8, ss * T))
        hv = res["track_hits"].view(np.float32).reshape(4, H) if H else np.zeros((4, 0), np.float32)
        res["hit_x"], res["hit_y"], res["hit_z"], res["hit_id"] = hv[0], hv[1], hv[2], hv[3].view(np.uint32)
        res["n_tracks"] = res["atomics"][:N]
        res["track_offsets"] = res["atomics"][N:2 * N + 1]
        res["T"], res["H"] = T, H
        return res, ms.value
    finally:
        L.ref_free(C.byref(out))


REF_PV_NBINS, REF_PV_MAX_VERTICES = 2400, 32


def ref_pv_run(atomics, track_hit_number, kalman_raw, n_events, reps=1):
    """The reference's beamline PV kernels (cuda/PV/beamlinePV) on consolidated VELO tracks:
    atomics[2N+1], track_hit_number[T+1], Kalman states as raw bytes (sizeof(VeloState) * T).
    Returns dict zhisto [N, 2400], zpeaks [N, 32], n_peaks [N], vertices (raw bytes,
    PV::Vertex [N, 32]), n_vertices [N], ms (device time of the four kernels, mean over
    reps - 1 repetitions after the first when reps > 1)."""
    L = ref_gpu_lib()
    N = int(n_events)
    a = np.ascontiguousarray(atomics, np.uint32)
    thn = np.ascontiguousarray(track_hit_number, np.uint32)
    kal = np.ascontiguousarray(kalman_raw, np.uint8)
    vs = L.ref_pv_vertex_size()
    out = dict(zhisto=np.zeros((N, REF_PV_NBINS), np.float32), zpeaks=np.zeros((N, REF_PV_MAX_VERTICES), np.float32),
               n_peaks=np.zeros(N, np.uint32), vertices=np.zeros(N * REF_PV_MAX_VERTICES * vs, np.uint8),
               n_vertices=np.zeros(N, np.uint32))
    ms = C.c_float()
    rc = L.ref_pv_run(a.ctypes.data, thn.ctypes.data, kal.ctypes.data, N, out["zhisto"].ctypes.data,
                      out["zpeaks"].ctypes.data, out["n_peaks"].ctypes.data, out["vertices"].ctypes.data,
                      out["n_vertices"].ctypes.data, int(reps), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_pv_run failed: {rc}")
    out["vertex_size"] = vs
    out["ms"] = ms.value
    return out


def ref_gec_run(ut_batch, scifi_batch, reps=1, timed=False):
    """The reference's global_event_cut kernel (GlobalEventCut.cu:3-55) on UT and SciFi
    batches (u32 offsets, as the reference takes them). Returns the selected events in the
    kernel's order (an atomic counter's: unspecified), and with timed=True also the mean
    device ms of one launch. Only for events whose UT hit total is below the cut (see
    ref_harness.cu); the caller checks that with gec_oracle first."""
    L = ref_gpu_lib()
    N = ut_batch.n_events
    ut_off = np.ascontiguousarray(ut_batch.offsets - ut_batch.offsets[0], np.uint32)
    sf_off = np.ascontiguousarray(scifi_batch.offsets - scifi_batch.offsets[0], np.uint32)
    ut = np.ascontiguousarray(ut_batch.raw[int(ut_batch.offsets[0]):int(ut_batch.offsets[-1])])
    sf = np.ascontiguousarray(scifi_batch.raw[int(scifi_batch.offsets[0]):int(scifi_batch.offsets[-1])])
    n_sel = np.zeros(1, np.uint32)
    lst = np.zeros(max(N, 1), np.uint32)
    ms = C.c_float()
    rc = L.ref_gec_run(ut.ctypes.data, ut_off.ctypes.data, sf.ctypes.data, sf_off.ctypes.data, N,
                       n_sel.ctypes.data, lst.ctypes.data, int(reps), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_gec_run failed: {rc}")
    return (lst[:int(n_sel[0])], ms.value) if timed else lst[:int(n_sel[0])]


def ref_event_clusters(res, e):
    out = []
    for m in range(NM):
        s, n = int(res["module_start"][e * NM + m]), int(res["module_num"][e * NM + m])
        out.append({k: res[k][s:s + n] for k in ("x", "y", "z", "phi", "id")})
    return out


def ref_decode_states(res, key):
    """SoA states of the reference (layout VeloConsolidated.cuh:68-144) -> dict of arrays."""
    T = res["T"]
    blob = res[key].tobytes()
    f = np.frombuffer(blob, dtype=np.float32, count=12 * T).reshape(12, T) if T else np.zeros((12, 0), np.float32)
    out = {k: f[i].copy() for i, k in enumerate(STATE_FIELDS[:12])}
    out["backward"] = np.frombuffer(blob, dtype=np.uint8, count=T, offset=48 * T).astype(bool) if T else np.zeros(0, bool)
    return out


# ---------------------------------------------------------------------------
# The reference's x86 clustering (oracle/_ref/libvelo_ref_x86.so)
# ---------------------------------------------------------------------------
_ref_x86 = None


def ref_x86_clustering(batch, geometry, algo=1, threads=0):
    """algo 0: clustering() (classic), 1: cuda_clustering_cpu_optimized(). Returns (counts, ids, id_offsets)."""
    global _ref_x86
    if _ref_x86 is None:
        if not os.path.exists(REF_X86_LIB):
            raise RuntimeError(f"{REF_X86_LIB} missing")
        _ref_x86 = C.CDLL(REF_X86_LIB)
        P = C.c_void_p
        _ref_x86.ref_x86_clustering.argtypes = [P, P, C.c_uint32, P, C.c_int, C.c_int, P, P, C.c_uint64, P]
        _ref_x86.ref_x86_clustering.restype = C.c_int
    N = batch.n_events
    off32 = batch.offsets.astype(np.uint32)
    counts = np.zeros(N, np.uint32)
    cap = int(batch.raw.size)
    ids = np.zeros(cap, np.uint32)
    io = np.zeros(N + 1, np.uint64)
    rc = _ref_x86.ref_x86_clustering(batch.raw.ctypes.data, off32.ctypes.data, N, geometry.ctypes.data, algo,
                                     threads, counts.ctypes.data, ids.ctypes.data, cap, io.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_x86_clustering failed: {rc}")
    return counts, ids, io


def ref_x86_sp_patterns():
    ref_x86_clustering  # noqa: B018 (library handle is created below)
    L = C.CDLL(REF_X86_LIB)
    P = C.c_void_p
    L.ref_x86_sp_patterns.argtypes = [P, P, P, P]
    pat = np.zeros(256, np.uint8)
    siz = np.zeros(256, np.uint8)
    fx = np.zeros(512, np.float32)
    fy = np.zeros(512, np.float32)
    L.ref_x86_sp_patterns(pat.ctypes.data, siz.ctypes.data, fx.ctypes.data, fy.ctypes.data)
    return pat, siz, fx, fy


_ref_checker = None


def ref_check_velo_tracks(batch, event_track_offsets, track_hit_offsets, hit_ids, max_categories=64):
    """The reference's own TrackCheckerVelo (oracle/_ref/libvelo_ref_checker.so, built from
    checker/tracking without ROOT) on consolidated tracks against the batch's MC_info blobs.
    Returns dict(categories={name: (reconstructible, found, clones)}, tracks, ghosts,
    ghost_per_event)."""
    global _ref_checker
    if _ref_checker is None:
        if not os.path.exists(REF_CHECKER_LIB):
            raise RuntimeError(f"{REF_CHECKER_LIB} missing: run oracle/build.py where the reference tree exists")
        L = C.CDLL(REF_CHECKER_LIB)
        P = C.c_void_p
        L.ref_check_velo_tracks.argtypes = [P, P, C.c_uint32, P, P, P, C.c_uint32, P, P, P, C.POINTER(C.c_float)]
        L.ref_check_velo_tracks.restype = C.c_int
        _ref_checker = L
    evt = np.ascontiguousarray(event_track_offsets, np.uint32)
    tho = np.ascontiguousarray(track_hit_offsets, np.uint32)
    ids = np.ascontiguousarray(hit_ids, np.uint32)
    mco = np.ascontiguousarray(batch.mc_offsets, np.uint64)
    names = np.zeros(64 * max_categories, np.uint8)
    counts = np.zeros(3 * max_categories, np.uint64)
    totals = np.zeros(2, np.uint64)
    gpe = C.c_float()
    n = _ref_checker.ref_check_velo_tracks(batch.mc.ctypes.data, mco.ctypes.data, batch.n_events, evt.ctypes.data,
                                           tho.ctypes.data, ids.ctypes.data, max_categories, names.ctypes.data,
                                           counts.ctypes.data, totals.ctypes.data, C.byref(gpe))
    cats = {}
    for i in range(min(n, max_categories)):
        name = bytes(names[64 * i:64 * (i + 1)]).split(b"\0")[0].decode()
        cats[name] = tuple(int(v) for v in counts[3 * i:3 * i + 3])
    return dict(categories=cats, tracks=int(totals[0]), ghosts=int(totals[1]), ghost_per_event=gpe.value)

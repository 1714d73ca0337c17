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

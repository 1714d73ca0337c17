"""Learned seed/extension scorer of the pruned search: trainer and weights over the C ABI.

The scorer is a 12 -> 64 -> 64 -> 2 MLP (include/velo_b200.h, VeloMlpWeights). It is
trained on the GPU by the library's own tensor-core kernels (velo_mlp_train / collect /
gradient / infer) on seeding candidates labelled by the plain search. There is no
counterpart in the reference; the plain search (search_by_triplet, TrackSeeding.cu:7-200)
is the fallback and the yardstick of what pruning costs.
"""
import ctypes as C

import numpy as np

from . import _lib

FEATURES = ("tx", "ty", "log_scatter", "dphi_01", "dphi_12", "module", "h0_window", "h2_window", "r1", "size_h1",
            "size_h0", "size_h2")


class MlpError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise MlpError(f"{what} failed with code {rc}")


def weights_to_dict(w):
    """VeloMlpWeights -> dict of numpy arrays (copies)."""
    return dict(mean=np.ctypeslib.as_array(w.mean).copy(), inv_std=np.ctypeslib.as_array(w.inv_std).copy(),
                w1=np.ctypeslib.as_array(w.w1).copy(), w2=np.ctypeslib.as_array(w.w2).copy(),
                w3=np.ctypeslib.as_array(w.w3).copy(), seed_threshold=float(w.seed_threshold),
                ext_threshold=float(w.ext_threshold), max_event_clusters=int(w.max_event_clusters),
                min_pairs=int(w.min_pairs), min_event_clusters=int(w.min_event_clusters))


def dict_to_weights(d):
    w = _lib.VeloMlpWeights()
    for k in ("mean", "inv_std", "w1", "w2", "w3"):
        np.ctypeslib.as_array(getattr(w, k))[...] = np.asarray(d[k], np.float32)
    w.seed_threshold = d.get("seed_threshold", 0.5)
    w.ext_threshold = d.get("ext_threshold", 0.0)
    w.max_event_clusters = d.get("max_event_clusters", 0xFFFFFFFF)
    w.min_pairs = d.get("min_pairs", 0)
    w.min_event_clusters = d.get("min_event_clusters", 0)
    return w


def save_weights(w, path):
    with open(path, "wb") as f:
        f.write(bytes(w))


def load_weights(path):
    with open(path, "rb") as f:
        blob = f.read()
    size = C.sizeof(_lib.VeloMlpWeights)
    if len(blob) == size - 4:  # files written before min_event_clusters: every event scored
        blob += bytes(4)
    if len(blob) != size:
        raise MlpError(f"{path}: {len(blob)} bytes, expected {size}")
    return _lib.VeloMlpWeights.from_buffer_copy(blob)


class MlpTrainer:
    """Holds training samples and the scorer's weights on one device."""

    def __init__(self, max_samples, device=0, seed=0):
        self.lib = _lib.gpu_lib()
        self.h = C.c_void_p()
        _check(self.lib.velo_mlp_trainer_create(device, int(max_samples), int(seed), C.byref(self.h)),
               "velo_mlp_trainer_create")

    def close(self):
        if self.h:
            self.lib.velo_mlp_trainer_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def collect(self, chain):
        """Adds the seeding candidates of the chain's last (plain, synced) run; returns the
        number of samples held."""
        n = C.c_uint64()
        _check(self.lib.velo_mlp_collect(self.h, chain.ctx, C.byref(n)), "velo_mlp_collect")
        return n.value

    def samples(self, first, n):
        f = np.empty((n, 12), np.float32)
        lab = np.empty(n, np.uint8)
        _check(self.lib.velo_mlp_samples(self.h, int(first), int(n), f.ctypes.data, lab.ctypes.data),
               "velo_mlp_samples")
        return f, lab

    def normalize(self):
        _check(self.lib.velo_mlp_normalize(self.h), "velo_mlp_normalize")

    def train(self, epochs, batch=16384, lr=2e-3):
        loss = C.c_float()
        _check(self.lib.velo_mlp_train(self.h, int(epochs), int(batch), float(lr), C.byref(loss)), "velo_mlp_train")
        return loss.value

    def weights(self):
        w = _lib.VeloMlpWeights()
        _check(self.lib.velo_mlp_get_weights(self.h, C.byref(w)), "velo_mlp_get_weights")
        return w

    def set_weights(self, w):
        _check(self.lib.velo_mlp_set_weights(self.h, C.byref(w)), "velo_mlp_set_weights")

    def gradient(self, features, labels):
        """Gradient of the mean cross-entropy over the given samples (training kernels)."""
        f = np.ascontiguousarray(features, np.float32)
        lab = np.ascontiguousarray(labels, np.uint8)
        g = _lib.VeloMlpWeights()
        loss = C.c_float()
        _check(self.lib.velo_mlp_gradient(self.h, f.ctypes.data, lab.ctypes.data, len(lab), C.byref(g),
                                          C.byref(loss)), "velo_mlp_gradient")
        d = weights_to_dict(g)
        return dict(w1=d["w1"], w2=d["w2"], w3=d["w3"]), loss.value

    def infer(self, features):
        """Logits [n][2] from the inference kernel code."""
        f = np.ascontiguousarray(features, np.float32)
        z = np.empty((len(f), 2), np.float32)
        _check(self.lib.velo_mlp_infer(self.h, f.ctypes.data, len(f), z.ctypes.data), "velo_mlp_infer")
        return z

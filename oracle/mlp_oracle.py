"""ORACLE — test infrastructure only (imported by tests/ and __graft_entry__.smoke(); never
by the product package). CPU restatement, in numpy, of the learned seed/extension scorer of
the pruned search (cuda_hlt_b200/csrc/velo_mlp.cuh, velo_mlp_train.cu): the proxy-triplet
features, the forward pass, the gradient of the training loss and the reference's phi
windows they start from. The scorer has no counterpart in the reference; the windows follow
cuda/velo/common/include/VeloTools.cuh:6-42 and FillCandidates.cu:8-70.

Two precisions:
  *_bf16   the device's arithmetic: bf16 operands (round to nearest even) at every GEMM
           input, fp32 accumulation, the same masks; agrees with the kernels up to the
           order of fp32 sums.
  *_f64    exact float64 maths of the same network, for stating the bf16 deviation and for
           finite-difference checks.
"""
import numpy as np

PHI_EXTRAPOLATION = np.float32(0.062)


def bf16(x):
    """Rounds float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out.reshape(np.shape(x))


def _unpack(w, dtype=np.float32):
    """dict of VeloMlpWeights fields (numpy) -> arrays of `dtype`."""
    return tuple(np.asarray(w[k], dtype) for k in ("mean", "inv_std", "w1", "w2", "w3"))


def forward_bf16(features, w):
    """Logits [n][2] and the intermediates of the device forward pass."""
    mean, inv_std, w1, w2, w3 = _unpack(w)
    n = len(features)
    x = bf16((np.asarray(features, np.float32) - mean) * inv_std)
    xa = np.concatenate([x, np.ones((n, 1), np.float32)], 1)
    d1 = xa @ bf16(w1).T
    h1 = bf16(np.maximum(d1, 0))
    h1a = np.concatenate([h1, np.ones((n, 1), np.float32)], 1)
    d2 = h1a @ bf16(w2).T
    h2 = bf16(np.maximum(d2, 0))
    h2a = np.concatenate([h2, np.ones((n, 1), np.float32)], 1)
    z = h2a @ bf16(w3).T
    return z, dict(xa=xa, d1=d1, h1a=h1a, d2=d2, h2a=h2a)


def loss_and_gradient_bf16(features, labels, w):
    """Mean cross-entropy over samples and both outputs, and its gradient (w1, w2, w3), with
    the device's roundings: dZ, dH2 and dH1 enter their GEMMs as bf16."""
    _, _, w1, w2, w3 = _unpack(w)
    z, t = forward_bf16(features, w)
    y = np.stack([(labels & 1), (labels >> 1) & 1], 1).astype(np.float32)
    n = len(z)
    loss = np.sum(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))) / (2 * n)
    dz = bf16((1 / (1 + np.exp(-z)) - y) * np.float32(1 / (2 * n)))
    dh2 = bf16((dz @ bf16(w3)[:, :64]) * (t["d2"] > 0))
    dh1 = bf16((dh2 @ bf16(w2)[:, :64]) * (t["d1"] > 0))
    g3 = dz.T @ t["h2a"]
    g2 = dh2.T @ t["h1a"]
    g1 = dh1.T @ t["xa"]
    return float(loss), dict(w1=g1, w2=g2, w3=g3)


def loss_f64(features, labels, w):
    mean, inv_std, w1, w2, w3 = _unpack(w, np.float64)
    x = (np.asarray(features, np.float64) - mean) * inv_std
    n = len(x)
    one = np.ones((n, 1))
    h1 = np.maximum(np.concatenate([x, one], 1) @ w1.T, 0)
    h2 = np.maximum(np.concatenate([h1, one], 1) @ w2.T, 0)
    z = np.concatenate([h2, one], 1) @ w3.T
    y = np.stack([(labels & 1), (labels >> 1) & 1], 1).astype(np.float64)
    return np.sum(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))) / (2 * n)


def gradient_f64(features, labels, w):
    """Exact gradient of loss_f64 (float64, no rounding)."""
    mean, inv_std, w1, w2, w3 = _unpack(w, np.float64)
    x = (np.asarray(features, np.float64) - mean) * inv_std
    n = len(x)
    one = np.ones((n, 1))
    xa = np.concatenate([x, one], 1)
    d1 = xa @ w1.T
    h1a = np.concatenate([np.maximum(d1, 0), one], 1)
    d2 = h1a @ w2.T
    h2a = np.concatenate([np.maximum(d2, 0), one], 1)
    z = h2a @ w3.T
    y = np.stack([(labels & 1), (labels >> 1) & 1], 1).astype(np.float64)
    dz = (1 / (1 + np.exp(-z)) - y) / (2 * n)
    dh2 = (dz @ w3[:, :64]) * (d2 > 0)
    dh1 = (dh2 @ w2[:, :64]) * (d1 > 0)
    return dict(w1=dh1.T @ xa, w2=dh2.T @ h1a, w3=dz.T @ h2a)


# ---------------------------------------------------------------------------
# Features (velo_mlp.cuh seed_features) from one event's phi-sorted clusters
# ---------------------------------------------------------------------------
def window_first(a, value, margin):
    """VeloTools.cuh:6-24 over a phi-sorted array (the "found" flag accumulates)."""
    found = False
    l, r = 0, len(a) - 1
    while l < r:
        m = (l + r) // 2
        e = a[m]
        found |= abs(np.float32(value - e)) < margin
        if np.float32(value - margin) > e:
            l = m + 1
        else:
            r = m
    found |= abs(np.float32(value - a[l])) < margin
    return l if found else -1


def window_second(a, value, margin):
    """VeloTools.cuh:26-42."""
    l, r = 0, len(a) - 1
    while l < r:
        m = (l + r) // 2
        if np.float32(value + margin) > a[m]:
            l = m + 1
        else:
            r = m
    return l + 1 if abs(np.float32(value - a[l])) < margin else l


def phi_window(phi, start, num, value):
    if num == 0:
        return -1, -1
    f = window_first(phi[start:start + num], value, PHI_EXTRAPOLATION)
    if f == -1:
        return -1, -1
    s = window_second(phi[start + f:start + num], value, PHI_EXTRAPOLATION)
    f += start
    return f, (f + 1 if s == 0 else f + s)


def _bracket(phi, f, l, p1):
    lo, hi = f, l
    while lo < hi:
        mid = (lo + hi) >> 1
        if phi[mid] < p1:
            lo = mid + 1
        else:
            hi = mid
    a = lo - 1 if lo - 1 >= f else lo
    b = lo if lo < l else lo - 1
    return a, b


def event_features(x, y, z, phi, size, module_num):
    """Features of every seeding candidate of one event, in hit order: (hit indices,
    windows [n][4], features [n][12]), hits event-relative in the per-module phi order."""
    x, y, z, phi = (np.asarray(a, np.float32) for a in (x, y, z, phi))
    ms = np.concatenate([[0], np.cumsum(np.asarray(module_num, np.int64))])
    idx, wins, feats = [], [], []
    for m in range(2, 50):
        for h in range(ms[m], ms[m + 1]):
            f0, l0 = phi_window(phi, ms[m + 2], ms[m + 3] - ms[m + 2], phi[h])
            f2, l2 = phi_window(phi, ms[m - 2], ms[m - 1] - ms[m - 2], phi[h])
            if f0 == -1 or f2 == -1:
                continue
            a0, b0 = _bracket(phi, f0, l0, phi[h])
            a2, b2 = _bracket(phi, f2, l2, phi[h])
            best, h0, h2 = np.float32(np.inf), a0, a2
            for c0 in (a0, b0):
                for c2 in (a2, b2):
                    z2_tz = np.float32((z[c2] - z[c0]) / (z[h] - z[c0]))
                    px = np.float32(x[c0] + (x[h] - x[c0]) * z2_tz)
                    py = np.float32(y[c0] + (y[h] - y[c0]) * z2_tz)
                    dx, dy = np.float32(px - x[c2]), np.float32(py - y[c2])
                    sc = np.float32((dx * dx + dy * dy) / ((z[c2] - z[h]) * (z[c2] - z[h])))
                    if sc < best:
                        best, h0, h2 = sc, c0, c2
            dz = z[h0] - z[h2]
            feats.append([(x[h0] - x[h2]) / dz, (y[h0] - y[h2]) / dz, np.log1p(min(best, 1e6) * 1000.0),
                          phi[h0] - phi[h], phi[h] - phi[h2], m, l0 - f0, l2 - f2, np.sqrt(x[h] ** 2 + y[h] ** 2),
                          size[h], size[h0], size[h2]])
            idx.append(h)
            wins.append((f0, l0, f2, l2))
    return (np.array(idx, np.int64), np.array(wins, np.int64).reshape(-1, 4),
            np.array(feats, np.float32).reshape(-1, 12))

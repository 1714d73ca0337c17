"""Comparison helpers for the parity tests: clusters per module in order, track hit-id
lists after a canonical sort, and fitted states matched by track."""
import numpy as np

NM = 52


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def compare_event_clusters(mods_a, mods_b, exact=True, tol=1e-5):
    """mods_*: list of 52 dicts (x, y, z, phi, id) in per-module order.
    Returns dict of mismatch counts. exact: float fields compared bit for bit."""
    r = dict(count=0, id=0, order=0, xyz=0, phi=0)
    for a, b in zip(mods_a, mods_b):
        if len(a["id"]) != len(b["id"]):
            r["count"] += 1
            continue
        if not np.array_equal(a["id"], b["id"]):
            if np.array_equal(np.sort(a["id"]), np.sort(b["id"])):
                r["order"] += 1
            else:
                r["id"] += 1
            continue
        for k in ("x", "y", "z"):
            if exact:
                if not np.array_equal(bits(a[k]), bits(b[k])):
                    r["xyz"] += 1
                    break
            elif not np.allclose(a[k], b[k], rtol=tol, atol=tol):
                r["xyz"] += 1
                break
        if exact:
            if not np.array_equal(bits(a["phi"]), bits(b["phi"])):
                r["phi"] += 1
        elif not np.allclose(a["phi"], b["phi"], rtol=tol, atol=tol):
            r["phi"] += 1
    return r


def canonical_tracks(tracks):
    return sorted(tracks)


def compare_event_tracks(ta, tb):
    """Track lists (tuples of LHCb ids). Returns (n_only_a, n_only_b)."""
    sa, sb = {}, {}
    for t in ta:
        sa[t] = sa.get(t, 0) + 1
    for t in tb:
        sb[t] = sb.get(t, 0) + 1
    only_a = sum(max(0, c - sb.get(t, 0)) for t, c in sa.items())
    only_b = sum(max(0, c - sa.get(t, 0)) for t, c in sb.items())
    return only_a, only_b


def track_index(tracks):
    idx = {}
    for i, t in enumerate(tracks):
        idx.setdefault(t, i)
    return idx


STATE_KEYS = ("x", "y", "tx", "ty", "c00", "c20", "c22", "c11", "c31", "c33", "chi2", "z")

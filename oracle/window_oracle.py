"""ORACLE — test infrastructure only (imported by tests/; never by the product package).

Vectorised numpy restatement of the phi windows of fill_candidates
(cuda/velo/search_by_triplet/src/FillCandidates.cu:8-70) with the two binary searches of
cuda/velo/common/include/VeloTools.cuh:6-42, probe for probe: every query runs the
reference's search loop on its own target range, in lockstep with the others, so the
"found" flag accumulates over exactly the elements the reference probes. float32 arithmetic
throughout (round to nearest, as the device's add and subtract under fast math).
`mlp_oracle.window_first` / `window_second` are the scalar form; tests check the two agree.
"""
import numpy as np

PHI_EXTRAPOLATION = np.float32(0.062)


def windows(phi, starts, nums, values, margin=PHI_EXTRAPOLATION):
    """Window [first, last) of each query (values[i] against phi[starts[i] : starts[i] +
    nums[i]], ascending), relative to its range, as phi_window returns it: first = last = -1
    when the search finds nothing or the range is empty."""
    phi = np.asarray(phi, np.float32)
    starts = np.asarray(starts, np.int64)
    nums = np.asarray(nums, np.int64)
    v = np.asarray(values, np.float32)
    margin = np.float32(margin)
    q = len(v)
    first = np.full(q, -1, np.int64)
    last = np.full(q, -1, np.int64)
    live = nums > 0
    if not live.any():
        return first, last
    s, n, v = starts[live], nums[live], v[live]
    lo_edge = (v - margin).astype(np.float32)
    hi_edge = (v + margin).astype(np.float32)
    # window_first (VeloTools.cuh:6-24)
    l = np.zeros(len(v), np.int64)
    r = n - 1
    found = np.zeros(len(v), bool)
    act = l < r
    while act.any():
        m = (l + r) // 2
        e = phi[s + np.where(act, m, 0)]
        found |= act & (np.abs((v - e).astype(np.float32)) < margin)
        go = lo_edge > e
        l = np.where(act & go, m + 1, l)
        r = np.where(act & ~go, m, r)
        act = l < r
    found |= np.abs((v - phi[s + l]).astype(np.float32)) < margin
    f = l
    # window_second (VeloTools.cuh:26-42) over [first, n)
    l2 = f.copy()
    r2 = n - 1
    act = found & (l2 < r2)
    while act.any():
        m = (l2 + r2) // 2
        e = phi[s + np.where(act, m, 0)]
        go = hi_edge > e
        l2 = np.where(act & go, m + 1, l2)
        r2 = np.where(act & ~go, m, r2)
        act = found & (l2 < r2)
    sec = np.where(np.abs((v - phi[s + l2]).astype(np.float32)) < margin, l2 + 1, l2) - f
    lst = np.where(sec == 0, f + 1, f + sec)
    first[live] = np.where(found, f, -1)
    last[live] = np.where(found, lst, -1)
    return first, last


def event_windows(phi, module_start, module_num, margin=PHI_EXTRAPOLATION):
    """fill_candidates of one event: for every hit h1 of modules 2..49 (phi-sorted, event
    indices), the h0 window in module m + 2 and the h2 window in module m - 2, as absolute
    [first, last) (-1, -1: none). Returns (h1 indices, first0, last0, first2, last2)."""
    h1 = np.concatenate([np.arange(module_start[m], module_start[m] + module_num[m]) for m in range(2, 50)])
    mod = np.concatenate([np.full(module_num[m], m) for m in range(2, 50)]).astype(np.int64)
    if len(h1) == 0:
        e = np.zeros(0, np.int64)
        return h1, e, e, e, e
    ms = np.asarray(module_start, np.int64)
    mn = np.asarray(module_num, np.int64)
    out = []
    for target in (mod + 2, mod - 2):
        f, l = windows(phi, ms[target], mn[target], phi[h1], margin)
        out += [np.where(f >= 0, f + ms[target], -1), np.where(f >= 0, l + ms[target], -1)]
    return (h1, *out)

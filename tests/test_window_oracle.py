"""The vectorised window oracle (oracle/window_oracle.py) against the scalar restatement of
the reference's searches (oracle/mlp_oracle.py, VeloTools.cuh:6-42), on random modules and on
modules built to sit on the window's edges: many equal phi, and values one or two float32
steps either side of phi +- margin, where the probe path decides the "found" flag."""
import numpy as np

from oracle import mlp_oracle, window_oracle

MARGIN = window_oracle.PHI_EXTRAPOLATION


def scalar_window(a, value):
    if len(a) == 0:
        return -1, -1
    f = mlp_oracle.window_first(a, value, MARGIN)
    if f == -1:
        return -1, -1
    s = mlp_oracle.window_second(a[f:], value, MARGIN)
    return f, (f + 1 if s == 0 else f + s)


def edge_values(rng, a, k):
    """Values at and around the window edges of elements of a."""
    picks = a[rng.integers(0, len(a), k)]
    side = np.where(rng.random(k) < 0.5, -1, 1).astype(np.float32)
    v = (picks + side * MARGIN).astype(np.float32)
    steps = rng.integers(-2, 3, k)
    for i in range(k):
        for _ in range(abs(int(steps[i]))):
            v[i] = np.nextafter(v[i], np.float32(np.inf if steps[i] > 0 else -np.inf), dtype=np.float32)
    return v


def module(rng, n, kind):
    a = rng.uniform(-3.3, 3.3, n).astype(np.float32)
    if kind == 1:  # few distinct values
        a = rng.choice(a[:max(1, n // 5)], n)
    elif kind == 2:  # a coarse grid: many ties at window distance
        a = (np.round(a / MARGIN) * MARGIN).astype(np.float32)
    return np.sort(a).astype(np.float32)


def test_vectorised_equals_scalar():
    rng = np.random.default_rng(11)
    checked = 0
    for trial in range(300):
        n = int(rng.integers(1, 120))
        a = module(rng, n, trial % 3)
        v = np.concatenate([rng.uniform(-3.5, 3.5, 20).astype(np.float32), a[rng.integers(0, n, 10)],
                            edge_values(rng, a, 30)])
        f, l = window_oracle.windows(a, np.zeros(len(v)), np.full(len(v), n), v)
        for i in range(len(v)):
            assert (f[i], l[i]) == scalar_window(a, v[i]), (trial, i, v[i])
            checked += 1
    assert checked == 300 * 60


def test_event_windows_equal_fill_candidates_loop():
    rng = np.random.default_rng(12)
    nums = rng.integers(0, 90, 52)
    nums[7] = 0  # an empty target module
    starts = np.concatenate([[0], np.cumsum(nums)[:-1]])
    phi = np.concatenate([module(rng, int(k), 0) if k else np.zeros(0, np.float32) for k in nums])
    h1, f0, l0, f2, l2 = window_oracle.event_windows(phi, starts, nums)
    i = 0
    for m in range(2, 50):
        for r in range(nums[m]):
            h = starts[m] + r
            assert h1[i] == h
            assert (f0[i], l0[i]) == mlp_oracle.phi_window(phi, starts[m + 2], nums[m + 2], phi[h])
            assert (f2[i], l2[i]) == mlp_oracle.phi_window(phi, starts[m - 2], nums[m - 2], phi[h])
            i += 1
    assert i == len(h1) == nums[2:50].sum()

"""CPU checks of the scorer's oracle (oracle/mlp_oracle.py): bf16 rounding, the float64
gradient against central finite differences, and the bf16 restatement against float64."""
import numpy as np
import pytest

from oracle import mlp_oracle


def weights(seed):
    rng = np.random.default_rng(seed)
    return dict(mean=rng.normal(0, 1, 12), inv_std=rng.uniform(0.5, 2, 12), w1=rng.normal(0, 0.4, (64, 13)),
                w2=rng.normal(0, 0.15, (64, 65)), w3=rng.normal(0, 0.3, (2, 65)))


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.01171875, 1.005859375, -3.0e-3, 65504.0, np.inf], np.float32)
    r = mlp_oracle.bf16(x)
    # bf16 spacing at 1 is 2^-7. 1 + 2^-8 and 1 + 3*2^-8 are halfway cases: ties to the even
    # mantissa (1 and 1 + 2^-6); 1 + 3*2^-9 rounds up to 1 + 2^-7
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[3] == 1.0078125
    assert r[4] == np.float32(-0.0030059814453125) and r[5] == 65536.0 and np.isinf(r[6])
    assert np.isnan(mlp_oracle.bf16(np.array([np.nan], np.float32)))[0]


def test_f64_gradient_matches_finite_differences():
    w = weights(1)
    rng = np.random.default_rng(2)
    f = rng.normal(0, 1.5, (64, 12))
    lab = rng.integers(0, 4, 64).astype(np.uint8)
    g = mlp_oracle.gradient_f64(f, lab, w)
    eps = 1e-6
    for k, shape in (("w1", (64, 13)), ("w2", (64, 65)), ("w3", (2, 65))):
        for idx in [tuple(rng.integers(0, s) for s in shape) for _ in range(12)]:
            wp = {kk: np.array(v, np.float64) for kk, v in w.items()}
            wm = {kk: np.array(v, np.float64) for kk, v in w.items()}
            wp[k][idx] += eps
            wm[k][idx] -= eps
            fd = (mlp_oracle.loss_f64(f, lab, wp) - mlp_oracle.loss_f64(f, lab, wm)) / (2 * eps)
            assert abs(fd - g[k][idx]) < 1e-6 + 1e-4 * abs(fd), (k, idx)


def test_bf16_gradient_close_to_f64():
    w = weights(3)
    rng = np.random.default_rng(4)
    f = rng.normal(0, 1.5, (512, 12)).astype(np.float32)
    lab = rng.integers(0, 4, 512).astype(np.uint8)
    loss, g = mlp_oracle.loss_and_gradient_bf16(f, lab, w)
    g64 = mlp_oracle.gradient_f64(f, lab, w)
    assert abs(loss - mlp_oracle.loss_f64(f, lab, w)) < 2e-2 * loss
    for k in ("w1", "w2", "w3"):
        assert np.linalg.norm(g[k] - g64[k]) < 0.1 * np.linalg.norm(g64[k]), k


def test_features_of_a_straight_track():
    """Three hits of a straight line from the origin plus noise hits: the proxy triplet is
    the line, its scatter is ~0 and the slopes are the line's."""
    tx, ty = 0.01, -0.02
    zs = {0: -287.5, 2: -262.5, 4: -237.5}
    x, y, z, phi, size, mnum = [], [], [], [], [], []
    rng = np.random.default_rng(5)
    for m in range(52):
        pts = []
        if m in zs:
            pts.append((tx * zs[m], ty * zs[m], zs[m], 2))
            for _ in range(3):
                a = rng.uniform(-np.pi, np.pi)
                r = rng.uniform(5, 40)
                pts.append((r * np.cos(a), r * np.sin(a), zs[m], 1))
        ph = [np.arctan2(p[1], p[0]) if m % 2 else np.arctan2(p[1], p[0]) % (2 * np.pi) for p in pts]
        order = np.argsort(ph, kind="stable")
        for i in order:
            x.append(pts[i][0]); y.append(pts[i][1]); z.append(pts[i][2]); size.append(pts[i][3]); phi.append(ph[i])
        mnum.append(len(pts))
    idx, wins, feats = mlp_oracle.event_features(x, y, z, phi, np.array(size), mnum)
    on_line = [i for i, h in enumerate(idx) if size[h] == 2]
    assert len(on_line) == 1
    fr = feats[on_line[0]]
    assert abs(fr[0] - tx) < 1e-5 and abs(fr[1] - ty) < 1e-5
    assert fr[2] < 1e-3 and fr[5] == 2 and fr[9] == 2 and fr[10] == 2 and fr[11] == 2


def test_committed_weights_file_and_old_format(tmp_path):
    """The committed scorer file holds the operating point; a file written before the event
    gate existed (4 bytes shorter) loads with the gate at 0 (every event scored)."""
    from cuda_hlt_b200 import mlp, train_scorer
    w = mlp.load_weights(train_scorer.DEFAULT_WEIGHTS)
    assert 0.0 < w.seed_threshold < 1.0
    assert w.min_event_clusters == train_scorer.BENCH_EVENT_GATE
    assert w.max_event_clusters > w.min_event_clusters
    old = tmp_path / "old.bin"
    old.write_bytes(bytes(w)[:-4])
    w_old = mlp.load_weights(str(old))
    assert w_old.min_event_clusters == 0 and w_old.min_pairs == w.min_pairs
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(w)[:-8])
    with pytest.raises(mlp.MlpError):
        mlp.load_weights(str(bad))

"""The beamline PV oracle (oracle/pv_oracle.py) on CPU, on the Kalman states of the CPU VELO
oracle: vertices sit on the beamline inside the luminous region, every kept vertex came from
a peak, and their number follows the pileup (on average about 0.7 nu visible primary
vertices are generated per event; vertices need 5 tracks in the event)."""
import numpy as np

from cuda_hlt_b200 import events
import oracle
from oracle import pv_oracle


def test_pv_oracle_on_oracle_tracks(geometry):
    counts = {}
    for nu in (3.0, 10.0):
        b = events.generate(seed=31, nu_min=nu, nu_max=nu, n_events=12, with_mc=False)
        r = oracle.run(b, geometry)
        names = ("x", "y", "tx", "ty", "c00", "c20", "c22", "c11", "c31", "c33", "chi2", "z")
        kal = {n: r.kal[:, i] for i, n in enumerate(names)}
        n_v = []
        for e in range(b.n_events):
            t0, t1 = int(r.event_track_offsets[e]), int(r.event_track_offsets[e + 1])
            p, vs = pv_oracle.event_pvs(kal, t0, t1)
            assert len(vs) <= min(len(p), 32)
            for v in vs:
                assert v["x"] ** 2 + v["y"] ** 2 < 0.09 and -300 < v["z"] < 300
                assert np.min(np.abs(p - v["z"])) < 5.0  # fitted near its seed
            n_v.append(len(vs))
        counts[nu] = float(np.mean(n_v))
    assert 1.0 <= counts[3.0] < counts[10.0] <= 10.0

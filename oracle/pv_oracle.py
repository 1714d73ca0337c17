"""ORACLE — test infrastructure only (imported by tests/). CPU restatement, in float32 numpy,
of the reference's beamline primary-vertex finder (cuda/PV/beamlinePV of the reference):

  extrapolate   pv_beamline_extrapolate.cu:3-30 with the PVTrack constructor of
                TrackBeamLineVertexFinder.cuh:9-31
  histogram     pv_beamline_histo.cu:3-76 (bins filled in track order)
  peaks         pv_beamline_peak.cu:3-147
  fit           pv_beamline_multi_fitter.cu:6-183 (sums over tracks in track order)

One event at a time, on the Kalman beamline states of its tracks. The reference computes in
fp32 on the GPU with fused multiply-adds, fast-math exp/sqrt/division and float atomics in
the histogram; this restatement rounds each operation separately, so it agrees with the
reference and with the CUDA stage to a tolerance, not bit for bit.
"""
import numpy as np

F = np.float32
ZMIN, ZMAX, NBINS, DZ = F(-300.0), F(300.0), 2400, F(0.25)
MAX_TRACK_Z0_ERR, MIN_DENSITY, MIN_DIP_DENSITY, MIN_TRACKS_IN_SEED = F(1.5), F(1.0), F(2.0), F(2.5)
MAX_VERTEX_RHO2, MAX_FIT_ITER, MAX_DELTA_CHI2, MIN_WEIGHT = F(0.09), 2, F(9.0), F(0.3)
ORDER, MIN_TRACKS_PER_VERTEX, MAX_VERTICES = 2, 5, 32

# Singular cases met since reset_singular(), by kind. The fp32 Kalman covariances of a few
# tracks are negative or zero (the simplified Kalman fit is ill-conditioned), so:
#   zweight    a track's z weight is not positive: the reference's 1/sqrt gives NaN or inf and
#              its "zerr < max" test drops the track; dropped here by an explicit test;
#   weight     a fit weight is not finite (exp overflows on a negative weight matrix): the
#              reference carries the NaN or inf into the vertex sums, and so does this code,
#              with the overflow counted instead of warned about.
SINGULAR = dict(zweight=0, weight=0)


def reset_singular():
    for k in SINGULAR:
        SINGULAR[k] = 0


def extrapolate(k):
    """k: dict of float32 arrays x, y, tx, ty, c00, c20, c22, c11, c31, c33, z of the event's
    tracks -> dict z, x, y, tx, ty, w00, w11 of the tracks at the beamline."""
    x, y, tx, ty = (np.asarray(k[n], F) for n in ("x", "y", "tx", "ty"))
    dz = (tx * (F(0) - x) + ty * (F(0) - y)) / (tx * tx + ty * ty)
    dz2 = dz * dz
    c00 = np.asarray(k["c00"], F) + (dz2 * np.asarray(k["c22"], F) + F(2) * dz * np.asarray(k["c20"], F))
    c11 = np.asarray(k["c11"], F) + (dz2 * np.asarray(k["c33"], F) + F(2) * dz * np.asarray(k["c31"], F))
    return dict(z=np.asarray(k["z"], F) + dz, x=x + dz * tx, y=y + dz * ty, tx=tx, ty=ty, w00=F(1) / c00,
                w11=F(1) / c11)


def _gauss_integral(v):
    a = np.sqrt(F(2 * ORDER + 3))
    xi = F(v) / a
    eta = F(1) - xi * xi
    return F(0.5) + xi * (F(0.5) + eta * (F(0.25) + eta * F(0.1875)))


def histogram(t):
    h = np.zeros(NBINS, F)
    a = np.sqrt(F(2 * ORDER + 3))
    for i in range(len(t["z"])):
        z = F(t["z"][i])
        if not (ZMIN < z < ZMAX):
            continue
        zbin = (z - ZMIN) / DZ
        zweight = F(t["tx"][i]) * F(t["tx"][i]) * F(t["w00"][i]) + F(t["ty"][i]) * F(t["ty"][i]) * F(t["w11"][i])
        if not zweight > F(0):  # 1/sqrt is NaN or inf: the reference's test below fails too
            SINGULAR["zweight"] += 1
            continue
        zerr = F(1) / np.sqrt(F(zweight))
        if not zerr < MAX_TRACK_Z0_ERR:
            continue
        half = a * zerr / DZ
        minbin = max(int(zbin - half), 1)
        maxbin = min(int(zbin + half), NBINS - 2)
        if maxbin < minbin:
            continue
        integral = F(0)
        for b in range(minbin, maxbin):
            this = _gauss_integral((ZMIN + F(b + 1) * DZ - z) / zerr)
            h[b] += this - integral
            integral = this
        h[maxbin] += F(1) - integral
    return h


def peaks(h):
    """z of the peak of every cluster of the histogram, in bin order (all of them; the
    reference keeps room for 32)."""
    threshold = DZ * (F(1) / (F(10) * MAX_TRACK_Z0_ERR))
    edges, prevempty, integral = [], True, F(h[0])
    for i in range(1, NBINS):
        integral += h[i]
        empty = h[i] < threshold
        if empty != prevempty:
            if prevempty or integral > MIN_TRACKS_IN_SEED:
                edges.append(i)
            else:
                edges.pop()
            prevempty = empty
            integral = F(0)
    mindip, minpeak = MIN_DIP_DENSITY * DZ, MIN_DENSITY * DZ
    izmax = []
    for c in range(len(edges) // 2):
        ibegin, iend = edges[2 * c], edges[2 * c + 1]
        ex = [(ibegin, F(h[ibegin]), F(h[ibegin]))]  # (index, value, integral)
        rising, integral = True, F(h[ibegin])
        for i in range(ibegin, iend):
            value = F(h[i])
            stillrising = h[i + 1] > value
            if rising and not stillrising and value >= minpeak:
                if len(ex) >= 2:
                    dv1 = ex[-2][1] - ex[-1][1]
                    dv2 = value - ex[-1][1]
                    if dv1 > mindip and dv2 > mindip:
                        ex.append((i, value, integral + F(0.5) * value))
                    elif dv1 > dv2:
                        ex.pop()
                    else:
                        del ex[-2:]
                        ex.append((i, value, integral + F(0.5) * value))
                else:
                    ex.append((i, value, integral + F(0.5) * value))
            elif rising != stillrising:
                ex.append((i, value, integral + F(0.5) * value))
            rising = stillrising
            integral += value
        ex.append((iend, F(h[iend]), integral))
        n = len(ex)
        sub = []
        if n > 3:
            for i in range(1, n // 2 + 1):
                if 2 * i < n and ex[2 * i][2] - ex[2 * i - 2][2] > MIN_TRACKS_IN_SEED:
                    sub.append(ex[2 * i - 1][0])
        if not sub:
            if ex[1][1] >= minpeak:
                izmax.append(ex[1][0])
        else:
            izmax += sub
    out = []
    for i in izmax:
        d1 = F(h[i]) - F(h[i - 1])
        d2 = F(h[i]) - F(h[i + 1])
        idz = F(0.5) * (d1 - d2) / (d1 + d2) if d1 + d2 > 0 else F(0)
        out.append(ZMIN + DZ * (F(i) + idz + F(0.5)))
    return np.array(out, F)


def fit(t, seeds):
    """Vertices of the kept seeds, in seed order: dicts x, y, z, chi2, n_tracks, cov[6]."""
    seeds = np.asarray(seeds, F)
    nt = len(t["z"])
    inz = (ZMIN <= t["z"]) & (t["z"] <= ZMAX)
    out = []
    for s in range(len(seeds)):
        vx, vy, vz = F(0), F(0), F(seeds[s])
        cov = np.zeros(6, F)
        chi2tot = F(0)
        converged = False
        for it in range(MAX_FIT_ITER):
            if converged:
                break
            a = np.zeros(5, F)  # 00, 11, 20, 21, 22
            g = np.zeros(3, F)
            chi2tot, nsel = F(0), 0
            cut = F(0.1) + F(0.01) * F(MAX_FIT_ITER) / F(it + 1)
            for i in np.nonzero(inz)[0]:
                tx, ty, w00, w11 = F(t["tx"][i]), F(t["ty"][i]), F(t["w00"][i]), F(t["w11"][i])
                dz = vz - F(t["z"][i])
                rx = vx - (F(t["x"][i]) + tx * dz)
                ry = vy - (F(t["y"][i]) + ty * dz)
                chi2 = rx * rx * w00 + ry * ry * w11
                if not chi2 < MAX_DELTA_CHI2:
                    continue
                nsel += 1
                odz = seeds - F(t["z"][i])
                ox = F(0) - (F(t["x"][i]) + tx * odz)
                oy = F(0) - (F(t["y"][i]) + ty * odz)
                with np.errstate(over="ignore", invalid="ignore"):
                    denom = np.exp(-cut * F(0.5)) + np.sum(np.exp(-(ox * ox * w00 + oy * oy * w11) * F(0.5)), dtype=F)
                    w = np.exp(-chi2 * F(0.5)) / denom
                if not (np.isfinite(denom) and np.isfinite(w)):
                    SINGULAR["weight"] += 1
                if w < MIN_WEIGHT:
                    continue
                g += np.array([rx * w00, ry * w11, -tx * rx * w00 - ty * ry * w11], F) * w
                h20, h21 = -tx, -ty
                a += w * np.array([w00, w11, h20 * w00, h21 * w11, h20 * h20 * w00 + h21 * h21 * w11], F)
                chi2tot += w * chi2
            if nsel < 2:
                break
            a00, a11, a20, a21, a22 = a
            det = a00 * (a22 * a11 - a21 * a21) + a20 * (-a11 * a20)
            inv = F(1) / det
            cov = np.array([(a22 * a11 - a21 * a21) * inv, -(-a20 * a21) * inv, (a22 * a00 - a20 * a20) * inv,
                            (-a20 * a11) * inv, -(a21 * a00) * inv, (a11 * a00) * inv], F)
            dx = -(cov[0] * g[0] + cov[1] * g[1] + cov[3] * g[2])
            dy = -(cov[1] * g[0] + cov[2] * g[1] + cov[4] * g[2])
            dzv = -(cov[3] * g[0] + cov[4] * g[1] + cov[5] * g[2])
            chi2tot += dx * g[0] + dy * g[1] + dzv * g[2]
            vx, vy, vz = vx + dx, vy + dy, vz + dzv
            converged = abs(dzv) < F(0.001)
        # the reference counts every track of the event (its fresh track copies have weight 1)
        if nt >= MIN_TRACKS_PER_VERTEX and vx * vx + vy * vy < MAX_VERTEX_RHO2:
            out.append(dict(x=vx, y=vy, z=vz, chi2=chi2tot, n_tracks=nt, cov=cov))
    return out


def event_pvs(kalman_fields, t0, t1):
    """(peaks, vertices) of one event whose tracks are [t0, t1) of the Kalman state arrays."""
    k = {n: np.asarray(kalman_fields[n][t0:t1], F) for n in
         ("x", "y", "tx", "ty", "c00", "c20", "c22", "c11", "c31", "c33", "z")}
    t = extrapolate(k)
    p = peaks(histogram(t))
    return p, fit(t, p[:MAX_VERTICES])

"""Host-side pieces: SuperPixel tables, generator, raw-format validation, MC checker."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from cuda_hlt_b200 import _lib, events


def test_sp_tables_match_oracle():
    pat, _, fx, fy = events.sp_luts()
    opat, ofx, ofy = oracle.sp_luts()
    assert np.array_equal(pat, opat)
    assert np.array_equal(fx.view(np.uint32), ofx.view(np.uint32))
    assert np.array_equal(fy.view(np.uint32), ofy.view(np.uint32))


@pytest.mark.skipif(not os.path.exists(oracle.REF_X86_LIB), reason="reference x86 build missing")
def test_sp_tables_match_reference_cache_sp_patterns():
    # x86/velo/clustering/src/ClusteringCommon.cpp:3-101, run from the reference build
    ref = oracle.ref_x86_sp_patterns()
    mine = events.sp_luts()
    for a, b in zip(ref, mine):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


def test_sp_table_properties():
    pat, sizes, fx, fy = events.sp_luts()
    for sp in range(1, 256):
        n0, n1 = sizes[sp] & 0xF, sizes[sp] >> 4
        assert n0 + n1 == bin(sp).count("1")
        assert bool(pat[sp] & 8) == (n1 > 0)
        assert 0 <= fx[2 * sp] < 1 and 0 <= fy[2 * sp] < 1


def test_generator_deterministic_and_splittable(geometry):
    a = events.generate(20, seed=7, nu_min=5, nu_max=9)
    b = events.generate(20, seed=7, nu_min=5, nu_max=9, threads=3)
    assert np.array_equal(a.raw, b.raw) and np.array_equal(a.offsets, b.offsets)
    assert np.array_equal(a.mc, b.mc)
    c = events.generate(10, first_event=10, seed=7, nu_min=5, nu_max=9)
    for i in range(10):
        assert np.array_equal(a.event(10 + i), c.event(i))
    d = events.generate(20, seed=8, nu_min=5, nu_max=9)
    assert not np.array_equal(a.raw[:1000], d.raw[:1000])


def test_generator_valid_and_sorted():
    b = events.generate_config("batched_500k", n_events=40)
    assert events.validate(b).all()
    for i in range(b.n_events):
        w = b.event(i).view(np.uint32)
        nb = w[0]
        offs = w[1:nb + 2] // 4
        pl = w[nb + 2:]
        for k in range(nb):
            cnt = pl[offs[k] + 1]
            words = pl[offs[k] + 2:offs[k] + 2 + cnt]
            addr = (words >> 8) & 0x7FFF
            assert np.all(np.diff(addr.astype(np.int64)) > 0)  # unique, address-sorted SPs


@pytest.mark.parametrize("name,lo,hi", [("plain_1k", 2150, 2650), ("high_occupancy_200k", 4500, 6000)])
def test_generator_cluster_counts(geometry, name, lo, hi):
    b = events.generate_config(name, n_events=100)
    r = oracle.run(b, geometry, stages=1)
    mean = r.module_num.sum() / b.n_events
    assert lo < mean < hi


def _event_with(words_per_bank):
    nb = 208
    payload = []
    offs = [0]
    for b in range(nb):
        ws = words_per_bank.get(b, [])
        payload += [b, len(ws)] + list(ws)
        offs.append(4 * len(payload))
    return np.array([nb] + offs + payload, dtype=np.uint32).view(np.uint8)


def test_validate_raw_edge_cases():
    lib = _lib.host_lib()
    good = _event_with({5: [0x80001203]})
    empty = _event_with({})
    assert lib.velo_validate_raw_event(good.ctypes.data, good.size) == 0
    assert lib.velo_validate_raw_event(empty.ctypes.data, empty.size) == 0
    assert lib.velo_validate_raw_event(good.ctypes.data, 0) != 0
    assert lib.velo_validate_raw_event(good.ctypes.data, good.size - 4) != 0  # truncated
    bad = good.view(np.uint32).copy()
    bad[0] = 207
    assert lib.velo_validate_raw_event(bad.ctypes.data, bad.nbytes) != 0  # wrong bank count
    bad = good.view(np.uint32).copy()
    pl = 1 + 209
    bad[pl + 2 * 3] = 4  # bank 3 claims sensor 4
    assert lib.velo_validate_raw_event(bad.ctypes.data, bad.nbytes) != 0
    bad = good.view(np.uint32).copy()
    bad[pl + 2 * 5 + 1] = 2  # bank 5 claims 2 SPs, holds 1
    assert lib.velo_validate_raw_event(bad.ctypes.data, bad.nbytes) != 0


def test_checker_truth_tracks(minbias):
    """Tracks made of the MC truth hits of each reconstructible particle: 100% efficiency, no ghosts."""
    lib = _lib.host_lib()
    b = events.generate_config("plain_1k", n_events=5)
    evt, tho, ids = [0], [0], []
    for e in range(b.n_events):
        m = b.mc[b.mc_offsets[e]:b.mc_offsets[e + 1]]
        n = int(m[:4].view(np.uint32)[0])
        p = 4
        for _ in range(n):
            has_velo = m[p + 26]
            p += 32
            k = int(m[p + 4:p + 8].view(np.uint32)[0])
            hits = m[p + 8:p + 8 + 4 * k].view(np.uint32)
            p += 8 + 4 * k + 8
            if has_velo:
                ids += hits.tolist()
                tho.append(len(ids))
        evt.append(len(tho) - 1)
    res = _lib.VeloCheckResult()
    evt = np.array(evt, np.uint32)
    tho = np.array(tho, np.uint32)
    ids = np.array(ids, np.uint32)
    assert lib.velo_check_tracks(b.mc.ctypes.data, b.mc_offsets.ctypes.data, b.n_events, evt.ctypes.data,
                                 tho.ctypes.data, ids.ctypes.data, C.byref(res)) == 0
    assert res.ghosts == 0
    assert res.velo_efficiency == 1.0 and res.long_efficiency == 1.0
    assert res.velo_clones == 0


def test_checker_reads_reference_mc_files(minbias):
    """The shipped MC_info files parse with the checker (layout MCEvent.cpp:16-92)."""
    lib = _lib.host_lib()
    N = minbias.n_events
    evt = np.zeros(N + 1, np.uint32)
    tho = np.zeros(1, np.uint32)
    ids = np.zeros(1, np.uint32)
    res = _lib.VeloCheckResult()
    assert lib.velo_check_tracks(minbias.mc.ctypes.data, minbias.mc_offsets.ctypes.data, N, evt.ctypes.data,
                                 tho.ctypes.data, ids.ctypes.data, C.byref(res)) == 0
    assert res.velo_reconstructible > 1000 and res.long_reconstructible > 100

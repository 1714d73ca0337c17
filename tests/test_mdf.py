"""The MDF reader (velo_mdf_read, counterpart of MDF::read_events in mdf/src/read_mdf.cpp for
the VP banks) on CPU.

* the reference's minbias MDF file (compressed, checksummed, all subdetectors' banks) gives,
  byte for byte, the VP raw events the reference ships for the same events as a bank folder,
  and the ODIN run/event numbers of their file names;
* skipping and limiting events;
* a corrupted byte fails the record checksum;
* records written here (uncompressed, and compressed in several ROOT zlib blocks) read back
  to the events they were written from, with foreign banks and an ODIN bank skipped over.
"""
import os
import struct
import zlib

import numpy as np
import pytest

from cuda_hlt_b200 import events

HERE = os.path.dirname(os.path.abspath(__file__))
MDF = os.path.join(HERE, "golden", "minbias", "mdf", "upgrade_mc_minbias_scifi_v5.mdf")
VP_FOLDER = os.path.join(HERE, "golden", "minbias", "VP")


def test_mdf_equals_bank_folder():
    m = events.read_mdf(MDF)
    f = events.read_bank_folder(VP_FOLDER)
    assert m.n_events == f.n_events == 10
    assert [n + ".bin" for n in m.names] == f.names
    assert np.array_equal(m.raw, f.raw)
    assert np.array_equal(m.offsets, f.offsets)
    assert events.validate(m).all()


def test_mdf_skip_and_limit():
    f = events.read_bank_folder(VP_FOLDER)
    m = events.read_mdf(MDF, first_event=3, max_events=4)
    assert m.n_events == 4
    for i in range(4):
        assert np.array_equal(m.event(i), f.event(3 + i))
    assert events.read_mdf(MDF, first_event=10).n_events == 0


def test_mdf_checksum(tmp_path):
    data = bytearray(open(MDF, "rb").read())
    data[200] ^= 0x01  # inside the first record's compressed payload
    p = tmp_path / "bad.mdf"
    p.write_bytes(bytes(data))
    with pytest.raises(ValueError):
        events.read_mdf(str(p))


# ---- an MDF writer for the tests (record layout of mdf/include/mdf_header.hpp) ----
def _hash32(b):
    h = 0
    for c in b:
        c = c - 256 if c >= 128 else c  # bytes read as signed char
        h = (h + c) & 0xFFFFFFFF
        h = (h + (h << 10)) & 0xFFFFFFFF
        h ^= h >> 6
    h = (h + (h << 3)) & 0xFFFFFFFF
    h ^= h >> 11
    h = (h + (h << 15)) & 0xFFFFFFFF
    return h


def _bank(btype, source, words, version=2):
    body = np.asarray(words, np.uint32).tobytes()
    b = struct.pack("<HHBBh", 0xCBCB, 8 + len(body), btype, version, source) + body
    return b + b"\0" * (-len(b) % 4)


def _vp_banks(event):
    w = event.view(np.uint32)
    n = int(w[0])
    offs = w[1:n + 2] // 4
    payload = w[n + 2:]
    return [_bank(63, int(payload[offs[i]]), payload[offs[i] + 1:offs[i + 1]]) for i in range(n)]


def _record(banks, run, evno, compress, blocks=1):
    body = b"".join(banks)
    if compress:
        parts = np.array_split(np.frombuffer(body, np.uint8), blocks)
        out = b""
        for p in parts:
            z = zlib.compress(p.tobytes())
            out += b"ZL\x08" + struct.pack("<I", len(z))[:3] + struct.pack("<I", p.size)[:3] + z
        body = out
    size = 48 + len(body)
    sub = struct.pack("<4I3I", *([0xFFFFFFFF] * 4), run, 0, 0)
    rec = bytearray(struct.pack("<3I", size, size, size) + b"\0\0\0\0" +
                    bytes([1 if compress else 0, 0x37, 1, 0]) + sub + body)
    struct.pack_into("<I", rec, 12, _hash32(bytes(rec[16:])))
    return bytes(rec)


@pytest.mark.parametrize("compress,blocks", [(False, 1), (True, 1), (True, 3)])
def test_mdf_written_records(tmp_path, compress, blocks):
    b = events.generate(seed=3, nu_min=2.0, nu_max=8.0, n_events=5, with_mc=False)
    recs = []
    for i in range(b.n_events):
        odin = _bank(16, 0, [1234, 0, 0, 0, 500 + i, 0, 0, 0, 0, 0], version=6)
        other = _bank(9, 7, [1, 2, 3])  # a bank of another subdetector, skipped
        recs.append(_record([odin, other] + _vp_banks(b.event(i)), 1234, 500 + i, compress, blocks))
    p = tmp_path / "written.mdf"
    p.write_bytes(b"".join(recs))
    m = events.read_mdf(str(p))
    assert m.names == [f"1234_{500 + i}" for i in range(b.n_events)]
    assert np.array_equal(m.raw, b.raw) and np.array_equal(m.offsets, b.offsets)

"""CPU checks of the BDIO writer (qed2d/bdio.py) with the independent reader in
tests/bdio_reader.py: header fields, record formats, user-info numbers, lengths,
payloads and the MD5 checksum records, for the record sequence the reference's
mc driver writes (main/MC.jl:87-100, 140-152)."""
import hashlib
import json
import struct

import numpy as np
import pytest

from bdio_reader import read_bdio


def test_writer_layout_roundtrip(tmp_path):
    from qed2d import bdio
    p = str(tmp_path / "x.bdio")
    fb = bdio.BDIOWriter(p, "protocol text", user="alice", host="box", now=1700000000)
    fb.start_record(bdio.ASC_GENERIC, 1, True)
    fb.write(b"hello\n")
    fb.write_hash()
    fb.start_record(bdio.BIN_F64LE, 2, False)
    a = np.array([1.5, -2.0, 3.25])
    fb.write(a)
    fb.write(a[::-1])
    fb.close()
    h, recs = read_bdio(p)
    assert h["version"] == 1 and h["dirinfo"] == (0, 0) and h["ctime"] == h["mtime"] == 1700000000
    assert (h["cuser"], h["muser"], h["chost"], h["mhost"], h["protocol"]) == \
        ("alice", "alice", "box", "box", "protocol text")
    assert [(r["fmt"], r["uinfo"], r["long"]) for r in recs] == [(0xA, 1, True), (0x0, 7, False), (0x9, 2, False)]
    assert recs[0]["data"] == b"hello\n"
    magic, digest = struct.unpack("<I16s", recs[1]["data"])
    assert magic == bdio.HASH_MAGIC and digest == hashlib.md5(b"hello\n").digest()
    assert np.array_equal(np.frombuffer(recs[2]["data"], "<f8"), np.concatenate([a, a[::-1]]))


def test_record_word_limits():
    from qed2d import bdio
    assert bdio.record_word(bdio.BIN_F64LE, 3, 80, False) == 1 | (9 << 4) | (3 << 8) | (80 << 12)
    assert bdio.record_word(bdio.BIN_F64LE, 3, 1 << 30, True) >> 12 == 1 << 30
    with pytest.raises(ValueError):
        bdio.record_word(bdio.BIN_F64LE, 3, 1 << 20, False)   # a short record holds < 1 MiB
    with pytest.raises(ValueError):
        bdio.record_word(16, 0, 8, False)


def test_mc_run_file_records(tmp_path):
    """The mc driver's record sequence: input file, [L1, L2, beta, ntraj], and the
    plaquette and Q series each written L1 times, every record long and hashed."""
    from qed2d import bdio
    from qed2d.drivers import _bdio_title
    inp = tmp_path / "mc.in"
    s = {"Run": {"user": "alberto", "host": "artemisa", "name": str(tmp_path / "run")},
         "Lattice": {"size": [8, 4], "beta": 11.25}, "HMC": {"ns": 10, "eps": 0.15, "nthm": 1, "ntraj": 3,
                                                             "Qzero": False}}
    inp.write_text(json.dumps(s))
    fb = bdio.open_run_file(s["Run"]["name"], s, str(inp), _bdio_title(11.25, 8, 4), 3)
    pl, qt = [0.9, 0.91, 0.92], [0.0, 1.0, -1.0]
    for uinfo, series in ((3, pl), (4, qt)):
        fb.start_record(bdio.BIN_F64LE, uinfo, True)
        for _ in range(8):
            fb.write(np.asarray(series))
        fb.write_hash()
    fb.close()
    h, recs = read_bdio(s["Run"]["name"] + ".bdio")
    assert h["protocol"] == "Data from Master field simulation in QED [2d]; beta = 11.25; 8 x 4"
    assert h["cuser"] == "alberto" and h["chost"] == "artemisa"
    data = [r for r in recs if r["uinfo"] != 7]
    hashes = [r for r in recs if r["uinfo"] == 7]
    assert [r["uinfo"] for r in data] == [1, 2, 3, 4] and len(hashes) == 4
    assert all(r["long"] for r in data) and [r["fmt"] for r in data] == [0xA, 0x9, 0x9, 0x9]
    assert data[0]["data"] == inp.read_bytes()
    assert np.array_equal(np.frombuffer(data[1]["data"], "<f8"), [8, 4, 11.25, 3])
    assert np.array_equal(np.frombuffer(data[2]["data"], "<f8"), np.tile(pl, 8))
    assert np.array_equal(np.frombuffer(data[3]["data"], "<f8"), np.tile(qt, 8))
    for k, r in enumerate(recs):
        if r["uinfo"] == 7:
            assert r["data"][4:] == hashlib.md5(recs[k - 1]["data"]).digest()


def test_err_avg_blocks():
    """err_avg of the master-field log (main/master_field.jl:41-56) on a field
    whose 16 x 16 block means are known."""
    from qed2d.drivers import _err_avg
    blocks = np.arange(256, dtype=float).reshape(16, 16)
    dfoo = np.kron(blocks, np.ones((3, 2)))
    m, e = _err_avg(dfoo)
    assert m == pytest.approx(blocks.mean()) and e == pytest.approx(blocks.std(ddof=1) / 16)

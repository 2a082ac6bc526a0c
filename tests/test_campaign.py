"""Campaign reference files ('PDMC' format) and the library's SHA-256, on the
CPU.  Cases follow the reference's cpp/tests/test_campaign_ref_io.cpp (known
digest of the empty string, round trip with M = 1000 and N = 50, a tampered
body rejected); the digest is also checked against Python's hashlib over
lengths around the 55/56/64-byte padding boundaries, and the file layout
against an independent struct parse of the reference's header
(cpp/include/pdmk/campaign_ref_io.hpp:20-36)."""
import hashlib
import os
import struct

import numpy as np
import pytest

import periodicdmk_b200 as pd
from periodicdmk_b200 import campaign

pytestmark = pytest.mark.skipif(not os.path.exists(pd.library_path()), reason="libpdmk_b200.so not built")

HEADER = struct.Struct("<6I2B2xIQQ32s")  # magic version endian header_len config_id N digits prec M seed body_len sha


def test_sha256_known_digests():
    assert campaign.sha256(b"").hex() == "e3b0c44298fc1c149afbf4c8996fb92427ae41e4649b934ca495991b7852b855"
    assert campaign.sha256(b"abc").hex() == "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"


def test_sha256_matches_hashlib():
    rng = np.random.default_rng(5)
    for n in list(range(0, 130)) + [1000, 4095, 4096, 4097, 100003]:
        b = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert campaign.sha256(b) == hashlib.sha256(b).digest(), n
    big = b"a" * 1_000_000
    assert campaign.sha256(big) == hashlib.sha256(big).digest()


def _system(n, seed):
    rng = np.random.default_rng(seed)
    return np.eye(3), rng.uniform(0, 1, (n, 3)), rng.uniform(0, 1, n)


def test_round_trip_and_layout(tmp_path):
    cell = np.array([[1.0, 0.3, 0.2], [0.0, 0.9, 0.25], [0.0, 0.0, 0.85]])
    _, pos, q = _system(50, 1)
    idx = np.arange(campaign.DEFAULT_M) % 50
    u = np.arange(campaign.DEFAULT_M) * 1e-3
    path = str(tmp_path / "ref.bin")
    campaign.write_ref(path, cell, pos, q, idx, u, config_id=7, digits=6, prec=1, seed=0xDEADBEEFCAFEBABE)
    d = campaign.read_ref(path)
    assert (d["config_id"], d["N"], d["M"], d["digits"], d["prec"]) == (7, 50, 1000, 6, 1)
    assert d["seed"] == 0xDEADBEEFCAFEBABE
    assert np.array_equal(d["cell"], cell) and np.array_equal(d["positions"], pos)
    assert np.array_equal(d["charges"], q) and np.array_equal(d["ref_idx"], idx) and np.array_equal(d["ref_u"], u)

    raw = open(path, "rb").read()
    assert len(raw) == 80 + 72 + 12 * 1000 + 32 * 50
    h = HEADER.unpack(raw[:80])
    assert raw[:4] == bytes([0x43, 0x4D, 0x44, 0x50])
    assert h[:6] == (0x50444D43, 1, 0x01020304, 80, 7, 50)
    assert h[6:11] == (6, 1, 1000, 0xDEADBEEFCAFEBABE, len(raw) - 80)
    body = raw[80:]
    assert h[11] == hashlib.sha256(body).digest()
    # body order: cell (column-major), ref_idx, ref_u, pos, chg
    assert np.array_equal(np.frombuffer(body[:72]).reshape(3, 3).T, cell)
    assert np.array_equal(np.frombuffer(body[72:72 + 4000], dtype="<u4"), idx)
    assert np.array_equal(np.frombuffer(body[4072:12072]), u)
    assert np.array_equal(np.frombuffer(body[12072:12072 + 1200]).reshape(50, 3), pos)
    assert np.array_equal(np.frombuffer(body[13272:]), q)


def test_reads_a_file_written_from_the_format_description(tmp_path):
    # a file assembled byte by byte from the reference's layout reads back
    cell, pos, q = _system(7, 2)
    idx = np.array([0, 3, 6], dtype=np.uint32)
    u = np.array([1.5, -2.0, 0.25])
    body = cell.T.ravel().tobytes() + idx.tobytes() + u.tobytes() + pos.tobytes() + q.tobytes()
    head = HEADER.pack(0x50444D43, 1, 0x01020304, 80, 3, 7, 9, 0, 3, 42, len(body), hashlib.sha256(body).digest())
    path = str(tmp_path / "hand.bin")
    open(path, "wb").write(head + body)
    d = campaign.read_ref(path)
    assert (d["config_id"], d["N"], d["M"], d["digits"], d["prec"], d["seed"]) == (3, 7, 3, 9, 0, 42)
    assert np.array_equal(d["positions"], pos) and np.array_equal(d["ref_u"], u)


def test_rejects_tampered_and_malformed(tmp_path):
    cell, pos, q = _system(10, 3)
    path = str(tmp_path / "t.bin")
    campaign.write_ref(path, cell, pos, q, np.zeros(campaign.DEFAULT_M, np.uint32), np.zeros(campaign.DEFAULT_M))
    good = open(path, "rb").read()

    def check_bad(data, msg):
        p = str(tmp_path / "bad.bin")
        open(p, "wb").write(data)
        with pytest.raises(RuntimeError, match=msg):
            campaign.read_ref(p)

    tampered = bytearray(good)
    tampered[80] ^= 0xFF  # first body byte
    check_bad(bytes(tampered), "sha256 mismatch")
    check_bad(b"XXXX" + good[4:], "bad magic")
    check_bad(good[:4] + struct.pack("<I", 2) + good[8:], "bad version")
    check_bad(good[:8] + struct.pack("<I", 0x04030201) + good[12:], "bad endian tag")
    check_bad(good[:-1], "short read")
    check_bad(good[:40], "header short read")
    with pytest.raises(RuntimeError, match="cannot open"):
        campaign.read_ref(str(tmp_path / "missing.bin"))
    with pytest.raises(ValueError):
        campaign.write_ref(path, cell, pos, q, [10], [0.0])  # index out of range

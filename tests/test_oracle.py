"""The CPU oracle against the reference's golden data and against zlib.

These pin the oracle before it is trusted as the checker of the CUDA path:
  * tests/golden synth-* fixtures (rebuilt with the reference corpus's own
    commands) decode to the reference's recorded SHA-256 (reference_sums.json);
  * the reference's committed fixtures themselves, when the reference tree is
    present;
  * the raw-DEFLATE known-answer vectors of the reference's miri_edge.rs;
  * the behaviours of the reference's pipeline/concat/nested/BGZF tests.
"""
import json
import os
import struct
import zlib

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, REFERENCE_CORPUS, ascii_payload, golden_fixtures, gzip_cli, sha256
from rusty_rapidgzip_b200 import workloads as W


@pytest.mark.parametrize("name,path,meta", golden_fixtures(), ids=[g[0] for g in golden_fixtures()])
@pytest.mark.parametrize("threads,chunk", [(1, 4 << 20), (4, 65536)])
def test_golden_fixture_sha(name, path, meta, threads, chunk):
    data = open(path, "rb").read()
    out = oracle.read_gz(data, num_threads=threads, chunk_size=chunk)
    assert len(out) == meta["raw_size"]
    assert sha256(out) == meta["sha256"]
    assert sha256(oracle.decode_all(data)) == meta["sha256"]


@pytest.mark.skipif(not os.path.isdir(REFERENCE_CORPUS), reason="reference tree not present")
def test_reference_committed_fixtures():
    sums = json.load(open(os.path.join(REFERENCE_CORPUS, "reference_sums.json")))
    checked = 0
    for name in sorted(os.listdir(REFERENCE_CORPUS)):
        if not name.endswith(".gz"):
            continue
        data = open(os.path.join(REFERENCE_CORPUS, name), "rb").read()
        for threads in (1, 4):
            out = oracle.read_gz(data, num_threads=threads, chunk_size=65536)
            assert sha256(out) == sums[name]["sha256"], (name, threads)
        checked += 1
    assert checked == 10


def test_miri_edge_vectors():
    vecs = json.load(open(os.path.join(GOLDEN, "miri_edge_vectors.json")))
    assert {v["name"] for v in vecs} == {"empty", "stored_block", "overlap_dist1", "repeat_dist3",
                                         "repeat_dist2", "longmatch", "mixed", "far_dist"}
    for v in vecs:
        out, end_bit = oracle.inflate_raw(bytes.fromhex(v["deflate"]))
        assert out == bytes.fromhex(v["plain"]), v["name"]
        assert (end_bit + 7) // 8 == len(v["deflate"]) // 2


def test_crc32_and_combine():
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 8, 9, 1000, 65537):
        a = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert oracle.crc32(a) == zlib.crc32(a)
        for m in (0, 1, 13, 4096):
            b = rng.integers(0, 256, m, dtype=np.uint8).tobytes()
            assert oracle.crc32_combine(zlib.crc32(a), zlib.crc32(b), m) == zlib.crc32(a + b)


@pytest.mark.parametrize("level", range(1, 10))
def test_all_levels(level):
    p = ascii_payload(300_000, level)
    gz = gzip_cli(p, level)
    for threads, chunk in ((1, 1 << 20), (4, 65536)):
        assert oracle.read_gz(gz, threads, chunk) == p


@pytest.mark.parametrize("size", [1024, 65_536, 250_000, 1_000_000])
def test_matrix_sizes_chunks_threads(size):
    p = ascii_payload(size, 7)
    gz = gzip_cli(p, 6)
    for cs in (64 * 1024, 1 << 20, 4 << 20):
        for nt in (1, 4):
            assert oracle.read_gz(gz, nt, cs) == p, (size, cs, nt)


def test_mixed_block_types():
    p = ascii_payload(200_000, 1) + np.random.default_rng(5).integers(0, 256, 200_000, dtype=np.uint8).tobytes() \
        + ascii_payload(200_000, 3)
    gz = gzip_cli(p, 1)
    assert oracle.read_gz(gz, 4, 256 * 1024) == p


def _stored_member(data: bytes) -> bytes:
    hdr = bytes([0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF])
    n = len(data)
    return hdr + bytes([1]) + struct.pack("<HH", n, n ^ 0xFFFF) + data + struct.pack("<II", zlib.crc32(data), n)


def _stored_bgzf(data: bytes) -> bytes:
    n = len(data)
    body = bytes([1]) + struct.pack("<HH", n, n ^ 0xFFFF) + data
    total = 18 + len(body) + 8
    hdr = bytes([0x1F, 0x8B, 8, 4, 0, 0, 0, 0, 0, 0xFF]) + struct.pack("<H", 6) + b"BC" + struct.pack("<HH", 2, total - 1)
    return hdr + body + struct.pack("<II", zlib.crc32(data), n)


@pytest.mark.parametrize("first,second", [("bgzf", "bgzf"), ("gz", "gz"), ("bgzf", "gz"), ("gz", "bgzf")])
def test_bgzf_gz_combinations(first, second):
    mk = {"gz": _stored_member, "bgzf": _stored_bgzf}
    data = mk[first](b"hello ") + mk[second](b"world")
    assert oracle.read_gz(data, 2, 1 << 20) == b"hello world"
    assert oracle.bgzf_block_size(_stored_bgzf(b"x")) == len(_stored_bgzf(b"x"))
    assert oracle.bgzf_block_size(_stored_member(b"x")) is None


def test_bgzf_generated():
    raw = W.fastq_like(3 << 20, 4)
    b = W.bgzf(raw, 5)
    assert oracle.read_gz(b, 4) == raw
    assert oracle.read_gz(b, 1) == raw


def test_concat_members_mid_chunk():
    parts = [ascii_payload(n, i) for i, n in enumerate([1, 100, 65_537, 1, 300_000, 7, 150_000])]
    gz = b"".join(gzip_cli(p, [6, 1, 9][i % 3]) for i, p in enumerate(parts))
    for nt in (1, 2, 4):
        assert oracle.read_gz(gz, nt, 65536) == b"".join(parts)


def test_concat_empty_and_many_small():
    parts = [b"", b"abc", b"", b"", b"def" * 1000, b""]
    gz = b"".join(gzip_cli(p) for p in parts)
    assert oracle.read_gz(gz, 4, 65536) == b"".join(parts)
    parts = [f"member-{i}-payload\n".encode() for i in range(500)]
    gz = b"".join(gzip_cli(p) for p in parts)
    assert oracle.read_gz(gz, 4, 65536) == b"".join(parts)


def test_nested_gzip_recovers_from_false_boundaries():
    # printable ASCII: the inner stream is dynamic blocks of near-incompressible
    # data, so the outer stream stores it and the finder meets real inner headers
    original = np.random.default_rng(0xC0FFEE).integers(32, 127, 4 << 20, dtype=np.uint8).tobytes()
    inner = gzip_cli(original, 6)
    outer = gzip_cli(inner, 6)
    out, st = oracle.read_gz(outer, 4, 65536, with_stats=True)
    assert out == inner
    assert st["speculation_failures"] > 0


def test_block_finder_finds_real_boundaries():
    raw = ascii_payload(600_000, 11)
    gz = gzip_cli(raw, 6)
    body = gz[10:]
    # walk real block starts: a chunk decode with end hint start+1 stops after one block
    starts = [0]
    while True:
        c = oracle.decode_chunk(body, starts[-1], starts[-1] + 1)
        if c.final_block or c.actual_end_bit >= len(body) * 8:
            break
        starts.append(c.actual_end_bit)
    assert len(starts) >= 3
    assert oracle.find_next_dynamic_block(body, 0, len(body) * 8) == 0
    f = oracle.find_next_dynamic_block(body, starts[1] - 7, len(body) * 8)
    assert f in starts
    # random garbage terminates
    g = np.random.default_rng(3).integers(0, 256, 4096, dtype=np.uint8).tobytes()
    oracle.find_next_dynamic_block(g, 0, len(g) * 8)


def test_speculative_chunk_markers_resolve_to_truth():
    raw = W.zipf_text(1 << 20, 2)
    gz = W.gzip_member(raw, 9)
    body = gz[10:]
    b = oracle.find_next_dynamic_block(body, 200_000 * 8, len(body) * 8)
    assert b is not None
    first = oracle.decode_chunk(body, 0, b)
    rest = oracle.decode_chunk(body, b, 1 << 62)
    assert len(first.marker_pos) == 0
    assert len(rest.marker_pos) > 0
    assert np.all(np.diff(rest.marker_pos.astype(np.int64)) > 0)
    assert rest.marker_off.max() < 32768
    assert first.actual_end_bit == b
    head = first.bytes
    assert head == raw[:len(head)]
    tail = head[-32768:]
    fixed = bytearray(rest.bytes)
    for pos, off in zip(rest.marker_pos, rest.marker_off):
        fixed[pos] = tail[len(tail) - 1 - off]
    assert bytes(fixed) == raw[len(head):]
    assert rest.final_block


def test_error_kinds():
    good = gzip_cli(b"some payload " * 100, 6)
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(b"\x00\x01" + good[2:], 2)
    assert e.value.code == 2
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(good[:2] + b"\x07" + good[3:], 2)
    assert e.value.code == 3
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(good[:3] + b"\x20" + good[4:], 2)
    assert e.value.code == 4
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(b"", 2)
    assert e.value.code == 5
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(good[:-4], 2)
    assert e.value.code in (5, 8)
    bad_crc = good[:-8] + bytes([good[-8] ^ 1]) + good[-7:]
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(bad_crc, 2)
    assert e.value.code == 6 and e.value.member == 0
    bad_isize = good[:-4] + struct.pack("<I", 5)
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(bad_isize, 2)
    assert e.value.code == 7
    two = gzip_cli(b"first") + bad_crc
    with pytest.raises(oracle.OracleError) as e:
        oracle.read_gz(two, 1)
    assert e.value.code == 6 and e.value.member == 1

"""Parity of the CUDA decoder (through the C ABI) with the CPU oracle.

Bit-exact bytes, identical block-finder offsets, identical speculative chunk
contents (bytes + markers + end offset), identical CRC32, identical error
kinds. Large inputs are checked through size-independent properties: the
SHA-256 of the whole stream and the per-member CRC32/ISIZE the decoder
verifies itself.
"""
import hashlib
import json
import os
import struct
import zlib

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, golden_fixtures, gzip_cli, sha256
from rusty_rapidgzip_b200 import workloads as W

pytestmark = pytest.mark.gpu


def dev(data: bytes):
    import torch
    t = torch.empty(max(len(data), 1), dtype=torch.uint8, device="cuda")
    if data:
        t[: len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    torch.cuda.synchronize()
    return t


@pytest.mark.parametrize("name,path,meta", golden_fixtures(), ids=[g[0] for g in golden_fixtures()])
@pytest.mark.parametrize("gpu_chunk", [0, 4096])
def test_golden_fixtures(gpu_decoder_factory, name, path, meta, gpu_chunk):
    d = gpu_decoder_factory(gpu_chunk_bytes=gpu_chunk)
    data = open(path, "rb").read()
    out = d.decompress(data)
    assert len(out) == meta["raw_size"]
    assert sha256(out) == meta["sha256"]


def test_raw_deflate_vectors(gpu_decoder_factory):
    d = gpu_decoder_factory()
    for v in json.load(open(os.path.join(GOLDEN, "miri_edge_vectors.json"))):
        plain = bytes.fromhex(v["plain"])
        gz = bytes([0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF]) + bytes.fromhex(v["deflate"]) + \
            struct.pack("<II", zlib.crc32(plain), len(plain))
        assert d.decompress(gz) == plain, v["name"]


MODES = [dict(), dict(warps_per_stream=-1), dict(boundary_mode=1), dict(warps_per_stream=-1, boundary_mode=1)]
MODE_IDS = ["warps-scan", "lanes-scan", "warps-targets", "lanes-targets"]


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("gpu_chunk", [8192, 65536, 0])
def test_fastq_level6(gpu_decoder_factory, gpu_chunk, mode):
    raw, gz = W.config0(8 << 20, seed=5)
    d = gpu_decoder_factory(gpu_chunk_bytes=gpu_chunk, **mode)
    out, st = d.count(gz)
    assert out == len(raw)
    got = d.decompress(gz)
    assert got == raw
    assert got == oracle.read_gz(gz, 4, 1 << 20)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("gpu_chunk", [16384, 0])
def test_zipf_level9(gpu_decoder_factory, gpu_chunk, mode):
    raw, gz = W.config1(24 << 20, seed=6)
    d = gpu_decoder_factory(gpu_chunk_bytes=gpu_chunk, **mode)
    out = d.decompress(gz)
    assert out == raw


def test_device_resident_matches_host(gpu_decoder_factory):
    import torch
    raw, gz = W.config1(16 << 20, seed=8)
    d = gpu_decoder_factory(gpu_chunk_bytes=32768)
    din = dev(gz)
    dout = torch.empty(len(raw) + 64, dtype=torch.uint8, device="cuda")
    n, st = d.decode_device(din, len(gz), dout, dout.numel())
    assert n == len(raw)
    assert bytes(dout[:n].cpu().numpy()) == raw
    assert st.gpu_chunks > 1 and st.markers > 0
    # too small an output buffer reports the size needed
    from rusty_rapidgzip_b200 import CapacityError
    small = torch.empty(1024, dtype=torch.uint8, device="cuda")
    with pytest.raises(CapacityError) as e:
        d.decode_device(din, len(gz), small, small.numel())
    assert e.value.required == len(raw)


def test_resolve_window_at_an_unaligned_output_start(gpu_decoder_factory):
    """Short sub-chunks into outputs at every alignment: the second sub-chunk's
    window begins at the output's first byte, whose aligned 16-byte word lies
    before the output."""
    import torch
    raw, gz = W.config0(90_000, seed=23)
    d = gpu_decoder_factory(gpu_chunk_bytes=8 << 10)
    din = dev(gz)
    for shift in range(16):
        dout = torch.full((len(raw) + 32,), 0xA5, dtype=torch.uint8, device="cuda")
        n, st = d.decode_device(din, len(gz), dout[shift:], len(raw))
        host = dout.cpu().numpy()
        assert n == len(raw) and host[shift:shift + n].tobytes() == raw, shift
        assert (host[:shift] == 0xA5).all() and (host[shift + n:] == 0xA5).all()
        assert st.gpu_chunks >= 2 and st.markers > 0


def test_block_finder_parity(gpu_decoder_factory):
    raw, gz = W.config0(4 << 20, seed=9)
    body = gz[10:]
    nbits = len(body) * 8
    targets = list(range(8 * 4096, nbits, 8 * 12288))
    limits = targets[1:] + [nbits]
    d = gpu_decoder_factory()
    got = d.find_blocks(dev(body), len(body), targets, limits)
    want = [oracle.find_next_dynamic_block(body, t, lim) for t, lim in zip(targets, limits)]
    assert got == want
    assert sum(x is not None for x in got) > len(got) // 2
    # exhaustive limits on random data must terminate and agree
    g = np.random.default_rng(1).integers(0, 256, 1 << 16, dtype=np.uint8).tobytes()
    t2 = list(range(0, len(g) * 8, 8 * 4096))
    l2 = [len(g) * 8] * len(t2)
    assert d.find_blocks(dev(g), len(g), t2, l2) == [oracle.find_next_dynamic_block(g, t, l) for t, l in zip(t2, l2)]


def test_speculative_chunk_parity(gpu_decoder_factory):
    raw, gz = W.config1(4 << 20, seed=10)
    body = gz[10:]
    d = gpu_decoder_factory()
    db = dev(body)
    b1 = oracle.find_next_dynamic_block(body, 300_000 * 8, len(body) * 8)
    b2 = oracle.find_next_dynamic_block(body, 700_000 * 8, len(body) * 8)
    for start, hint in ((0, b1), (b1, b2), (b2, 1 << 62)):
        want = oracle.decode_chunk(body, start, hint)
        got_bytes, mp, mo, end, fin = d.decode_chunk(db, len(body), start, hint)
        assert got_bytes == want.bytes
        assert np.array_equal(mp, want.marker_pos)
        assert np.array_equal(mo, want.marker_off)
        assert end == want.actual_end_bit
        assert fin == want.final_block


def test_resolve_markers_parity(gpu_decoder_factory):
    import torch
    raw, gz = W.config1(2 << 20, seed=11)
    body = gz[10:]
    b1 = oracle.find_next_dynamic_block(body, 200_000 * 8, len(body) * 8)
    first = oracle.decode_chunk(body, 0, b1)
    rest = oracle.decode_chunk(body, b1, 1 << 62)
    tail = first.bytes[-32768:]
    d = gpu_decoder_factory()
    dbytes = dev(rest.bytes)
    dpos = torch.tensor(rest.marker_pos.astype(np.int64), dtype=torch.int64, device="cuda").to(torch.int32)
    doff = torch.tensor(rest.marker_off.astype(np.int32), device="cuda").to(torch.int16)
    torch.cuda.synchronize()
    d.resolve_markers(dbytes, len(rest.bytes), dpos, doff, len(rest.marker_pos), dev(tail), len(tail))
    torch.cuda.synchronize()
    assert bytes(dbytes[: len(rest.bytes)].cpu().numpy()) == raw[len(first.bytes):]


@pytest.mark.parametrize("n", [0, 1, 7, 4096, (1 << 20) + 13, 40 << 20])
def test_crc32_parity(gpu_decoder_factory, n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    d = gpu_decoder_factory()
    assert d.crc32(dev(data), n) == zlib.crc32(data)


@pytest.mark.parametrize("mode", MODES[:2], ids=MODE_IDS[:2])
def test_bgzf(gpu_decoder_factory, mode):
    raw = W.fastq_like(12 << 20, 12)
    b = W.bgzf(raw, 5)
    d = gpu_decoder_factory(**mode)
    assert d.decompress(b) == raw
    out, st = d.count(b)
    assert out == len(raw) and st.members == (len(raw) + 65279) // 65280


def _stored_member(data: bytes) -> bytes:
    n = len(data)
    return bytes([0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF, 1]) + struct.pack("<HH", n, n ^ 0xFFFF) + data + \
        struct.pack("<II", zlib.crc32(data), n)


def _stored_bgzf(data: bytes) -> bytes:
    n = len(data)
    body = bytes([1]) + struct.pack("<HH", n, n ^ 0xFFFF) + data
    hdr = bytes([0x1F, 0x8B, 8, 4, 0, 0, 0, 0, 0, 0xFF]) + struct.pack("<H", 6) + b"BC" + \
        struct.pack("<HH", 2, 18 + len(body) + 8 - 1)
    return hdr + body + struct.pack("<II", zlib.crc32(data), n)


@pytest.mark.parametrize("first,second", [("bgzf", "bgzf"), ("gz", "gz"), ("bgzf", "gz"), ("gz", "bgzf")])
def test_bgzf_gz_combinations(gpu_decoder_factory, first, second):
    mk = {"gz": _stored_member, "bgzf": _stored_bgzf}
    d = gpu_decoder_factory()
    assert d.decompress(mk[first](b"hello ") + mk[second](b"world")) == b"hello world"


def test_batch_of_files(gpu_decoder_factory):
    import torch
    files = W.config3_files(n_files=12, seed=4, lo=4 << 10, hi=2 << 20)
    blobs = [gz for _, gz in files]
    offs = np.cumsum([0] + [len(b) for b in blobs])[:-1].tolist()
    raws = [r for r, _ in files]
    ooffs = np.cumsum([0] + [len(r) for r in raws])[:-1].tolist()
    din = dev(b"".join(blobs))
    dout = torch.empty(sum(len(r) for r in raws) + 16, dtype=torch.uint8, device="cuda")
    d = gpu_decoder_factory()
    lens, status, st = d.decode_batch(din, offs, [len(b) for b in blobs], dout, ooffs, [len(r) for r in raws])
    assert status == [0] * len(files)
    assert lens == [len(r) for r in raws]
    host = dout.cpu().numpy().tobytes()
    for r, o in zip(raws, ooffs):
        assert host[o:o + len(r)] == r


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_concat_members(gpu_decoder_factory, mode):
    parts = [W.fastq_like(n, i) for i, n in enumerate([1, 100, 65_537, 1, 300_000, 7, 1_000_000])]
    gz = b"".join(gzip_cli(p, [6, 1, 9][i % 3]) for i, p in enumerate(parts))
    for gc in (4096, 65536):
        d = gpu_decoder_factory(gpu_chunk_bytes=gc, **mode)
        assert d.decompress(gz) == b"".join(parts)
    parts = [b"", b"abc", b"", b"", b"def" * 1000, b""] + [f"member-{i}-payload\n".encode() for i in range(500)]
    gz = b"".join(gzip_cli(p) for p in parts)
    d = gpu_decoder_factory(gpu_chunk_bytes=4096)
    assert d.decompress(gz) == b"".join(parts)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_nested_gzip(gpu_decoder_factory, mode):
    original = np.random.default_rng(0xC0FFEE).integers(32, 127, 2 << 20, dtype=np.uint8).tobytes()
    inner = gzip_cli(original, 6)
    outer = gzip_cli(inner, 6)
    d = gpu_decoder_factory(gpu_chunk_bytes=16384, **mode)
    out, st = [], None
    st = d.decode_host(outer, out.append)
    assert b"".join(out) == inner
    assert st.speculation_failures > 0


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_mixed_block_types(gpu_decoder_factory, mode):
    p = W.fastq_like(300_000, 1) + W.random_bytes(300_000, 5) + W.zipf_text(300_000, 3)
    gz = gzip_cli(p, 1)
    d = gpu_decoder_factory(gpu_chunk_bytes=16384, **mode)
    assert d.decompress(gz) == p


def _expect(code, fn):
    from rusty_rapidgzip_b200 import RrgError
    with pytest.raises(RrgError) as e:
        fn()
    return e.value


def test_error_kinds_match_oracle(gpu_decoder_factory):
    d = gpu_decoder_factory()
    good = gzip_cli(W.fastq_like(200_000, 3), 6)
    cases = {
        "magic": b"\x00\x01" + good[2:],
        "method": good[:2] + b"\x07" + good[3:],
        "flags": good[:3] + b"\x20" + good[4:],
        "empty": b"",
        "crc": good[:-8] + bytes([good[-8] ^ 1]) + good[-7:],
        "isize": good[:-4] + struct.pack("<I", 5),
        "second_crc": gzip_cli(b"first") + good[:-8] + bytes([good[-8] ^ 1]) + good[-7:],
    }
    for name, data in cases.items():
        with pytest.raises(oracle.OracleError) as oe:
            oracle.read_gz(data, 2)
        err = _expect(None, lambda: d.decompress(data))
        assert err.code == oe.value.code, name
        if name in ("crc", "second_crc"):
            assert err.member == oe.value.member
            assert err.expected == oe.value.expected and err.got_crc == oe.value.got_crc
    # truncation: an error either way (EOF or Truncated, like the reference)
    err = _expect(None, lambda: d.decompress(good[:-4]))
    assert err.code in (5, 8)


def test_read_gz_path_sink_and_close(tmp_path, gpu_decoder_factory):
    from rusty_rapidgzip_b200 import SinkClosed, read_gz, Config
    raw, gz = W.config0(6 << 20, seed=13)
    p = tmp_path / "x.gz"
    p.write_bytes(gz)
    chunks = []
    st = read_gz(p, chunks.append, Config(device=0, chunk_size_bytes=1 << 20))
    assert b"".join(chunks) == raw
    assert st.uncompressed_bytes == len(raw) and st.compressed_bytes == len(gz)
    assert st.chunks_decoded == len(chunks) and len(chunks) > 1
    got = []

    def closing(b):
        got.append(b)
        raise SinkClosed()

    st2 = read_gz(p, closing, Config(device=0, chunk_size_bytes=1 << 20))
    assert len(got) == 1 and raw.startswith(got[0])
    z = tmp_path / "zero.gz"
    z.write_bytes(b"")
    from rusty_rapidgzip_b200 import GzipError
    with pytest.raises(GzipError) as e:
        read_gz(z, lambda b: None, Config(device=0))
    assert e.value.kind == "Truncated"


def test_large_stream_properties(gpu_decoder_factory):
    """256 MiB of the Zipf-text shape: SHA-256 of the whole stream plus the
    decoder's own CRC32/ISIZE check; device and host entry points agree."""
    import torch
    raw, gz = W.config1(256 << 20, seed=14)
    d = gpu_decoder_factory()
    din = dev(gz)
    dout = torch.empty(len(raw) + 64, dtype=torch.uint8, device="cuda")
    n, st = d.decode_device(din, len(gz), dout, dout.numel())
    assert n == len(raw)
    h = hashlib.sha256(dout[:n].cpu().numpy().tobytes()).hexdigest()
    assert h == sha256(raw)
    assert st.members == 1 and st.gpu_chunks > 100
    # every sub-chunk start is a real block start: no speculative decode is redone
    assert st.speculation_failures == 0


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["chain", "false-headers", "then-plain", "truncated", "crc"])
def test_bgzf_device_walk(gpu_decoder_factory, case):
    """The device BGZF member walk (scan, compaction, chain) against the oracle,
    including the error kind, member index and trailer position."""
    from conftest import bgzf_cases
    from rusty_rapidgzip_b200 import RrgError
    data = bgzf_cases()[case]
    d = gpu_decoder_factory()
    try:
        want = oracle.read_gz(data, 2)
    except oracle.OracleError as oe:
        with pytest.raises(RrgError) as ge:
            d.decompress(data)
        assert (ge.value.code, ge.value.member, ge.value.trailer_byte) == (oe.code, oe.member, oe.trailer_byte)
        return
    assert d.decompress(data) == want
    # a second decode of the same layout replays the captured graph
    import numpy as np
    import torch
    din = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda()
    dout = torch.empty(len(want) + 64, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        n, st = d.decode_device(din, len(data), dout, dout.numel())
        assert n == len(want) and bytes(dout[:n].cpu().numpy()) == want
    assert st.graph_launches == 1


@pytest.mark.gpu
@pytest.mark.parametrize("plan", [0, -1], ids=["device-planned", "host-planned"])
@pytest.mark.parametrize("budget", [0, 1], ids=["one-wave", "waves"])
def test_batch_mixed(gpu_decoder_factory, budget, plan):
    """A batch mixing multi-chunk, single-chunk, multi-member and BGZF files, a
    corrupt file and a too-small output range; per-item status and bytes against
    the oracle, in one wave and in several, on the device-planned route (whose
    unfinished jobs go the checked route) and on the host-planned one."""
    import torch
    from test_emu import batch_items, expected_status, run_batch

    def devbuf(data, out_n):
        din = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda()
        dout = torch.zeros(out_n, dtype=torch.uint8, device="cuda")
        return din, dout, lambda: dout.cpu().numpy().tobytes()

    items = batch_items()
    d = gpu_decoder_factory(hbm_budget_bytes=budget, batch_plan=plan)
    outs, lens, status = run_batch(d, items, devbuf)
    for (raw, gz, cap), got, n, stt in zip(items, outs, lens, status):
        want = expected_status(gz)
        if want == 0 and raw is not None and len(raw) > cap:
            assert stt == 24 and n == len(raw)
        else:
            assert stt == want
            if want == 0:
                assert got == raw


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [0, 65536], ids=["auto-spacing", "64KiB"])
def test_batch_graph_replay(gpu_decoder_factory, chunk):
    """A batch of single-member files of uneven size on the device-planned
    route: the first call runs its launches directly, the second (the same
    shape again) captures and launches the graph, the third replays it, each
    into a zeroed output whose every file's bytes come back; the host-planned
    route decodes the same bytes."""
    import torch
    files = W.config3_files(n_files=40, seed=21, lo=4 << 10, hi=6 << 20)
    blobs = [gz for _, gz in files]
    raws = [r for r, _ in files]
    offs = np.cumsum([0] + [len(b) for b in blobs])[:-1].tolist()
    ooffs = np.cumsum([0] + [len(r) for r in raws])[:-1].tolist()
    din = dev(b"".join(blobs))
    dout = torch.zeros(sum(len(r) for r in raws) + 16, dtype=torch.uint8, device="cuda")
    d = gpu_decoder_factory(gpu_chunk_bytes=chunk)
    for call in range(3):
        dout.zero_()
        lens, status, st = d.decode_batch(din, offs, [len(b) for b in blobs], dout, ooffs, [len(r) for r in raws])
        assert status == [0] * len(files) and lens == [len(r) for r in raws]
        assert st.graph_launches == (1 if call else 0) and st.members == len(files)
        host = dout.cpu().numpy().tobytes()
        for r, o in zip(raws, ooffs):
            assert host[o:o + len(r)] == r
    assert st.gpu_chunks > len(files)  # the larger files were split
    h = gpu_decoder_factory(gpu_chunk_bytes=chunk, batch_plan=-1)
    dout.zero_()
    lens, status, st = h.decode_batch(din, offs, [len(b) for b in blobs], dout, ooffs, [len(r) for r in raws])
    assert status == [0] * len(files) and st.graph_launches == 0
    assert dout.cpu().numpy().tobytes()[:sum(len(r) for r in raws)] == b"".join(raws)


@pytest.mark.gpu
def test_autotune(gpu_decoder_factory):
    """The sweep (sub-chunk size, boundary search and scan tile, warps per BGZF
    member) on a sample batch, then the batch decodes exactly under the chosen
    setting."""
    import torch
    from test_emu import run_batch
    raw_a, gz_a = W.config1(6 << 20, seed=8)
    raw_b = W.fastq_like(3 << 20, 9)
    items = [(raw_a, gz_a, len(raw_a)), (raw_b, W.bgzf(raw_b, 5), len(raw_b))]

    def devbuf(data, out_n):
        din = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda()
        dout = torch.zeros(out_n, dtype=torch.uint8, device="cuda")
        return din, dout, lambda: dout.cpu().numpy().tobytes()

    d = gpu_decoder_factory()
    blobs = [gz for _, gz, _ in items]
    offs = np.cumsum([0] + [len(b) for b in blobs])[:-1].tolist()
    caps = [cap for _, _, cap in items]
    ooffs = np.cumsum([0] + caps)[:-1].tolist()
    din, dout, _ = devbuf(b"".join(blobs), sum(caps) + 64)
    t = d.autotune(din, offs, [len(b) for b in blobs], dout, ooffs, caps)
    assert t["trials"] >= 12 and 0 < t["best_ms"] <= t["default_ms"] * 1.0001
    assert t["boundary_mode"] in (0, 1) and 1 <= t["warps_per_member"] <= 4
    outs, lens, status = run_batch(d, items, devbuf)
    assert status == [0, 0] and outs == [raw_a, raw_b]


@pytest.mark.gpu
def test_serving_alone_and_in_the_mix(gpu_decoder_factory):
    """Serving loop: each request's bytes and status are the same decoded alone
    and in the mix; requests queue for a 256 MiB budget, batches hold several
    requests (continuous batching) and both engines run at once (overlap)."""
    from conftest import run_serving, serve_requests
    reqs = serve_requests(40, seed=12, hi=24 << 20)
    alone = gpu_decoder_factory()
    want = {}
    for i, gz in enumerate(reqs):
        try:
            want[i] = (0, alone.decompress(gz))
        except Exception as e:  # noqa: BLE001 - compared by status code below
            want[i] = (e.code, None)
    budget = 256 << 20
    d = gpu_decoder_factory(hbm_budget_bytes=budget)
    d.serve_start(engines=2, max_ready=8)
    got = run_serving(d, reqs, seed=2, gap_s=0.002, copy=False)  # zero-copy submits
    assert got == want
    st = d.serve_stats()
    assert st["completed"] == len(reqs) and d.pending() == 0
    assert st["max_batch"] >= 2 and st["max_engines_busy"] == 2
    assert st["peak_in_use_bytes"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("stripe", [4 << 20, 0], ids=["4MiB-stripes", "default-stripes"])
def test_read_stream_gpu(gpu_decoder_factory, stripe):
    """A 64 MiB Zipf member and a multi-member stream read forward stripe by
    stripe: bytes equal the generator's, counts equal the input's."""
    import io
    raw, gz = W.config1(64 << 20, seed=11)
    d = gpu_decoder_factory()
    h, n = hashlib.sha256(), [0]

    def sink(b):
        h.update(b)
        n[0] += len(b)

    st = d.read_stream(io.BytesIO(gz), sink, stripe_bytes=stripe)
    assert n[0] == len(raw) and h.digest() == hashlib.sha256(raw).digest()
    assert st.compressed_bytes == len(gz) and st.speculation_failures == 0
    rnd = np.random.default_rng(12).integers(0, 256, 3 << 20, dtype=np.uint8).tobytes()
    parts = [raw[: 20 << 20], rnd, b"", raw[20 << 20:]]
    multi = b"".join(W.gzip_member(p, 6) for p in parts)
    out = []
    st = d.read_stream(io.BytesIO(multi), out.append, stripe_bytes=stripe)
    assert b"".join(out) == b"".join(parts) and st.members == 4


@pytest.mark.gpu
def test_read_stream_gpu_errors(gpu_decoder_factory):
    """A CRC32 error in a member spanning stripes and a truncated stream give
    the oracle's error (code; member and trailer offset for CRC32)."""
    import io
    from rusty_rapidgzip_b200 import RrgError
    raw, gz = W.config1(8 << 20, seed=13)
    bad = bytearray(gz)
    bad[-8] ^= 1
    d = gpu_decoder_factory()
    for data in (bytes(bad), gz[: len(gz) // 2]):
        with pytest.raises(oracle.OracleError) as oe:
            oracle.read_gz(data, 4)
        with pytest.raises(RrgError) as ge:
            d.read_stream(io.BytesIO(data), None, stripe_bytes=1 << 20)
        assert ge.value.code == oe.value.code
        if oe.value.code == 6:
            assert (ge.value.member, ge.value.trailer_byte) == (oe.value.member, oe.value.trailer_byte)


@pytest.mark.gpu
def test_read_gz_pipe_gpu(gpu_decoder_factory, tmp_path):
    """read_gz on a named pipe decodes through the stripe route."""
    import threading
    raw, gz = W.config0(32 << 20, seed=14)
    fifo = str(tmp_path / "in.gz")
    os.mkfifo(fifo)

    def writer():
        with open(fifo, "wb") as f:
            f.write(gz)

    t = threading.Thread(target=writer)
    t.start()
    out = []
    st = gpu_decoder_factory().read_gz(fifo, out.append)
    t.join()
    assert b"".join(out) == raw and st.compressed_bytes == len(gz)


@pytest.mark.gpu
def test_seek_index_gpu(gpu_decoder_factory):
    """Seek index of a 128 MiB Zipf member plus a FASTQ member: random ranges
    read from checkpoints equal the generator's bytes."""
    raw, gz = W.config1(128 << 20, seed=16)
    tail = W.fastq_like(8 << 20, 16)
    data = gz + W.gzip_member(tail, 6)
    whole = raw + tail
    d = gpu_decoder_factory()
    idx = d.build_index(data)
    pts = idx.points()
    assert idx.total_out == len(whole) and len(pts) >= 30
    rng = np.random.default_rng(16)
    cases = [(0, 4096), (len(raw) - 100_000, 300_000), (pts[-1][0], len(whole) - pts[-1][0])]
    cases += [(int(o), int(n)) for o, n in zip(rng.integers(0, len(whole), 6), rng.integers(1, 9 << 20, 6))]
    for off, n in cases:
        n = min(n, len(whole) - off)
        assert d.read_range(data, idx, off, n) == whole[off:off + n], (off, n)


@pytest.mark.parametrize("size", [4 << 20, 128 << 20])
def test_fixed_huffman_blocks(gpu_decoder_factory, size):
    """Fixed-Huffman blocks only (zlib level 1, Z_FIXED): block starts come
    from the fixed-code walk, so the member splits into many sub-chunks with
    no re-decode, device-resident and through the pipelined host path."""
    import torch
    raw, gz = W.fixed_blocks(size, seed=21)
    if size <= 4 << 20:
        assert oracle.read_gz(gz, 4, 1 << 20) == raw
    d = gpu_decoder_factory()
    src = dev(gz)
    out = torch.empty(len(raw) + (1 << 20), dtype=torch.uint8, device="cuda")
    n, st = d.decode_device(src.data_ptr(), len(gz), out.data_ptr(), out.numel())
    assert n == len(raw)
    assert hashlib.sha256(out[:n].cpu().numpy().tobytes()).hexdigest() == sha256(raw)
    assert st.gpu_chunks >= 32 and st.speculation_failures == 0
    got = []
    d2 = gpu_decoder_factory(host_pipeline=2)  # two overlapped waves where the input is large enough
    st2 = d2.decode_host(gz, got.append)
    assert b"".join(got) == raw
    assert st2.gpu_chunks >= 32 and st2.speculation_failures == 0
    assert st2.pipeline_waves == (2 if size > 64 << 20 else 0)


def test_device_planned_member_falls_back_gpu(gpu_decoder_factory):
    """decode_device takes the device-planned route for members of 16 MiB or
    more and replays it as a graph when the call repeats; two concatenated
    members and trailing bytes fall back to the checked route, with the
    oracle's bytes and error code."""
    import torch
    from rusty_rapidgzip_b200 import RrgError
    r1, g1 = W.config0(48 << 20, seed=41)
    r2 = b"second member " * 4096
    g2 = gzip_cli(r2, 6)
    d = gpu_decoder_factory()

    def device(gz, cap, reuse=None):
        src = reuse[0] if reuse else dev(gz)
        out = reuse[1] if reuse else torch.empty(cap + 64, dtype=torch.uint8, device="cuda")
        n, st = d.decode_device(src.data_ptr(), len(gz), out.data_ptr(), out.numel())
        return out[:n].cpu().numpy().tobytes(), st, (src, out)

    got, st, bufs = device(g1, len(r1))
    assert got == r1 and st.members == 1 and st.speculation_failures == 0
    for _ in range(2):
        got, st, _ = device(g1, len(r1), reuse=bufs)
        assert got == r1
    assert st.graph_launches == 1
    got, st, _ = device(g1 + g2, len(r1) + len(r2))
    assert got == r1 + r2 and st.members == 2
    bad = g1 + b"\x1f\x8b\x08\x00garbage"
    with pytest.raises(RrgError) as ge:
        device(bad, len(r1))
    with pytest.raises(oracle.OracleError) as oe:
        oracle.read_gz(bad, 4, 1 << 20)
    assert ge.value.code == oe.value.code

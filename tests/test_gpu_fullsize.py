"""Parity of the CUDA decoder at (or near) the benchmark configurations' full
sizes, through the C ABI: every output is compared with the generator's bytes
by SHA-256, and the decoder checks every member's CRC32/ISIZE itself.

* FASTQ-like text, 64 MiB, zlib level 6, one member (the plain path);
* Zipf text, 256 MiB, one plain zlib level-9 stream (no sync-flush points);
* Zipf text, 1 GiB, one member, through the pipelined host path;
* BGZF, 256 MiB of FASTQ-like text at level 5 (> 4,000 members), through the
  captured decode graph, replayed;
* a batch of 100 files with one 64 MiB file of each content kind, decoded in
  several waves;
* serving with a 512 MiB request, alone and in a mix of smaller ones.
"""
import hashlib

import numpy as np
import pytest

from rusty_rapidgzip_b200 import workloads as W

pytestmark = pytest.mark.gpu


def sha(b) -> str:
    return hashlib.sha256(b).hexdigest()


def dev(data: bytes):
    import torch
    t = torch.empty(max(len(data), 1), dtype=torch.uint8, device="cuda")
    if data:
        t[: len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    torch.cuda.synchronize()
    return t


def host_sha(d, gz):
    """decode_host into a hashing sink: (sha256, bytes, stats)."""
    h = hashlib.sha256()
    n = [0]

    def sink(b):
        h.update(b)
        n[0] += len(b)

    st = d.decode_host(gz, sink)
    return h.hexdigest(), n[0], st


def device_sha(d, gz, n_out):
    import torch
    din = dev(gz)
    dout = torch.empty(n_out + 64, dtype=torch.uint8, device="cuda")
    n, st = d.decode_device(din, len(gz), dout, dout.numel())
    return sha(dout[:n].cpu().numpy().tobytes()), n, st


def test_fastq_64mib_level6(gpu_decoder_factory):
    raw, gz = W.config0(64 << 20, seed=0)
    d = gpu_decoder_factory()
    h, n, st = host_sha(d, gz)
    assert (h, n) == (sha(raw), len(raw)) and st.members == 1
    h2, n2, st2 = device_sha(d, gz, len(raw))
    assert (h2, n2) == (sha(raw), len(raw)) and st2.gpu_chunks > 1000


def test_zipf_plain_zlib_stream_256mib(gpu_decoder_factory):
    """One zlib level-9 stream as zlib writes it (no pieces, no sync flushes):
    every sub-chunk starts at a dynamic block the boundary scan verified."""
    raw = W.zipf_text(256 << 20, 31)
    gz = W.gzip_member(raw, 9, parallel_threshold=1 << 62)
    d = gpu_decoder_factory()
    h, n, st = device_sha(d, gz, len(raw))
    assert (h, n) == (sha(raw), len(raw))
    assert st.members == 1 and st.gpu_chunks > 1000 and st.speculation_failures == 0
    h2, n2, _ = host_sha(d, gz)
    assert (h2, n2) == (sha(raw), len(raw))


def test_zipf_1gib_pipelined_host_path(gpu_decoder_factory):
    """The benchmark's 1 GiB member from host memory: decoded in waves with the
    copy to the host overlapped, no fallback; the same bytes on the checked path."""
    raw, gz = W.config1(1 << 30, seed=1)
    d = gpu_decoder_factory()
    h, n, st = host_sha(d, gz)
    assert (h, n) == (sha(raw), len(raw))
    assert st.pipeline_waves >= 2 and st.pipeline_fallbacks == 0 and st.members == 1
    plain = gpu_decoder_factory(host_pipeline=-1)
    h2, n2, st2 = host_sha(plain, gz)
    assert (h2, n2) == (sha(raw), len(raw)) and st2.pipeline_waves == 0


def test_bgzf_256mib_graph_replay(gpu_decoder_factory):
    """More than 4,000 BGZF members in one captured graph; the second decode
    replays it; both outputs equal the generator's."""
    import torch
    raw = W.fastq_like(256 << 20, 5)
    gz = W.bgzf(raw, 5)
    d = gpu_decoder_factory()
    # the same buffers both times: a decode graph is kept per shape and buffers
    din = dev(gz)
    dout = torch.empty(len(raw) + 64, dtype=torch.uint8, device="cuda")
    for k in range(2):
        dout.fill_(0)
        n, st = d.decode_device(din, len(gz), dout, dout.numel())
        assert (sha(dout[:n].cpu().numpy().tobytes()), n) == (sha(raw), len(raw))
        assert st.members >= 4000
    assert st.graph_launches >= 1
    h, n, _ = host_sha(d, gz)
    assert (h, n) == (sha(raw), len(raw))


def test_batch_100_files_with_64mib_of_each_kind(gpu_decoder_factory):
    """96 files of log-uniform size (4 KiB to 4 MiB, mixed content) and one
    64 MiB file of each content kind (FASTQ-like level 6, Zipf level 9, random
    bytes level 1, sparse binary level 6), in one batch whose budget forces
    several waves; every file's bytes and status."""
    import torch
    small = W.config3_files(n_files=96, seed=40, lo=4 << 10, hi=4 << 20)
    big = []
    for i, kind in enumerate(W.CONTENT_KINDS):
        r = W.make_content(kind, 64 << 20, 900 + i)
        big.append((r, W.gzip_member(r, W.CONTENT_LEVEL[kind])))
    files = small[:24] + big[:2] + small[24:72] + big[2:] + small[72:]
    blobs = [gz for _, gz in files]
    offs = np.cumsum([0] + [len(b) for b in blobs])[:-1].tolist()
    caps = [len(r) for r, _ in files]
    ooffs = np.cumsum([0] + caps)[:-1].tolist()
    din = torch.from_numpy(np.frombuffer(b"".join(blobs), dtype=np.uint8).copy()).cuda()
    dout = torch.zeros(sum(caps) + 64, dtype=torch.uint8, device="cuda")
    d = gpu_decoder_factory(hbm_budget_bytes=1 << 30)
    for call in range(2):  # the second call replays each wave's captured graph
        dout.zero_()
        lens, status, st = d.decode_batch(din, offs, [len(b) for b in blobs], dout, ooffs, caps)
        assert status == [0] * len(files) and lens == caps
        out = dout.cpu().numpy()
        for (r, _), o in zip(files, ooffs):
            assert sha(out[o:o + len(r)].tobytes()) == sha(r)
        assert st.members == len(files) and (call == 0 or st.graph_launches >= 2)


def test_serving_512mib_request_alone_and_in_the_mix(gpu_decoder_factory):
    """A 512 MiB request among 20 smaller ones arriving at random gaps: every
    result equals the same request decoded alone."""
    from conftest import run_serving
    big_raw = W.fastq_like(512 << 20, 41)
    big = W.gzip_member(big_raw, 6)
    reqs = [gz for _, gz in W.config3_files(n_files=20, seed=42, lo=64 << 10, hi=16 << 20)]
    reqs.insert(7, big)
    alone = gpu_decoder_factory()
    want = {i: (0, sha(alone.decompress(gz))) for i, gz in enumerate(reqs)}
    assert want[7][1] == sha(big_raw)
    d = gpu_decoder_factory()
    d.serve_start(engines=2, max_ready=8)
    got = run_serving(d, reqs, seed=3, gap_s=0.01, copy=False)
    assert {i: (s, sha(b) if b is not None else None) for i, (s, b) in got.items()} == want
    st = d.serve_stats()
    assert st["completed"] == len(reqs) and d.pending() == 0


def test_member_split_in_four_ranges(gpu_decoder_factory):
    """The member-split path on one GPU: 256 MiB of Zipf text in four ranges,
    each decoded by its own context (phase 1), the windows composed from the
    ranges' maps, then each range resolved (phase 2); the joined bytes and the
    combined CRC32/ISIZE equal the member's."""
    from rusty_rapidgzip_b200.sharding import gzip_body_offset
    raw, gz = W.config1(256 << 20, seed=44)
    body = gzip_body_offset(gz)
    nbits = (len(gz) - body - 8) * 8
    world = 4
    decs = [gpu_decoder_factory() for _ in range(world)]
    infos, maps = [], []
    for r in range(world):
        stop = nbits * (r + 1) // world if r + 1 < world else (1 << 64) - 1
        info, m = decs[r].split_begin(gz, body, nbits * r // world, stop)
        infos.append(info)
        maps.append(m)
    for a, b in zip(infos, infos[1:]):
        assert b["start_bit"] == a["end_bit"]
    win = np.full(32768, 0x4000, dtype=np.uint16)
    h = hashlib.sha256()
    crc, total = 0, 0
    for r in range(world):
        wlen = min(32768, sum(i["out_len"] for i in infos[:r]))
        w = win[32768 - wlen:]
        assert (w < 0x100).all()
        c, n = decs[r].split_finish(w.astype(np.uint8).tobytes(), h.update)
        crc = decs[0].crc32_combine(crc, c, n) if r else c
        total += n
        win = np.where(maps[r] & 0x8000, win[maps[r] & 0x7FFF], maps[r]).astype(np.uint16)
    assert h.hexdigest() == sha(raw) and total == len(raw)
    assert infos[-1]["has_trailer"] and crc == infos[-1]["crc"] and total & 0xFFFFFFFF == infos[-1]["isize"]

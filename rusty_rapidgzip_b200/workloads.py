"""Seeded synthetic inputs shaped like the benchmark configurations.

* ``fastq_like``   — 4-line records: ``@r<index>``, 150 bases uniform over ACGT
  with 1% N, ``+``, 150 quality chars from '!'..'J' (triangular, mode 'F').
* ``zipf_text``    — 50,000-word vocabulary of random lowercase words (length
  uniform 2..12) sampled with Zipf exponent 1.1; words separated by spaces with
  a newline every 8..20 words.
* ``random_bytes`` — uniform bytes (level 1 gives stored/fixed blocks).
* ``sparse_binary``— 90% zero bytes in runs of geometric length (mean 64),
  uniform random bytes elsewhere.

Compression uses zlib. ``gzip_member`` writes ONE gzip member; above
``parallel_threshold`` it compresses 32 MiB pieces on threads, each primed with
the previous piece's last 32 KiB as a preset dictionary and ended with a sync
flush (the pigz construction), so the result is still a single member of
ordinary zlib blocks. ``bgzf`` writes BGZF members (<= 65280 input bytes each,
``BC`` extra subfield).
"""
from __future__ import annotations

import struct
import zlib
from concurrent.futures import ThreadPoolExecutor

import numpy as np

# ---------------------------------------------------------------- generators


def _fastq_segment(n_bytes: int, rng, first_index: int) -> np.ndarray:
    """FASTQ-like records, truncated to exactly ``n_bytes``."""
    out = []
    total = 0
    idx = first_index
    while total < n_bytes:
        digits = len(str(idx))
        # records whose index has the same number of digits share one layout
        limit = 10 ** digits
        rec_len = 2 + digits + 1 + 150 + 1 + 2 + 150 + 1
        want = (n_bytes - total + rec_len - 1) // rec_len
        n = int(min(limit - idx, max(want, 1), 1 << 20))
        rec = np.empty((n, rec_len), dtype=np.uint8)
        rec[:, 0] = ord("@")
        rec[:, 1] = ord("r")
        ids = np.arange(idx, idx + n, dtype=np.int64)
        for d in range(digits):
            rec[:, 2 + d] = ord("0") + (ids // 10 ** (digits - 1 - d)) % 10
        p = 2 + digits
        rec[:, p] = ord("\n")
        p += 1
        bases = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, size=(n, 150))]
        bases[rng.random((n, 150)) < 0.01] = ord("N")
        rec[:, p:p + 150] = bases
        p += 150
        rec[:, p] = ord("\n")
        rec[:, p + 1] = ord("+")
        rec[:, p + 2] = ord("\n")
        p += 3
        q = np.floor(rng.triangular(33.0, 70.5, 75.0, size=(n, 150)))
        rec[:, p:p + 150] = np.clip(q, 33, 74).astype(np.uint8)
        p += 150
        rec[:, p] = ord("\n")
        out.append(rec.reshape(-1))
        total += rec.size
        idx += n
    return np.concatenate(out)[:n_bytes]


def _zipf_vocab(rng):
    lens = rng.integers(2, 13, size=50_000)
    vocab = rng.integers(ord("a"), ord("z") + 1, size=(50_000, 12), dtype=np.uint8)
    p = np.arange(1, 50_001, dtype=np.float64) ** -1.1
    cdf = np.cumsum(p / p.sum())
    return vocab, lens, cdf


def _zipf_segment(n_bytes: int, rng, vocab_rng_seed: int) -> np.ndarray:
    vocab, lens, cdf = _zipf_vocab(np.random.default_rng(vocab_rng_seed))
    # flat vocabulary: word i occupies flat[wstart[i] : wstart[i] + lens[i] + 1]
    wstart = np.concatenate(([0], np.cumsum(lens + 1)[:-1])).astype(np.int64)
    flat = np.zeros(int(wstart[-1] + lens[-1] + 1), dtype=np.uint8)
    for L in range(2, 13):
        sel = np.nonzero(lens == L)[0]
        cols = wstart[sel][:, None] + np.arange(L)
        flat[cols] = vocab[sel, :L]
    out = np.empty(n_bytes, dtype=np.uint8)
    filled = 0
    carry = int(rng.integers(8, 21))  # words left in the current line
    block_words = 1 << 20
    while filled < n_bytes:
        ranks = np.minimum(np.searchsorted(cdf, rng.random(block_words), side="right"), 49_999)
        wl = lens[ranks]
        # line ends: the current line ends after `carry` words, then every 8..20
        line_lens = rng.integers(8, 21, size=block_words // 8 + 2)
        ends = carry - 1 + np.concatenate(([0], np.cumsum(line_lens)))
        inside = ends < block_words
        sep = np.full(block_words, ord(" "), dtype=np.uint8)
        sep[ends[inside]] = ord("\n")
        carry = int(ends[inside.sum()] - block_words + 1)
        tok = (wl + 1).astype(np.int64)
        pos = np.cumsum(tok) - tok
        total = int(pos[-1] + tok[-1])
        take = min(total, n_bytes - filled)
        # byte b of token t is flat[wstart[rank_t] + (b - pos_t)]; one 1-D gather
        idx = np.repeat(wstart[ranks] - pos, tok)[:take] + np.arange(take, dtype=np.int64)
        byte = flat[idx]
        sp = pos + wl
        keep = sp < take
        byte[sp[keep]] = sep[keep]
        out[filled:filled + take] = byte
        filled += take
    return out


SEGMENT = 16 << 20


def _segmented(fn, n_bytes: int, seed: int) -> bytes:
    """Concatenate independently seeded SEGMENT-sized pieces made on threads."""
    nseg = max(1, (n_bytes + SEGMENT - 1) // SEGMENT)
    out = np.empty(n_bytes, dtype=np.uint8)

    def work(k):
        s = k * SEGMENT
        e = min(n_bytes, s + SEGMENT)
        out[s:e] = fn(e - s, np.random.default_rng([seed, k]), k)

    with ThreadPoolExecutor() as ex:
        list(ex.map(work, range(nseg)))
    return out.tobytes()


def fastq_like(n_bytes: int, seed: int = 0) -> bytes:
    """FASTQ-like records; record indices run on across segments."""
    per_seg = SEGMENT // 300 + 1
    return _segmented(lambda n, rng, k: _fastq_segment(n, rng, k * per_seg), n_bytes, seed)


def zipf_text(n_bytes: int, seed: int = 1) -> bytes:
    """Zipf(1.1) word text over one 50,000-word vocabulary (seeded by ``seed``)."""
    return _segmented(lambda n, rng, k: _zipf_segment(n, rng, seed), n_bytes, seed)


def random_bytes(n_bytes: int, seed: int = 2) -> bytes:
    return np.random.default_rng(seed).integers(0, 256, size=n_bytes, dtype=np.uint8).tobytes()


def sparse_binary(n_bytes: int, seed: int = 3) -> bytes:
    """90% zeros in geometric runs (mean 64), uniform random bytes elsewhere."""
    rng = np.random.default_rng(seed)
    out = np.empty(n_bytes, dtype=np.uint8)
    filled = 0
    while filled < n_bytes:
        k = 1 << 16
        zr = rng.geometric(1 / 64.0, size=k)
        # random runs sized so zeros are ~90% of bytes: mean random run = 64/9
        rr = rng.geometric(9 / 64.0, size=k)
        seg = np.empty(2 * k, dtype=np.int64)
        seg[0::2] = zr
        seg[1::2] = rr
        ends = np.cumsum(seg)
        total = int(ends[-1])
        buf = np.zeros(total, dtype=np.uint8)
        starts = ends - seg
        mask = np.zeros(total + 1, dtype=np.int32)
        np.add.at(mask, starts[1::2], 1)
        np.add.at(mask, ends[1::2], -1)
        is_rand = np.cumsum(mask[:-1]) > 0
        buf[is_rand] = rng.integers(0, 256, size=int(is_rand.sum()), dtype=np.uint8)
        take = min(total, n_bytes - filled)
        out[filled:filled + take] = buf[:take]
        filled += take
    return out.tobytes()


CONTENT_KINDS = ("fastq", "zipf", "random", "sparse")
CONTENT_LEVEL = {"fastq": 6, "zipf": 9, "random": 1, "sparse": 6}


def make_content(kind: str, n_bytes: int, seed: int) -> bytes:
    if kind == "fastq":
        return fastq_like(n_bytes, seed)
    if kind == "zipf":
        return zipf_text(n_bytes, seed)
    if kind == "random":
        return random_bytes(n_bytes, seed)
    if kind == "sparse":
        return sparse_binary(n_bytes, seed)
    raise ValueError(kind)


# --------------------------------------------------------------- compressors

GZIP_HEADER = bytes([0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF])


def _crc32(data: bytes) -> int:
    return zlib.crc32(data) & 0xFFFFFFFF


def gzip_member(data: bytes, level: int = 6, parallel_threshold: int = 64 << 20,
                piece: int = 32 << 20, threads: int | None = None,
                strategy: int = zlib.Z_DEFAULT_STRATEGY) -> bytes:
    """One gzip member (RFC 1952) of ``data`` at zlib ``level`` and ``strategy``
    (``zlib.Z_FIXED``: every block fixed-Huffman)."""
    mv = memoryview(data)
    if len(data) <= parallel_threshold:
        c = zlib.compressobj(level, zlib.DEFLATED, -15, 8, strategy)
        body = c.compress(mv) + c.flush(zlib.Z_FINISH)
    else:
        starts = list(range(0, len(data), piece))

        def work(i):
            s = starts[i]
            e = min(len(data), s + piece)
            if i == 0:
                c = zlib.compressobj(level, zlib.DEFLATED, -15, 8, strategy)
            else:
                c = zlib.compressobj(level, zlib.DEFLATED, -15, 8, strategy,
                                     zdict=bytes(mv[max(0, s - 32768):s]))
            last = e == len(data)
            return c.compress(mv[s:e]) + c.flush(zlib.Z_FINISH if last else zlib.Z_SYNC_FLUSH)

        with ThreadPoolExecutor(max_workers=threads) as ex:
            body = b"".join(ex.map(work, range(len(starts))))
    return GZIP_HEADER + body + struct.pack("<II", _crc32(data), len(data) & 0xFFFFFFFF)


def bgzf(data: bytes, level: int = 5, block: int = 65280, threads: int | None = None) -> bytes:
    """BGZF: independent gzip members of <= ``block`` input bytes, each with the
    ``BC`` FEXTRA subfield holding BSIZE = member size - 1."""
    mv = memoryview(data)
    starts = list(range(0, len(data), block)) or [0]

    def member(s):
        e = min(len(data), s + block)
        c = zlib.compressobj(level, zlib.DEFLATED, -15, 8)
        body = c.compress(mv[s:e]) + c.flush(zlib.Z_FINISH)
        total = 18 + len(body) + 8
        hdr = bytes([0x1F, 0x8B, 8, 4, 0, 0, 0, 0, 0, 0xFF]) + struct.pack("<H", 6) + b"BC" + \
            struct.pack("<HH", 2, total - 1)
        return hdr + body + struct.pack("<II", _crc32(bytes(mv[s:e])), (e - s) & 0xFFFFFFFF)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        return b"".join(ex.map(member, starts, chunksize=64))


# ----------------------------------------------------------- configurations


def config0(n_bytes: int = 64 << 20, seed: int = 0):
    """FASTQ-like text, zlib level 6, one gzip member."""
    raw = fastq_like(n_bytes, seed)
    return raw, gzip_member(raw, 6)


def config1(n_bytes: int = 1 << 30, seed: int = 1):
    """Zipf text, zlib level 9, one gzip member."""
    raw = zipf_text(n_bytes, seed)
    return raw, gzip_member(raw, 9)


def fixed_blocks(n_bytes: int = 64 << 20, seed: int = 1):
    """Zipf text, zlib level 1 with the Z_FIXED strategy: one gzip member made
    of fixed-Huffman blocks only (16,383 symbols each), which no dynamic-block
    finder can split."""
    raw = zipf_text(n_bytes, seed)
    return raw, gzip_member(raw, 1, strategy=zlib.Z_FIXED)


def config2(n_bytes: int = 4 << 30, seed: int = 0):
    """FASTQ-like text as BGZF at level 5."""
    raw = fastq_like(n_bytes, seed)
    return raw, bgzf(raw, 5)


def config3_sizes(n_files: int = 2000, seed: int = 3, lo: int = 4 << 10, hi: int = 256 << 20):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_files)).astype(np.int64)
    kinds = rng.integers(0, 4, size=n_files)
    return [(int(s), CONTENT_KINDS[int(k)], int(seed * 1_000_003 + i)) for i, (s, k) in
            enumerate(zip(sizes, kinds))]


def config3_files(n_files: int = 2000, seed: int = 3, lo: int = 4 << 10, hi: int = 256 << 20):
    """Independent single-member gzip files of log-uniform size and mixed content."""
    return [(raw, gz) for raw, gz in config3_stream(n_files, seed, lo, hi)]


def config3_stream(n_files: int = 2000, seed: int = 3, lo: int = 4 << 10, hi: int = 256 << 20,
                   threads: int | None = None, only=None):
    """config3_files generated in parallel, yielded in order as (raw, gz);
    with ``only`` (indices), just those files."""
    import os
    spec = config3_sizes(n_files, seed, lo, hi)
    if only is not None:
        spec = [spec[i] for i in only]

    def one(t):
        size, kind, s = t
        raw = make_content(kind, size, s)
        return raw, gzip_member(raw, CONTENT_LEVEL[kind])

    with ThreadPoolExecutor(max_workers=threads or os.cpu_count()) as ex:
        yield from ex.map(one, spec)

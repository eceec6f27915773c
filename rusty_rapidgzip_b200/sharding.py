"""Multi-GPU work split for the batch and serving paths.

Independent files (or BGZF members, or requests) need no data exchange
between GPUs: each rank decodes a contiguous run of the inputs whose
compressed bytes are about 1/world of the total, and the outputs stay in input
order when the runs are concatenated by rank. The only collectives are the
host-side gather of per-file results and the max over ranks of the timed
region (torch.distributed, NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import bisect
from typing import Sequence


def shard_by_bytes(sizes: Sequence[int], world: int) -> list[range]:
    """Contiguous index ranges, one per rank, whose byte sums are as close to
    total/world as the item boundaries allow. Every item lands in exactly one
    range; ranges are in input order (rank r's range precedes rank r+1's)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    n = len(sizes)
    prefix = [0]
    for s in sizes:
        prefix.append(prefix[-1] + int(s))
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        i = min(bisect.bisect_left(prefix, target), n)  # prefix[i] >= target
        # the cut nearer the target, never before the previous cut
        if i > 0 and target - prefix[i - 1] <= prefix[i] - target:
            i -= 1
        cuts.append(max(cuts[-1], i))
    cuts.append(n)
    return [range(cuts[r], cuts[r + 1]) for r in range(world)]


def _buffers(decoder, data: bytes, out_n: int):
    """(input buffer, output buffer, output-to-host) on the decoder's device:
    torch CUDA tensors on a GPU, host arrays for the CPU-emulated build
    (device -1, whose "device" addresses are host addresses)."""
    import numpy as np
    if decoder.config.device >= 0:
        import torch
        din = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).to(f"cuda:{decoder.config.device}")
        dout = torch.empty(max(out_n, 1), dtype=torch.uint8, device=din.device)
        return din, dout, lambda: dout.cpu().numpy()
    din = np.frombuffer(data, dtype=np.uint8).copy()
    dout = np.empty(max(out_n, 1), dtype=np.uint8)
    keep = (din, dout)  # the addresses below stay valid while the closure lives
    return din.ctypes.data, dout.ctypes.data, lambda: keep[1]


def decode_shard(decoder, blobs: Sequence[bytes], shard: range) -> list[tuple[int, int, bytes | None]]:
    """Decode this rank's files with `decoder` (a Decoder) as ONE batch
    (rrg_gpu_decode_batch: one launch per stage for all of them, in waves under
    the decoder's device budget): [(index, status, bytes or None)] in input
    order. Output ranges are sized from each file's trailer ISIZE; a file whose
    output is larger (several members) is decoded again with the size the batch
    reported."""
    from ._abi import ERR_CAPACITY
    idx = list(shard)
    if not idx:
        return []
    gzs = [blobs[i] for i in idx]
    caps = [int.from_bytes(g[-4:], "little") if len(g) >= 18 else 0 for g in gzs]
    status = [None] * len(idx)
    outs = [None] * len(idx)
    todo = list(range(len(idx)))
    for _ in range(2):
        if not todo:
            break
        part = [gzs[k] for k in todo]
        pcap = [max(caps[k], 1) for k in todo]
        offs = [0]
        for g in part[:-1]:
            offs.append(offs[-1] + len(g))
        ooffs = [0]
        for c in pcap[:-1]:
            ooffs.append(ooffs[-1] + c)
        din, dout, host = _buffers(decoder, b"".join(part), sum(pcap) + 64)
        lens, st, _ = decoder.decode_batch(din, offs, [len(g) for g in part], dout, ooffs, pcap)
        out = host()
        retry = []
        for q, k in enumerate(todo):
            if st[q] == ERR_CAPACITY and caps[k] < lens[q]:
                caps[k] = lens[q]
                retry.append(k)
                continue
            status[k] = int(st[q])
            outs[k] = out[ooffs[q]:ooffs[q] + lens[q]].tobytes() if st[q] == 0 else None
        todo = retry
    return [(i, status[k] if status[k] is not None else ERR_CAPACITY, outs[k]) for k, i in enumerate(idx)]


def gzip_body_offset(data: bytes) -> int:
    """Byte offset of a gzip member's deflate body (RFC 1952 header: FEXTRA,
    FNAME, FCOMMENT, FHCRC), as gzip.rs:252-300 parse_header reads it."""
    if len(data) < 10 or data[0] != 0x1F or data[1] != 0x8B or data[2] != 8:
        raise ValueError("not a deflate gzip member")
    flg, p = data[3], 10
    if flg & 4:
        p += 2 + int.from_bytes(data[p:p + 2], "little")
    for bit in (8, 16):
        if flg & bit:
            p = data.index(b"\0", p) + 1
    if flg & 2:
        p += 2
    return p


def decode_member_split(decoder, data: bytes, rank: int, world: int, sink=None, group=None) -> dict:
    """Decode ONE gzip member on `world` GPUs, this rank's share: the body is cut
    into `world` ranges at dynamic block starts near equal shares of its bits;
    every rank decodes its range at once (phase 1), the ranks exchange their
    ranges' end bits and 32 KiB window maps (the only exchange), each rank
    composes the window before its range from the earlier ranges' maps and
    resolves its range (phase 2), and the (CRC32, length) of every range are
    combined and checked against the member trailer. A range whose start is not
    where the previous range ended (a false block start) is decoded again from
    that exact bit, so every rank takes the same rounds. This rank's bytes go to
    `sink`. Returns {"ok", "total", "crc", "out_len", "rounds"}; raises on
    corrupt data. Uses torch.distributed (NCCL on GPUs, gloo on CPUs)."""
    import numpy as np
    import torch.distributed as dist
    body = gzip_body_offset(data)
    nbits = (len(data) - body - 8) * 8
    start_t = nbits * rank // world
    stop_t = nbits * (rank + 1) // world if rank + 1 < world else (1 << 64) - 1
    empty = (1 << 64) - 1  # start and end bit of a range with no block start after its target
    failed = (1 << 64) - 2  # start bit of a range whose guessed start did not decode

    def begin(start, exact):
        # a guessed start may be false (a dynamic header inside stored data):
        # its failure is a broken link the exchange repairs; a failure from an
        # exact start is an error of the stream, raised on every rank together
        try:
            i, m = decoder.split_begin(data, body, start, stop_t, exact=exact)
            return i, m, None
        except Exception as ex:  # noqa: BLE001 - passed to every rank below
            if not exact and start != 0:
                return {"start_bit": failed, "end_bit": failed, "out_len": 0, "has_trailer": 0, "crc": 0,
                        "isize": 0, "trailer_byte": 0}, np.zeros(32768, dtype=np.uint16), None
            return None, None, ex

    info, emap, error = begin(start_t, start_t == 0)
    rounds = 1
    for _ in range(world + 1):
        ends = [None] * world
        dist.all_gather_object(ends, (None, None, repr(error)) if error else
                               (info["start_bit"], info["end_bit"], None), group=group)
        errs = [e for _, _, e in ends if e]
        if errs:
            raise error if error else RuntimeError(f"split decode failed on another rank: {errs[0]}")
        # every non-empty range must start where the previous non-empty one ended
        live = [r for r in range(world) if ends[r][0] != empty]
        broken = [b for a, b in zip(live, live[1:]) if ends[b][0] != ends[a][1] or ends[a][1] == failed]
        if not broken:
            break
        first = broken[0]
        prev = max(r for r in live if r < first)
        if ends[prev][1] == failed:  # the previous range must be repaired first
            first, prev = prev, max([r for r in live if r < prev], default=None)
        if rank == first:  # from the previous range's exact end
            info, emap, error = begin(ends[prev][1] if prev is not None else 0, True)
        rounds += 1
    else:
        raise RuntimeError("split ranges did not chain")
    maps = [None] * world
    dist.all_gather_object(maps, (emap.tobytes(), info["out_len"]), group=group)
    win = np.full(32768, 0x4000, dtype=np.uint16)  # before the stream: nothing
    for r in range(rank):
        m = np.frombuffer(maps[r][0], dtype=np.uint16)
        win = np.where(m & 0x8000, win[m & 0x7FFF], m).astype(np.uint16)
    wlen = min(32768, sum(maps[r][1] for r in range(rank)))
    w = win[32768 - wlen:]
    if (w >= 0x100).any():
        raise ValueError("a back-reference reaches before the stream")
    crc, n = decoder.split_finish(w.astype(np.uint8).tobytes(), sink)
    parts = [None] * world
    dist.all_gather_object(parts, (crc, n, info["has_trailer"], info["crc"], info["isize"]), group=group)
    total_crc, total = parts[0][0], parts[0][1]
    for c, ln, _, _, _ in parts[1:]:
        total_crc = decoder.crc32_combine(total_crc, c, ln)
        total += ln
    last = [p for p in parts if p[2]]
    ok = len(last) == 1 and total_crc == last[0][3] and (total & 0xFFFFFFFF) == last[0][4]
    return {"ok": ok, "total": total, "crc": total_crc, "out_len": n, "rounds": rounds}

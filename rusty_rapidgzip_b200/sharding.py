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

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


def decode_shard(decoder, blobs: Sequence[bytes], shard: range) -> list[tuple[int, int, bytes | None]]:
    """Decode this rank's files one after another with `decoder` (a Decoder):
    [(index, status, bytes or None)] in input order."""
    out = []
    for i in shard:
        try:
            out.append((i, 0, decoder.decompress(blobs[i])))
        except Exception as e:  # noqa: BLE001 - the status is the result
            out.append((i, int(getattr(e, "code", -1)), None))
    return out

"""Multi-GPU split of independent files, checked on the CPU: the byte-balanced
contiguous shards, and two gloo ranks that each decode their shard (with the
emulated build) and gather the results in input order, plus the max-over-ranks
reduction of the timed region."""
import os
import socket

import pytest

from rusty_rapidgzip_b200.sharding import shard_by_bytes


def test_shards_cover_in_order_and_balance():
    sizes = [5, 100, 3, 3, 50, 50, 7, 1, 200, 9]
    for world in (1, 2, 3, 4, 7):
        sh = shard_by_bytes(sizes, world)
        assert len(sh) == world
        assert [i for r in sh for i in r] == list(range(len(sizes)))
    sh = shard_by_bytes([10] * 100, 4)
    assert [len(r) for r in sh] == [25, 25, 25, 25]
    assert shard_by_bytes([], 3) == [range(0, 0)] * 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, lib, blobs, q):
    import time
    import torch.distributed as dist
    from rusty_rapidgzip_b200 import Config, Decoder
    from rusty_rapidgzip_b200.sharding import decode_shard, shard_by_bytes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = Decoder(Config(device=-1), lib=lib)
        shard = shard_by_bytes([len(b) for b in blobs], world)[rank]
        t0 = time.perf_counter()
        mine = decode_shard(d, blobs, shard)
        t = time.perf_counter() - t0
        import torch
        tt = torch.tensor([t], dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            q.put(([x for part in gathered for x in part], float(tt.item()), t))
        d.close()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_decode_their_shards():
    import multiprocessing as mp
    import oracle
    from conftest import build_emu_lib, gzip_cli
    from rusty_rapidgzip_b200 import workloads as W
    lib = build_emu_lib()
    raws = [W.fastq_like(9000 + 2000 * i, i) for i in range(5)] + [b"", b"x" * 3000]
    blobs = [gzip_cli(r) for r in raws]
    bad = bytearray(blobs[2])
    bad[-8] ^= 1
    blobs[2] = bytes(bad)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, lib, blobs, q)) for r in range(2)]
    for p in procs:
        p.start()
    results, t_max, t0 = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [i for i, _, _ in results] == list(range(len(blobs)))
    for i, status, data in results:
        try:
            want = oracle.read_gz(blobs[i], 2)
            assert status == 0 and data == want
        except oracle.OracleError as e:
            assert status == e.code and data is None
    assert t_max >= t0 > 0

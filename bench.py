#!/usr/bin/env python3
"""Decompressed GB/s of the B200 gzip/DEFLATE decoder.

Default workload: 1 GiB of seeded Zipf(1.1) word text (50,000-word vocabulary,
newline every 8-20 words) compressed at zlib level 9 as ONE gzip member,
decoded on one GPU (input resident in HBM, output to HBM). A step is one
whole-file decode through rrg_gpu_decode_device.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload zipf1g|zipf_plain|fixed|fastq64m|bgzf|files|serve|stream]

With N > 1 (torchrun, one rank per GPU) every rank decodes its own copy of the
workload (independent files: weak scaling, no collective on the data path);
value = all ranks' bytes / the slowest rank's time.

--impl reference times the reference algorithm's CPU path (the C restatement in
oracle/, rusty_rapidgzip's Rust crate cannot be built here) on all host cores
on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CACHE = os.environ.get("RRG_BENCH_CACHE", "/tmp/rrg_bench_cache")
GEN_VERSION = 2


def workload(name: str, size: int | None):
    """(raw, compressed, description) — cached on local disk between runs."""
    from rusty_rapidgzip_b200 import workloads as W
    if name == "zipf1g":
        n = size or (1 << 30)
        key, make = f"zipf_{n}_s1_v{GEN_VERSION}", lambda: W.config1(n, seed=1)
        desc = {"workload": "zipf_text_level9_single_member", "uncompressed_bytes": n, "zlib_level": 9,
                "vocabulary": 50000, "zipf_exponent": 1.1}
    elif name == "zipf_plain":
        # the same text as one zlib stream written by a single compressor (no
        # 32 MiB pieces, no sync-flush points); slow to make at 1 GiB
        n = size or (256 << 20)

        def make():
            raw = W.zipf_text(n, 1)
            return raw, W.gzip_member(raw, 9, parallel_threshold=1 << 62)

        key = f"zipfplain_{n}_s1_v{GEN_VERSION}"
        desc = {"workload": "zipf_text_level9_single_member_one_zlib_stream", "uncompressed_bytes": n,
                "zlib_level": 9, "vocabulary": 50000, "zipf_exponent": 1.1}
    elif name == "fixed":
        # one member of fixed-Huffman blocks only (zlib level 1, Z_FIXED): its
        # sub-chunk starts come from the fixed-code walk
        n = size or (256 << 20)
        key, make = f"fixed_{n}_s1_v{GEN_VERSION}", lambda: W.fixed_blocks(n, seed=1)
        desc = {"workload": "zipf_text_level1_fixed_huffman_single_member", "uncompressed_bytes": n,
                "zlib_level": 1, "zlib_strategy": "Z_FIXED", "vocabulary": 50000, "zipf_exponent": 1.1}
    elif name == "fastq64m":
        n = size or (64 << 20)
        key, make = f"fastq_{n}_s0_v{GEN_VERSION}", lambda: W.config0(n, seed=0)
        desc = {"workload": "fastq_like_level6_single_member", "uncompressed_bytes": n, "zlib_level": 6}
    elif name == "bgzf":
        n = size or (4 << 30)
        key, make = f"bgzf_{n}_s0_v{GEN_VERSION}", lambda: W.config2(n, seed=0)
        desc = {"workload": "fastq_like_bgzf_level5", "uncompressed_bytes": n, "zlib_level": 5,
                "member_max_input": 65280}
    else:
        raise SystemExit(f"unknown workload {name}")
    os.makedirs(CACHE, exist_ok=True)
    pr, pc = os.path.join(CACHE, key + ".raw"), os.path.join(CACHE, key + ".gz")
    if os.path.exists(pr) and os.path.exists(pc) and os.path.getsize(pr) == n:
        return open(pr, "rb").read(), open(pc, "rb").read(), desc
    raw, gz = make()
    try:
        with open(pr + ".tmp", "wb") as f:
            f.write(raw)
        with open(pc + ".tmp", "wb") as f:
            f.write(gz)
        os.replace(pr + ".tmp", pr)
        os.replace(pc + ".tmp", pc)
    except OSError:
        pass
    return raw, gz, desc


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_time_oracle(gz: bytes, n_raw: int, threads: int, min_reps: int = 3, min_seconds: float = 3.0):
    import oracle
    times = []
    t_start = time.perf_counter()
    while len(times) < min_reps or time.perf_counter() - t_start < min_seconds:
        t0 = time.perf_counter()
        n, _ = oracle.read_gz_count(gz, num_threads=threads, chunk_size=4 << 20)
        times.append(time.perf_counter() - t0)
        assert n == n_raw
        if len(times) >= 20:
            break
    return times


def run_reference(args, raw, gz, desc):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_time_oracle(gz, len(raw), threads, min_reps=1, min_seconds=0)
    times = []
    for _ in range(args.steps):
        times += cpu_time_oracle(gz, len(raw), threads, min_reps=1, min_seconds=0)
    total = sum(times)
    value = len(raw) * len(times) / total / 1e9
    line = {
        "metric": "decompressed GB/s", "value": round(value, 3), "unit": "GB/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * total / len(times), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": dict(desc, compressed_bytes=len(gz), parallelism="cpu threads"),
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": "whole workload file per step, all host threads, oracle/ C restatement of the "
                                   "reference pipeline (rusty_rapidgzip's Rust crate has no toolchain here)"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, raw, gz, desc):
    import torch
    import torch.distributed as dist
    from rusty_rapidgzip_b200 import Config, Decoder, kernel_launch_count
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    dec = Decoder(Config(device=local, gpu_chunk_bytes=args.gpu_chunk, warps_per_stream=args.warps_per_stream,
                         boundary_mode=args.boundary_mode, host_pipeline=args.pipeline_waves, verbose=False))
    stream = torch.cuda.Stream()
    din = torch.empty(len(gz), dtype=torch.uint8, device="cuda")
    din.copy_(torch.frombuffer(bytearray(gz), dtype=torch.uint8))
    dout = torch.empty(len(raw) + 64, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    tuning = None
    if args.workload == "bgzf" and args.warps_per_stream == 0 and not args.no_autotune:
        # autotune (untimed) on the file's first 2048 members
        off, k = 0, 0
        while k < 2048 and off + 18 <= len(gz):
            off += int.from_bytes(gz[off + 16:off + 18], "little") + 1
            k += 1
        s_out = torch.empty(k * 65536 + 64, dtype=torch.uint8, device="cuda")
        tuning = dec.autotune(din, [0], [off], s_out, [0], [s_out.numel()])
        del s_out

    def step():
        n, st = dec.decode_device(din, len(gz), dout, dout.numel(), stream=stream.cuda_stream)
        assert n == len(raw)
        return st

    for _ in range(max(args.warmup, 1)):
        step()
    # correctness of the measured path (outside the timed region)
    torch.cuda.synchronize()
    import hashlib
    ok = hashlib.sha256(dout[: len(raw)].cpu().numpy().tobytes()).digest() == hashlib.sha256(raw).digest()
    if not ok:
        raise SystemExit("decoded bytes differ from the generator output")

    def barrier():
        if world > 1:
            dist.barrier()

    # ---------------- device-resident timed region
    barrier()
    torch.cuda.synchronize()
    stats = []
    with ClockSampler(local) as clk:
        l0 = kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            stats.append(step())
        e1.record(stream)
        torch.cuda.synchronize()
        launches = kernel_launch_count() - l0
    barrier()
    t = e0.elapsed_time(e1) / 1000.0
    if world > 1:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    value = world * len(raw) * args.steps / t / 1e9

    # ---------------- BGZF: the plain per-member path on the file's first 4,096
    # members (each a complete gzip file: one decode_device call per member)
    plain = None
    if args.workload == "bgzf":
        offs, off = [], 0
        while len(offs) < 4096 and off + 18 <= len(gz):
            bs = int.from_bytes(gz[off + 16:off + 18], "little") + 1
            offs.append((off, bs, int.from_bytes(gz[off + bs - 4:off + bs], "little")))
            off += bs
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        u = 0
        for o, bs, isz in offs:
            m, _ = dec.decode_device(din[o:], bs, dout[u:], isz, stream=stream.cuda_stream)
            assert m == isz
            u += isz
        p1.record(stream)
        torch.cuda.synchronize()
        plain = {"members": len(offs), "uncompressed_bytes": u,
                 "gbs": round(u / (p0.elapsed_time(p1) / 1000.0) / 1e9, 3)}

    # ---------------- end to end through the C ABI with host buffers
    pinned = torch.empty(len(gz), dtype=torch.uint8, pin_memory=True)
    pinned.copy_(torch.frombuffer(bytearray(gz), dtype=torch.uint8))
    buf = pinned.numpy()
    n, _ = dec.count(buf)  # warm the host-path buffers
    assert n == len(raw)
    barrier()
    e2e_times = []
    e2e_st = None
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n, e2e_st = dec.count(buf)
        e2e_times.append(time.perf_counter() - t0)
        assert n == len(raw)
    te = sum(e2e_times)
    if world > 1:
        tt = torch.tensor([te], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    e2e_value = world * len(raw) * args.steps / te / 1e9

    # ---------------- roofline of the dominant kernel
    kern = {k: statistics.mean(s.timings_ms[k] for s in stats) for k in ("finder", "inflate", "resolve", "crc")}
    dominant = max(kern, key=kern.get)
    C_, U_ = len(gz), len(raw)
    algo = {"inflate": C_ + 2 * U_,          # compressed read once + u16 cells written
            "resolve": 3 * U_,                # u16 cells read + bytes written
            "crc": U_,                        # bytes read
            "finder": C_}                     # upper bound: every compressed byte scanned once
    peak, peak_kind = measured_peak_hbm()
    achieved = algo[dominant] / (kern[dominant] / 1000.0) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(f"{args.workload}:{dominant}")
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        times = cpu_time_oracle(gz, len(raw), threads)
        cpu = {"value": round(len(raw) / statistics.median(times) / 1e9, 3), "unit": "GB/s", "cores": threads,
               "kind": "port",
               "sample": f"whole workload file, median of {len(times)} runs, oracle/ C restatement of the reference "
                         "pipeline on all host threads"}
    if rank == 0:
        ms = stats[-1]
        line = {
            "metric": "decompressed GB/s", "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * t / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator)",
            "config": dict(desc, compressed_bytes=C_, parallelism=f"replicas x{world}",
                           l2="inputs (compressed + output) larger than L2; no flush",
                           gpu_chunk_bytes=args.gpu_chunk or "auto", gpu_chunks=ms.gpu_chunks,
                           inflate="lane-per-chunk" if args.warps_per_stream < 0 else "warp-per-chunk",
                           boundaries="per target" if args.boundary_mode == 1 else "every offset",
                           markers=ms.markers, speculation_failures=ms.speculation_failures,
                           graph_launches=ms.graph_launches, autotuned=tuning,
                           **({"plain_per_member": plain} if plain else {})),
            "e2e": {"value": round(e2e_value, 3), "unit": "GB/s", "h2d_bytes_per_step": C_,
                    "d2h_bytes_per_step": U_, "pipeline_waves": e2e_st.pipeline_waves if e2e_st else None},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 2), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "algorithmic_bytes_per_launch": algo[dominant]},
            "kernels_ms": {k: round(v, 3) for k, v in kern.items()},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    dec.close()


def run_serve(args):
    """Serving: open-loop Poisson arrivals of decode requests (sizes log-uniform
    64 KiB - 1 GiB, content mixed as in the many-files workload) at each rate
    for --duration seconds, through submit/poll with the HBM budget. At most
    --max-outstanding requests may be waiting (later arrivals are counted as
    rejected) so host memory stays bounded when a rate exceeds capacity."""
    import hashlib
    import random
    import threading
    import ctypes as C
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from rusty_rapidgzip_b200 import Config, Decoder
    from rusty_rapidgzip_b200 import workloads as W
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    n_pool = args.size or 48
    t_gen = time.perf_counter()
    pool, sums, lens = [], [], []
    for raw, gz in W.config3_stream(n_pool, seed=4, lo=64 << 10, hi=1 << 30):
        pool.append(gz)
        sums.append(hashlib.sha256(raw).digest())
        lens.append(len(raw))
    t_gen = time.perf_counter() - t_gen
    # the requests sit in page-locked host memory, as a server's receive
    # buffers would, and are submitted in place: a read-only bytes object
    # would be copied by the Python binding on every submit
    pinned = []
    for i, gz in enumerate(pool):
        t = torch.empty(len(gz), dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = np.frombuffer(gz, dtype=np.uint8)
        pinned.append(t)
        pool[i] = t.numpy()
    rates = [float(x) for x in args.rates.split(",")]
    dec = Decoder(Config(device=0))
    dec.serve_start(engines=args.engines, max_ready=16)
    # warm-up: every pool item once (untimed; grows the engines' resident scratch)
    for gz in pool:
        dec.submit(gz, copy=False)
    for _ in pool:
        while dec.poll(timeout_ms=1000) is None:
            pass
    per_rate = []
    # every result is checked against its SHA-256 before it is freed: enough
    # threads that the checks keep up with the decoder (held results would
    # make the library allocate more page-locked result buffers)
    hasher = ThreadPoolExecutor(max_workers=max(4, min(8, (os.cpu_count() or 8) // 2)))
    for rate in rates:
        rng = random.Random(int(rate * 1000))
        sched, lock = {}, threading.Lock()
        done, bad = [], []
        rejected = [0]

        def feeder():
            t0 = time.perf_counter()
            t = t0
            while True:
                t += rng.expovariate(rate)
                if t - t0 > args.duration:
                    break
                now = time.perf_counter()
                if t > now:
                    time.sleep(t - now)
                k = rng.randrange(n_pool)
                if dec.pending() >= args.max_outstanding:
                    rejected[0] += 1
                    continue
                rid = dec.submit(pool[k], copy=False)
                with lock:
                    sched[rid] = (t, k)

        def check(addr, n, k):
            ok = n == lens[k] and hashlib.sha256((C.c_uint8 * n).from_address(addr)).digest() == sums[k]
            dec.free(addr)
            return ok

        th = threading.Thread(target=feeder)
        t_start = time.perf_counter()
        th.start()
        futs = []
        while th.is_alive() or dec.pending() > 0:
            r = dec.poll_raw(timeout_ms=100)
            if r is None:
                continue
            now = time.perf_counter()
            rid, addr, n, status, _ = r
            while True:
                with lock:
                    if rid in sched:
                        t_arr, k = sched.pop(rid)
                        break
                time.sleep(0.0005)
            done.append((now - t_arr, lens[k], now))
            if status != 0:
                bad.append(status)
                dec.free(addr)
            else:
                futs.append(hasher.submit(check, addr, n, k))
        th.join()
        ok = all(f.result() for f in futs)
        if bad or not ok:
            raise SystemExit(f"serving produced wrong results at {rate} req/s: statuses {bad[:5]}, bytes ok {ok}")
        lat = sorted(x[0] * 1000 for x in done)
        span = max(x[2] for x in done) - t_start
        per_rate.append({"rate_req_s": rate, "completed": len(done), "rejected": rejected[0],
                         "offered_gbs": round(rate * statistics.mean(lens) / 1e9, 3),
                         "sustained_gbs": round(sum(x[1] for x in done) / span / 1e9, 3),
                         "p50_ms": round(lat[len(lat) // 2], 2), "p99_ms": round(lat[min(len(lat) - 1, int(len(lat) * 0.99))], 2)})
    hasher.shutdown()
    st = dec.serve_stats()
    dec.close()
    top = per_rate[-1]
    line = {"metric": "decompressed GB/s", "value": top["sustained_gbs"], "unit": "GB/s", "n_gpus": 1,
            "steps": len(rates), "warmup": 1, "ms_per_step": round(args.duration * 1000, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
            "config": {"workload": "serving_poisson_requests_log_uniform_64KiB_1GiB_mixed_content",
                       "pool_requests": n_pool, "pool_uncompressed_bytes": sum(lens),
                       "duration_s_per_rate": args.duration, "hbm_budget_bytes": st["budget_bytes"], "engines": args.engines,
                       "max_outstanding": args.max_outstanding, "per_rate": per_rate,
                       "serve_stats": st, "generation_s": round(t_gen, 1)},
            "e2e": {"value": top["sustained_gbs"], "unit": "GB/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "the serving path itself is end to end: host request bytes in, host result bytes out"},
            "latency_ms": {"p50": top["p50_ms"], "p99": top["p99_ms"]}}
    print(json.dumps(line), flush=True)


def cpu_files_baseline(files):
    """The oracle on a size-stratified sample of independent files (every 10th
    file in size order, about a tenth of the bytes): files of 16 MiB or more one
    after another with every host thread (read_gz's own parallel pipeline), the
    smaller ones by a persistent pool of one thread per host core, each decoding
    whole files on the serial path. Returns (GB/s, output bytes, files, threads)."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    threads = os.cpu_count() or 1
    pick = sorted(files, key=lambda f: f[0])[5::10] or list(files)
    big = [f for f in pick if f[0] >= (16 << 20)]
    small = [f for f in pick if f[0] < (16 << 20)]
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda f: oracle.read_gz_count(f[1], num_threads=1), small[:threads]))  # warm
        t0 = time.perf_counter()
        got = [oracle.read_gz_count(f[1], num_threads=threads)[0] for f in big]
        got += list(ex.map(lambda f: oracle.read_gz_count(f[1], num_threads=1)[0], small))
        dt = time.perf_counter() - t0
    assert got == [n for n, _ in big] + [n for n, _ in small]
    nb = sum(got)
    return nb / dt / 1e9, nb, len(pick), threads


def run_files_reference(args):
    """Reference arm of the many-files workload: the oracle port over a
    size-stratified sample of the files (every 10th by size) per step, one file
    per host thread from a persistent pool."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from rusty_rapidgzip_b200 import workloads as W
    n_all = args.size or 2000
    files = [(len(raw), gz) for raw, gz in W.config3_stream(n_all, seed=3)]
    for _ in range(args.warmup):
        cpu_files_baseline(files)
    runs = [cpu_files_baseline(files) for _ in range(args.steps)]
    nb = sum(r[1] for r in runs)
    t_all = sum(r[1] / (r[0] * 1e9) for r in runs)
    value = nb / t_all / 1e9
    threads = runs[0][3]
    line = {"metric": "decompressed GB/s", "value": round(value, 3), "unit": "GB/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * t_all / args.steps, 3), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
            "config": {"workload": "independent_gzip_files_log_uniform_4KiB_256MiB_mixed_content",
                       "files": n_all, "parallelism": "cpu threads"},
            "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                             "sample": f"{runs[0][2]} files ({runs[0][1]} output bytes, every 10th file by size) "
                                       "per step: files >= 16 MiB one after another on all threads, smaller "
                                       "ones one per thread from a persistent pool; oracle/ C restatement"},
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_files(args):
    """Many independent gzip files (log-uniform 4 KiB - 256 MiB, four content
    kinds) decoded as one batch per step: device-resident batch time (value),
    the plain path (one decode_device per file) for comparison, and end to end
    with host buffers."""
    import hashlib
    import torch
    import torch.distributed as dist
    from rusty_rapidgzip_b200 import Config, Decoder, kernel_launch_count
    from rusty_rapidgzip_b200 import workloads as W
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    n_files_all = args.size or 2000
    # with several ranks each one takes a contiguous run of the files holding
    # about 1/world of the output bytes (strong scaling: the job is fixed)
    from rusty_rapidgzip_b200.sharding import shard_by_bytes
    mine = shard_by_bytes([s for s, _, _ in W.config3_sizes(n_files_all, seed=3)], world)[rank]
    n_files = len(mine)
    t_gen = time.perf_counter()
    gzs, sums, lens = [], [], []
    sample = []  # (raw, gz) of a few files for the tuner
    strata = []  # (output bytes, gz) of every file, for the CPU baseline's size-stratified sample
    for i, (raw, gz) in enumerate(W.config3_stream(n_files_all, seed=3, only=list(mine))):
        gzs.append(gz)
        sums.append(hashlib.sha256(raw).digest())
        lens.append(len(raw))
        if len(raw) < (32 << 20) and len(sample) < 64 and i % 3 == 0:
            sample.append((raw, gz))
        strata.append((len(raw), gz))
    t_gen = time.perf_counter() - t_gen
    in_off = np.cumsum([0] + [len(g) for g in gzs])[:-1].tolist()
    in_len = [len(g) for g in gzs]
    out_off = np.cumsum([0] + lens)[:-1].tolist()
    C_, U_ = sum(in_len), sum(lens)
    blob = np.empty(C_, dtype=np.uint8)
    for g, o in zip(gzs, in_off):
        blob[o:o + len(g)] = np.frombuffer(g, dtype=np.uint8)
    del gzs
    din = torch.from_numpy(blob).cuda()
    dout = torch.empty(U_ + 64, dtype=torch.uint8, device="cuda")
    dec = Decoder(Config(device=local))
    stream = torch.cuda.Stream()
    # ---- autotune on a sample (untimed; --no-autotune keeps the defaults, for
    # profiler runs whose own slowdown would steer the sweep)
    tuning = None
    if not args.no_autotune:
        s_gz = [g for _, g in sample]
        s_raw = [r for r, _ in sample]
        s_in = torch.from_numpy(np.frombuffer(b"".join(s_gz), dtype=np.uint8).copy()).cuda()
        s_out = torch.empty(sum(len(r) for r in s_raw) + 64, dtype=torch.uint8, device="cuda")
        tuning = dec.autotune(s_in, np.cumsum([0] + [len(g) for g in s_gz])[:-1].tolist(), [len(g) for g in s_gz],
                              s_out, np.cumsum([0] + [len(r) for r in s_raw])[:-1].tolist(), [len(r) for r in s_raw])
        del s_in, s_out

    def step():
        got, status, st = dec.decode_batch(din, in_off, in_len, dout, out_off, lens, stream=stream.cuda_stream)
        assert status == [0] * n_files, [x for x in status if x][:5]
        return st

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    host = dout.cpu().numpy()
    for o, n, h in zip(out_off, lens, sums):
        if hashlib.sha256(host[o:o + n].tobytes()).digest() != h:
            raise SystemExit("decoded bytes differ from the generator output")
    del host
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        l0 = kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        stats = [step() for _ in range(args.steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        launches = kernel_launch_count() - l0
    t = e0.elapsed_time(e1) / 1000.0
    U_all = U_
    if world > 1:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
        uu = torch.tensor([U_], device="cuda", dtype=torch.float64)
        dist.all_reduce(uu, op=dist.ReduceOp.SUM)
        U_all = int(uu.item())
    value = U_all * args.steps / t / 1e9
    # ---- plain path: one device-resident decode per file, same buffers
    plain = None
    if not args.no_plain:
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for o, n, io, il in zip(out_off, lens, in_off, in_len):
            m, _ = dec.decode_device(din[io:], il, dout[o:], n, stream=stream.cuda_stream)
            assert m == n
        p1.record(stream)
        torch.cuda.synchronize()
        plain = round(U_ / (p0.elapsed_time(p1) / 1000.0) / 1e9, 3)
    # ---- end to end: pinned host input -> batch -> pinned host output, every step
    e2e = None
    try:
        pin_in = torch.from_numpy(blob).pin_memory()
        pin_out = torch.empty(U_ + 64, dtype=torch.uint8, pin_memory=True)
        times = []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            din.copy_(pin_in, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            step()
            pin_out.copy_(dout, non_blocking=True)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        te = sum(times)
        if world > 1:
            tt = torch.tensor([te], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt.item())
        e2e = {"value": round(U_all * args.steps / te / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": C_,
               "d2h_bytes_per_step": U_ + 64}
        del pin_in, pin_out
    except RuntimeError as ex:  # pinned memory unavailable for this size
        e2e = {"value": None, "unit": "GB/s", "note": f"pinned buffers unavailable: {ex}"[:200]}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        value_cpu, nb, nf, threads = cpu_files_baseline(strata)
        cpu = {"value": round(value_cpu, 3), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"{nf} files ({nb} output bytes, every 10th file by size): files >= 16 MiB one after "
                         f"another on all {threads} threads, smaller ones one per thread from a persistent pool; "
                         "oracle/ C restatement of the reference pipeline"}
    if rank == 0:
        st = stats[-1]
        kern = {k: round(statistics.mean(s_.timings_ms[k] for s_ in stats), 3)
                for k in ("finder", "inflate", "resolve", "crc")}
        line = {
            "metric": "decompressed GB/s", "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * t / args.steps, 3),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator)",
            "config": {"workload": "independent_gzip_files_log_uniform_4KiB_256MiB_mixed_content",
                       "files": n_files_all, "uncompressed_bytes": U_all, "rank0_files": n_files,
                       "rank0_compressed_bytes": C_,
                       "parallelism": f"file shards x{world} (byte-balanced)", "l2": "inputs larger than L2; no flush",
                       "plain_per_file_gbs": plain, "autotuned": tuning,
                       "gpu_chunks": st.gpu_chunks, "generation_s": round(t_gen, 1)},
            "e2e": e2e, "gpu_launches": int(launches), "kernels_ms": kern,
            "clocks": clk.summary(), "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    dec.close()


def run_stream(args, raw, gz, desc):
    """Non-seekable input: rrg_gpu_read_stream pulls the member from a file
    object and pushes the output to a sink stripe by stripe. Host buffers on
    both ends, so the line's value is already end to end (one GPU)."""
    import io
    import torch
    from rusty_rapidgzip_b200 import Config, Decoder, kernel_launch_count
    torch.cuda.set_device(0)
    dec = Decoder(Config(device=0))

    def step():  # the sink takes the bytes without a Python copy; the count comes back in the stats
        st = dec.read_stream(io.BytesIO(gz), None, stripe_bytes=args.stripe)
        assert st.uncompressed_bytes == len(raw)
        return st

    for _ in range(max(args.warmup, 1)):
        step()
    times, stats = [], []
    with ClockSampler(0) as clk:
        l0 = kernel_launch_count()
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            stats.append(step())
            times.append(time.perf_counter() - t0)
        launches = kernel_launch_count() - l0
    t = sum(times)
    value = len(raw) * args.steps / t / 1e9
    kern = {k: statistics.mean(s.timings_ms[k] for s in stats) for k in ("finder", "inflate", "resolve", "crc")}
    peak, peak_kind = measured_peak_hbm()
    algo = len(gz) + 2 * len(raw)
    achieved = algo / (kern["inflate"] / 1000.0) / 1e9
    line = {
        "metric": "decompressed GB/s", "value": round(value, 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1000 * t / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": dict(desc, compressed_bytes=len(gz), gpu_chunks=stats[-1].gpu_chunks,
                       speculation_failures=stats[-1].speculation_failures, l2="inputs larger than L2; no flush",
                       timing="wall clock around each read_stream call"),
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": len(gz), "d2h_bytes_per_step": len(raw)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "inflate", "achieved": round(achieved, 2), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "algorithmic_bytes_per_launch": algo},
        "kernels_ms": {k: round(v, 3) for k, v in kern.items()},
        "clocks": clk.summary(),
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    dec.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="zipf1g",
                    choices=["zipf1g", "zipf_plain", "fixed", "fastq64m", "bgzf", "files", "serve", "stream"])
    ap.add_argument("--rates", default="10,50,200", help="serve: request rates (req/s)")
    ap.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals per rate")
    ap.add_argument("--max-outstanding", type=int, default=32, help="serve: waiting requests before rejecting")
    ap.add_argument("--engines", type=int, default=4, help="serve: decode engines (sub-contexts with their own stream)")
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--gpu-chunk", type=int, default=0)
    ap.add_argument("--warps-per-stream", type=int, default=0, help="-1: one decoder per lane")
    ap.add_argument("--boundary-mode", type=int, default=0, help="1: one finder search per target")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="files: leave out the plain per-file comparison arm")
    ap.add_argument("--no-autotune", action="store_true", help="files, bgzf: keep the default tunables")
    ap.add_argument("--pipeline-waves", type=int, default=0,
                    help="end-to-end leg: waves of the pipelined host path (0: automatic, -1: off)")
    ap.add_argument("--stripe", type=int, default=0, help="stream: compressed bytes per stripe (0: 256 MiB)")
    args = ap.parse_args()
    if args.warmup < 3:
        print("note: fewer than 3 warm-up steps", file=sys.stderr)
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop"}))
        else:
            run_serve(args)
        return
    if args.workload == "files":
        if args.impl == "reference":
            run_files_reference(args)
        else:
            run_files(args)
        return
    if args.workload == "stream":
        raw, gz, desc = workload("zipf1g", args.size)
        desc = dict(desc, workload="zipf_text_level9_non_seekable_stream", stripe_bytes=args.stripe or (256 << 20))
        if args.impl == "reference":
            run_reference(args, raw, gz, desc)
        else:
            run_stream(args, raw, gz, desc)
        return
    raw, gz, desc = workload(args.workload, args.size)
    if args.impl == "reference":
        run_reference(args, raw, gz, desc)
    else:
        run_ours(args, raw, gz, desc)


if __name__ == "__main__":
    main()

import hashlib
import json
import os
import subprocess
import sys

import numpy as np

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# The rusty_rapidgzip checkout whose committed corpus pins the oracle: set
# RRG_REFERENCE_DIR to its root (the pinning test skips where it is absent).
REFERENCE_DIR = os.environ.get("RRG_REFERENCE_DIR", "/root/reference")
REFERENCE_CORPUS = os.path.join(REFERENCE_DIR, "tests", "corpus")
EMU_DIR = os.path.join(ROOT, "tests", "emu")
EMU_LIB = os.path.join(EMU_DIR, "librrg_gpu_emu.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built librrg_gpu.so")
    config.addinivalue_line("markers", "slow: longer CPU tests")


def sha256(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def golden_fixtures():
    sums = json.load(open(os.path.join(GOLDEN, "sums.json")))
    return [(name, os.path.join(GOLDEN, name), meta) for name, meta in sorted(sums.items())]


def ascii_payload(n: int, seed: int) -> bytes:
    """Seeded printable-ASCII LCG payload (the reference tests' generator shape)."""
    import numpy as np
    out = np.empty(n, dtype=np.uint8)
    s = (seed | 1) & 0xFFFFFFFFFFFFFFFF
    # vectorised LCG: s_{k} = a^k s_0 + c (a^k - 1)/(a - 1) is awkward in numpy; step in blocks
    a, c = 6364136223846793005, 1442695040888963407
    mask = (1 << 64) - 1
    i = 0
    block = []
    while i < n:
        s = (s * a + c) & mask
        block.append(((s >> 56) % 95) + 32)
        i += 1
        if len(block) == 65536 or i == n:
            out[i - len(block):i] = block
            block = []
    return out.tobytes()


def gzip_cli(data: bytes, level: int = 6) -> bytes:
    return subprocess.run(["gzip", f"-{level}", "-n", "-c"], input=data, stdout=subprocess.PIPE,
                          check=True).stdout


def build_emu_lib() -> str:
    """Compile the product sources against the CPU warp emulation (tests only)."""
    srcs = [os.path.join(ROOT, "rusty_rapidgzip_b200", "csrc", f) for f in
            ("rrg_gpu.cu", "rrg_kernels.cuh", "rrg_common.h")] + [os.path.join(EMU_DIR, "cuda_emu.h"),
                                                                  os.path.join(ROOT, "include", "rrg_gpu.h")]
    if not os.path.exists(EMU_LIB) or any(os.path.getmtime(s) > os.path.getmtime(EMU_LIB) for s in srcs):
        subprocess.check_call([
            "g++", "-std=c++20", "-O2", "-g", "-Werror=return-type", "-x", "c++", "-DRRG_EMU", "-include",
            os.path.join(EMU_DIR, "cuda_emu.h"), "-I", os.path.join(ROOT, "include"), "-I",
            os.path.join(ROOT, "rusty_rapidgzip_b200", "csrc"), "-fPIC", "-shared", "-pthread",
            "-o", EMU_LIB, os.path.join(ROOT, "rusty_rapidgzip_b200", "csrc", "rrg_gpu.cu")])
    return EMU_LIB


@pytest.fixture(scope="session")
def emu_decoder_factory():
    lib = build_emu_lib()
    from rusty_rapidgzip_b200 import Config, Decoder

    def make(**kw):
        kw.setdefault("device", -1)
        return Decoder(Config(**kw), lib=lib)

    return make


@pytest.fixture(scope="session")
def gpu_lib():
    """The real CUDA build; GPU tests fail loudly when it is missing."""
    import torch
    assert torch.cuda.is_available(), "GPU test needs CUDA"
    from rusty_rapidgzip_b200 import build as B
    path = B.build()
    assert os.path.exists(path), "librrg_gpu.so was not built"
    return path


@pytest.fixture()
def gpu_decoder_factory(gpu_lib):
    from rusty_rapidgzip_b200 import Config, Decoder
    made = []

    def make(**kw):
        kw.setdefault("device", 0)
        d = Decoder(Config(**kw), lib=gpu_lib)
        made.append(d)
        return d

    yield make
    for d in made:
        d.close()


def bgzf_cases():
    """BGZF inputs that exercise the device member walk: chains longer than a
    warp's 32-hit step, an EOF block, header-like bytes stored verbatim inside
    members (hits that are not on the chain), a plain member after the BGZF
    members, truncation inside a member and a corrupt trailer CRC."""
    from rusty_rapidgzip_b200 import workloads as W
    rng = np.random.default_rng(7)
    small = W.bgzf(W.fastq_like(70_000, 3), 5, block=1000)  # ~70 members
    eof = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")
    inner = W.bgzf(rng.integers(0, 256, 3000, dtype=np.uint8).tobytes(), 1, block=700)
    fake = W.bgzf(inner * 3, 0, block=4000)  # stored blocks: inner headers appear verbatim
    plain = gzip_cli(b"trailing plain member " * 50)
    cut = small[: len(small) - 300]
    bad = bytearray(small)
    m0 = int.from_bytes(bad[16:18], "little") + 1  # first member's size
    m1 = m0 + int.from_bytes(bad[m0 + 16:m0 + 18], "little") + 1
    bad[m1 - 8] ^= 0x40  # second member's CRC
    return {"chain": small + eof, "false-headers": fake, "then-plain": small + plain, "truncated": cut,
            "crc": bytes(bad)}


def serve_requests(n: int, seed: int, hi: int):
    """Mixed decode requests for the serving loop: the four content kinds of the
    many-files workload at log-uniform sizes up to `hi` bytes, plus a BGZF file,
    a two-member file and a request with a corrupt CRC."""
    from rusty_rapidgzip_b200 import workloads as W
    reqs = [gz for _, gz in W.config3_files(n_files=n, seed=seed, lo=4 << 10, hi=hi)]
    reqs.append(W.bgzf(W.fastq_like(min(200_000, 2 * hi), seed), 5, block=20_000))
    reqs.append(gzip_cli(b"first member " * 500) + gzip_cli(b"second member " * 4000))
    bad = bytearray(gzip_cli(b"payload with a broken trailer " * 100))
    bad[-8] ^= 0x10
    reqs.append(bytes(bad))
    return reqs


def run_serving(d, reqs, seed: int, gap_s: float, copy: bool = True):
    """Submit `reqs` from a thread at random gaps (open loop) while this thread
    polls; returns {request index: (status, bytes or None)}."""
    import random
    import threading
    import time
    rng = random.Random(seed)
    ids = {}
    order = list(range(len(reqs)))

    def feeder():
        for i in order:
            ids[d.submit(reqs[i], copy=copy)] = i
            time.sleep(rng.random() * gap_s)

    th = threading.Thread(target=feeder)
    th.start()
    got = {}
    deadline = time.time() + 600
    while len(got) < len(reqs) and time.time() < deadline:
        r = d.poll(timeout_ms=200)
        if r is None:
            continue
        rid, data, status, lat = r
        while rid not in ids:
            time.sleep(0.001)
        got[ids[rid]] = (status, data)
        if status:
            print(f"request {ids[rid]}: status {status}: {d.last_poll_error}")
    th.join()
    return got

"""The allocation-free CRC32 entry point, for callers that own all device
memory through their own pool and cannot let the library call cudaMalloc.
Its result must equal the context-based rrg_gpu_crc32 on consecutive calls
(the shared scratch keeps the previous call's contents), and oversized inputs
must be refused before any device work. Collected last on purpose."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(data: bytes):
    import torch
    t = torch.empty(max(len(data), 1), dtype=torch.uint8, device="cuda")
    if data:
        t[: len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    torch.cuda.synchronize()
    return t


def test_noalloc_crc_matches_context_entry_point(gpu_lib):
    import torch
    from rusty_rapidgzip_b200 import CapacityError, Config, Decoder
    from rusty_rapidgzip_b200._abi import crc32_noalloc
    rng = np.random.default_rng(2024)
    big = rng.integers(0, 256, (3 << 20) + 5, dtype=np.uint8).tobytes()
    small = rng.integers(0, 256, 1000, dtype=np.uint8).tobytes()
    with Decoder(Config(device=0), lib=gpu_lib) as d:
        for data in (big, small, b"", big[:262144]):  # consecutive calls reuse the scratch
            buf = _dev(data)
            want = d.crc32(buf, len(data))
            got = crc32_noalloc(buf, len(data), lib=gpu_lib)
            assert got == want == zlib.crc32(data)
        stream = torch.cuda.Stream()
        buf = _dev(big)
        assert crc32_noalloc(buf, len(big), stream=stream.cuda_stream, lib=gpu_lib) == zlib.crc32(big)
        # unaligned starts: every 256 KiB piece keeps the input's misalignment
        for shift in (1, 3, 7):
            n = len(big) - shift
            assert crc32_noalloc(buf[shift:], n, lib=gpu_lib) == d.crc32(buf[shift:], n) == zlib.crc32(big[shift:])
        with pytest.raises(CapacityError, match="at most"):
            crc32_noalloc(buf, (4 << 30) + 1, lib=gpu_lib)


def test_noalloc_crc_at_its_size_limit(gpu_lib):
    """Exactly 4 GiB is accepted and agrees with the context-based entry point
    (whose kernels differ); one byte more is refused."""
    import torch
    from rusty_rapidgzip_b200 import CapacityError, Config, Decoder
    from rusty_rapidgzip_b200._abi import crc32_noalloc
    n = 4 << 30
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    buf = torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda", generator=g)
    torch.cuda.synchronize()
    with Decoder(Config(device=0), lib=gpu_lib) as d:
        want = d.crc32(buf, n)
    for _ in range(2):
        assert crc32_noalloc(buf, n, lib=gpu_lib) == want
    with pytest.raises(CapacityError, match="at most"):
        crc32_noalloc(buf, n + 1, lib=gpu_lib)

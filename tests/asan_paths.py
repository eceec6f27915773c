"""Runs the batch, BGZF, member, stream, seek-index and serving paths of the emulated build under
AddressSanitizer with exact device-buffer sizes (RRG_STRICT_ALLOC), so that an
index past the end of any device buffer fails here rather than on a GPU.
Started by test_emu.py::test_address_sanitizer in its own process."""
import sys

import numpy as np

sys.path.insert(0, sys.argv[2])
from conftest import bgzf_cases, run_serving, serve_requests  # noqa: E402
from rusty_rapidgzip_b200 import Config, Decoder  # noqa: E402
from rusty_rapidgzip_b200 import workloads as W  # noqa: E402
from test_emu import batch_items, haddr, run_batch  # noqa: E402

lib = sys.argv[1]
d = Decoder(Config(device=-1, gpu_chunk_bytes=8192), lib=lib)
raw, gz = W.config1(40 << 10, seed=3)
assert d.decompress(gz) == raw
for case, data in bgzf_cases().items():
    if case in ("chain", "truncated", "crc"):
        try:
            d.decompress(data)
        except Exception:  # noqa: BLE001 - error cases are expected; only memory safety is checked here
            pass
import io  # noqa: E402

raw2, gz2 = W.config1(200 << 10, seed=4)
out = []
d.read_stream(io.BytesIO(gz2), out.append, stripe_bytes=65536)  # several stripes
assert b"".join(out) == raw2
idx = d.build_index(gz2, spacing=32 << 10)  # seek index and range reads
pts = idx.points()
assert d.read_range(gz2, idx, pts[1][0] - 10, 50_000) == raw2[pts[1][0] - 10:pts[1][0] + 49_990]
assert d.read_range(gz2, idx, len(raw2) - 100, 100) == raw2[-100:]
keep = []


def dev(data, out_n):
    a = np.frombuffer(data, dtype=np.uint8).copy()
    o = np.zeros(out_n, dtype=np.uint8)
    keep.extend([a, o])
    return haddr(a), haddr(o), lambda: o.tobytes()


small = [(r, g, c) for r, g, c in batch_items() if len(g) < 100_000]
b = Decoder(Config(device=-1, hbm_budget_bytes=1), lib=lib)  # several waves
run_batch(b, small, dev)
# one wave through the device-planned route, split files included
b = Decoder(Config(device=-1, gpu_chunk_bytes=16384), lib=lib)
outs, lens, status = run_batch(b, batch_items(), dev)
assert status[:4] == [0, 0, 0, 0] and outs[0] == batch_items()[0][0]
s = Decoder(Config(device=-1, hbm_budget_bytes=4 << 20), lib=lib)
s.serve_start(engines=2, max_ready=2)
got = run_serving(s, serve_requests(1, seed=5, hi=16 << 10), seed=3, gap_s=0.0)
assert len(got) == 4
s.close()
print("asan paths ok")

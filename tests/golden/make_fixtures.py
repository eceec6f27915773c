"""Regenerate the golden fixtures under tests/golden/.

1. ``synth-*.gz`` — the reference corpus's synthetic fixtures, rebuilt with
   the commands its manifest records (tests/corpus/corpus.json: system
   ``gzip -n`` over fixed payloads). Each output SHA-256 is pinned to the
   reference's tests/corpus/reference_sums.json. ``synth-random-1m`` comes
   from /dev/urandom upstream and cannot be rebuilt; a seeded 1 MiB random
   payload at gzip -6 stands in for it (its hash is computed here).
2. ``miri_edge_vectors.json`` — the raw-DEFLATE known-answer vectors of
   crates/rusty-rapidgzip/tests/miri_edge.rs, read from that file as text.
3. ``sums.json`` — file -> {sha256, raw_size, pinned_to_reference}.

Run with the reference checkout's root as the argument, or in
RRG_REFERENCE_DIR:
    python tests/golden/make_fixtures.py [/path/to/rusty_rapidgzip]
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RRG_REFERENCE_DIR", "/root/reference")

PAYLOADS = {
    "synth-empty.gz": (b"", 6),
    "synth-single-byte.gz": (b"A", 6),
    "synth-zeros-1m.gz": (b"\x00" * 1048576, 6),
    "synth-repeated-pattern.gz": (b"ABCDEFGH" * 131072, 6),
    "synth-spaces-1m.gz": (b" " * 1048576, 6),
    "synth-0xff-1m.gz": (b"\xff" * 1048576, 6),
    "synth-level1.gz": (bytes(range(256)) * 40960, 1),
    "synth-level9.gz": (bytes(range(256)) * 40960, 9),
}


def gzip_cli(data: bytes, level: int) -> bytes:
    return subprocess.run(["gzip", f"-{level}", "-n", "-c"], input=data, stdout=subprocess.PIPE,
                          check=True).stdout


def main():
    ref_sums = {}
    p = os.path.join(REF, "tests/corpus/reference_sums.json")
    if os.path.exists(p):
        ref_sums = json.load(open(p))
    sums = {}
    for name, (payload, level) in PAYLOADS.items():
        gz = gzip_cli(payload, level)
        open(os.path.join(HERE, name), "wb").write(gz)
        h = hashlib.sha256(payload).hexdigest()
        pinned = name in ref_sums
        if pinned and ref_sums[name]["sha256"] != h:
            raise SystemExit(f"{name}: payload hash {h} != reference {ref_sums[name]['sha256']}")
        sums[name] = {"sha256": h, "raw_size": len(payload), "pinned_to_reference": pinned}
    # concatenated members: (printf 'Hello' | gzip -n; printf 'World' | gzip -n)
    gz = gzip_cli(b"Hello", 6) + gzip_cli(b"World", 6)
    open(os.path.join(HERE, "synth-concat-members.gz"), "wb").write(gz)
    h = hashlib.sha256(b"HelloWorld").hexdigest()
    if "synth-concat-members.gz" in ref_sums:
        assert ref_sums["synth-concat-members.gz"]["sha256"] == h
    sums["synth-concat-members.gz"] = {"sha256": h, "raw_size": 10,
                                       "pinned_to_reference": "synth-concat-members.gz" in ref_sums}
    # seeded stand-in for the urandom fixture
    import numpy as np
    payload = np.random.default_rng(20240611).integers(0, 256, 1048576, dtype=np.uint8).tobytes()
    open(os.path.join(HERE, "seeded-random-1m.gz"), "wb").write(gzip_cli(payload, 6))
    sums["seeded-random-1m.gz"] = {"sha256": hashlib.sha256(payload).hexdigest(), "raw_size": len(payload),
                                   "pinned_to_reference": False}
    json.dump(sums, open(os.path.join(HERE, "sums.json"), "w"), indent=1, sort_keys=True)

    # raw-DEFLATE vectors from the reference test file
    src = os.path.join(REF, "crates/rusty-rapidgzip/tests/miri_edge.rs")
    if os.path.exists(src):
        text = open(src).read()
        body = text[text.index("vec!["):text.index("#[test]")]
        vecs = []
        for m in re.finditer(r'\(\s*"(\w+)",\s*vec!\[([^\]]*)\],\s*vec!\[([^\]]*)\],?\s*\)', body, re.S):
            name, stream, plain = m.group(1), m.group(2), m.group(3)
            nums = lambda s: [int(x) for x in re.findall(r"\d+", s)]
            vecs.append({"name": name, "deflate": bytes(nums(stream)).hex(), "plain": bytes(nums(plain)).hex()})
        # the empty vector is written with a tuple of empty vecs on one line
        if not any(v["name"] == "empty" for v in vecs):
            m = re.search(r'\("empty",\s*vec!\[([^\]]*)\],\s*vec!\[\]\)', body)
            if m:
                vecs.insert(0, {"name": "empty", "deflate": bytes(int(x) for x in re.findall(r"\d+", m.group(1))).hex(),
                                "plain": ""})
        json.dump(vecs, open(os.path.join(HERE, "miri_edge_vectors.json"), "w"), indent=0)
        print(f"{len(vecs)} raw-deflate vectors")
    print(f"{len(sums)} gzip fixtures")


if __name__ == "__main__":
    main()

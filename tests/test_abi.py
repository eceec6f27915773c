"""The C ABI boundary: the built library loads without a GPU, exports every
function include/rrg_gpu.h declares, and the Python mirror's struct layouts
match the C ones."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, build_emu_lib

HEADER = os.path.join(ROOT, "include", "rrg_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rrg_gpu_\w+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("rrg_gpu_create", "rrg_gpu_destroy", "rrg_gpu_read_gz", "rrg_gpu_decode_host",
                 "rrg_gpu_decode_device", "rrg_gpu_decode_batch", "rrg_gpu_find_blocks", "rrg_gpu_crc32",
                 "rrg_gpu_resolve_markers", "rrg_gpu_decode_chunk", "rrg_gpu_submit", "rrg_gpu_poll"):
        assert must in names


def _exports(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], stdout=subprocess.PIPE, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_cuda_library_exports_every_declared_symbol():
    from rusty_rapidgzip_b200 import build as B
    path = B.build()
    exported = _exports(path)
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    # loads on a machine without a GPU (no compute call is made)
    lib = C.CDLL(path)
    lib.rrg_gpu_version.restype = C.c_char_p
    assert b"sm_100a" in lib.rrg_gpu_version()


def test_emulated_library_exports_the_same_symbols():
    exported = _exports(build_emu_lib())
    assert not [n for n in declared_functions() if n not in exported]


def test_struct_layouts_match_c(tmp_path):
    from rusty_rapidgzip_b200 import _abi
    src = tmp_path / "sz.c"
    src.write_text('#include "rrg_gpu.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(rrg_error), sizeof(rrg_config), '
                   'sizeof(rrg_stats), offsetof(rrg_stats, finder_ms), offsetof(rrg_stats, graph_launches), '
                   'sizeof(rrg_tuning), offsetof(rrg_tuning, best_ms));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    e, c, s, off, goff, t, toff = map(int, subprocess.run([str(exe)], stdout=subprocess.PIPE,
                                                         text=True).stdout.split())
    assert C.sizeof(_abi._Error) == e
    assert C.sizeof(_abi._Config) == c
    assert C.sizeof(_abi._Stats) == s
    assert _abi._Stats.finder_ms.offset == off
    assert _abi._Stats.graph_launches.offset == goff
    assert C.sizeof(_abi._Tuning) == t
    assert _abi._Tuning.best_ms.offset == toff


def test_missing_library_fails_loudly(tmp_path):
    from rusty_rapidgzip_b200 import Config, Decoder
    with pytest.raises(ImportError, match="no CPU fallback"):
        Decoder(Config(), lib=str(tmp_path / "absent.so"))

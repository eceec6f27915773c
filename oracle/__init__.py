"""CPU oracle for the gzip/DEFLATE decode path (ctypes over librrg_oracle.so).

TEST INFRASTRUCTURE ONLY. The C library restates rusty_rapidgzip's decode
path (see rrg_oracle.h for the function-by-function reference map). It is the
parity checker for the CUDA decoder and the timed CPU baseline. Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg and reference arm
import it; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librrg_oracle.so")
SRC = os.path.join(HERE, "rrg_oracle.c")


def build(force: bool = False) -> str:
    """Compile librrg_oracle.so next to its source (gcc, -O2, pthreads)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "rrg_oracle.h"))
    ):
        subprocess.check_call(
            ["gcc", "-O2", "-Wall", "-fPIC", "-shared", "-pthread", "-o", LIB_PATH, SRC]
        )
    return LIB_PATH


class OrcError(C.Structure):
    _fields_ = [
        ("code", C.c_int32),
        ("member", C.c_uint32),
        ("expected", C.c_uint32),
        ("got_crc", C.c_uint32),
        ("got", C.c_uint64),
        ("uncompressed", C.c_uint64),
        ("trailer_byte", C.c_uint64),
        ("message", C.c_char * 160),
    ]


class OrcStats(C.Structure):
    _fields_ = [
        ("compressed_bytes", C.c_uint64),
        ("uncompressed_bytes", C.c_uint64),
        ("chunks_decoded", C.c_uint64),
        ("speculation_failures", C.c_uint64),
        ("n_chunks", C.c_uint64),
        ("n_markers", C.c_uint64),
    ]


class OrcMemberBoundary(C.Structure):
    _fields_ = [
        ("byte_offset_in_chunk", C.c_uint64),
        ("crc_expected", C.c_uint32),
        ("isize_expected", C.c_uint32),
        ("trailer_input_byte", C.c_uint64),
    ]


class OrcChunk(C.Structure):
    _fields_ = [
        ("bytes", C.POINTER(C.c_uint8)),
        ("n_bytes", C.c_uint64),
        ("marker_pos", C.POINTER(C.c_uint32)),
        ("marker_off", C.POINTER(C.c_uint16)),
        ("n_markers", C.c_uint64),
        ("mbs", C.POINTER(OrcMemberBoundary)),
        ("n_mbs", C.c_uint64),
        ("start_bit", C.c_uint64),
        ("end_bit_hint", C.c_uint64),
        ("actual_end_bit", C.c_uint64),
        ("final_block", C.c_int32),
        ("status", C.c_int32),
    ]


SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t)

_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        u8p = C.POINTER(C.c_uint8)
        L.orc_crc32.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t]
        L.orc_crc32.restype = C.c_uint32
        L.orc_crc32_combine.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
        L.orc_crc32_combine.restype = C.c_uint32
        L.orc_parse_header.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.orc_bgzf_block_size.argtypes = [C.c_void_p, C.c_size_t]
        L.orc_bgzf_block_size.restype = C.c_int64
        L.orc_find_next_dynamic_block.argtypes = [
            C.c_void_p, C.c_size_t, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
        L.orc_verify_candidate.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64]
        L.orc_inflate_raw.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(u8p),
                                      C.POINTER(C.c_size_t), C.POINTER(C.c_uint64),
                                      C.POINTER(OrcError)]
        L.orc_decode_all.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(u8p),
                                     C.POINTER(C.c_size_t), C.POINTER(OrcError)]
        L.orc_decode_chunk.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, C.c_uint64,
                                       C.POINTER(OrcChunk), C.POINTER(OrcError)]
        L.orc_chunk_free.argtypes = [C.POINTER(OrcChunk)]
        L.orc_resolve_markers.argtypes = [C.POINTER(OrcChunk), C.c_void_p, C.c_size_t,
                                          C.POINTER(OrcError)]
        L.orc_build_prev_tail.argtypes = [C.POINTER(OrcChunk), C.c_void_p, C.c_size_t, C.c_void_p]
        L.orc_build_prev_tail.restype = C.c_size_t
        L.orc_read_gz_buffer.argtypes = [C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint64, SINK,
                                         C.c_void_p, C.POINTER(OrcStats), C.POINTER(OrcError)]
        L.orc_read_gz_to_buffer.argtypes = [C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint64,
                                            C.POINTER(u8p), C.POINTER(C.c_size_t),
                                            C.POINTER(OrcStats), C.POINTER(OrcError)]
        L.orc_free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


class OracleError(Exception):
    def __init__(self, code: int, err: OrcError | None = None):
        self.code = int(code)
        self.member = err.member if err else 0
        self.expected = err.expected if err else 0
        self.got_crc = err.got_crc if err else 0
        self.got = err.got if err else 0
        self.uncompressed = err.uncompressed if err else 0
        self.trailer_byte = err.trailer_byte if err else 0
        self.message = err.message.decode(errors="replace") if err else ""
        super().__init__(f"oracle status {self.code}: {self.message}")


def _buf(data):
    """(pointer, length, keepalive) for bytes-like or numpy input."""
    if isinstance(data, np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.uint8)
    else:
        a = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, (bytes, bytearray, memoryview)) \
            else np.frombuffer(data, dtype=np.uint8)
    return a.ctypes.data if a.size else None, a.size, a


def _take(ptr, n) -> bytes:
    try:
        return C.string_at(ptr, n) if n else b""
    finally:
        lib().orc_free(C.cast(ptr, C.c_void_p))


def crc32(data, crc: int = 0) -> int:
    p, n, _k = _buf(data)
    return lib().orc_crc32(crc, p, n)


def crc32_combine(crc_a: int, crc_b: int, len_b: int) -> int:
    return lib().orc_crc32_combine(crc_a, crc_b, len_b)


def parse_header(data) -> int:
    p, n, _k = _buf(data)
    out = C.c_size_t()
    r = lib().orc_parse_header(p, n, C.byref(out))
    if r:
        raise OracleError(r)
    return out.value


def bgzf_block_size(data):
    p, n, _k = _buf(data)
    v = lib().orc_bgzf_block_size(p, n)
    return None if v < 0 else v


def find_next_dynamic_block(data, from_bit: int, until_bit: int):
    p, n, _k = _buf(data)
    out = C.c_uint64()
    ok = lib().orc_find_next_dynamic_block(p, n, from_bit, until_bit, C.byref(out))
    return out.value if ok else None


def verify_candidate(data, pos: int) -> bool:
    p, n, _k = _buf(data)
    return bool(lib().orc_verify_candidate(p, n, pos))


def inflate_raw(data):
    """Whole raw-DEFLATE stream -> (bytes, end_bit)."""
    p, n, _k = _buf(data)
    out = C.POINTER(C.c_uint8)()
    olen = C.c_size_t()
    end = C.c_uint64()
    err = OrcError()
    r = lib().orc_inflate_raw(p, n, C.byref(out), C.byref(olen), C.byref(end), C.byref(err))
    if r:
        raise OracleError(r, err)
    return _take(out, olen.value), end.value


def decode_all(data) -> bytes:
    p, n, _k = _buf(data)
    out = C.POINTER(C.c_uint8)()
    olen = C.c_size_t()
    err = OrcError()
    r = lib().orc_decode_all(p, n, C.byref(out), C.byref(olen), C.byref(err))
    if r:
        raise OracleError(r, err)
    return _take(out, olen.value)


@dataclass
class Chunk:
    bytes: bytes
    marker_pos: np.ndarray
    marker_off: np.ndarray
    member_boundaries: list
    start_bit: int
    end_bit_hint: int
    actual_end_bit: int
    final_block: bool


def decode_chunk(body, start_bit: int, end_bit_hint: int) -> Chunk:
    """decode_one_chunk: speculative decode of [start_bit, end_bit_hint)."""
    p, n, _k = _buf(body)
    ch = OrcChunk()
    err = OrcError()
    r = lib().orc_decode_chunk(p, n, start_bit, end_bit_hint, C.byref(ch), C.byref(err))
    if r:
        raise OracleError(r, err)
    try:
        b = C.string_at(ch.bytes, ch.n_bytes) if ch.n_bytes else b""
        mp = np.ctypeslib.as_array(ch.marker_pos, (ch.n_markers,)).copy() if ch.n_markers else \
            np.zeros(0, np.uint32)
        mo = np.ctypeslib.as_array(ch.marker_off, (ch.n_markers,)).copy() if ch.n_markers else \
            np.zeros(0, np.uint16)
        mbs = [(ch.mbs[i].byte_offset_in_chunk, ch.mbs[i].crc_expected, ch.mbs[i].isize_expected,
                ch.mbs[i].trailer_input_byte) for i in range(ch.n_mbs)]
        return Chunk(b, mp, mo, mbs, ch.start_bit, ch.end_bit_hint, ch.actual_end_bit,
                     bool(ch.final_block))
    finally:
        lib().orc_chunk_free(C.byref(ch))


def read_gz(data, num_threads: int = 0, chunk_size: int = 4 << 20, with_stats: bool = False):
    """lib.rs read_gz over an in-memory file; returns the decompressed bytes."""
    p, n, _k = _buf(data)
    out = C.POINTER(C.c_uint8)()
    olen = C.c_size_t()
    st = OrcStats()
    err = OrcError()
    r = lib().orc_read_gz_to_buffer(p, n, num_threads, chunk_size, C.byref(out), C.byref(olen),
                                    C.byref(st), C.byref(err))
    if r:
        raise OracleError(r, err)
    data_out = _take(out, olen.value)
    if with_stats:
        return data_out, {f: getattr(st, f) for f, _ in OrcStats._fields_}
    return data_out


def read_gz_count(data, num_threads: int = 0, chunk_size: int = 4 << 20):
    """read_gz with a sink that only counts bytes (for timing the CPU path).
    Returns (uncompressed_bytes, stats dict)."""
    p, n, _k = _buf(data)
    st = OrcStats()
    err = OrcError()
    total = [0]

    def _sink(_u, _ptr, ln):
        total[0] += ln
        return 0

    cb = SINK(_sink)
    r = lib().orc_read_gz_buffer(p, n, num_threads, chunk_size, cb, None, C.byref(st), C.byref(err))
    if r:
        raise OracleError(r, err)
    return total[0], {f: getattr(st, f) for f, _ in OrcStats._fields_}

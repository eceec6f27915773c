"""ctypes binding of include/rrg_gpu.h and the Python mirror of the reference API.

The reference's drop-in surface (crates/rusty-rapidgzip/src/lib.rs):

    read_gz(path, sink: Sender<Arc<Vec<u8>>>, config: Config) -> Result<DecodeStats, Error>

is mirrored by :func:`read_gz` here: ``sink`` receives the decompressed stream
in order as ``bytes`` pieces (a callable, or any object with ``send``/``put``,
e.g. ``queue.Queue``); a sink returning ``False`` (or whose ``send``/``put``
raises :class:`SinkClosed`) closes the channel and decoding stops early with
success, as a dropped receiver does in the reference (pipeline.rs:1028-1030).
Errors raise :class:`RrgError` subclasses mirroring ``Error::{Io, Gzip, Deflate}``.

All work runs in the CUDA library ``librrg_gpu.so`` built next to this file.
There is no CPU fallback: if the library is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "librrg_gpu.so"
DEFAULT_LIB = os.path.join(HERE, LIB_NAME)

# enum rrg_status
OK = 0
ERR_IO = 1
ERR_BAD_MAGIC = 2
ERR_UNSUPPORTED_METHOD = 3
ERR_RESERVED_FLAGS = 4
ERR_TRUNCATED = 5
ERR_CRC_MISMATCH = 6
ERR_ISIZE_MISMATCH = 7
ERR_DEFLATE_EOF = 8
ERR_DEFLATE_INVALID = 9
ERR_CUDA = 20
ERR_OUT_OF_MEMORY = 21
ERR_INVALID_ARGUMENT = 22
ERR_TIMEOUT = 23
ERR_CAPACITY = 24

GZIP_KINDS = {
    ERR_BAD_MAGIC: "BadMagic",
    ERR_UNSUPPORTED_METHOD: "UnsupportedMethod",
    ERR_RESERVED_FLAGS: "ReservedFlags",
    ERR_TRUNCATED: "Truncated",
    ERR_CRC_MISMATCH: "CrcMismatch",
    ERR_ISIZE_MISMATCH: "IsizeMismatch",
}


class _Error(C.Structure):
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


class _Config(C.Structure):
    _fields_ = [
        ("num_threads", C.c_uint32),
        ("chunk_size_bytes", C.c_uint64),
        ("verbose", C.c_int32),
        ("device", C.c_int32),
        ("gpu_chunk_bytes", C.c_uint64),
        ("finder_tile_bits", C.c_uint64),
        ("warps_per_stream", C.c_int32),
        ("boundary_mode", C.c_int32),
        ("hbm_budget_bytes", C.c_uint64),
        ("host_pipeline", C.c_int32),
        ("batch_plan", C.c_int32),
    ]


_STAT_U64 = ["compressed_bytes", "uncompressed_bytes", "chunks_decoded", "speculation_failures",
             "gpu_chunks", "markers", "members", "kernel_launches"]
_STAT_F64 = ["finder_ms", "inflate_ms", "resolve_ms", "crc_ms", "h2d_ms", "d2h_ms", "total_ms"]


class _SplitInfo(C.Structure):
    _fields_ = [("start_bit", C.c_uint64), ("end_bit", C.c_uint64), ("out_len", C.c_uint64),
                ("has_trailer", C.c_uint32), ("crc", C.c_uint32), ("isize", C.c_uint32), ("pad", C.c_uint32),
                ("trailer_byte", C.c_uint64)]


class _Tuning(C.Structure):
    _fields_ = [("gpu_chunk_bytes", C.c_uint64), ("boundary_mode", C.c_int32), ("warps_per_member", C.c_int32),
                ("finder_tile_bits", C.c_uint64), ("best_ms", C.c_double), ("default_ms", C.c_double),
                ("trials", C.c_uint32)]


class _ServeStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "batches", "max_batch", "engines_busy",
                                          "max_engines_busy", "in_use_bytes", "peak_in_use_bytes", "budget_bytes",
                                          "waiting", "bytes_out")] + [
        (n, C.c_double) for n in ("h2d_ms", "decode_ms", "d2h_ms")]


class _Stats(C.Structure):
    _fields_ = ([(n, C.c_uint64) for n in _STAT_U64] + [(n, C.c_double) for n in _STAT_F64]
                + [("graph_launches", C.c_uint64), ("pipeline_waves", C.c_uint64),
                   ("pipeline_fallbacks", C.c_uint64)])


SINK_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t)
BUF_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t))
READ_FN = C.CFUNCTYPE(C.c_int64, C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t)


# ------------------------------------------------------------------ API types
@dataclass
class Config:
    """Mirrors Config (lib.rs:50-100) plus device tunables (0 = autotuned)."""
    num_threads: int = 0
    chunk_size_bytes: int = 4 << 20
    verbose: int = 0  # 0 off, 1 per-call summary, 2 also every re-decoded sub-chunk
    device: int = -1
    gpu_chunk_bytes: int = 0
    finder_tile_bits: int = 0
    warps_per_stream: int = 0
    boundary_mode: int = 0
    hbm_budget_bytes: int = 0
    host_pipeline: int = 0  # -1: the host path never decodes in overlapped waves; N >= 2: N waves
    batch_plan: int = 0  # -1: decode_batch never takes the device-planned graph route

    def _c(self) -> _Config:
        c = _Config()
        c.num_threads = self.num_threads
        c.chunk_size_bytes = self.chunk_size_bytes
        c.verbose = int(self.verbose)
        c.device = self.device
        c.gpu_chunk_bytes = self.gpu_chunk_bytes
        c.finder_tile_bits = self.finder_tile_bits
        c.warps_per_stream = self.warps_per_stream
        c.boundary_mode = self.boundary_mode
        c.hbm_budget_bytes = self.hbm_budget_bytes
        c.host_pipeline = self.host_pipeline
        c.batch_plan = self.batch_plan
        return c


@dataclass
class DecodeStats:
    """Mirrors DecodeStats (lib.rs:103-108) plus device-path counters."""
    compressed_bytes: int = 0
    uncompressed_bytes: int = 0
    chunks_decoded: int = 0
    speculation_failures: int = 0
    gpu_chunks: int = 0
    markers: int = 0
    members: int = 0
    kernel_launches: int = 0
    graph_launches: int = 0
    pipeline_waves: int = 0
    pipeline_fallbacks: int = 0
    timings_ms: dict = field(default_factory=dict)

    @classmethod
    def _from(cls, s: _Stats) -> "DecodeStats":
        return cls(**{n: int(getattr(s, n)) for n in _STAT_U64}, graph_launches=int(s.graph_launches),
                   pipeline_waves=int(s.pipeline_waves), pipeline_fallbacks=int(s.pipeline_fallbacks),
                   timings_ms={n[:-3]: float(getattr(s, n)) for n in _STAT_F64})


class RrgError(Exception):
    """Base of the decoder errors (Error in lib.rs:111-118)."""

    def __init__(self, e: _Error):
        self.code = int(e.code)
        self.member = int(e.member)
        self.expected = int(e.expected)
        self.got_crc = int(e.got_crc)
        self.got = int(e.got)
        self.uncompressed = int(e.uncompressed)
        self.trailer_byte = int(e.trailer_byte)
        self.message = e.message.decode(errors="replace")
        super().__init__(self.message or f"status {self.code}")


class IoError(RrgError):
    """Error::Io"""


class GzipError(RrgError):
    """Error::Gzip(GzipError::...); ``kind`` names the variant."""

    @property
    def kind(self) -> str:
        return GZIP_KINDS.get(self.code, "Unknown")


class DeflateError(RrgError):
    """Error::Deflate(DeflateError::UnexpectedEof | Invalid(&str))."""

    @property
    def kind(self) -> str:
        return "UnexpectedEof" if self.code == ERR_DEFLATE_EOF else "Invalid"


class DeviceError(RrgError):
    """CUDA runtime failure, device memory exhausted, or bad ABI argument."""


class CapacityError(RrgError):
    """Caller-provided output buffer too small."""


class SinkClosed(Exception):
    """Raise from a sink to close it (the reference's disconnected receiver)."""


def _raise(e: _Error):
    code = int(e.code)
    if code == OK:
        return
    if code == ERR_IO:
        raise IoError(e)
    if code in GZIP_KINDS:
        raise GzipError(e)
    if code in (ERR_DEFLATE_EOF, ERR_DEFLATE_INVALID):
        raise DeflateError(e)
    if code == ERR_CAPACITY:
        raise CapacityError(e)
    raise DeviceError(e)


# ------------------------------------------------------------------ library
_lib_cache: dict = {}
_lib_lock = threading.Lock()


def library_path() -> str:
    return os.environ.get("RRG_GPU_LIB", DEFAULT_LIB)


def load_library(path: str | None = None):
    """Load and type the decoder library; raises if it has not been built."""
    path = path or library_path()
    with _lib_lock:
        if path in _lib_cache:
            return _lib_cache[path]
        if not os.path.exists(path):
            raise ImportError(
                f"{path} not found: build the CUDA library first "
                "(python -m rusty_rapidgzip_b200.build); there is no CPU fallback")
        L = C.CDLL(path)
        vp, sz, u64, i32 = C.c_void_p, C.c_size_t, C.c_uint64, C.c_int32
        E, S = C.POINTER(_Error), C.POINTER(_Stats)
        L.rrg_gpu_create.argtypes = [C.POINTER(_Config), E]
        L.rrg_gpu_create.restype = vp
        L.rrg_gpu_destroy.argtypes = [vp]
        L.rrg_gpu_read_gz.argtypes = [vp, C.c_char_p, SINK_FN, vp, S, E]
        L.rrg_gpu_decode_host.argtypes = [vp, vp, sz, SINK_FN, vp, S, E]
        L.rrg_gpu_decode_host_into.argtypes = [vp, vp, sz, BUF_FN, SINK_FN, vp, S, E]
        L.rrg_gpu_split_begin.argtypes = [vp, vp, sz, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32,
                                          C.POINTER(C.c_uint16), C.POINTER(_SplitInfo), E]
        L.rrg_gpu_split_finish.argtypes = [vp, vp, sz, SINK_FN, vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), E]
        L.rrg_crc32_combine.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
        L.rrg_crc32_combine.restype = C.c_uint32
        L.rrg_gpu_read_gz_into.argtypes = [vp, C.c_char_p, BUF_FN, SINK_FN, vp, S, E]
        L.rrg_gpu_read_stream.argtypes = [vp, READ_FN, vp, SINK_FN, vp, u64, S, E]
        L.rrg_gpu_index_build.argtypes = [vp, vp, sz, u64, C.POINTER(vp), S, E]
        L.rrg_gpu_read_range.argtypes = [vp, vp, sz, vp, u64, u64, vp, E]
        L.rrg_index_total_out.argtypes = [vp]
        L.rrg_index_total_out.restype = u64
        L.rrg_index_count.argtypes = [vp]
        L.rrg_index_count.restype = sz
        L.rrg_index_point.argtypes = [vp, sz, C.POINTER(u64), C.POINTER(u64)]
        L.rrg_index_serialize.argtypes = [vp, vp, sz]
        L.rrg_index_serialize.restype = sz
        L.rrg_index_deserialize.argtypes = [vp, sz, E]
        L.rrg_index_deserialize.restype = vp
        L.rrg_index_free.argtypes = [vp]
        L.rrg_index_free.restype = None
        L.rrg_gpu_decode_device.argtypes = [vp, vp, sz, vp, sz, C.POINTER(sz), vp, S, E]
        L.rrg_gpu_decode_batch.argtypes = [vp, vp, C.POINTER(u64), C.POINTER(u64), vp, C.POINTER(u64),
                                           C.POINTER(u64), C.POINTER(u64), C.POINTER(i32), sz, vp, S, E]
        L.rrg_gpu_autotune.argtypes = [vp, vp, C.POINTER(u64), C.POINTER(u64), vp, C.POINTER(u64), C.POINTER(u64),
                                       sz, vp, C.POINTER(_Tuning), E]
        L.rrg_gpu_find_blocks.argtypes = [vp, vp, sz, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), sz, E]
        L.rrg_gpu_crc32.argtypes = [vp, vp, sz, C.POINTER(C.c_uint32), E]
        L.rrg_gpu_resolve_markers.argtypes = [vp, vp, sz, vp, vp, sz, vp, sz, E]
        L.rrg_gpu_decode_chunk.argtypes = [vp, vp, sz, u64, u64, vp, C.POINTER(sz), vp, vp, C.POINTER(sz),
                                           C.POINTER(u64), C.POINTER(i32), E]
        L.rrg_gpu_submit.argtypes = [vp, vp, sz, E]
        L.rrg_gpu_submit.restype = C.c_int64
        L.rrg_gpu_submit_nocopy.argtypes = [vp, vp, sz, E]
        L.rrg_gpu_submit_nocopy.restype = C.c_int64
        L.rrg_gpu_poll.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(sz),
                                   C.POINTER(i32), C.POINTER(C.c_double), i32, E]
        L.rrg_gpu_serve_start.argtypes = [vp, C.c_uint32, C.c_uint32, E]
        L.rrg_gpu_serve_stop.argtypes = [vp]
        L.rrg_gpu_serve_stop.restype = None
        L.rrg_gpu_serve_stats.argtypes = [vp, C.POINTER(_ServeStats)]
        L.rrg_gpu_pending.argtypes = [vp]
        L.rrg_gpu_pending.restype = C.c_int64
        L.rrg_gpu_crc32_noalloc.argtypes = [vp, sz, C.POINTER(C.c_uint32), vp, E]
        L.rrg_gpu_free.argtypes = [vp]
        L.rrg_gpu_version.restype = C.c_char_p
        L.rrg_gpu_kernel_launch_count.restype = C.c_uint64
        _lib_cache[path] = L
        return L


def _ptr(x) -> int:
    """Address of a device buffer: an int, or an object with data_ptr() (torch)."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    raise TypeError(f"expected a device pointer, got {type(x).__name__}")


def _host_buffer(data):
    """(address, length, keepalive) of a host bytes-like object, in place: the
    library only reads it. A read-only object (bytes, a read-only mmap) is not
    copied either; the keepalive holds it for as long as the call needs it."""
    if isinstance(data, bytes):
        return (C.cast(C.c_char_p(data), C.c_void_p).value if data else None), len(data), (data,)
    mv = memoryview(data).cast("B")
    if not len(mv):
        return None, 0, (mv,)
    if mv.readonly:
        import numpy as np  # exposes a read-only buffer's address without a copy
        arr = np.frombuffer(mv, dtype=np.uint8)
        return arr.ctypes.data, len(mv), (arr, mv)
    buf = (C.c_char * len(mv)).from_buffer(mv)
    return C.addressof(buf), len(mv), (buf, mv)


def _as_sink(sink):
    if sink is None:
        return None
    if callable(sink):
        return sink
    for m in ("send", "put"):
        if hasattr(sink, m):
            return getattr(sink, m)
    raise TypeError("sink must be callable or have send()/put()")


class SeekIndex:
    """Checkpoints of one member stream for random access (rrg_index)."""

    def __init__(self, lib, ptr: int):
        self._L, self._p = lib, ptr

    @classmethod
    def load(cls, blob: bytes, lib: str | None = None) -> "SeekIndex":
        L = load_library(lib)
        e = _Error()
        p = L.rrg_index_deserialize(blob, len(blob), C.byref(e))
        _raise(e)
        return cls(L, p)

    @property
    def total_out(self) -> int:
        return int(self._L.rrg_index_total_out(self._p))

    def points(self) -> list[tuple[int, int]]:
        """(output offset, file-absolute bit) of every checkpoint."""
        pts = []
        for k in range(int(self._L.rrg_index_count(self._p))):
            o, b = C.c_uint64(), C.c_uint64()
            self._L.rrg_index_point(self._p, k, C.byref(o), C.byref(b))
            pts.append((o.value, b.value))
        return pts

    def serialize(self) -> bytes:
        n = self._L.rrg_index_serialize(self._p, None, 0)
        buf = (C.c_char * n)()
        self._L.rrg_index_serialize(self._p, C.addressof(buf), n)
        return buf.raw

    def close(self):
        if self._p:
            self._L.rrg_index_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Decoder:
    """A decoding context on one GPU (rrg_gpu_create). One decode at a time."""

    def __init__(self, config: Config | None = None, lib: str | None = None):
        self.config = config or Config()
        self._L = load_library(lib)
        e = _Error()
        self._ctx = self._L.rrg_gpu_create(C.byref(self.config._c()), C.byref(e))
        if not self._ctx:
            _raise(e)
        import threading
        self._inflight: dict = {}      # zero-copy requests: id -> the bytes the engines read
        self._polled_early: set = set()
        self._inflight_lock = threading.Lock()

    def close(self):
        if getattr(self, "_ctx", None):
            self._L.rrg_gpu_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- streaming
    def _run(self, fn, *args, sink=None) -> DecodeStats:
        target = _as_sink(sink)
        failure = []

        def cb(_u, p, n):
            if target is None:
                return 0
            try:
                r = target(C.string_at(p, n))
            except SinkClosed:
                return 1
            except BaseException as ex:  # surfaced after the call returns
                failure.append(ex)
                return 1
            return 1 if r is False else 0

        st, e = _Stats(), _Error()
        fn(self._ctx, *args, SINK_FN(cb), None, C.byref(st), C.byref(e))
        if failure:
            raise failure[0]
        _raise(e)
        return DecodeStats._from(st)

    def read_gz(self, path, sink) -> DecodeStats:
        """read_gz (lib.rs:366-496) for a file path."""
        return self._run(self._L.rrg_gpu_read_gz, os.fsencode(os.fspath(path)), sink=sink)

    def _run_into(self, fn, arg0, arg1, recycle, sink) -> DecodeStats:
        """`recycle(want) -> (address, capacity) | None` supplies destination
        buffers (Config::recycle_rx); `sink(address, length)` then receives
        each filled buffer (the consumer's; hand it back through `recycle`)."""
        failure = []

        def get(_u, want, cap):
            try:
                r = recycle(int(want))
            except BaseException as ex:  # surfaced after the call returns
                failure.append(ex)
                r = None
            if not r:
                return None
            cap[0] = int(r[1])
            return int(r[0])

        def cb(_u, p, n):
            try:
                r = sink(C.cast(p, C.c_void_p).value, int(n))
            except SinkClosed:
                return 1
            except BaseException as ex:
                failure.append(ex)
                return 1
            return 1 if r is False else 0

        st, e = _Stats(), _Error()
        fn(self._ctx, arg0, arg1, BUF_FN(get), SINK_FN(cb), None, C.byref(st), C.byref(e))
        if failure:
            raise failure[0]
        _raise(e)
        return DecodeStats._from(st)

    def crc32_combine(self, crc_a: int, crc_b: int, len_b: int) -> int:
        """CRC32 of A||B from CRC32(A), CRC32(B) and |B| (rrg_crc32_combine)."""
        return int(self._L.rrg_crc32_combine(crc_a, crc_b, len_b))

    # ------------------------------------------------------- split member
    def split_begin(self, data, body_off: int, start_target: int, stop_target: int, exact: bool = False):
        """Phase 1 of one range of a member decoded on several GPUs
        (rrg_gpu_split_begin): -> (info dict, end_map as a numpy uint16 array)."""
        import numpy as np
        addr, n, keep = _host_buffer(data)
        m = np.empty(32768, dtype=np.uint16)
        info, e = _SplitInfo(), _Error()
        self._L.rrg_gpu_split_begin(self._ctx, addr, n, body_off, start_target, stop_target, 1 if exact else 0,
                                    m.ctypes.data_as(C.POINTER(C.c_uint16)), C.byref(info), C.byref(e))
        del keep
        _raise(e)
        return {f: int(getattr(info, f)) for f, _ in _SplitInfo._fields_ if f != "pad"}, m

    def split_finish(self, window: bytes, sink) -> tuple[int, int]:
        """Phase 2 (rrg_gpu_split_finish): resolve with the 32 KiB before the
        range; the bytes go to `sink`; -> (CRC32, length) of the range."""
        target = _as_sink(sink)
        failure = []

        def cb(_u, p, n):
            try:
                if target is not None:
                    target(C.string_at(p, n))
            except BaseException as ex:  # noqa: BLE001 - surfaced below
                failure.append(ex)
                return 1
            return 0

        crc, ln, e = C.c_uint32(), C.c_uint64(), _Error()
        self._L.rrg_gpu_split_finish(self._ctx, window if window else None, len(window), SINK_FN(cb), None,
                                     C.byref(crc), C.byref(ln), C.byref(e))
        if failure:
            raise failure[0]
        _raise(e)
        return int(crc.value), int(ln.value)

    def decode_host_into(self, data, recycle, sink) -> DecodeStats:
        """decode_host whose output pieces land in buffers from `recycle`."""
        addr, n, keep = _host_buffer(data)
        stats = self._run_into(self._L.rrg_gpu_decode_host_into, addr, n, recycle, sink)
        del keep
        return stats

    def read_gz_into(self, path, recycle, sink) -> DecodeStats:
        """read_gz whose output pieces land in buffers from `recycle`."""
        p = os.fsencode(os.fspath(path))
        L = self._L

        def fn(ctx, path_, _unused, get, cb, user, st, e):
            return L.rrg_gpu_read_gz_into(ctx, path_, get, cb, user, st, e)

        return self._run_into(fn, p, None, recycle, sink)

    def read_stream(self, source, sink, stripe_bytes: int = 0) -> DecodeStats:
        """read_gz's non-seekable route (lib.rs:378-431, streaming.rs:389-614):
        `source` is a binary file object (readinto/read) or a callable
        taking a byte count and returning bytes (b"" at the end). Decoding
        runs stripe by stripe as the input is read."""
        failure = []
        if hasattr(source, "readinto"):
            def pull(buf, cap):
                return source.readinto(memoryview(buf).cast("B")[:cap]) or 0
        else:
            reader = source.read if hasattr(source, "read") else source

            def pull(buf, cap):
                b = reader(cap)
                C.memmove(buf, b, len(b))
                return len(b)

        def rcb(_u, p, cap):
            try:
                arr = (C.c_uint8 * cap).from_address(C.addressof(p.contents))
                return int(pull(arr, cap))
            except BaseException as ex:  # surfaced after the call returns
                failure.append(ex)
                return -1

        target = _as_sink(sink)

        def cb(_u, p, n):
            if target is None:
                return 0
            try:
                r = target(C.string_at(p, n))
            except SinkClosed:
                return 1
            except BaseException as ex:
                failure.append(ex)
                return 1
            return 1 if r is False else 0

        st, e = _Stats(), _Error()
        self._L.rrg_gpu_read_stream(self._ctx, READ_FN(rcb), None, SINK_FN(cb), None, int(stripe_bytes),
                                    C.byref(st), C.byref(e))
        if failure:
            raise failure[0]
        _raise(e)
        return DecodeStats._from(st)

    def build_index(self, data, spacing: int = 0) -> "SeekIndex":
        """Seek index of a member stream in host memory (no reference
        counterpart): checkpoints at least `spacing` output bytes apart (0:
        4 MiB) with their 32 KiB windows, from one CRC-checked decode."""
        addr, n, keep = _host_buffer(data)
        out, st, e = C.c_void_p(), _Stats(), _Error()
        self._L.rrg_gpu_index_build(self._ctx, addr, n, int(spacing), C.byref(out), C.byref(st), C.byref(e))
        del keep
        _raise(e)
        return SeekIndex(self._L, out.value)

    def read_range(self, data, index: "SeekIndex", off: int, n: int) -> bytes:
        """Output bytes [off, off + n) of `data` (the file `index` was built on)."""
        addr, ln, keep = _host_buffer(data)
        dst = (C.c_char * max(n, 1))()
        e = _Error()
        self._L.rrg_gpu_read_range(self._ctx, addr, ln, index._p, int(off), int(n), C.addressof(dst), C.byref(e))
        del keep
        _raise(e)
        return dst.raw[:n]

    def decode_host(self, data, sink) -> DecodeStats:
        """read_gz over a gzip file already in host memory."""
        addr, n, keep = _host_buffer(data)
        stats = self._run(self._L.rrg_gpu_decode_host, addr, n, sink=sink)
        del keep
        return stats

    def decompress(self, data) -> bytes:
        out = []
        self.decode_host(data, out.append)
        return b"".join(out)

    def count(self, data) -> tuple[int, DecodeStats]:
        """Decode, delivering to a sink that only counts bytes (no Python copy)."""
        addr, n, keep = _host_buffer(data)
        total = [0]

        def cb(_u, _p, ln):
            total[0] += ln
            return 0

        st, e = _Stats(), _Error()
        self._L.rrg_gpu_decode_host(self._ctx, addr, n, SINK_FN(cb), None, C.byref(st), C.byref(e))
        del keep
        _raise(e)
        return total[0], DecodeStats._from(st)

    # -------------------------------------------------------------- device
    def decode_device(self, d_in, length: int, d_out, out_cap: int, stream=None) -> tuple[int, DecodeStats]:
        """Device-resident decode; returns (bytes written, stats)."""
        out_len = C.c_size_t()
        st, e = _Stats(), _Error()
        self._L.rrg_gpu_decode_device(self._ctx, _ptr(d_in), length, _ptr(d_out), out_cap, C.byref(out_len),
                                      _ptr(stream), C.byref(st), C.byref(e))
        if e.code == ERR_CAPACITY:
            err = CapacityError(e)
            err.required = int(out_len.value)
            raise err
        _raise(e)
        return int(out_len.value), DecodeStats._from(st)

    def decode_batch(self, d_in, in_off, in_len, d_out, out_off, out_cap, stream=None):
        """Batched member decode; returns (out_len list, status list, stats).
        Raises nothing for per-item failures (see the status list)."""
        n = len(in_off)
        A = C.c_uint64 * max(n, 1)
        io, il, oo, oc = A(*in_off), A(*in_len), A(*out_off), A(*out_cap)
        ol = A()
        stv = (C.c_int32 * max(n, 1))()
        st, e = _Stats(), _Error()
        self._L.rrg_gpu_decode_batch(self._ctx, _ptr(d_in), io, il, _ptr(d_out), oo, oc, ol, stv, n,
                                     _ptr(stream), C.byref(st), C.byref(e))
        if e.code not in (OK,) and e.code >= ERR_CUDA and e.code != ERR_CAPACITY:
            _raise(e)
        return [int(ol[i]) for i in range(n)], [int(stv[i]) for i in range(n)], DecodeStats._from(st)

    def autotune(self, d_in, in_off, in_len, d_out, out_off, out_cap, stream=None) -> dict:
        """Sweep the tunables on a sample batch (decode_batch's arguments) and keep
        the fastest setting in this decoder; returns the chosen setting."""
        n = len(in_off)
        A = C.c_uint64 * max(n, 1)
        t, e = _Tuning(), _Error()
        self._L.rrg_gpu_autotune(self._ctx, _ptr(d_in), A(*in_off), A(*in_len), _ptr(d_out), A(*out_off),
                                 A(*out_cap), n, _ptr(stream), C.byref(t), C.byref(e))
        _raise(e)
        return {f: getattr(t, f) for f, _ in _Tuning._fields_}

    # -------------------------------------------------------------- kernels
    def find_blocks(self, d_body, body_len: int, targets, limits):
        n = len(targets)
        A = C.c_uint64 * max(n, 1)
        t, lim, f = A(*targets), A(*limits), A()
        e = _Error()
        self._L.rrg_gpu_find_blocks(self._ctx, _ptr(d_body), body_len, t, lim, f, n, C.byref(e))
        _raise(e)
        return [None if f[i] == 0xFFFFFFFFFFFFFFFF else int(f[i]) for i in range(n)]

    def crc32(self, d_data, length: int) -> int:
        out = C.c_uint32()
        e = _Error()
        self._L.rrg_gpu_crc32(self._ctx, _ptr(d_data), length, C.byref(out), C.byref(e))
        _raise(e)
        return int(out.value)

    def resolve_markers(self, d_bytes, n_bytes, d_out_pos, d_prefix_offset, n_markers, d_tail, tail_len):
        e = _Error()
        self._L.rrg_gpu_resolve_markers(self._ctx, _ptr(d_bytes), n_bytes, _ptr(d_out_pos),
                                        _ptr(d_prefix_offset), n_markers, _ptr(d_tail), tail_len, C.byref(e))
        _raise(e)

    def decode_chunk(self, d_body, body_len: int, start_bit: int, end_bit_hint: int,
                     max_bytes: int = 64 << 20, max_markers: int = 16 << 20):
        """Speculative chunk decode -> (bytes, marker_pos list, marker_off list, actual_end_bit, final)."""
        import numpy as np
        nb, nm = C.c_size_t(max_bytes), C.c_size_t(max_markers)
        b = np.zeros(max_bytes, np.uint8)
        mp = np.zeros(max_markers, np.uint32)
        mo = np.zeros(max_markers, np.uint16)
        end, fin = C.c_uint64(), C.c_int32()
        e = _Error()
        self._L.rrg_gpu_decode_chunk(self._ctx, _ptr(d_body), body_len, start_bit, end_bit_hint,
                                     b.ctypes.data, C.byref(nb), mp.ctypes.data, mo.ctypes.data, C.byref(nm),
                                     C.byref(end), C.byref(fin), C.byref(e))
        _raise(e)
        return (b[:nb.value].tobytes(), mp[:nm.value].copy(), mo[:nm.value].copy(), int(end.value),
                bool(fin.value))

    # -------------------------------------------------------------- serving
    def submit(self, data, copy: bool = True) -> int:
        """Queue a decode request. With copy=False the library reads `data` in
        place; this decoder keeps a reference to it until poll returns it."""
        addr, n, keep = _host_buffer(data)
        e = _Error()
        fn = self._L.rrg_gpu_submit if copy else self._L.rrg_gpu_submit_nocopy
        rid = fn(self._ctx, addr, n, C.byref(e))
        if rid < 0:
            _raise(e)
        if not copy:
            with self._inflight_lock:
                if int(rid) in self._polled_early:  # already finished and polled
                    self._polled_early.discard(int(rid))
                else:
                    self._inflight[int(rid)] = (data, keep)
        del keep
        return int(rid)

    def _release(self, rid: int):
        with self._inflight_lock:
            if self._inflight.pop(rid, None) is None:
                self._polled_early.add(rid)

    def poll(self, timeout_ms: int = 0):
        """-> None, or (request_id, bytes | None, status, latency_ms)."""
        rid = C.c_int64()
        out = C.POINTER(C.c_uint8)()
        n = C.c_size_t()
        stv = C.c_int32()
        lat = C.c_double()
        e = _Error()
        r = self._L.rrg_gpu_poll(self._ctx, C.byref(rid), C.byref(out), C.byref(n), C.byref(stv), C.byref(lat),
                                 timeout_ms, C.byref(e))
        if r < 0:
            _raise(e)
        if r == 0:
            return None
        self._release(int(rid.value))
        self.last_poll_error = e.message.decode(errors="replace") if stv.value else ""
        data = None
        if out:
            data = C.string_at(out, n.value)
            self._L.rrg_gpu_free(out)
        return int(rid.value), data, int(stv.value), float(lat.value)

    def poll_raw(self, timeout_ms: int = 0):
        """Like poll, without copying the result: -> None, or (request_id,
        address, length, status, latency_ms); release the address with free()."""
        rid = C.c_int64()
        out = C.POINTER(C.c_uint8)()
        n = C.c_size_t()
        stv = C.c_int32()
        lat = C.c_double()
        e = _Error()
        r = self._L.rrg_gpu_poll(self._ctx, C.byref(rid), C.byref(out), C.byref(n), C.byref(stv), C.byref(lat),
                                 timeout_ms, C.byref(e))
        if r < 0:
            _raise(e)
        if r == 0:
            return None
        self._release(int(rid.value))
        addr = C.cast(out, C.c_void_p).value or 0
        return int(rid.value), addr, int(n.value), int(stv.value), float(lat.value)

    def free(self, addr: int):
        if addr:
            self._L.rrg_gpu_free(addr)

    def pending(self) -> int:
        return int(self._L.rrg_gpu_pending(self._ctx))

    def serve_start(self, engines: int = 0, max_ready: int = 0):
        """Start the serving loop (rrg_gpu_serve_start); submit() starts it with defaults."""
        e = _Error()
        self._L.rrg_gpu_serve_start(self._ctx, engines, max_ready, C.byref(e))
        _raise(e)

    def serve_stop(self):
        self._L.rrg_gpu_serve_stop(self._ctx)

    def serve_stats(self) -> dict:
        st = _ServeStats()
        self._L.rrg_gpu_serve_stats(self._ctx, C.byref(st))
        return {f: (round(getattr(st, f), 3) if f.endswith("_ms") else int(getattr(st, f)))
                for f, _ in _ServeStats._fields_}


def read_gz(path, sink, config: Config | None = None) -> DecodeStats:
    """Decode `path` and stream decompressed bytes to `sink` in stream order.

    Blocks until EOF or the first error (lib.rs:366-496)."""
    with Decoder(config) as d:
        return d.read_gz(path, sink)


def decompress(data, config: Config | None = None) -> bytes:
    with Decoder(config) as d:
        return d.decompress(data)


def crc32_noalloc(d_data, length: int, stream=None, lib: str | None = None) -> int:
    """CRC32 of a device buffer through rrg_gpu_crc32_noalloc: no device
    memory is allocated (fixed library scratch; at most 4 GiB per call; calls
    that overlap on the GPU race)."""
    out = C.c_uint32()
    e = _Error()
    load_library(lib).rrg_gpu_crc32_noalloc(_ptr(d_data), length, C.byref(out), _ptr(stream), C.byref(e))
    _raise(e)
    return int(out.value)


def crc32_combine(crc_a: int, crc_b: int, len_b: int, lib: str | None = None) -> int:
    """CRC32 of A||B from CRC32(A), CRC32(B) and |B| (rrg_crc32_combine)."""
    return int(load_library(lib).rrg_crc32_combine(crc_a, crc_b, len_b))


def kernel_launch_count(lib: str | None = None) -> int:
    return int(load_library(lib).rrg_gpu_kernel_launch_count())

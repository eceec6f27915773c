"""rusty_rapidgzip_b200 — gzip/DEFLATE decoding on one NVIDIA B200.

Drop-in for rusty_rapidgzip's streaming decode path
(``read_gz(path, Sender<Arc<Vec<u8>>>, Config)``): hand-written sm_100a CUDA
kernels (block finder, speculative marker inflate, marker resolution,
CRC32/ISIZE combine) behind the C ABI in include/rrg_gpu.h.
"""
from ._abi import (  # noqa: F401
    CapacityError,
    Config,
    DecodeStats,
    Decoder,
    DeflateError,
    DeviceError,
    GzipError,
    IoError,
    RrgError,
    SeekIndex,
    SinkClosed,
    decompress,
    kernel_launch_count,
    library_path,
    load_library,
    read_gz,
)

__all__ = [
    "CapacityError", "Config", "DecodeStats", "Decoder", "DeflateError", "DeviceError", "GzipError",
    "IoError", "RrgError", "SeekIndex", "SinkClosed", "decompress", "kernel_launch_count", "library_path",
    "load_library", "read_gz",
]

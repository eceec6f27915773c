/*
 * rrg_gpu.h — C ABI of the B200 gzip/DEFLATE decoder.
 *
 * This is the drop-in boundary for rusty_rapidgzip's streaming decode path:
 *
 *   pub fn read_gz(path, sink: Sender<Arc<Vec<u8>>>, config: Config)
 *       -> Result<DecodeStats, Error>                (crates/rusty-rapidgzip/src/lib.rs:366-370)
 *
 * Every entry point takes plain pointers and sizes. Device pointers are
 * ordinary CUDA global-memory addresses on the context's device; host
 * pointers are ordinary process memory. No entry point takes a torch or any
 * other framework type.
 *
 * Threading: a context runs one decode at a time (calls on one context must
 * not overlap); independent contexts are fully independent. The sink callback
 * runs on the calling thread, in stream order.
 */
#ifndef RRG_GPU_H
#define RRG_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. 1..9 mirror the reference's error enums:
 *   Error::Io                       (lib.rs:111-118)            -> RRG_ERR_IO
 *   GzipError::BadMagic             (gzip.rs:26-61)             -> RRG_ERR_BAD_MAGIC
 *   GzipError::UnsupportedMethod(u8)                            -> RRG_ERR_UNSUPPORTED_METHOD
 *   GzipError::ReservedFlags(u8)                                -> RRG_ERR_RESERVED_FLAGS
 *   GzipError::Truncated                                        -> RRG_ERR_TRUNCATED
 *   GzipError::CrcMismatch{..}                                  -> RRG_ERR_CRC_MISMATCH
 *   GzipError::IsizeMismatch{..}                                -> RRG_ERR_ISIZE_MISMATCH
 *   DeflateError::UnexpectedEof     (deflate/mod.rs:23-28)      -> RRG_ERR_DEFLATE_EOF
 *   DeflateError::Invalid(&str)                                 -> RRG_ERR_DEFLATE_INVALID
 * 20.. are conditions of the device path that the CPU reference cannot hit. */
enum rrg_status {
    RRG_OK = 0,
    RRG_ERR_IO = 1,
    RRG_ERR_BAD_MAGIC = 2,
    RRG_ERR_UNSUPPORTED_METHOD = 3,
    RRG_ERR_RESERVED_FLAGS = 4,
    RRG_ERR_TRUNCATED = 5,
    RRG_ERR_CRC_MISMATCH = 6,
    RRG_ERR_ISIZE_MISMATCH = 7,
    RRG_ERR_DEFLATE_EOF = 8,
    RRG_ERR_DEFLATE_INVALID = 9,
    RRG_ERR_CUDA = 20,             /* a CUDA runtime call failed (message holds the CUDA error string) */
    RRG_ERR_OUT_OF_MEMORY = 21,    /* device allocation or HBM budget exceeded */
    RRG_ERR_INVALID_ARGUMENT = 22, /* bad pointer/size/flag passed to the ABI */
    RRG_ERR_TIMEOUT = 23,          /* a bounded device-side wait gave up */
    RRG_ERR_CAPACITY = 24          /* caller-provided output buffer too small */
};

/* Error detail; fields follow GzipError::CrcMismatch / IsizeMismatch (gzip.rs:36-58). */
typedef struct rrg_error {
    int32_t code;          /* enum rrg_status */
    uint32_t member;       /* 0-based member index (CRC/ISIZE errors) */
    uint32_t expected;     /* trailer CRC32 or ISIZE; method/flag byte for codes 3/4 */
    uint32_t got_crc;      /* computed CRC32 (CRC errors) */
    uint64_t got;          /* computed uncompressed length (ISIZE errors) */
    uint64_t uncompressed; /* member's uncompressed bytes */
    uint64_t trailer_byte; /* byte offset of the member's trailer in the input file */
    char message[160];     /* human-readable; DeflateError::Invalid's text for code 9 */
} rrg_error;

/* Mirrors Config (lib.rs:50-100). */
typedef struct rrg_config {
    uint32_t num_threads;        /* host threads that read a regular file in rrg_gpu_read_gz, in parallel,
                                    into page-locked memory; 0 = one per core, at most 16
                                    (Config::num_threads: the host side's parallelism) */
    uint64_t chunk_size_bytes;   /* sink delivery granularity in compressed bytes; 0 = 4 MiB (Config::chunk_size_bytes) */
    int32_t verbose;             /* 0 = Verbosity::Off, 1 = Verbosity::On (stderr lines) */
    int32_t device;              /* CUDA device ordinal; -1 = current device */
    uint64_t gpu_chunk_bytes;    /* speculative sub-chunk size on the GPU; 0 = autotuned */
    uint64_t finder_tile_bits;   /* block-finder tile width in bits; 0 = autotuned */
    int32_t warps_per_stream;    /* 0 or 1 = one chunk per warp; -1 = one decoder per lane (32 chunks per warp) */
    int32_t boundary_mode;       /* 0 = test every bit offset of the body and keep verified block starts
                                    >= gpu_chunk_bytes apart; 1 = one search per target as
                                    find_next_dynamic_block does (block_finder.rs:109) */
    uint64_t hbm_budget_bytes;   /* serving admission budget; 0 = 120 GB */
    int32_t host_pipeline;       /* rrg_gpu_decode_host/read_gz: 0 = decode a large single-member stream
                                    in waves with the copy to the host overlapped (falls back to the
                                    checked path on any irregularity), up to 4 waves; N >= 2 = N waves
                                    where every sub-chunk keeps at least 8 KiB; -1 = always the
                                    checked path */
    int32_t batch_plan;          /* rrg_gpu_decode_batch, and rrg_gpu_decode_device for member streams of
                                    16 MiB or more: 0 = the member route planned and checked on the device
                                    (sub-chunk starts, item list, anchored chain, resolve, CRC) as one
                                    captured graph, with the jobs it cannot finish decoded on the checked
                                    path; -1 = always the host-planned checked path */
} rrg_config;

/* Mirrors DecodeStats (lib.rs:103-108), plus device-path counters. */
typedef struct rrg_stats {
    uint64_t compressed_bytes;
    uint64_t uncompressed_bytes;
    uint64_t chunks_decoded;       /* sink pieces delivered */
    uint64_t speculation_failures; /* chunks re-decoded because a guessed start was false */
    uint64_t gpu_chunks;           /* speculative sub-chunks decoded on the device */
    uint64_t markers;              /* unresolved back-reference cells resolved by the marker kernel */
    uint64_t members;              /* gzip members verified */
    uint64_t kernel_launches;      /* kernels launched by this call */
    double finder_ms, inflate_ms, resolve_ms, crc_ms, h2d_ms, d2h_ms, total_ms;
    uint64_t graph_launches;       /* captured decode graphs launched by this call (BGZF route, device-planned batch) */
    uint64_t pipeline_waves;       /* waves of the pipelined host path (0: not taken) */
    uint64_t pipeline_fallbacks;   /* 1 when the pipelined path handed the rest to the checked path */
} rrg_stats;

/* Sink: called in stream order with consecutive pieces of decompressed output.
 * The pointer is valid only for the duration of the call. Return 0 to continue,
 * non-zero to close the sink (decoding stops early and the call returns RRG_OK,
 * like a disconnected Sender in pipeline.rs:1028-1030). */
typedef int (*rrg_sink_fn)(void* user, const uint8_t* data, size_t len);

/* Destination provider (Config::recycle_rx, lib.rs:58-69: the reference's
 * decode workers pull warm output buffers with try_recv, pipeline.rs:603-607).
 * Called before a piece of output leaves the device, with the piece's size:
 * returns a buffer of at least `want` bytes (its capacity in *cap), into which
 * the piece is copied straight from the device and which the following sink
 * call receives as `data`. The consumer owns it from then on and may hand it
 * back through later calls (the recycle_tx side). NULL, or a capacity below
 * `want`, makes the library use its own staging for that piece. Page-locked
 * buffers (cudaMallocHost, cudaHostRegister) are filled at the link's rate;
 * pageable ones are staged by the CUDA runtime. Called on the decoding thread,
 * in stream order, at most a few pieces ahead of the sink. */
typedef uint8_t* (*rrg_buffer_fn)(void* user, size_t want, size_t* cap);

typedef struct rrg_ctx rrg_ctx;

/* Context lifetime. Allocates the device workspace lazily on first use.
 * Replaces constructing Config + the worker pools (pipeline.rs:580-625). */
rrg_ctx* rrg_gpu_create(const rrg_config* cfg, rrg_error* err);
void rrg_gpu_destroy(rrg_ctx* ctx);

/* Drop-in for read_gz (lib.rs:366-496): open `path`, route BGZF vs plain member
 * decode (lib.rs:463), decode on the GPU, verify CRC32/ISIZE per member and
 * stream the bytes to `sink` in order. A zero-byte file is RRG_ERR_TRUNCATED. */
int rrg_gpu_read_gz(rrg_ctx* ctx, const char* path, rrg_sink_fn sink, void* user,
                    rrg_stats* stats, rrg_error* err);

/* Compressed input for rrg_gpu_read_stream: copy up to `cap` bytes into `buf`
 * and return the count, 0 at the end of the input, or a negative value on a
 * read error (the call then returns RRG_ERR_IO). */
typedef int64_t (*rrg_read_fn)(void* user, uint8_t* buf, size_t cap);

/* Non-seekable input (pipe, stdin, socket): replaces the streaming routes of
 * read_gz (lib.rs:378-431; streaming.rs:389-614 read_gz_streaming_parallel).
 * The stream is read forward and decoded in stripes of about `stripe_bytes`
 * compressed bytes (0: 256 MiB) plus a lookahead; only the open member's last
 * 32 KiB of output, its running CRC32/length and the unread input carry over
 * between stripes, so memory is bounded by a few stripes. Output reaches
 * `sink` in order. rrg_gpu_read_gz takes this route for paths that are not
 * regular files. Errors, stats and the sink contract are those of
 * rrg_gpu_read_gz; stats->compressed_bytes counts the bytes read. `read_fn`
 * is called from a thread of the library, one call at a time, so that the
 * next stripe is read while the GPU decodes the current one; when the call
 * returns early (an error, a closed sink) it first waits for a read in flight. */
int rrg_gpu_read_stream(rrg_ctx* ctx, rrg_read_fn read_fn, void* read_user, rrg_sink_fn sink, void* user,
                        uint64_t stripe_bytes, rrg_stats* stats, rrg_error* err);

/* Seek index of a member stream (the reference has none; README.md:45 lists
 * random access as absent). rrg_gpu_index_build decodes the file once (CRC32
 * and ISIZE checked) and keeps block starts at least `spacing` output bytes
 * apart (0: 4 MiB), each with the 32 KiB of output before it. BGZF files are
 * refused (RRG_ERR_INVALID_ARGUMENT): each member is already a seek point. */
typedef struct rrg_index rrg_index;
int rrg_gpu_index_build(rrg_ctx* ctx, const uint8_t* data, size_t len, uint64_t spacing, rrg_index** out,
                        rrg_stats* stats, rrg_error* err);
/* Output bytes [off, off + n) of the file the index was built on (`data`,
 * `len`: the same file in host memory) into host `dst`. Decodes from the
 * checkpoint at or before `off` to the first at or past `off + n`, in
 * parallel like any stripe. Members are decoded only in part, so CRC32/ISIZE
 * are not checked here. */
int rrg_gpu_read_range(rrg_ctx* ctx, const uint8_t* data, size_t len, const rrg_index* idx, uint64_t off,
                       uint64_t n, uint8_t* dst, rrg_error* err);
uint64_t rrg_index_total_out(const rrg_index* idx);  /* decompressed size of the file */
size_t rrg_index_count(const rrg_index* idx);        /* checkpoints */
/* Checkpoint k: its output offset and the file-absolute bit where its block starts. */
int rrg_index_point(const rrg_index* idx, size_t k, uint64_t* out_off, uint64_t* in_bit);
/* Byte image of the index: returns the size needed; writes it when `cap` suffices. */
size_t rrg_index_serialize(const rrg_index* idx, uint8_t* buf, size_t cap);
rrg_index* rrg_index_deserialize(const uint8_t* buf, size_t n, rrg_error* err);
void rrg_index_free(rrg_index* idx);

/* Same as rrg_gpu_read_gz for a gzip file already in host memory (`data` may be
 * pageable or pinned). Replaces read_gz's mmap'd InputBytes (pipeline.rs:47-50). */
int rrg_gpu_decode_host(rrg_ctx* ctx, const uint8_t* data, size_t len, rrg_sink_fn sink,
                        void* user, rrg_stats* stats, rrg_error* err);

/* One range of a single-member stream decoded on one of several GPUs (the
 * reference's tail chain, pipeline.rs:1045-1078, spread over ranks: ranges
 * decode in parallel and the only exchange is one 32 KiB window map per range).
 * Phase 1, rrg_gpu_split_begin: `data` is the whole file in host memory and
 * `body_off` its first member's deflate body. The range starts at the first
 * dynamic block at or after body bit `start_target` (exactly there with
 * RRG_SPLIT_EXACT_START; 0 is the body's start) and stops at the first block
 * edge at or after the first dynamic block at or after `stop_target` (or at the
 * member's end for ~0). It is decoded and its output laid out on the device;
 * `end_map` (32768 entries) receives the range's last 32 KiB as a map of its
 * first 32 KiB: a value below 0x100 is that byte, 0x8000|j is byte j of the
 * window before the range, 0x4000 lies before the stream. `info` gets the exact
 * start and end bits (a range is valid only if it starts where the previous
 * non-empty one ended), its output length and the member trailer when it lies
 * in this range. With no dynamic block after `start_target` the range is empty
 * (start and end bits ~0, no output, identity map): the previous range, whose
 * stop search finds the same nothing, decodes to the member's end.
 * A range in which a member ends before its last block is refused
 * (RRG_ERR_INVALID_ARGUMENT): split decoding takes one-member streams.
 * Phase 2, rrg_gpu_split_finish: given the 32 KiB of output before the range
 * (`window_len` < 32768 only near the stream's start; 0 for the first range),
 * resolves the range, streams its bytes to `sink` and returns their CRC32 and
 * length, which the ranks combine (crc32_combine) and compare with the trailer.
 * One split range per context at a time. */
#define RRG_SPLIT_EXACT_START 1u
/* CRC32 of A||B from CRC32(A), CRC32(B) and |B| (crc32fast's combine, used by
 * the reference's output stage, pipeline.rs:885-916), for joining the ranges'
 * CRC32s. Host only. */
uint32_t rrg_crc32_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b);
typedef struct rrg_split_info {
    uint64_t start_bit, end_bit; /* body-relative */
    uint64_t out_len;
    uint32_t has_trailer, crc, isize, pad;
    uint64_t trailer_byte;       /* file offset of the trailer (when has_trailer) */
} rrg_split_info;
int rrg_gpu_split_begin(rrg_ctx* ctx, const uint8_t* data, size_t len, uint64_t body_off,
                        uint64_t start_target, uint64_t stop_target, uint32_t flags,
                        uint16_t* end_map, rrg_split_info* info, rrg_error* err);
int rrg_gpu_split_finish(rrg_ctx* ctx, const uint8_t* window, size_t window_len, rrg_sink_fn sink,
                         void* user, uint32_t* crc_out, uint64_t* len_out, rrg_error* err);

/* rrg_gpu_decode_host and rrg_gpu_read_gz with a destination provider (read_gz
 * with Config::recycle_rx/recycle_tx set, lib.rs:58-69): each piece of output
 * is copied from the device into a buffer `get` returns, and `sink` receives
 * that buffer. `user` is passed to both. */
int rrg_gpu_decode_host_into(rrg_ctx* ctx, const uint8_t* data, size_t len, rrg_buffer_fn get,
                             rrg_sink_fn sink, void* user, rrg_stats* stats, rrg_error* err);
int rrg_gpu_read_gz_into(rrg_ctx* ctx, const char* path, rrg_buffer_fn get, rrg_sink_fn sink,
                         void* user, rrg_stats* stats, rrg_error* err);

/* Device-resident decode: `d_in` (device, `len` bytes) is a whole gzip file;
 * the decompressed stream is written contiguously to `d_out` (device, capacity
 * `out_cap`). Returns RRG_ERR_CAPACITY with *out_len = the required size when
 * `out_cap` is too small. All work is ordered on `stream` (a cudaStream_t, or
 * NULL for the context's own stream); the call returns after the stream's work
 * for this decode has completed. Covers parallel_decode_member (pipeline.rs:468)
 * and parallel_decode_bgzf (pipeline.rs:1357) without any host round trip of
 * the payload. */
int rrg_gpu_decode_device(rrg_ctx* ctx, const uint8_t* d_in, size_t len, uint8_t* d_out,
                          size_t out_cap, size_t* out_len, void* stream, rrg_stats* stats,
                          rrg_error* err);

/* Batched decode of `n` independent gzip files already on the device (the
 * per-file work of read_gz, lib.rs:366-496, for many files at once; BGZF files
 * as in pipeline.rs:1357-1636). Headers are parsed on the device. BGZF files
 * take the device member walk and one persistent decode per file (a captured
 * CUDA graph). All other files share one boundary scan, one persistent inflate
 * launch over a device work queue, one resolve and one CRC pass; a file small
 * enough for one sub-chunk decodes straight to its output bytes. Files are
 * processed in waves whose reserved scratch fits rrg_config.hbm_budget_bytes
 * (and the free device memory). Input i is d_in[in_off[i] .. +in_len[i]); its
 * output goes to d_out[out_off[i] ..] with room for out_cap[i] bytes; out_len[i]
 * and status[i] (enum rrg_status) are written to host arrays; RRG_ERR_CAPACITY
 * leaves the size needed in out_len[i]. in_off/in_len/out_off/out_cap are host
 * arrays. Returns the first failing status (RRG_OK if all passed). */
int rrg_gpu_decode_batch(rrg_ctx* ctx, const uint8_t* d_in, const uint64_t* in_off,
                         const uint64_t* in_len, uint8_t* d_out, const uint64_t* out_off,
                         const uint64_t* out_cap, uint64_t* out_len, int32_t* status, size_t n,
                         void* stream, rrg_stats* stats, rrg_error* err);

/* Settings chosen by rrg_gpu_autotune. */
typedef struct rrg_tuning {
    uint64_t gpu_chunk_bytes;   /* speculative sub-chunk size; 0 = one wave of resident decoders */
    int32_t boundary_mode;      /* 0 = boundary scan of every bit offset, 1 = one search per target */
    int32_t warps_per_member;   /* BGZF: 1 = one warp decodes a whole member; 2-4 = sub-chunks per member */
    uint64_t finder_tile_bits;  /* boundary-scan tile width (8192, 16384 or 32768 bits) */
    double best_ms;             /* batch time on the sample with the chosen settings */
    double default_ms;          /* batch time on the sample with the settings before tuning */
    uint32_t trials;            /* settings timed */
} rrg_tuning;

/* Autotuner. Decodes the sample batch (same arguments as rrg_gpu_decode_batch)
 * under a coordinate sweep of sub-chunk size, boundary search and scan tile
 * width, and warps per BGZF member, three runs each, and keeps the fastest
 * setting in the context for later calls. The reference has no autotuner
 * (its chunk size is a fixed Config field, lib.rs:50-100). */
int rrg_gpu_autotune(rrg_ctx* ctx, const uint8_t* d_in, const uint64_t* in_off, const uint64_t* in_len,
                     uint8_t* d_out, const uint64_t* out_off, const uint64_t* out_cap, size_t n, void* stream,
                     rrg_tuning* result, rrg_error* err);

/* ---- kernel-level entry points (each replaces one reference function) ---- */

/* Block finder over a raw DEFLATE body on the device. For each target bit
 * offset targets[i] (host array), writes to found[i] (host array) the first
 * bit offset >= targets[i] and < limits[i] that find_next_dynamic_block
 * (deflate/block_finder.rs:109-141) would return with until_bit = limits[i],
 * or UINT64_MAX if none. */
int rrg_gpu_find_blocks(rrg_ctx* ctx, const uint8_t* d_body, size_t body_len,
                        const uint64_t* targets, const uint64_t* limits, uint64_t* found,
                        size_t n, rrg_error* err);

/* CRC32 (IEEE, as crc32fast::hash) of a device buffer; replaces the crc32fast
 * pieces + combine of pipeline.rs:712-732 and :885-916. */
int rrg_gpu_crc32(rrg_ctx* ctx, const uint8_t* d_data, size_t len, uint32_t* crc_out,
                  rrg_error* err);

/* Marker resolution (deflate/speculative.rs:175-213): for each marker
 * (out_pos[i], prefix_offset[i]) set d_bytes[out_pos[i]] =
 * d_tail[tail_len - 1 - prefix_offset[i]]. All arrays are on the device. Fails
 * with RRG_ERR_DEFLATE_INVALID if any prefix_offset >= tail_len. */
int rrg_gpu_resolve_markers(rrg_ctx* ctx, uint8_t* d_bytes, size_t n_bytes,
                            const uint32_t* d_out_pos, const uint16_t* d_prefix_offset,
                            size_t n_markers, const uint8_t* d_tail, size_t tail_len,
                            rrg_error* err);

/* Speculative decode of one chunk of a raw DEFLATE body on the device, with
 * the output contract of decode_one_chunk + decode_until_u16 (pipeline.rs:1080-1185,
 * deflate/fast_inflate.rs:1794-1888): host receives the chunk's bytes (marker
 * bytes = 0), its markers sorted by out_pos, and the bit offset where decoding
 * stopped. `*n_bytes`/`*n_markers` are in: capacity, out: count. */
int rrg_gpu_decode_chunk(rrg_ctx* ctx, const uint8_t* d_body, size_t body_len,
                         uint64_t start_bit, uint64_t end_bit_hint, uint8_t* bytes,
                         size_t* n_bytes, uint32_t* marker_pos, uint16_t* marker_off,
                         size_t* n_markers, uint64_t* actual_end_bit, int32_t* final_block,
                         rrg_error* err);

/* ---- serving loop (continuous batching under an HBM budget) ---- */

/* The reference has no serving loop; this is the request path a service puts
 * on top of read_gz (lib.rs:366-496). Engines are sub-contexts, each with its
 * own stream, device scratch (resident across requests) and host thread. An
 * idle engine takes the oldest waiting requests whose device bytes (input,
 * output from the trailer's ISIZE, decode scratch) fit the HBM budget
 * (rrg_config.hbm_budget_bytes) next to the requests already admitted, and
 * decodes them as one batch (rrg_gpu_decode_batch's path). Requests submitted
 * while other batches run join the next batch an engine takes, so several
 * batches overlap on the device. Finished requests wait in a bounded
 * completion queue; engines take no new work while it is full. */

/* Counters of the serving loop. */
typedef struct rrg_serve_stats {
    uint64_t submitted, completed, batches;
    uint64_t max_batch;          /* most requests decoded together in one batch */
    uint64_t engines_busy, max_engines_busy;
    uint64_t in_use_bytes, peak_in_use_bytes, budget_bytes;
    uint64_t waiting;            /* submitted, not yet admitted */
    uint64_t bytes_out;          /* decompressed bytes finished */
    double h2d_ms, decode_ms, d2h_ms;  /* engine time copying requests in, decoding, copying results out (summed over engines) */
} rrg_serve_stats;

/* Start the serving loop with `engines` engines (0 = 2) and a completion queue
 * of `max_ready` entries (0 = 64). rrg_gpu_submit starts it with the defaults
 * if it is not running. */
int rrg_gpu_serve_start(rrg_ctx* ctx, uint32_t engines, uint32_t max_ready, rrg_error* err);

/* Stop the engines (waits for the batches on the device); unpolled results are
 * dropped. rrg_gpu_destroy calls it. */
void rrg_gpu_serve_stop(rrg_ctx* ctx);

int rrg_gpu_serve_stats(rrg_ctx* ctx, rrg_serve_stats* out);

/* Submit a whole gzip file held in host memory (copied at submit). Returns a
 * request id >= 0, or -1 on error. */
int64_t rrg_gpu_submit(rrg_ctx* ctx, const uint8_t* data, size_t len, rrg_error* err);

/* Same, without the copy: the engine reads `data` in place, so the caller
 * keeps it valid and unchanged until rrg_gpu_poll has returned this request.
 * For servers whose request bodies already sit in memory they own: the copy
 * costs more host time than the decode of a large request. */
int64_t rrg_gpu_submit_nocopy(rrg_ctx* ctx, const uint8_t* data, size_t len, rrg_error* err);

/* Collect one finished request, waiting up to `timeout_ms`. Returns 1 and
 * fills the outputs, 0 if none finished in time, or a negative rrg_status on
 * failure. `*out` is a malloc'd buffer the caller frees with rrg_gpu_free;
 * `*latency_ms` is submit-to-finish wall time. A request that failed returns 1
 * with *status != RRG_OK and *out == NULL. */
int rrg_gpu_poll(rrg_ctx* ctx, int64_t* request_id, uint8_t** out, size_t* out_len,
                 int32_t* status, double* latency_ms, int32_t timeout_ms, rrg_error* err);

/* Number of requests submitted but not yet returned by rrg_gpu_poll. */
int64_t rrg_gpu_pending(rrg_ctx* ctx);

/* CRC32 (IEEE, as crc32fast::hash) of `len` bytes at device address `d_data`,
 * written to the host word *crc_out, for callers that cannot let a library
 * allocate device memory (an application that owns the GPU's memory through
 * its own pool allocator, where a hidden cudaMalloc can fail and a cudaFree
 * synchronises the device; a latency-critical path that must not stall on
 * allocation). No counterpart in the reference: it has no device memory.
 * It calls no cudaMalloc/cudaFree and needs no context. All scratch lives in
 * one fixed device array of about 336 KB inside this library, which every GPU
 * that loads the library holds until the process exits; that bounds `len` to
 * 4 GiB (4294967296 bytes), and longer inputs fail with RRG_ERR_CAPACITY. The
 * first call on a device looks up that array and loads the CRC tables; make
 * it before any stream capture. A new CUDA context on the device (after
 * cudaDeviceReset) gets a fresh copy of the array, and the next call there
 * repeats that set-up. Work is ordered on `stream` (a cudaStream_t,
 * or NULL for the legacy default stream) and the call returns once the result
 * is on the host. Every call shares the same array, so calls that overlap on
 * the GPU (from several host threads or streams) race and must be serialised
 * by the caller. */
int rrg_gpu_crc32_noalloc(const uint8_t* d_data, size_t len, uint32_t* crc_out, void* stream,
                          rrg_error* err);

/* Release a result buffer returned by rrg_gpu_poll. Buffers of 1 MiB and more
 * return to the library's pool (at most 32 GiB held idle) and are reused for
 * later results, whose pages are then already mapped. */
void rrg_gpu_free(void* p);

/* Library version string and the number of kernels this library has launched
 * in this process (for launch accounting). */
const char* rrg_gpu_version(void);
uint64_t rrg_gpu_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* RRG_GPU_H */

/*
 * rrg_oracle.h — CPU restatement of rusty_rapidgzip's gzip/DEFLATE decode path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker for the CUDA
 * decoder and the timed CPU baseline. It is loaded by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg and reference arm,
 * and by nothing on the product path.
 *
 * Each function names the reference function it restates (paths relative to
 * the rusty_rapidgzip repository; rrg/ = crates/rusty-rapidgzip/).
 * Status codes are the enum rrg_status values of include/rrg_gpu.h.
 */
#ifndef RRG_ORACLE_H
#define RRG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_error {
    int32_t code;
    uint32_t member;
    uint32_t expected;
    uint32_t got_crc;
    uint64_t got;
    uint64_t uncompressed;
    uint64_t trailer_byte;
    char message[160];
} orc_error; /* same layout as rrg_error */

typedef struct orc_stats {
    uint64_t compressed_bytes;
    uint64_t uncompressed_bytes;
    uint64_t chunks_decoded;
    uint64_t speculation_failures;
    uint64_t n_chunks;
    uint64_t n_markers;
} orc_stats;

typedef int (*orc_sink_fn)(void* user, const uint8_t* data, size_t len);

/* crc32fast::Hasher::update semantics: crc32(crc, data) with the standard
 * pre/post inversion; orc_crc32(0, p, n) == crc32fast::hash(p[..n]). */
uint32_t orc_crc32(uint32_t crc, const uint8_t* data, size_t len);
/* crc32fast::Hasher::combine: CRC of A||B from crc(A), crc(B), len(B). */
uint32_t orc_crc32_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b);

/* gzip.rs:252-300 parse_header. Returns status; *hdr_len on success. */
int orc_parse_header(const uint8_t* in, size_t len, size_t* hdr_len);
/* gzip.rs:311-351 parse_bgzf_block_size. Returns BSIZE+1, or -1 for None. */
int64_t orc_bgzf_block_size(const uint8_t* in, size_t len);

/* block_finder.rs:109-141 find_next_dynamic_block. Returns 1 and *found when
 * a block is found, 0 otherwise. */
int orc_find_next_dynamic_block(const uint8_t* data, size_t len, uint64_t from_bit,
                                uint64_t until_bit, uint64_t* found);
/* block_finder.rs:175-189 verify_candidate (strict header + 64-symbol trial). */
int orc_verify_candidate(const uint8_t* data, size_t len, uint64_t pos);

/* Raw DEFLATE decode of a whole stream with a real window (safe_inflate.rs:617-645
 * semantics). *out is malloc'd (free with orc_free). *end_bit = bits consumed. */
int orc_inflate_raw(const uint8_t* in, size_t len, uint8_t** out, size_t* out_len,
                    uint64_t* end_bit, orc_error* err);

/* gzip.rs:65-77 decode_all: every member serially, CRC32/ISIZE checked. */
int orc_decode_all(const uint8_t* in, size_t len, uint8_t** out, size_t* out_len,
                   orc_error* err);

/* A member transition inside a chunk (pipeline.rs:419-428). */
typedef struct orc_member_boundary {
    uint64_t byte_offset_in_chunk;
    uint32_t crc_expected;
    uint32_t isize_expected;
    uint64_t trailer_input_byte; /* relative to the start of `body` */
} orc_member_boundary;

/* Output of one speculative chunk decode (SpeculativeChunk + WorkResult). */
typedef struct orc_chunk {
    uint8_t* bytes;
    uint64_t n_bytes;
    uint32_t* marker_pos;    /* Marker::out_pos, ascending */
    uint16_t* marker_off;    /* Marker::prefix_offset */
    uint64_t n_markers;
    orc_member_boundary* mbs;
    uint64_t n_mbs;
    uint64_t start_bit;
    uint64_t end_bit_hint;
    uint64_t actual_end_bit;
    int32_t final_block;
    int32_t status;
} orc_chunk;

/* pipeline.rs:1080-1185 decode_one_chunk with the first member decoded by
 * fast_inflate.rs:1794-1888 decode_until_u16 (u16 marker cells, hand-off to
 * byte decoding once the live window is marker-free) and later members by the
 * u8 kernel with a fresh window. Fills *out; release with orc_chunk_free. */
int orc_decode_chunk(const uint8_t* body, size_t body_len, uint64_t start_bit,
                     uint64_t end_bit_hint, orc_chunk* out, orc_error* err);
void orc_chunk_free(orc_chunk* c);

/* speculative.rs:175-213 resolve_markers. */
int orc_resolve_markers(orc_chunk* c, const uint8_t* prev_tail, size_t tail_len, orc_error* err);

/* pipeline.rs:1045-1078 build_prev_tail_fast. `new_tail` must hold 32768
 * bytes; returns the new tail length. */
size_t orc_build_prev_tail(const orc_chunk* c, const uint8_t* prev_tail, size_t prev_len,
                           uint8_t* new_tail);

/* lib.rs:366-496 read_gz over an in-memory file: BGZF route
 * (pipeline.rs:1357-1636) or the speculative member pipeline
 * (pipeline.rs:468-1041; serial_decode_member :1211 when num_threads == 1).
 * num_threads 0 = all online CPUs; chunk_size 0 = 4 MiB. */
int orc_read_gz_buffer(const uint8_t* file, size_t len, uint32_t num_threads,
                       uint64_t chunk_size, orc_sink_fn sink, void* user, orc_stats* stats,
                       orc_error* err);

/* Convenience: decode into one malloc'd buffer through orc_read_gz_buffer. */
int orc_read_gz_to_buffer(const uint8_t* file, size_t len, uint32_t num_threads,
                          uint64_t chunk_size, uint8_t** out, size_t* out_len,
                          orc_stats* stats, orc_error* err);

void orc_free(void* p);

#ifdef __cplusplus
}
#endif

#endif

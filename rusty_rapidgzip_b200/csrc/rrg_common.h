// rrg_common.h — records shared by the host orchestration and the kernels.
#pragma once
#include <stdint.h>

namespace rrg {

// Kernel status values: 0 and 1..9 are enum rrg_status (include/rrg_gpu.h);
// the DS_* values above 100 are device-internal conditions the host resolves.
enum : int32_t {
    DS_OK = 0,
    DS_BAD_MAGIC = 2,
    DS_METHOD = 3,
    DS_FLAGS = 4,
    DS_TRUNCATED = 5,
    DS_CRC = 6,
    DS_ISIZE = 7,
    DS_EOF = 8,
    DS_INVALID = 9,
    DS_OVERFLOW = 101,  // output slot too small; n_cells holds the size needed
    DS_PENDING = 102,   // item not processed (work queue gave up)
};

// Message codes for DS_INVALID (text table in the host code).
enum : int32_t {
    MSG_NONE = 0,
    MSG_RESERVED_BTYPE,
    MSG_STORED_NLEN,
    MSG_LITLEN_RANGE,
    MSG_DIST_RANGE,
    MSG_NO_CODE,
    MSG_OVERSUB,
    MSG_HLIT_HDIST,
    MSG_CODE16_FIRST,
    MSG_CODE16_OVER,
    MSG_CODE17_OVER,
    MSG_CODE18_OVER,
    MSG_BAD_CL_SYM,
    MSG_EOB_ZERO,
    MSG_DIST_FAR,
    MSG_MARKER_WINDOW,
    MSG_COUNT
};

// One unit of inflate work: a bit range of a DEFLATE body.
struct ChunkItem {
    uint64_t in_off;     // byte offset of the body in the kernel's input buffer
    uint64_t in_len;     // body bytes readable from in_off
    uint64_t start_bit;  // relative to the body start
    uint64_t end_hint;   // stop at the first block boundary >= this (UINT64_MAX: until BFINAL)
    uint64_t out_off;    // first output cell in the slot arena
    uint64_t out_cap;    // output cells available
    uint32_t flags;      // ITEM_* below
    uint32_t id;         // caller's index, echoed into member-boundary records
};
enum : uint32_t {
    ITEM_MARKERS = 1u,      // the first member may reference bytes before the chunk (u16 markers)
    ITEM_ONE_MEMBER = 2u,   // input is exactly one gzip member with its header (batch mode)
    ITEM_STORED_START = 4u, // host only: the start is a stored-block header byte of zeros
    ITEM_EMPTY_STORED = 8u, // host only: ... of an empty stored block (LEN = 0)
    ITEM_SKIP = 16u,        // no work: an unused sub-chunk of a device-planned job (empty result)
};

struct ChunkResult {
    uint64_t n_cells;         // output cells produced (needed, when DS_OVERFLOW)
    uint64_t actual_end_bit;  // bit offset (body-relative) where decoding stopped
    int32_t status;
    int32_t msg;
    int32_t final_block;      // reached EOF after the last member's trailer
    uint32_t n_members;       // member trailers passed inside this item
    uint64_t markers;         // marker cells emitted
    uint64_t err_bit;         // body-relative bit position of the failure
};

// Member trailer met inside an item (pipeline.rs:419-428 MemberBoundary).
struct MemberRec {
    uint32_t item;        // ChunkItem::id
    uint32_t seq;         // order within the item
    uint64_t cell_off;    // cells of the item before this member's end
    uint32_t crc;         // trailer CRC32
    uint32_t isize;       // trailer ISIZE
    uint64_t trailer_byte;  // body-relative byte offset of the trailer
};

// Output tile for the resolve kernel: cells [cell_begin, cell_end) of chunk `chunk`.
struct ResolveChunk {
    uint64_t out_start;   // global output byte of the chunk's first cell
    uint64_t slot_off;    // first cell in the slot arena
    uint64_t n_cells;
    uint64_t member_start;  // global output byte where the chunk's first member began
    uint64_t job_out;       // first output byte of the chunk's job: bytes in [member_start, job_out)
                            // were written by earlier calls (a stripe's prefix) and are read from the output
};

// A CRC piece: output bytes [start, start+len) all belonging to one member.
struct CrcPiece {
    uint64_t start;
    uint64_t len;
};

constexpr uint32_t MARKER16 = 0x8000u;
constexpr uint32_t WINDOW = 32768u;

}  // namespace rrg

// rrg_kernels.cuh — device code of the B200 gzip/DEFLATE decoder.
//
// Kernels (each names the reference function whose result it reproduces;
// paths are relative to the rusty_rapidgzip repository, rrg/ = crates/rusty-rapidgzip/):
//   k_find_blocks  — rrg/src/deflate/block_finder.rs:109-141 find_next_dynamic_block
//   k_inflate      — rrg/src/pipeline.rs:1080-1185 decode_one_chunk with
//                    rrg/src/deflate/fast_inflate.rs:1794-2234 (u16 marker cells), or a
//                    whole member into final bytes (gzip.rs:197-249 decode_one_indexed_fast)
//   k_win_maps / k_win_supers / k_win_bases / k_win_expand / k_res_tails / k_res_heads —
//                    rrg/src/deflate/speculative.rs:175-213
//                    resolve_markers together with the tail chain of rrg/src/pipeline.rs:1045-1078,
//                    fused with the chunk compaction
//   k_crc_pieces / k_crc_members — crc32fast hashing + combine (rrg/src/pipeline.rs:712-732, :885-916)
//
// This header is compiled by nvcc for sm_100a (rrg_kernels.cu) and, for the
// CPU test build only, by g++ against a warp-emulation shim.
#pragma once
#include "rrg_common.h"

#ifndef FULLMASK
#define FULLMASK 0xffffffffu
#endif

#if defined(__CUDA_ARCH__)
#define RRG_PREFETCH_L1(p) asm volatile("prefetch.global.L1 [%0];" ::"l"(p))
#else
#define RRG_PREFETCH_L1(p) ((void)(p))
#endif

#ifdef RRG_EMU
#define RRG_DYN_SMEM(name) unsigned char* name = emu::dyn_smem()
#else
#define RRG_DYN_SMEM(name) extern __shared__ __align__(16) unsigned char name[]
#endif

namespace rrg {

// ---------------------------------------------------------------- constants
__constant__ uint16_t c_len_base[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                         31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint8_t c_len_extra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                        2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint16_t c_dist_base[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                         33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                         1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
__constant__ uint8_t c_dist_extra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                         6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
__constant__ uint8_t c_cl_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
// x^(2^k) mod P (reflected CRC-32), k = 0..66; uploaded by the host.
__constant__ uint32_t c_x2k[67];

constexpr int LUT_BITS = 10;
constexpr int LUT_SIZE = 1 << LUT_BITS;
constexpr int PRE_BITS = 7;
constexpr int DIST_BITS = 8;  // inflate's distance LUT; longer codes (~1% of distances) take long_decode
constexpr int DIST_SIZE = 1 << DIST_BITS;
constexpr int NB = 32;  // symbols per decode batch
constexpr int MAT_GROUPS = 4;  // 32-cell groups whose loads a materialisation pass issues together

// ------------------------------------------------------- warp helpers
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
    return v;
}
__device__ __forceinline__ uint64_t bcast64(uint64_t v) {
    uint32_t lo = __shfl_sync(FULLMASK, (uint32_t)v, 0);
    uint32_t hi = __shfl_sync(FULLMASK, (uint32_t)(v >> 32), 0);
    return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ int32_t bcast32(int32_t v) { return __shfl_sync(FULLMASK, v, 0); }

// ------------------------------------------------------- bounded byte source
// Bytes [lo, hi) relative to a 4-byte-aligned base are readable. Whole words
// inside the range use one aligned load; edge words are assembled from bytes
// so no access leaves the caller's buffer.
struct Src {
    const uint8_t* base;
    uint64_t lo, hi;
};
__device__ __forceinline__ Src make_src(const uint8_t* p, uint64_t len) {
    Src s;
    uintptr_t a = (uintptr_t)p;
    s.base = (const uint8_t*)(a & ~(uintptr_t)3);
    s.lo = a & 3;
    s.hi = s.lo + len;
    return s;
}
__device__ __forceinline__ uint32_t src_word(const Src& s, uint64_t w) {
    uint64_t b = w * 4;
    if (b >= s.lo && b + 4 <= s.hi) return __ldg((const uint32_t*)(s.base + b));
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) {
        uint64_t p = b + k;
        if (p >= s.lo && p < s.hi) v |= (uint32_t)__ldg(s.base + p) << (8 * k);
    }
    return v;
}
__device__ __forceinline__ uint32_t src_byte(const Src& s, uint64_t rel) {  // rel: from s.lo
    uint64_t p = s.lo + rel;
    return p < s.hi ? (uint32_t)__ldg(s.base + p) : 0u;
}

// ------------------------------------------------------- bit reader (one lane)
// LSB-first (RFC 1951 §3.1.1). `nw` is the next 32-bit word to load; after a
// refill at least 33 bits are buffered. Bits past the end read as zero; the
// caller compares tell() with the end to report EOF exactly.
struct BR {
    Src s;
    uint64_t nw;
    uint64_t buf;
    uint32_t bits;
};
__device__ __forceinline__ void br_refill(BR& b) {
    if (b.bits <= 32) {
        if ((b.nw & 31) == 0 && (b.nw + 128) * 4 < b.s.hi) RRG_PREFETCH_L1(b.s.base + (b.nw + 128) * 4);
        b.buf |= (uint64_t)src_word(b.s, b.nw) << b.bits;
        b.nw++;
        b.bits += 32;
    }
}
__device__ __forceinline__ void br_consume(BR& b, uint32_t n) {
    b.buf >>= n;
    b.bits -= n;
}
// absolute bit position relative to base
__device__ __forceinline__ uint64_t br_tell_abs(const BR& b) { return b.nw * 32 - b.bits; }
__device__ __forceinline__ uint64_t br_tell(const BR& b) { return br_tell_abs(b) - b.s.lo * 8; }
__device__ __forceinline__ void br_seek(BR& b, uint64_t rel_bit) {
    uint64_t a = rel_bit + b.s.lo * 8;
    b.nw = a >> 5;
    b.buf = 0;
    b.bits = 0;
    br_refill(b);
    br_consume(b, (uint32_t)(a & 31));
    br_refill(b);
}
__device__ __forceinline__ uint32_t br_read(BR& b, uint32_t n) {  // n <= 32
    br_refill(b);
    uint32_t v = (uint32_t)(b.buf & ((1ull << n) - 1));
    br_consume(b, n);
    return v;
}
__device__ __forceinline__ bool br_past_end(const BR& b) { return br_tell_abs(b) > b.s.hi * 8; }

// ------------------------------------------------------- Huffman tables
// LUT entry (u32): bits 0-3 code length (0 = not in the LUT), bits 4-5 kind,
// bits 8-11 extra-bit count, bits 16-31 value.
//   litlen kind: 1 length (value = base), 2 end of block, 3 invalid (286/287)
//   dist kind:   0 distance (value = base), 3 invalid (30/31)
//   precode:     value = symbol
// A litlen literal is 0x80000000 | code length << 12 | code length << 8 | byte:
// the sign bit tells it apart in one test, and masked with 0x800000ff it is the
// batch entry itself. pair_literals() turns a literal whose LUT index also
// holds the whole code of a second literal into a pair: bit 24 set, bits 8-11
// the two codes' total length, bits 16-23 the second byte (bits 0-7 and 12-15
// still describe the first literal alone).
enum { TK_LITLEN = 0, TK_DIST = 1, TK_PRE = 2 };
constexpr uint32_t LIT_FLAG = 0x80000000u;
constexpr uint32_t LIT_PAIR = 1u << 24;

__device__ __forceinline__ uint32_t entry_len(uint32_t e) {  // code length of any entry (first literal of a pair)
    return (int32_t)e < 0 ? (e >> 12) & 15u : e & 15u;
}

__device__ __forceinline__ uint32_t make_entry(int kind, uint32_t sym, uint32_t len) {
    if (kind == TK_LITLEN) {
        if (sym < 256) return LIT_FLAG | (len << 12) | (len << 8) | sym;
        if (sym == 256) return (2u << 4) | len;
        if (sym <= 285)
            return ((uint32_t)c_len_base[sym - 257] << 16) | ((uint32_t)c_len_extra[sym - 257] << 8) | (1u << 4) | len;
        return (3u << 4) | len;
    }
    if (kind == TK_DIST) {
        if (sym < 30) return ((uint32_t)c_dist_base[sym] << 16) | ((uint32_t)c_dist_extra[sym] << 8) | len;
        return (3u << 4) | len;
    }
    return (sym << 16) | len;
}

struct Table {
    uint32_t* lut;
    uint16_t* sorted;  // symbols in canonical order
    uint16_t* first;   // [16] first canonical code of each length
    uint16_t* count;   // [16]
    uint16_t* off;     // [16] index of each length's first symbol in `sorted`
};

// Canonical code construction (RFC 1951 §3.2.2), warp-parallel. Rejects an
// oversubscribed tree with >= 2 symbols (huffman.rs:238-249); with `strict`
// also an incomplete one (the block finder's strict build). Returns MSG_NONE
// or MSG_OVERSUB (uniform across the warp).
__device__ int warp_build(const uint8_t* len, int n, const Table& T, int lut_bits, int kind, uint16_t* run,
                          int lane, bool strict = false) {
    const uint32_t lut_size = 1u << lut_bits;
    for (uint32_t i = lane; i < lut_size; i += 32) T.lut[i] = 0;
    uint32_t cnt = 0;
    if (lane >= 1 && lane <= 15)
        for (int s = 0; s < n; s++) cnt += (len[s] == (uint32_t)lane);
    uint32_t kraft = (lane >= 1 && lane <= 15) ? (cnt << (15 - lane)) : 0u;
    uint32_t ksum = warp_sum(kraft), nsym = warp_sum(cnt);
    if (nsym >= 2 && (ksum > 32768u || (strict && ksum != 32768u))) {
        __syncwarp();
        return MSG_OVERSUB;
    }
    uint32_t f = 0, o = 0;
    for (int i = 1; i < 16; i++) {
        uint32_t ci = __shfl_sync(FULLMASK, cnt, i);
        if (i < lane) {
            f = (f + ci) << 1;
            o += ci;
        }
    }
    if (lane < 16) {
        T.first[lane] = (uint16_t)f;
        T.count[lane] = (uint16_t)(lane ? cnt : 0);
        T.off[lane] = (uint16_t)o;
        run[lane] = 0;
    }
    __syncwarp();
    for (int g = 0; g < n; g += 32) {
        int s = g + lane;
        uint32_t l = (s < n) ? len[s] : 0u;
        unsigned same = __match_any_sync(FULLMASK, l);
        unsigned rank = __popc(same & ((1u << lane) - 1u));
        uint32_t base = run[l];
        __syncwarp();
        if (l && (same >> lane) == 1u) run[l] = (uint16_t)(base + __popc(same));
        __syncwarp();
        if (s < n && l) {
            uint32_t idx = base + rank;
            uint32_t code = T.first[l] + idx;
            T.sorted[T.off[l] + idx] = (uint16_t)s;
            if ((int)l <= lut_bits) {
                uint32_t e = make_entry(kind, (uint32_t)s, l);
                uint32_t rev = __brev(code) >> (32 - l);
                for (uint32_t i = rev; i < lut_size; i += (1u << l)) T.lut[i] = e;
            }
        }
    }
    __syncwarp();
    return MSG_NONE;
}

// Two-literal entries for a built litlen LUT of LUT_BITS bits: where the bits
// after a literal's code (the index shifted by its length) decode to another
// literal within the LUT's width, one lookup yields both. Entries keep the
// first literal's byte and length, so the pass reads entries that other lanes
// may already have paired.
__device__ void pair_literals(uint32_t* lut, int lane) {
    for (uint32_t i = lane; i < (uint32_t)LUT_SIZE; i += 32) {
        const uint32_t e = lut[i];
        uint32_t ne = e;
        if ((int32_t)e < 0) {
            const uint32_t c1 = (e >> 12) & 15u;
            const uint32_t e2 = lut[i >> c1];
            if ((int32_t)e2 < 0) {
                const uint32_t c2 = (e2 >> 12) & 15u;
                if (c1 + c2 <= (uint32_t)LUT_BITS)
                    ne = (e & 0x8000f0ffu) | ((c1 + c2) << 8) | ((e2 & 0xffu) << 16) | LIT_PAIR;
            }
        }
        __syncwarp();
        lut[i] = ne;
        __syncwarp();
    }
}

// Codes longer than the LUT: canonical decode over lengths lut_bits+1..15.
// Returns 0 when no code matches.
__device__ __noinline__ uint32_t long_decode(uint64_t buf, const Table& T, int lut_bits, int kind) {
    uint32_t rv = __brev((uint32_t)buf);
    for (int l = lut_bits + 1; l <= 15; l++) {
        uint32_t code = rv >> (32 - l);
        uint32_t d = code - T.first[l];
        if (d < T.count[l]) return make_entry(kind, T.sorted[T.off[l] + d], (uint32_t)l);
    }
    return 0;
}

// ------------------------------------------------------- inflate kernel
struct WarpSmem {
    uint32_t lit_lut[LUT_SIZE];
    union {  // the precode table is dead once the distance table is built
        uint32_t dist_lut[DIST_SIZE];
        uint32_t pre_lut[1 << PRE_BITS];
    };
    uint2 ep[NB];  // per batch symbol: x = entry (literal flag|byte, or dist<<9|length), y = output offset
    uint16_t lit_sorted[288];
    uint16_t dist_sorted[32];
    uint16_t pre_sorted[32];
    uint16_t lit_first[16], lit_count[16], lit_off[16];
    uint16_t dist_first[16], dist_count[16], dist_off[16];
    uint16_t pre_first[16], pre_count[16], pre_off[16];
    uint16_t run[16];
    uint8_t lengths[320];
    uint8_t pre_len[20];
    int32_t fixed_loaded;
    int32_t pad[3];
};

struct InflateArgs {
    const uint8_t* in;       // compressed input base
    const ChunkItem* items;
    ChunkResult* results;
    uint32_t n_items;
    const uint32_t* n_items_dev;  // when set, the item count is read here (device-built work lists)
    const uint32_t* order;   // optional permutation of the work queue (largest first)
    uint32_t* queue;         // work-queue head
    void* out;               // cell arena (u16) or byte output (u8)
    MemberRec* mbs;
    uint32_t* mb_count;
    uint32_t mb_cap;
};

// Per-item decode state (identical in every lane except the bit reader,
// which only lane 0 advances).
struct ItemState {
    BR br;
    uint64_t cur;           // cells produced
    uint64_t cap;           // cells available
    uint64_t member_start;  // cell where the current member began
    uint64_t markers;
    int32_t status, msg;
    bool markers_ok;
    bool counting;          // output full: keep decoding only to measure the size
};

__device__ __forceinline__ Table lit_table(WarpSmem& S) {
    return Table{S.lit_lut, S.lit_sorted, S.lit_first, S.lit_count, S.lit_off};
}
__device__ __forceinline__ Table dist_table(WarpSmem& S) {
    return Table{S.dist_lut, S.dist_sorted, S.dist_first, S.dist_count, S.dist_off};
}
__device__ __forceinline__ Table pre_table(WarpSmem& S) {
    return Table{S.pre_lut, S.pre_sorted, S.pre_first, S.pre_count, S.pre_off};
}

__device__ __forceinline__ int find_entry(const uint2* ep, int n, uint32_t j) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ep[mid].y <= j) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Dynamic block header (inflate.rs:74-145 read_dynamic_header) -> tables.
__device__ void read_dynamic(WarpSmem& S, ItemState& st, int lane) {
    int status = 0, msg = 0;
    uint32_t hlit = 0, hdist = 0;
    if (lane == 0) {
        hlit = br_read(st.br, 5) + 257;
        hdist = br_read(st.br, 5) + 1;
        uint32_t hclen = br_read(st.br, 4) + 4;
        for (int i = 0; i < 19; i++) S.pre_len[i] = 0;
        if (hlit > 286 || hdist > 30) {
            status = DS_INVALID;
            msg = MSG_HLIT_HDIST;
        } else {
            for (uint32_t i = 0; i < hclen; i++) S.pre_len[c_cl_order[i]] = (uint8_t)br_read(st.br, 3);
            if (br_past_end(st.br)) status = DS_EOF;
        }
    }
    status = bcast32(status);
    msg = bcast32(msg);
    hlit = (uint32_t)bcast32((int32_t)hlit);
    hdist = (uint32_t)bcast32((int32_t)hdist);
    if (status) {
        st.status = status;
        st.msg = msg;
        return;
    }
    __syncwarp();
    msg = warp_build(S.pre_len, 19, pre_table(S), PRE_BITS, TK_PRE, S.run, lane);
    if (msg) {
        st.status = DS_INVALID;
        st.msg = msg;
        return;
    }
    for (int i = lane; i < 320; i += 32) S.lengths[i] = 0;
    __syncwarp();
    if (lane == 0) {
        uint32_t total = hlit + hdist, i = 0;
        while (i < total) {
            br_refill(st.br);
            uint32_t e = S.pre_lut[st.br.buf & ((1u << PRE_BITS) - 1)];
            uint32_t cl = e & 15;
            if (!cl) {
                status = DS_INVALID;
                msg = MSG_NO_CODE;
                break;
            }
            br_consume(st.br, cl);
            uint32_t sym = e >> 16;
            if (sym <= 15) {
                S.lengths[i++] = (uint8_t)sym;
            } else if (sym == 16) {
                if (i == 0) {
                    status = DS_INVALID;
                    msg = MSG_CODE16_FIRST;
                    break;
                }
                uint32_t r = br_read(st.br, 2) + 3;
                if (i + r > total) {
                    status = DS_INVALID;
                    msg = MSG_CODE16_OVER;
                    break;
                }
                uint8_t prev = S.lengths[i - 1];
                for (uint32_t j = 0; j < r; j++) S.lengths[i + j] = prev;
                i += r;
            } else if (sym == 17) {
                uint32_t r = br_read(st.br, 3) + 3;
                if (i + r > total) {
                    status = DS_INVALID;
                    msg = MSG_CODE17_OVER;
                    break;
                }
                i += r;
            } else {
                uint32_t r = br_read(st.br, 7) + 11;
                if (i + r > total) {
                    status = DS_INVALID;
                    msg = MSG_CODE18_OVER;
                    break;
                }
                i += r;
            }
            if (br_past_end(st.br)) {
                status = DS_EOF;
                break;
            }
        }
        if (!status && S.lengths[256] == 0) {
            status = DS_INVALID;
            msg = MSG_EOB_ZERO;
        }
    }
    status = bcast32(status);
    msg = bcast32(msg);
    if (status) {
        st.status = status;
        st.msg = msg;
        return;
    }
    __syncwarp();
    msg = warp_build(S.lengths, (int)hlit, lit_table(S), LUT_BITS, TK_LITLEN, S.run, lane);
    if (!msg) pair_literals(S.lit_lut, lane);
    if (!msg) msg = warp_build(S.lengths + hlit, (int)hdist, dist_table(S), DIST_BITS, TK_DIST, S.run, lane);
    if (msg) {
        st.status = DS_INVALID;
        st.msg = msg;
    }
    if (lane == 0) S.fixed_loaded = 0;
    __syncwarp();
}

__device__ void load_fixed(WarpSmem& S, int lane) {
    if (S.fixed_loaded) return;  // uniform (shared value)
    for (int i = lane; i < 288; i += 32) S.lengths[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : 8;
    for (int i = lane; i < 30; i += 32) S.lengths[288 + i] = 5;
    __syncwarp();
    warp_build(S.lengths, 288, lit_table(S), LUT_BITS, TK_LITLEN, S.run, lane);
    warp_build(S.lengths + 288, 30, dist_table(S), DIST_BITS, TK_DIST, S.run, lane);
    if (lane == 0) S.fixed_loaded = 1;
    __syncwarp();
}

// Stored block (inflate.rs:38-53): byte-align, LEN/NLEN, LEN raw bytes.
template <typename CellT>
__device__ void stored_block(WarpSmem& S, ItemState& st, CellT* out, int lane) {
    int status = 0, msg = 0;
    uint64_t bp = 0;
    uint32_t len = 0;
    if (lane == 0) {
        br_consume(st.br, st.br.bits & 7);
        len = br_read(st.br, 16);
        uint32_t nlen = br_read(st.br, 16);
        if ((len ^ 0xffffu) != nlen) {
            status = DS_INVALID;
            msg = MSG_STORED_NLEN;
        } else {
            bp = br_tell(st.br) >> 3;  // relative to the source start
            if (st.br.s.lo + bp + len > st.br.s.hi) status = DS_EOF;
        }
    }
    status = bcast32(status);
    msg = bcast32(msg);
    len = (uint32_t)bcast32((int32_t)len);
    bp = bcast64(bp);
    if (status) {
        st.status = status;
        st.msg = msg;
        return;
    }
    if (!st.counting && st.cur + len > st.cap) st.counting = true;
    if (!st.counting) {
        // bounds were checked above: plain byte loads, 16 per lane in flight,
        // each load and store instruction covering 32 consecutive bytes/cells
        const uint8_t* src = st.br.s.base + st.br.s.lo + bp;
        CellT* dst = out + st.cur;
        uint32_t i = 0;
        for (; i + 512 <= len; i += 512) {
            uint32_t v[16];
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = __ldg(src + i + 32 * k + lane);
#pragma unroll
            for (int k = 0; k < 16; k++) dst[i + 32 * k + lane] = (CellT)v[k];
        }
        for (i += lane; i < len; i += 32) dst[i] = (CellT)__ldg(src + i);
    }
    st.cur += len;
    if (lane == 0) br_seek(st.br, (bp + len) * 8);
    __syncwarp();
}

// Huffman-coded block body: lane 0 decodes up to NB symbols into the batch,
// the warp materialises the batch's bytes in parallel.
template <typename CellT>
__device__ void decode_codes(WarpSmem& S, ItemState& st, CellT* out, int lane) {
    const Table LT = lit_table(S), DT = dist_table(S);
    for (;;) {
        int n = 0, stop = 0, status = 0, msg = 0, fast_flag = 0;
        uint32_t pos = 0;
        if (lane == 0) {
            uint64_t room = st.counting ? ~0ull : (st.cap > st.cur ? st.cap - st.cur : 0);
            BR b = st.br;
            // Fast path: the batch surely fits the slot (<= NB * 258 cells) and every
            // word it can load (a batch consumes <= NB * 48 bits) lies inside the input.
            const bool fast = room >= (uint64_t)NB * 258 && (b.nw + 56) * 4 <= b.s.hi && b.nw * 4 >= b.s.lo;
            fast_flag = fast ? 1 : 0;
            bool handoff = false;
            if (fast) {
                const uint32_t* base_w = reinterpret_cast<const uint32_t*>(b.s.base);
                const uint32_t* wp = base_w + b.nw;
                uint64_t buf = b.buf;
                uint32_t bits = b.bits;
                while (n < NB - 1) {  // a pair may add two entries
                    if (bits <= 32) {
                        buf |= (uint64_t)__ldg(wp) << bits;
                        wp++;
                        bits += 32;
                    }
                    uint32_t e = S.lit_lut[(uint32_t)buf & (LUT_SIZE - 1)];
                    if ((int32_t)e < 0) {  // literal (or two): the entry is the batch entry
                        const uint32_t cl = (e >> 8) & 15u;
                        buf >>= cl;
                        bits -= cl;
                        S.ep[n].x = e & 0x800000ffu;
                        S.ep[n + 1].x = LIT_FLAG | ((e >> 16) & 0xffu);  // kept only for a pair
                        n += 1 + ((e >> 24) & 1u);
                        continue;
                    }
                    if (!e) {  // a code longer than the LUT: the checked path takes this symbol
                        handoff = true;
                        break;
                    }
                    const uint32_t cl = e & 15u;
                    const uint32_t kind = (e >> 4) & 3;
                    if (kind == 1) {
                        const uint32_t ex = (e >> 8) & 15;
                        const uint32_t length = (e >> 16) + ((uint32_t)(buf >> cl) & ((1u << ex) - 1u));
                        buf >>= cl + ex;
                        bits -= cl + ex;
                        if (bits <= 32) {
                            buf |= (uint64_t)__ldg(wp) << bits;
                            wp++;
                            bits += 32;
                        }
                        uint32_t de = S.dist_lut[(uint32_t)buf & (DIST_SIZE - 1)];
                        uint32_t dl = de & 15;
                        if (!dl) {
                            de = long_decode(buf, DT, DIST_BITS, TK_DIST);
                            dl = de & 15;
                            if (!dl) {
                                status = DS_INVALID;
                                msg = MSG_NO_CODE;
                                break;
                            }
                        }
                        if (((de >> 4) & 3) == 3) {
                            status = DS_INVALID;
                            msg = MSG_DIST_RANGE;
                            break;
                        }
                        const uint32_t dx = (de >> 8) & 15;
                        const uint32_t dist = (de >> 16) + ((uint32_t)(buf >> dl) & ((1u << dx) - 1u));
                        buf >>= dl + dx;
                        bits -= dl + dx;
                        S.ep[n].x = (dist << 9) | length;
                        n++;
                    } else if (kind == 2) {
                        buf >>= cl;
                        bits -= cl;
                        stop = 1;
                        break;
                    } else {
                        status = DS_INVALID;
                        msg = MSG_LITLEN_RANGE;
                        break;
                    }
                }
                b.nw = (uint64_t)(wp - base_w);
                b.buf = buf;
                b.bits = bits;
                if (!status && br_past_end(b)) status = DS_EOF;
                if (handoff && !status) {
                    // the checked path finishes the batch: it needs the entries'
                    // offsets, which the fast path leaves to the warp
                    fast_flag = 0;
                    for (int k = 0; k < n; k++) {
                        const uint32_t x = S.ep[k].x;
                        S.ep[k].y = pos;
                        pos += (x & LIT_FLAG) ? 1u : (x & 511u);
                    }
                }
            }
            while ((!fast || (handoff && !status)) && n < NB) {
                const BR save = b;
                br_refill(b);
                uint32_t e = S.lit_lut[b.buf & (LUT_SIZE - 1)];
                if (!e) {
                    e = long_decode(b.buf, LT, LUT_BITS, TK_LITLEN);
                    if (!e) {
                        status = br_past_end(b) ? DS_EOF : DS_INVALID;
                        msg = MSG_NO_CODE;
                        break;
                    }
                }
                const uint32_t cl = entry_len(e);
                const uint32_t kind = (int32_t)e < 0 ? 0u : (e >> 4) & 3;
                if (kind == 0) {
                    if (pos + 1 > room) {  // output full: this symbol is re-read in counting mode
                        b = save;
                        stop = 3;
                        break;
                    }
                    br_consume(b, cl);
                    S.ep[n] = make_uint2(e & 0x800000ffu, pos);
                    pos += 1;
                    n++;
                } else if (kind == 1) {
                    uint32_t ex = (e >> 8) & 15;
                    uint32_t length = (e >> 16) + ((uint32_t)(b.buf >> cl) & ((1u << ex) - 1u));
                    br_consume(b, cl + ex);
                    br_refill(b);
                    uint32_t de = S.dist_lut[b.buf & (DIST_SIZE - 1)];
                    uint32_t dl = de & 15;
                    if (!dl) {
                        de = long_decode(b.buf, DT, DIST_BITS, TK_DIST);
                        dl = de & 15;
                        if (!dl) {
                            status = br_past_end(b) ? DS_EOF : DS_INVALID;
                            msg = MSG_NO_CODE;
                            break;
                        }
                    }
                    if (((de >> 4) & 3) == 3) {
                        status = DS_INVALID;
                        msg = MSG_DIST_RANGE;
                        break;
                    }
                    if (pos + length > room) {
                        b = save;
                        stop = 3;
                        break;
                    }
                    uint32_t dx = (de >> 8) & 15;
                    uint32_t dist = (de >> 16) + ((uint32_t)(b.buf >> dl) & ((1u << dx) - 1u));
                    br_consume(b, dl + dx);
                    S.ep[n] = make_uint2((dist << 9) | length, pos);
                    pos += length;
                    n++;
                } else if (kind == 2) {
                    br_consume(b, cl);
                    stop = 1;
                } else {
                    status = DS_INVALID;
                    msg = MSG_LITLEN_RANGE;
                    break;
                }
                if (br_past_end(b)) {
                    status = DS_EOF;
                    break;
                }
                if (stop) break;
            }
            st.br = b;
        }
        n = bcast32(n);
        pos = (uint32_t)bcast32((int32_t)pos);
        stop = bcast32(stop);
        status = bcast32(status);
        msg = bcast32(msg);
        const int fast_batch = bcast32(fast_flag);
        __syncwarp();
        if (fast_batch) {
            // the fast path stores entries only: their output offsets are a warp prefix sum
            const uint32_t x = lane < n ? S.ep[lane].x : 0u;
            const uint32_t len = lane < n ? ((x & LIT_FLAG) ? 1u : (x & 511u)) : 0u;
            uint32_t incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULLMASK, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane < n) S.ep[lane].y = incl - len;
            pos = __shfl_sync(FULLMASK, incl, 31);
            __syncwarp();
        }
        if (!st.counting && n) {
            uint32_t bad = 0, mk = 0;
            const uint64_t cur = st.cur;
            // Lane k holds the start of entry k. For each 32-cell group one OR
            // over the warp marks the entries that start inside it, so a lane's
            // entry is (entries started before the group) + (starts at or below
            // the lane) - 1: no search.
            // A pass covers MAT_GROUPS groups: every cell is first resolved to a
            // byte, a marker or an output position written by an earlier batch;
            // the loads of those positions are issued together, then the cells
            // are stored (a batch never reads its own cells from memory: sources
            // inside the batch are followed through its entries).
            const uint32_t my_start = lane < n ? S.ep[lane].y : 0xffffffffu;
            uint32_t before = 0;
            for (uint32_t p0 = 0; p0 < pos; p0 += 32u * MAT_GROUPS) {
                uint32_t cell[MAT_GROUPS];
                int64_t from[MAT_GROUPS];  // >= 0: output position to load
#pragma unroll
                for (int g = 0; g < MAT_GROUPS; g++) {
                    cell[g] = 0;
                    from[g] = -1;
                    const uint32_t j0 = p0 + 32u * g;
                    if (j0 >= pos) continue;  // warp-uniform
                    const uint32_t j = j0 + lane;
                    const uint32_t rel = my_start - j0;
                    const uint32_t starts = __reduce_or_sync(FULLMASK, rel < 32u ? (1u << rel) : 0u);
                    int k = (int)(before + __popc(starts & (0xffffffffu >> (31 - lane)))) - 1;
                    before += __popc(starts);
                    if (j >= pos) continue;
                    uint32_t jj = j;
                    for (;;) {
                        uint32_t e = S.ep[k].x;
                        if (e & 0x80000000u) {
                            cell[g] = e & 0xffu;
                            break;
                        }
                        uint32_t d = e >> 9;
                        const uint32_t ek = S.ep[k].y;
                        uint32_t t = jj - ek;
                        if (t >= d) t %= d;
                        int64_t src = (int64_t)ek - (int64_t)d + (int64_t)t;
                        if (src >= 0) {
                            jj = (uint32_t)src;
                            k = find_entry(S.ep, k, jj);
                            continue;
                        }
                        int64_t a = (int64_t)cur + src;
                        if (a >= (int64_t)st.member_start) {
                            from[g] = a;
                            break;
                        }
                        if (st.markers_ok && a < 0) {
                            cell[g] = MARKER16 | (uint32_t)(-a - 1);
                            mk++;
                            break;
                        }
                        bad = 1;
                        break;
                    }
                }
#pragma unroll
                for (int g = 0; g < MAT_GROUPS; g++)
                    if (from[g] >= 0) cell[g] = (uint32_t)out[from[g]];
#pragma unroll
                for (int g = 0; g < MAT_GROUPS; g++) {
                    const uint32_t j = p0 + 32u * g + lane;
                    if (j < pos) out[cur + j] = (CellT)cell[g];
                }
            }
            bad = warp_sum(bad);
            mk = warp_sum(mk);
            st.markers += mk;
            if (bad && !status) {
                status = DS_INVALID;
                msg = MSG_DIST_FAR;
            }
        }
        st.cur += pos;
        __syncwarp();
        if (status) {
            st.status = status;
            st.msg = msg;
            return;
        }
        if (stop == 1) return;
        if (stop == 3) st.counting = true;
    }
}

__device__ __forceinline__ uint32_t le32_at(const Src& s, uint64_t rel) {
    return src_byte(s, rel) | (src_byte(s, rel + 1) << 8) | (src_byte(s, rel + 2) << 16) | (src_byte(s, rel + 3) << 24);
}

// gzip.rs:252-300 parse_header, on the device (lane 0 only).
__device__ int dev_parse_header(const Src& s, uint64_t at, uint64_t* hl, int* msg) {
    uint64_t n = s.hi - s.lo;
    *msg = 0;
    if (at + 10 > n) return DS_TRUNCATED;
    if (src_byte(s, at) != 0x1f || src_byte(s, at + 1) != 0x8b) return DS_BAD_MAGIC;
    uint32_t cm = src_byte(s, at + 2);
    if (cm != 8) {
        *msg = (int)cm;
        return DS_METHOD;
    }
    uint32_t flg = src_byte(s, at + 3);
    if (flg & 0xe0) {
        *msg = (int)flg;
        return DS_FLAGS;
    }
    uint64_t pos = at + 10;
    if (flg & 4) {
        if (pos + 2 > n) return DS_TRUNCATED;
        uint64_t xlen = src_byte(s, pos) | (src_byte(s, pos + 1) << 8);
        pos += 2 + xlen;
        if (pos > n) return DS_TRUNCATED;
    }
    for (uint32_t f = 8; f <= 16; f <<= 1) {
        if (flg & f) {
            while (pos < n && src_byte(s, pos) != 0) pos++;
            if (pos >= n) return DS_TRUNCATED;
            pos++;
        }
    }
    if (flg & 2) {
        if (pos + 2 > n) return DS_TRUNCATED;
        pos += 2;
    }
    *hl = pos - at;
    return DS_OK;
}

template <typename CellT>
__device__ void inflate_item(WarpSmem& S, const InflateArgs& A, uint32_t item_idx, int lane) {
    const ChunkItem it = A.items[item_idx];
    if (it.flags & ITEM_SKIP) {
        if (lane == 0) A.results[item_idx] = ChunkResult{0, it.start_bit, DS_OK, 0, 0, 0, 0, 0};
        __syncwarp();
        return;
    }
    CellT* out = (CellT*)A.out + it.out_off;
    ItemState st;
    st.br.s = make_src(A.in + it.in_off, it.in_len);
    st.br.nw = 0;
    st.br.buf = 0;
    st.br.bits = 0;
    st.cur = 0;
    st.cap = it.out_cap;
    st.member_start = 0;
    st.markers = 0;
    st.status = 0;
    st.msg = 0;
    st.markers_ok = (it.flags & ITEM_MARKERS) != 0 && sizeof(CellT) == 2;
    st.counting = false;
    const uint64_t body_len = it.in_len;
    uint64_t start = it.start_bit;
    uint32_t trailer_crc = 0, trailer_isize = 0;
    if (it.flags & ITEM_ONE_MEMBER) {
        int status = 0, msg = 0;
        uint64_t hl = 0;
        if (lane == 0) status = dev_parse_header(st.br.s, 0, &hl, &msg);
        status = bcast32(status);
        msg = bcast32(msg);
        hl = bcast64(hl);
        if (status) {
            st.status = status;
            st.msg = msg;
        }
        start = hl * 8;
    }
    if (lane == 0) {
        if (start > body_len * 8) st.status = DS_EOF;
        else br_seek(st.br, start);
        S.fixed_loaded = 0;
    }
    st.status = bcast32(st.status);
    __syncwarp();
    bool final_block = false;
    uint32_t n_members = 0;
    uint64_t end_bit = 0;
    while (!st.status) {
        int at_end = 0;
        if (lane == 0) at_end = br_tell(st.br) >= it.end_hint;
        if (bcast32(at_end)) break;
        // one member: blocks until BFINAL or the chunk boundary
        int bfinal = 0;
        for (;;) {
            uint32_t bt = 0;
            int status = 0;
            if (lane == 0) {
                bfinal = (int)br_read(st.br, 1);
                bt = br_read(st.br, 2);
                if (br_past_end(st.br)) status = DS_EOF;
            }
            bfinal = bcast32(bfinal);
            bt = (uint32_t)bcast32((int32_t)bt);
            status = bcast32(status);
            if (status) {
                st.status = status;
                break;
            }
            if (bt == 0) {
                stored_block<CellT>(S, st, out, lane);
            } else if (bt == 1) {
                load_fixed(S, lane);
                decode_codes<CellT>(S, st, out, lane);
            } else if (bt == 2) {
                read_dynamic(S, st, lane);
                if (!st.status) decode_codes<CellT>(S, st, out, lane);
            } else {
                st.status = DS_INVALID;
                st.msg = MSG_RESERVED_BTYPE;
            }
            if (st.status || bfinal) break;
            int past = 0;
            if (lane == 0) past = br_tell(st.br) >= it.end_hint;
            if (bcast32(past)) break;
        }
        if (st.status || !bfinal) break;
        // member trailer (pipeline.rs:1124-1165)
        int status = 0, msg = 0, fin = 0;
        uint64_t after = 0, hl = 0;
        if (lane == 0) {
            br_consume(st.br, st.br.bits & 7);
            uint64_t tb = br_tell(st.br) >> 3;
            if (tb + 8 > body_len) {
                status = DS_TRUNCATED;
            } else {
                trailer_crc = le32_at(st.br.s, tb);
                trailer_isize = le32_at(st.br.s, tb + 4);
                if (!(it.flags & ITEM_ONE_MEMBER)) {
                    uint32_t slot = atomicAdd(A.mb_count, 1u);
                    if (slot < A.mb_cap) {
                        MemberRec r;
                        r.item = it.id;
                        r.seq = n_members;
                        r.cell_off = st.cur;
                        r.crc = trailer_crc;
                        r.isize = trailer_isize;
                        r.trailer_byte = tb;
                        A.mbs[slot] = r;
                    }
                }
                after = tb + 8;
                if (after >= body_len || (it.flags & ITEM_ONE_MEMBER)) {
                    fin = 1;
                } else {
                    status = dev_parse_header(st.br.s, after, &hl, &msg);
                    if (!status) br_seek(st.br, (after + hl) * 8);
                }
            }
        }
        status = bcast32(status);
        msg = bcast32(msg);
        fin = bcast32(fin);
        after = bcast64(after);
        n_members++;
        if (status) {
            st.status = status;
            st.msg = msg;
            break;
        }
        if (fin) {
            final_block = true;
            end_bit = after * 8;
            break;
        }
        st.member_start = st.cur;
        st.markers_ok = false;
    }
    if (lane == 0) {
        ChunkResult r;
        r.n_cells = st.cur;
        r.actual_end_bit = final_block ? end_bit : br_tell(st.br);
        r.status = st.status ? st.status : (st.counting ? DS_OVERFLOW : DS_OK);
        r.msg = st.msg;
        r.final_block = final_block ? 1 : 0;
        r.n_members = n_members;
        r.markers = st.markers;
        r.err_bit = br_tell(st.br);
        if (it.flags & ITEM_ONE_MEMBER) {
            // batch mode: the trailer fields travel in place of the marker count
            r.markers = ((uint64_t)trailer_isize << 32) | trailer_crc;
        }
        A.results[item_idx] = r;
    }
    __syncwarp();
}

#ifndef RRG_INFLATE_MIN_BLOCKS
#define RRG_INFLATE_MIN_BLOCKS 6
#endif
// 128 threads (4 warps) per block, >= RRG_INFLATE_MIN_BLOCKS blocks per SM
template <typename CellT>
__global__ void __launch_bounds__(128, RRG_INFLATE_MIN_BLOCKS) k_inflate(InflateArgs A) {
    RRG_DYN_SMEM(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpSmem& S = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
    for (;;) {
        uint32_t idx = 0;
        if (lane == 0) idx = atomicAdd(A.queue, 1u);
        idx = (uint32_t)bcast32((int32_t)idx);
        if (idx >= (A.n_items_dev ? *A.n_items_dev : A.n_items)) break;
        uint32_t item = A.order ? A.order[idx] : idx;
        inflate_item<CellT>(S, A, item, lane);
    }
}

// ------------------------------------------------------- lane-per-chunk inflate
// Every thread is a whole decoder for one work item (the same item contract
// as k_inflate): 32 chunks advance per warp instruction, which is what a
// single-member file split at block boundaries, or a BGZF file, offers in
// the thousands. Tables are per lane in shared memory: a 9-bit litlen LUT and
// an 8-bit distance LUT of 16-bit entries plus canonical data for longer
// codes; code lengths and symbol lists live in a per-thread global scratch.
constexpr int LL_BITS = 9;
constexpr int DL_BITS = 8;
constexpr int LANE_THREADS = 64;

struct LaneTab {
    uint16_t lit[1 << LL_BITS];
    uint16_t dist[1 << DL_BITS];
    uint16_t lfirst[16], lcount[16], loff[16];
    uint16_t dfirst[16], dcount[16], doff[16];
};

struct LaneScratch {
    uint8_t lengths[320];
    uint16_t lsorted[288];
    uint16_t dsorted[32];
};

struct LaneConsts {
    uint16_t lbase[32];
    uint16_t dbase[32];
    uint8_t lextra[32];
    uint8_t dextra[32];
};

// lane LUT entries (u16): bits 0-3 code length (0 = not in the LUT),
// bits 4-5 kind, bits 8-15 value.
//   litlen: kind 0 literal (value = byte), 1 length (value = length code 0..28), 2 EOB, 3 invalid
//   dist:   kind 0 (value = distance code 0..29), 1 invalid (30/31)
//   precode: value = symbol
__device__ __forceinline__ uint16_t lane_entry(int kind, uint32_t s, uint32_t l) {
    if (kind == TK_LITLEN) {
        if (s < 256) return (uint16_t)((s << 8) | l);
        if (s == 256) return (uint16_t)((2u << 4) | l);
        if (s <= 285) return (uint16_t)(((s - 257) << 8) | (1u << 4) | l);
        return (uint16_t)((3u << 4) | l);
    }
    if (kind == TK_DIST) return (uint16_t)(s < 30 ? ((s << 8) | l) : ((1u << 4) | l));
    return (uint16_t)((s << 8) | l);
}

// Canonical table build for one lane (RFC 1951 §3.2.2); non-strict like
// huffman.rs build_into: only an oversubscribed tree (>= 2 symbols) fails.
__device__ int lane_build(const uint8_t* len, int n, uint16_t* lut, int lut_bits, uint16_t* first, uint16_t* count,
                          uint16_t* off, uint16_t* sorted, int kind) {
    uint16_t cnt[16], next[16];
    for (int l = 0; l < 16; l++) cnt[l] = 0;
    for (int s = 0; s < n; s++) cnt[len[s] & 15]++;
    cnt[0] = 0;
    uint32_t kraft = 0, nsym = 0;
    for (int l = 1; l < 16; l++) {
        kraft += (uint32_t)cnt[l] << (15 - l);
        nsym += cnt[l];
    }
    if (nsym >= 2 && kraft > 32768u) return MSG_OVERSUB;
    uint32_t f = 0, o = 0;
    first[0] = count[0] = off[0] = 0;
    for (int l = 1; l < 16; l++) {
        f = (f + cnt[l - 1]) << 1;
        first[l] = (uint16_t)f;
        next[l] = (uint16_t)f;
        count[l] = cnt[l];
        off[l] = (uint16_t)o;
        o += cnt[l];
    }
    const uint32_t size = 1u << lut_bits;
    uint32_t* lut32 = reinterpret_cast<uint32_t*>(lut);
    for (uint32_t i = 0; i < size / 2; i++) lut32[i] = 0;
    for (int s = 0; s < n; s++) {
        const uint32_t l = len[s];
        if (!l) continue;
        const uint32_t code = next[l]++;
        sorted[off[l] + (code - first[l])] = (uint16_t)s;
        if ((int)l <= lut_bits) {
            const uint16_t e = lane_entry(kind, (uint32_t)s, l);
            const uint32_t rev = __brev(code) >> (32 - l);
            for (uint32_t i = rev; i < size; i += 1u << l) lut[i] = e;
        }
    }
    return MSG_NONE;
}

// Longer codes: canonical decode over lengths lut_bits+1..15. Returns the
// symbol and sets *l, or returns -1.
__device__ __forceinline__ int lane_long(uint64_t buf, const uint16_t* first, const uint16_t* count,
                                         const uint16_t* off, const uint16_t* sorted, int lut_bits, uint32_t* l) {
    const uint32_t rv = __brev((uint32_t)buf);
    for (int k = lut_bits + 1; k <= 15; k++) {
        const uint32_t code = rv >> (32 - k);
        const uint32_t d = code - first[k];
        if (d < count[k]) {
            *l = (uint32_t)k;
            return sorted[off[k] + d];
        }
    }
    return -1;
}

struct LaneState {
    BR br;
    uint64_t cur, cap, member_start, markers;
    int32_t status, msg;
    bool markers_ok, counting;
};

// Huffman-coded block body for one lane.
template <typename CellT>
__device__ void lane_codes(LaneState& st, LaneTab& T, const LaneScratch* scr, const LaneConsts& K, CellT* out) {
    BR b = st.br;
    uint64_t cur = st.cur;
    uint64_t cap = st.counting ? ~0ull : st.cap;
    const uint64_t hi_bits = b.s.hi * 8;
    for (;;) {
        br_refill(b);
        uint32_t e = T.lit[b.buf & ((1u << LL_BITS) - 1)];
        uint32_t cl = e & 15;
        if (!cl) {
            const int s = lane_long(b.buf, T.lfirst, T.lcount, T.loff, scr->lsorted, LL_BITS, &cl);
            if (s < 0) {
                st.status = br_past_end(b) ? DS_EOF : DS_INVALID;
                st.msg = MSG_NO_CODE;
                break;
            }
            e = lane_entry(TK_LITLEN, (uint32_t)s, cl);
        }
        const uint32_t kind = (e >> 4) & 3;
        if (kind == 0) {
            if (cur >= cap) {  // output full: the rest is only measured (this symbol again)
                st.counting = true;
                cap = ~0ull;
                continue;
            }
            if (!st.counting) out[cur] = (CellT)(e >> 8);
            cur++;
            br_consume(b, cl);
        } else if (kind == 1) {
            const uint32_t li = e >> 8;
            const uint32_t ex = K.lextra[li];
            const uint32_t length = K.lbase[li] + ((uint32_t)(b.buf >> cl) & ((1u << ex) - 1u));
            const BR save = b;
            br_consume(b, cl + ex);
            br_refill(b);
            uint32_t de = T.dist[b.buf & ((1u << DL_BITS) - 1)];
            uint32_t dl = de & 15;
            if (!dl) {
                const int s = lane_long(b.buf, T.dfirst, T.dcount, T.doff, scr->dsorted, DL_BITS, &dl);
                if (s < 0) {
                    st.status = br_past_end(b) ? DS_EOF : DS_INVALID;
                    st.msg = MSG_NO_CODE;
                    break;
                }
                de = lane_entry(TK_DIST, (uint32_t)s, dl);
            }
            if (de & 0x10u) {
                st.status = DS_INVALID;
                st.msg = MSG_DIST_RANGE;
                break;
            }
            const uint32_t di = de >> 8;
            const uint32_t dx = K.dextra[di];
            const uint32_t d = K.dbase[di] + ((uint32_t)(b.buf >> dl) & ((1u << dx) - 1u));
            if (cur + length > cap) {
                b = save;  // output full: re-read this match, measuring only
                st.counting = true;
                cap = ~0ull;
                continue;
            }
            br_consume(b, dl + dx);
            if (!st.counting) {
                const int64_t c0 = (int64_t)cur;
                const int64_t ms = (int64_t)st.member_start;
                int64_t k = 0;
                // references before the member start: markers (first member of a
                // speculative chunk) or an error
                for (; k < (int64_t)length && c0 + k - (int64_t)d < ms; k++) {
                    const int64_t src = c0 + k - (int64_t)d;
                    if (st.markers_ok && src < 0) {
                        out[c0 + k] = (CellT)(MARKER16 | (uint32_t)(-src - 1));
                        st.markers++;
                    } else {
                        st.status = DS_INVALID;
                        st.msg = MSG_DIST_FAR;
                        break;
                    }
                }
                if (st.status) break;
                CellT* dst = out + c0;
                const CellT* src = out + c0 - d;
                if (d >= (uint32_t)length) {
                    for (; k + 4 <= (int64_t)length; k += 4) {
                        const CellT v0 = src[k], v1 = src[k + 1], v2 = src[k + 2], v3 = src[k + 3];
                        dst[k] = v0;
                        dst[k + 1] = v1;
                        dst[k + 2] = v2;
                        dst[k + 3] = v3;
                    }
                }
                for (; k < (int64_t)length; k++) dst[k] = src[k];
            }
            cur += length;
        } else if (kind == 2) {
            br_consume(b, cl);
            break;
        } else {
            st.status = DS_INVALID;
            st.msg = MSG_LITLEN_RANGE;
            break;
        }
        if (br_tell_abs(b) > hi_bits) {
            st.status = DS_EOF;
            break;
        }
    }
    st.br = b;
    st.cur = cur;
}

// Dynamic header (inflate.rs:74-145) for one lane.
__device__ void lane_dynamic(LaneState& st, LaneTab& T, LaneScratch* scr) {
    BR& b = st.br;
    const uint32_t hlit = br_read(b, 5) + 257, hdist = br_read(b, 5) + 1, hclen = br_read(b, 4) + 4;
    if (hlit > 286 || hdist > 30) {
        st.status = DS_INVALID;
        st.msg = MSG_HLIT_HDIST;
        return;
    }
    uint8_t pre[19];
    for (int i = 0; i < 19; i++) pre[i] = 0;
    for (uint32_t i = 0; i < hclen; i++) pre[c_cl_order[i]] = (uint8_t)br_read(b, 3);
    if (br_past_end(b)) {
        st.status = DS_EOF;
        return;
    }
    // precode table (7 bits) in the distance LUT's space
    for (int i = 0; i < 19; i++) scr->lengths[i] = pre[i];
    int m = lane_build(scr->lengths, 19, T.dist, PRE_BITS, T.dfirst, T.dcount, T.doff, scr->dsorted, TK_PRE);
    if (m) {
        st.status = DS_INVALID;
        st.msg = m;
        return;
    }
    const uint32_t total = hlit + hdist;
    for (uint32_t i = 0; i < total; i++) scr->lengths[i] = 0;
    uint32_t i = 0;
    while (i < total) {
        br_refill(b);
        const uint32_t e = T.dist[b.buf & ((1u << PRE_BITS) - 1)];
        const uint32_t cl = e & 15;
        if (!cl) {
            st.status = DS_INVALID;
            st.msg = MSG_NO_CODE;
            return;
        }
        br_consume(b, cl);
        const uint32_t sym = e >> 8;
        if (sym <= 15) {
            scr->lengths[i++] = (uint8_t)sym;
        } else if (sym == 16) {
            if (i == 0) {
                st.status = DS_INVALID;
                st.msg = MSG_CODE16_FIRST;
                return;
            }
            const uint32_t r = br_read(b, 2) + 3;
            if (i + r > total) {
                st.status = DS_INVALID;
                st.msg = MSG_CODE16_OVER;
                return;
            }
            const uint8_t prev = scr->lengths[i - 1];
            for (uint32_t j = 0; j < r; j++) scr->lengths[i + j] = prev;
            i += r;
        } else if (sym == 17) {
            const uint32_t r = br_read(b, 3) + 3;
            if (i + r > total) {
                st.status = DS_INVALID;
                st.msg = MSG_CODE17_OVER;
                return;
            }
            i += r;
        } else {
            const uint32_t r = br_read(b, 7) + 11;
            if (i + r > total) {
                st.status = DS_INVALID;
                st.msg = MSG_CODE18_OVER;
                return;
            }
            i += r;
        }
        if (br_past_end(b)) {
            st.status = DS_EOF;
            return;
        }
    }
    if (scr->lengths[256] == 0) {
        st.status = DS_INVALID;
        st.msg = MSG_EOB_ZERO;
        return;
    }
    m = lane_build(scr->lengths, (int)hlit, T.lit, LL_BITS, T.lfirst, T.lcount, T.loff, scr->lsorted, TK_LITLEN);
    if (!m)
        m = lane_build(scr->lengths + hlit, (int)hdist, T.dist, DL_BITS, T.dfirst, T.dcount, T.doff, scr->dsorted,
                       TK_DIST);
    if (m) {
        st.status = DS_INVALID;
        st.msg = m;
    }
}

__device__ void lane_fixed(LaneState& st, LaneTab& T, LaneScratch* scr) {
    for (int i = 0; i < 288; i++) scr->lengths[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : 8;
    for (int i = 0; i < 30; i++) scr->lengths[288 + i] = 5;
    lane_build(scr->lengths, 288, T.lit, LL_BITS, T.lfirst, T.lcount, T.loff, scr->lsorted, TK_LITLEN);
    lane_build(scr->lengths + 288, 30, T.dist, DL_BITS, T.dfirst, T.dcount, T.doff, scr->dsorted, TK_DIST);
    (void)st;
}

template <typename CellT>
__device__ void lane_stored(LaneState& st, CellT* out) {
    BR& b = st.br;
    br_consume(b, b.bits & 7);
    const uint32_t len = br_read(b, 16), nlen = br_read(b, 16);
    if ((len ^ 0xffffu) != nlen) {
        st.status = DS_INVALID;
        st.msg = MSG_STORED_NLEN;
        return;
    }
    const uint64_t bp = br_tell(b) >> 3;
    if (b.s.lo + bp + len > b.s.hi) {
        st.status = DS_EOF;
        return;
    }
    if (!st.counting && st.cur + len > st.cap) st.counting = true;
    if (!st.counting)
        for (uint32_t i = 0; i < len; i++) out[st.cur + i] = (CellT)src_byte(b.s, bp + i);
    st.cur += len;
    br_seek(b, (bp + len) * 8);
}

template <typename CellT>
__device__ void lane_item(const InflateArgs& A, uint32_t item_idx, LaneTab& T, LaneScratch* scr, const LaneConsts& K) {
    const ChunkItem it = A.items[item_idx];
    if (it.flags & ITEM_SKIP) {
        A.results[item_idx] = ChunkResult{0, it.start_bit, DS_OK, 0, 0, 0, 0, 0};
        return;
    }
    CellT* out = (CellT*)A.out + it.out_off;
    LaneState st;
    st.br.s = make_src(A.in + it.in_off, it.in_len);
    st.br.nw = 0;
    st.br.buf = 0;
    st.br.bits = 0;
    st.cur = 0;
    st.cap = it.out_cap;
    st.member_start = 0;
    st.markers = 0;
    st.status = 0;
    st.msg = 0;
    st.markers_ok = (it.flags & ITEM_MARKERS) != 0 && sizeof(CellT) == 2;
    st.counting = false;
    const uint64_t body_len = it.in_len;
    uint64_t start = it.start_bit;
    uint32_t trailer_crc = 0, trailer_isize = 0;
    if (it.flags & ITEM_ONE_MEMBER) {
        uint64_t hl = 0;
        int msg = 0;
        st.status = dev_parse_header(st.br.s, 0, &hl, &msg);
        st.msg = msg;
        start = hl * 8;
    }
    if (!st.status) {
        if (start > body_len * 8) st.status = DS_EOF;
        else br_seek(st.br, start);
    }
    bool final_block = false, fixed_loaded = false;
    uint32_t n_members = 0;
    uint64_t end_bit = 0;
    while (!st.status) {
        if (br_tell(st.br) >= it.end_hint) break;
        uint32_t bfinal = 0;
        for (;;) {
            bfinal = br_read(st.br, 1);
            const uint32_t bt = br_read(st.br, 2);
            if (br_past_end(st.br)) {
                st.status = DS_EOF;
                break;
            }
            if (bt == 0) {
                lane_stored<CellT>(st, out);
            } else if (bt == 1) {
                if (!fixed_loaded) lane_fixed(st, T, scr);
                fixed_loaded = true;
                lane_codes<CellT>(st, T, scr, K, out);
            } else if (bt == 2) {
                fixed_loaded = false;
                lane_dynamic(st, T, scr);
                if (!st.status) lane_codes<CellT>(st, T, scr, K, out);
            } else {
                st.status = DS_INVALID;
                st.msg = MSG_RESERVED_BTYPE;
            }
            if (st.status || bfinal) break;
            if (br_tell(st.br) >= it.end_hint) break;
        }
        if (st.status || !bfinal) break;
        br_consume(st.br, st.br.bits & 7);
        const uint64_t tb = br_tell(st.br) >> 3;
        if (tb + 8 > body_len) {
            st.status = DS_TRUNCATED;
            break;
        }
        trailer_crc = le32_at(st.br.s, tb);
        trailer_isize = le32_at(st.br.s, tb + 4);
        if (!(it.flags & ITEM_ONE_MEMBER)) {
            const uint32_t slot = atomicAdd(A.mb_count, 1u);
            if (slot < A.mb_cap) {
                MemberRec r;
                r.item = it.id;
                r.seq = n_members;
                r.cell_off = st.cur;
                r.crc = trailer_crc;
                r.isize = trailer_isize;
                r.trailer_byte = tb;
                A.mbs[slot] = r;
            }
        }
        n_members++;
        const uint64_t after = tb + 8;
        if (after >= body_len || (it.flags & ITEM_ONE_MEMBER)) {
            final_block = true;
            end_bit = after * 8;
            break;
        }
        uint64_t hl = 0;
        int msg = 0;
        st.status = dev_parse_header(st.br.s, after, &hl, &msg);
        st.msg = msg;
        if (st.status) break;
        br_seek(st.br, (after + hl) * 8);
        st.member_start = st.cur;
        st.markers_ok = false;
    }
    ChunkResult r;
    r.n_cells = st.cur;
    r.actual_end_bit = final_block ? end_bit : br_tell(st.br);
    r.status = st.status ? st.status : (st.counting ? DS_OVERFLOW : DS_OK);
    r.msg = st.msg;
    r.final_block = final_block ? 1 : 0;
    r.n_members = n_members;
    r.markers = (it.flags & ITEM_ONE_MEMBER) ? (((uint64_t)trailer_isize << 32) | trailer_crc) : st.markers;
    r.err_bit = br_tell(st.br);
    A.results[item_idx] = r;
}

template <typename CellT>
__global__ void __launch_bounds__(LANE_THREADS) k_inflate_lanes(InflateArgs A, LaneScratch* scratch) {
    RRG_DYN_SMEM(smem_raw);
    __shared__ LaneConsts K;
    for (int i = threadIdx.x; i < 32; i += blockDim.x) {
        K.lbase[i] = i < 29 ? c_len_base[i] : 0;
        K.lextra[i] = i < 29 ? c_len_extra[i] : 0;
        K.dbase[i] = i < 30 ? c_dist_base[i] : 0;
        K.dextra[i] = i < 30 ? c_dist_extra[i] : 0;
    }
    __syncthreads();
    LaneTab& T = reinterpret_cast<LaneTab*>(smem_raw)[threadIdx.x];
    LaneScratch* scr = scratch + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (;;) {
        const uint32_t idx = atomicAdd(A.queue, 1u);
        if (idx >= (A.n_items_dev ? *A.n_items_dev : A.n_items)) break;
        lane_item<CellT>(A, A.order ? A.order[idx] : idx, T, scr, K);
    }
}

// ------------------------------------------------------- block finder
// One warp per target; the search runs over tiles of 1024 bit offsets that
// start at the current skip-chain position. For its 32 offsets each lane
// computes, from five register-resident input words:
//   * the 13-bit prefilter skip of block_finder.rs:60-101 (BFINAL=0, BTYPE=2,
//     HLIT<=29, HDIST<=29; 0 = candidate), and
//   * for candidates, the strict Kraft test of the HCLEN precode lengths.
// The rare offsets that pass both get the full strict verification of
// block_finder.rs:175-301 (precode, code lengths, complete litlen/dist trees,
// EOB length, 64 trial symbols) done by the whole warp with shared-memory
// tables. The reference walks the skip chain one offset at a time; here each
// lane turns its 32-offset segment into a transfer table (for every entry
// offset 0..12: exit offset into the next segment, or the first verified
// offset met), and lane 0 composes the 32 tables. The result is exactly the
// offset find_next_dynamic_block returns.
constexpr int FIND_TILE = 1024;
constexpr uint32_t STEP_END = 14;  // offset + 13 > limit: the scan stops

struct FindArgs {
    const uint8_t* body;
    uint64_t body_len;
    const uint64_t* targets;
    const uint64_t* limits;
    uint64_t* found;
    uint32_t n;
    uint32_t* queue;
    const uint8_t* next_lut;  // 8192 entries
    uint32_t tile;            // unused (tile width is fixed at 1024 offsets)
};

struct FindSmem {
    uint32_t lit_lut[LUT_SIZE];
    uint32_t dist_lut[LUT_SIZE];
    uint32_t pre_lut[1 << PRE_BITS];
    uint16_t lit_sorted[288];
    uint16_t dist_sorted[32];
    uint16_t pre_sorted[32];
    uint16_t lit_first[16], lit_count[16], lit_off[16];
    uint16_t dist_first[16], dist_count[16], dist_off[16];
    uint16_t pre_first[16], pre_count[16], pre_off[16];
    uint16_t run[16];
    uint8_t lengths[320];
    uint8_t pre_len[20];
    uint8_t trans[32][16];
};

// 32 bits starting at bit b (b < 128) of the 5-word register window W.
__device__ __forceinline__ uint32_t win_bits(const uint32_t W[5], uint32_t b) {
    const uint32_t q = b >> 5, r = b & 31;
    const uint32_t lo = q == 0 ? W[0] : q == 1 ? W[1] : q == 2 ? W[2] : W[3];
    const uint32_t hi = q == 0 ? W[1] : q == 1 ? W[2] : q == 2 ? W[3] : W[4];
    return r ? ((lo >> r) | (hi << (32 - r))) : lo;
}

// bits [pos, pos+n) of the source (n <= 25)
__device__ __forceinline__ uint32_t peek_at(const Src& s, uint64_t pos, uint32_t n) {
    const uint64_t a = pos + s.lo * 8;
    const uint64_t w = a >> 5;
    const uint64_t v = (uint64_t)src_word(s, w) | ((uint64_t)src_word(s, w + 1) << 32);
    return (uint32_t)(v >> (a & 31)) & ((1u << n) - 1u);
}

// Reference-exact reads on lane 0: a read of n bits needs n bits left.
struct VC {
    const Src* s;
    uint64_t pos, total;
    bool ok;
    __device__ uint32_t read(uint32_t n) {
        if (!ok || pos + n > total) {
            ok = false;
            return 0;
        }
        uint32_t v = n ? peek_at(*s, pos, n) : 0;
        pos += n;
        return v;
    }
    // HuffmanDecoder::decode (huffman.rs:356-389): 10 bits must be available
    // for the LUT probe, 15 for a long code.
    __device__ uint32_t sym(const Table& T, int lut_bits) {
        if (!ok || pos + 10 > total) {
            ok = false;
            return 0;
        }
        const uint32_t avail = total - pos >= 25 ? 25u : (uint32_t)(total - pos);
        const uint32_t bits = peek_at(*s, pos, avail);
        uint32_t e = T.lut[bits & ((1u << lut_bits) - 1u)];
        if (!(e & 15)) {
            if (pos + 15 > total) {
                ok = false;
                return 0;
            }
            e = long_decode(bits, T, lut_bits, TK_PRE);
            if (!(e & 15)) {
                ok = false;
                return 0;
            }
        }
        pos += e & 15;
        return e >> 16;
    }
};

// Full strict verification of one candidate offset (warp-uniform call).
// With `next_header`, a trial that meets the end-of-block code also reads the
// header of the block that must follow (BFINAL is 0 in every candidate):
// BTYPE 3, HLIT > 286, HDIST > 30 or a stored LEN/NLEN mismatch reject the
// candidate. The reference's trial stops at the end-of-block code; a false
// header whose trees reach it within a few symbols then passes (one such
// offset is in 256 MiB of level-9 text), so the boundary scan, whose
// survivors only become sub-chunk starts, asks for this check; the
// reference-exact finder does not.
__device__ __noinline__ bool verify_heavy(FindSmem& S, const Src& src, uint64_t total_bits, uint64_t pos, int lane,
                                          bool next_header = false) {
    int ok = 1;
    uint32_t hlit = 0, hdist = 0;
    uint64_t cur = 0;
    if (lane == 0) {
        VC c{&src, pos, total_bits, true};
        c.read(3);
        hlit = c.read(5) + 257;
        hdist = c.read(5) + 1;
        uint32_t hclen = c.read(4) + 4;
        for (int i = 0; i < 19; i++) S.pre_len[i] = 0;
        if (hlit > 286 || hdist > 30) c.ok = false;
        for (uint32_t i = 0; i < hclen && c.ok; i++) S.pre_len[c_cl_order[i]] = (uint8_t)c.read(3);
        ok = c.ok ? 1 : 0;
        cur = c.pos;
    }
    ok = bcast32(ok);
    hlit = (uint32_t)bcast32((int32_t)hlit);
    hdist = (uint32_t)bcast32((int32_t)hdist);
    cur = bcast64(cur);
    if (!ok) return false;
    __syncwarp();
    const Table PT{S.pre_lut, S.pre_sorted, S.pre_first, S.pre_count, S.pre_off};
    if (warp_build(S.pre_len, 19, PT, PRE_BITS, TK_PRE, S.run, lane, true)) return false;
    for (int i = lane; i < 320; i += 32) S.lengths[i] = 0;
    __syncwarp();
    if (lane == 0) {
        VC c{&src, cur, total_bits, true};
        const uint32_t total = hlit + hdist;
        uint32_t i = 0;
        while (i < total && c.ok) {
            uint32_t sym = c.sym(PT, PRE_BITS);
            if (!c.ok) break;
            if (sym <= 15) {
                S.lengths[i++] = (uint8_t)sym;
            } else if (sym == 16) {
                if (i == 0) c.ok = false;
                uint32_t r = c.read(2) + 3;
                if (!c.ok || i + r > total) {
                    c.ok = false;
                    break;
                }
                for (uint32_t j = 0; j < r; j++) S.lengths[i + j] = S.lengths[i - 1];
                i += r;
            } else if (sym == 17) {
                uint32_t r = c.read(3) + 3;
                if (!c.ok || i + r > total) c.ok = false;
                i += r;
            } else if (sym == 18) {
                uint32_t r = c.read(7) + 11;
                if (!c.ok || i + r > total) c.ok = false;
                i += r;
            } else {
                c.ok = false;
            }
        }
        if (c.ok && S.lengths[256] == 0) c.ok = false;
        ok = c.ok ? 1 : 0;
        cur = c.pos;
    }
    ok = bcast32(ok);
    cur = bcast64(cur);
    if (!ok) return false;
    __syncwarp();
    const Table LT{S.lit_lut, S.lit_sorted, S.lit_first, S.lit_count, S.lit_off};
    const Table DT{S.dist_lut, S.dist_sorted, S.dist_first, S.dist_count, S.dist_off};
    if (warp_build(S.lengths, (int)hlit, LT, LUT_BITS, TK_PRE, S.run, lane, true)) return false;
    if (warp_build(S.lengths + hlit, (int)hdist, DT, LUT_BITS, TK_PRE, S.run, lane, true)) return false;
    if (lane == 0) {
        VC c{&src, cur, total_bits, true};
        bool done = false;
        for (int k = 0; k < 64 && c.ok && !done; k++) {
            uint32_t sym = c.sym(LT, LUT_BITS);
            if (!c.ok) break;
            if (sym < 256) continue;
            if (sym == 256) {
                done = true;
                if (next_header) {
                    c.read(1);
                    const uint32_t bt = c.read(2);
                    if (bt == 3) {
                        c.ok = false;
                    } else if (bt == 2) {
                        const uint32_t hl = c.read(5) + 257, hd = c.read(5) + 1;
                        if (hl > 286 || hd > 30) c.ok = false;
                    } else if (bt == 0) {
                        c.read((uint32_t)((8 - (c.pos & 7)) & 7));
                        const uint32_t len = c.read(16), nlen = c.read(16);
                        if ((len ^ nlen) != 0xffffu) c.ok = false;
                    }
                }
                break;
            }
            if (sym > 285) {
                c.ok = false;
                break;
            }
            c.read(c_len_extra[sym - 257]);
            uint32_t ds = c.sym(DT, LUT_BITS);
            if (!c.ok || ds >= 30) {
                c.ok = false;
                break;
            }
            c.read(c_dist_extra[ds]);
        }
        ok = c.ok ? 1 : 0;
    }
    ok = bcast32(ok);
    __syncwarp();
    return ok != 0;
}

__global__ void __launch_bounds__(128) k_find_blocks(FindArgs A) {
    RRG_DYN_SMEM(smem_raw);
    __shared__ uint8_t lut[8192];
    for (int i = threadIdx.x; i < 8192; i += blockDim.x) lut[i] = A.next_lut[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    FindSmem& S = reinterpret_cast<FindSmem*>(smem_raw)[warp];
    const Src src = make_src(A.body, A.body_len);
    const uint64_t total_bits = A.body_len * 8;
    for (;;) {
        uint32_t idx = 0;
        if (lane == 0) idx = atomicAdd(A.queue, 1u);
        idx = (uint32_t)bcast32((int32_t)idx);
        if (idx >= A.n) break;
        const uint64_t from = A.targets[idx];
        const uint64_t limit = A.limits[idx] < total_bits ? A.limits[idx] : total_bits;
        uint64_t result = ~0ull;
        uint64_t pos = from;
        bool done = from >= limit || from + 13 > limit;
        while (!done) {
            const uint64_t tb = pos;
            // ---- per-offset prefilter + precode test for this lane's 32 offsets
            const uint64_t seg = tb + 32ull * lane;
            const uint64_t a = seg + src.lo * 8;
            const uint64_t w0 = a >> 5;
            const uint32_t sh = (uint32_t)(a & 31);
            uint32_t W[5];
            for (int q = 0; q < 5; q++) W[q] = src_word(src, w0 + q);
            uint64_t stepA = 0, stepB = 0;
            uint32_t pre = 0;
            for (uint32_t i = 0; i < 32; i++) {
                uint32_t st;
                if (seg + i + 13 > limit) {
                    st = STEP_END;
                } else {
                    const uint32_t b = sh + i;
                    st = lut[win_bits(W, b) & 0x1fffu];
                    if (st == 0) {
                        const uint32_t hclen = (win_bits(W, b + 13) & 15u) + 4;
                        const uint32_t y = win_bits(W, b + 17), z = win_bits(W, b + 47);
                        uint32_t kraft = 0, nsym = 0;
#pragma unroll
                        for (uint32_t j = 0; j < 19; j++) {
                            const uint32_t l = j < 10 ? (y >> (3 * j)) & 7u : (z >> (3 * (j - 10))) & 7u;
                            if (j < hclen && l) {
                                kraft += 128u >> l;
                                nsym++;
                            }
                        }
                        if (nsym < 2 || kraft == 128u) pre |= 1u << i;
                    }
                }
                if (i < 16) stepA |= (uint64_t)st << (4 * i);
                else stepB |= (uint64_t)st << (4 * (i - 16));
            }
            // ---- full verification of the offsets that passed the precode test
            uint32_t okm = 0;
            unsigned todo = __ballot_sync(FULLMASK, pre != 0);
            while (todo) {
                const int L = __ffs(todo) - 1;
                uint32_t m = __shfl_sync(FULLMASK, pre, L);
                while (m) {
                    const int i = __ffs(m) - 1;
                    m &= m - 1;
                    const bool ok = verify_heavy(S, src, total_bits, tb + 32ull * L + i, lane);
                    if (ok && lane == L) okm |= 1u << i;
                }
                todo &= todo - 1;
            }
            // ---- transfer table of this lane's segment for entry offsets 0..12
            for (uint32_t e = 0; e < 13; e++) {
                uint32_t p = e, res = 0xFFu;
                while (p < 32) {
                    const uint32_t st = (uint32_t)((p < 16 ? stepA >> (4 * p) : stepB >> (4 * (p - 16))) & 15u);
                    if (st == STEP_END) {
                        res = 0xFEu;
                        break;
                    }
                    if (st == 0) {
                        if ((okm >> p) & 1u) {
                            res = 0x80u | p;
                            break;
                        }
                        p += 1;
                    } else {
                        p += st;
                    }
                }
                S.trans[lane][e] = (uint8_t)(res == 0xFFu ? p - 32 : res);
            }
            __syncwarp();
            int d = 0;
            uint64_t np = 0, res = ~0ull;
            if (lane == 0) {
                uint32_t e = 0;
                for (int sgi = 0; sgi < 32; sgi++) {
                    const uint32_t t = S.trans[sgi][e];
                    if (t == 0xFEu) {
                        d = 1;
                        break;
                    }
                    if (t & 0x80u) {
                        res = tb + 32ull * sgi + (t & 0x7fu);
                        d = 1;
                        break;
                    }
                    e = t;
                }
                np = tb + FIND_TILE + e;
            }
            d = bcast32(d);
            np = bcast64(np);
            res = bcast64(res);
            __syncwarp();
            if (d) {
                result = res;
                done = true;
            }
            pos = np;
            if (pos + 13 > limit) done = true;
        }
        if (lane == 0) A.found[idx] = result;
        __syncwarp();
    }
}

// ------------------------------------------------------- full-stream candidate scan
// The decode path needs many block boundaries, not the reference's one per
// target, so it tests every bit offset of the body: 4 KiB tiles staged in
// shared memory with 16-byte loads, each thread testing the 128 offsets of
// its 16 bytes (prefilter BFINAL=0, BTYPE=2, HLIT<=29, HDIST<=29, then the
// strict Kraft test of the precode). A tile's survivors are appended to a
// shared-memory list with shared atomics and copied out with one global
// atomicAdd per tile.
// k_verify_light then applies the strict code-length checks of
// read_dynamic_header_strict_into (block_finder.rs:196-262) per thread, and
// the last survivors get verify_heavy (tables + 64 trial symbols).
constexpr int SCAN_HALO = 48;  // the last thread reads up to 2.5 words past its 16 bytes

struct ScanArgs {
    const uint8_t* body;
    uint64_t body_len;
    uint64_t* cand;
    uint32_t* n_cand;
    uint32_t cap;
    uint64_t* stored;       // stored-block starts (bit offsets), appended
    uint32_t* n_stored;
    uint32_t stored_cap;
    uint64_t tile_lo, tile_hi;  // the tiles this launch covers (input that has arrived)
    const uint32_t* tile_list;  // when set: only these tiles (sorted), n_list of them
    uint32_t n_list;
};

// 32 bits of the staged tile starting at bit b (b + 32 <= 8 * tile bytes)
__device__ __forceinline__ uint32_t tile_bits(const uint32_t* tw, uint32_t b) {
    const uint32_t q = b >> 5, r = b & 31;
    return __funnelshift_r(tw[q], tw[q + 1], r);
}

constexpr int SCAN_LIST = 1024;  // candidates a tile stages in shared memory before one global append

// ST threads per block; a tile is ST * 16 bytes (the finder tile width knob)
template <int ST>
__global__ void __launch_bounds__(ST) k_scan_candidates(ScanArgs A) {
    constexpr int TILE = ST * 16;
    __shared__ __align__(16) uint32_t tile[(TILE + SCAN_HALO) / 4];
    __shared__ uint32_t s_list[SCAN_LIST];
    __shared__ uint32_t s_n, s_base;
    __shared__ uint32_t s_kt[64];  // two precode lengths -> Kraft weight (128 >> l) | count << 16
    if (threadIdx.x < 64) {
        const uint32_t l1 = threadIdx.x & 7u, l2 = threadIdx.x >> 3;
        s_kt[threadIdx.x] = (l1 ? 128u >> l1 : 0u) + (l2 ? 128u >> l2 : 0u) + (((l1 ? 1u : 0u) + (l2 ? 1u : 0u)) << 16);
    }
    const uintptr_t addr = (uintptr_t)A.body;
    const uint8_t* base = (const uint8_t*)(addr & ~(uintptr_t)15);
    const uint64_t lo = addr & 15, hi = lo + A.body_len;
    const uint64_t n_tiles = (hi + TILE - 1) / TILE;
    const uint64_t t_end = A.tile_hi < n_tiles ? A.tile_hi : n_tiles;
    uint8_t* tb = reinterpret_cast<uint8_t*>(tile);
    const uint64_t n_iter = A.tile_list ? A.n_list : (t_end > A.tile_lo ? t_end - A.tile_lo : 0);
    for (uint64_t it = blockIdx.x; it < n_iter; it += gridDim.x) {
        const uint64_t t = A.tile_list ? A.tile_list[it] : A.tile_lo + it;
        if (t >= n_tiles) continue;  // uniform over the block
        const uint64_t t0 = t * TILE;
        if (threadIdx.x == 0) s_n = 0;
        for (uint32_t q = threadIdx.x; q < (TILE + SCAN_HALO) / 16; q += blockDim.x) {
            const uint64_t b0 = t0 + 16ull * q;
            if (b0 >= lo && b0 + 16 <= hi) {
                *reinterpret_cast<uint4*>(tb + 16 * q) = __ldg(reinterpret_cast<const uint4*>(base + b0));
            } else {
                for (int k = 0; k < 16; k++) {
                    const uint64_t p = b0 + k;
                    tb[16 * q + k] = (p >= lo && p < hi) ? __ldg(base + p) : 0;
                }
            }
        }
        __syncthreads();
        // stored blocks (no reference counterpart: its finder looks for dynamic
        // blocks only). A stored block that follows a stored block, or an empty
        // sync-flush block, starts at a byte: header byte 0x00 (BFINAL=0,
        // BTYPE=00, zero padding), then LEN and NLEN = ~LEN. To keep chance
        // matches inside compressed data (about one per 8 MB) from becoming
        // chunk starts, a non-empty block counts only if another stored block
        // header follows its data. This thread tests the header byte at each of
        // its 16 bytes, so LEN..NLEN reach 4 bytes into the halo. A false start
        // would only cost the anchored chain a re-decode.
        {
            const uint32_t b0 = threadIdx.x * 16;
#pragma unroll 4
            for (uint32_t k = 0; k < 16; k++) {
                const uint32_t j = b0 + k;
                const uint64_t g = t0 + j;  // header byte, relative to `base`
                if (tb[j] == 0u && g >= lo && g + 5 <= hi) {
                    const uint32_t len = tb[j + 1] | ((uint32_t)tb[j + 2] << 8);
                    const uint32_t nlen = tb[j + 3] | ((uint32_t)tb[j + 4] << 8);
                    bool ok = (len ^ nlen) == 0xffffu;
                    if (ok && len) {
                        const uint64_t q = g + 5 + len;  // the next block's header byte
                        ok = q + 5 <= hi && __ldg(base + q) <= 1u &&
                             ((__ldg(base + q + 1) | ((uint32_t)__ldg(base + q + 2) << 8)) ^
                              (__ldg(base + q + 3) | ((uint32_t)__ldg(base + q + 4) << 8))) == 0xffffu;
                    }
                    if (ok) {  // bit 0 of the (byte-aligned) offset marks an empty block
                        const uint32_t slot = atomicAdd(A.n_stored, 1u);
                        if (slot < A.stored_cap) A.stored[slot] = (g - lo) * 8 + (len ? 0u : 1u);
                    }
                }
            }
        }
        // phase 1: prefilter every offset of this thread's 16 bytes (4 groups of 32)
        const uint64_t tile_bit0 = t0 * 8;
        const uint32_t w0 = threadIdx.x * 4;
        uint32_t mask[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t a = tile[w0 + q], b = tile[w0 + q + 1];
            // bit-sliced over the 32 offsets: bit r of f(k) is header bit k at offset r.
            // BFINAL=0, BTYPE=2 (bits 0,1,2 = 0,0,1); HLIT <= 29 and HDIST <= 29
            // (not bits 4-7 all set, not bits 9-12 all set)
#define RRG_F(k) __funnelshift_r(a, b, k)
            uint32_t m = ~RRG_F(0) & ~RRG_F(1) & RRG_F(2) & ~(RRG_F(4) & RRG_F(5) & RRG_F(6) & RRG_F(7)) &
                         ~(RRG_F(9) & RRG_F(10) & RRG_F(11) & RRG_F(12));
#undef RRG_F
            // only offsets p with lo*8 <= p and p + 13 <= hi*8 are tested
            const uint64_t g0 = tile_bit0 + 32ull * (w0 + q);
            if (g0 < lo * 8 || g0 + 32 + 13 > hi * 8) {
                for (int r = 0; r < 32; r++) {
                    const uint64_t pa = g0 + r;
                    if (pa < lo * 8 || pa + 13 > hi * 8) m &= ~(1u << r);
                }
            }
            mask[q] = m;
        }
        // phase 2: strict precode Kraft test of each candidate
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint32_t m = mask[q];
            while (m) {
                const uint32_t r = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t boff = 32 * (w0 + q) + r;  // bit offset inside the tile
                const uint32_t hclen = (tile_bits(tile, boff + 13) & 15u) + 4;
                uint32_t y = tile_bits(tile, boff + 17), z = tile_bits(tile, boff + 47);
                // lengths past HCLEN are absent: clear their fields, then sum
                // the Kraft weights and counts two 3-bit lengths per lookup
                if (hclen <= 10) {
                    y &= (1u << (3 * hclen)) - 1u;
                    z = 0;
                } else {
                    y &= (1u << 30) - 1u;
                    z &= (1u << (3 * (hclen - 10))) - 1u;
                }
                uint32_t acc = 0;
#pragma unroll
                for (int j = 0; j < 5; j++) acc += s_kt[(y >> (6 * j)) & 63u] + s_kt[(z >> (6 * j)) & 63u];
                const uint32_t kraft = acc & 0xffffu, nsym = acc >> 16;
                if (nsym < 2 || kraft == 128u) {
                    const uint32_t k = atomicAdd(&s_n, 1u);
                    if (k < SCAN_LIST) {
                        s_list[k] = boff;
                    } else {  // a crowded tile: straight to the global list
                        const uint32_t slot = atomicAdd(A.n_cand, 1u);
                        if (slot < A.cap) A.cand[slot] = tile_bit0 + boff - lo * 8;
                    }
                }
            }
        }
        // one global append per tile for the staged candidates
        __syncthreads();
        const uint32_t ns = s_n < SCAN_LIST ? s_n : SCAN_LIST;
        if (threadIdx.x == 0) s_base = ns ? atomicAdd(A.n_cand, ns) : 0u;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x)
            if (s_base + i < A.cap) A.cand[s_base + i] = tile_bit0 + s_list[i] - lo * 8;
        __syncthreads();
    }
}

struct VerifyArgs {
    const uint8_t* body;
    uint64_t body_len;
    const uint64_t* cand;
    const uint32_t* n_ptr;  // number of candidates (device word written by the previous kernel)
    uint32_t cap;           // entries of `cand` that exist
    uint64_t* out;          // survivors, appended
    uint32_t* n_out;
    uint32_t out_cap;
    uint8_t* ok;            // k_verify_heavy: per-survivor verdict
    uint32_t* queue;
    const uint32_t* lo_ptr;  // k_verify_light: candidates before this index are done (null: none)
};

// strict code-length parse without building tables: litlen and distance Kraft
// sums are accumulated as the lengths are decoded.
__device__ bool verify_light(const Src& s, uint64_t total_bits, uint64_t pos, uint8_t* lut) {
    VC c{&s, pos, total_bits, true};
    c.read(3);
    const uint32_t hlit = c.read(5) + 257, hdist = c.read(5) + 1, hclen = c.read(4) + 4;
    if (!c.ok || hlit > 286 || hdist > 30) return false;
    // precode lengths, 3 bits per symbol, and the count of each length (5-bit fields)
    uint64_t cl = 0;
    for (uint32_t i = 0; i < hclen; i++) cl |= (uint64_t)c.read(3) << (3 * c_cl_order[i]);
    if (!c.ok) return false;
    uint64_t cnt = 0;
    uint32_t k = 0, ns = 0;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const uint32_t l = (uint32_t)(cl >> (3 * i)) & 7u;
        if (l) {
            cnt += 1ull << (5 * l);
            k += 128u >> l;
            ns++;
        }
    }
    if (ns >= 2 && k != 128u) return false;
    // 7-bit decode table: entry = symbol << 3 | length (0 = no code). Canonical
    // codes (RFC 1951 3.2.2) in symbol order; next codes in 8-bit fields.
    uint64_t next = 0;
    {
        uint32_t code = 0;
#pragma unroll
        for (int l = 1; l <= 7; l++) {
            code = (code + (l > 1 ? (uint32_t)(cnt >> (5 * (l - 1))) & 31u : 0u)) << 1;
            next |= (uint64_t)code << (8 * l);
        }
    }
    for (int i = 0; i < 128; i += 16) *reinterpret_cast<uint4*>(lut + i) = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const uint32_t l = (uint32_t)(cl >> (3 * i)) & 7u;
        if (l) {
            const uint32_t code = (uint32_t)(next >> (8 * l)) & 0xffu;
            next += 1ull << (8 * l);
            const uint32_t rev = __brev(code) >> (32 - l);
            for (uint32_t x = rev; x < 128u; x += 1u << l) lut[x] = (uint8_t)((i << 3) | l);
        }
    }
    const uint32_t total = hlit + hdist;
    uint32_t i = 0, prev = 0, len256 = 0;
    uint32_t kl = 0, nl = 0, kd = 0, nd = 0;
    auto put = [&](uint32_t L) {
        if (i < hlit) {
            if (L) {
                kl += 1u << (15 - L);
                nl++;
            }
            if (i == 256) len256 = L;
        } else if (L) {
            kd += 1u << (15 - L);
            nd++;
        }
        i++;
    };
    while (i < total) {
        // precode symbol: HuffmanDecoder::decode needs 10 bits available
        if (c.pos + 10 > c.total) return false;
        const uint32_t e = lut[peek_at(s, c.pos, 7)];
        if (!e) return false;
        // an oversubscribed code stays oversubscribed (the final test needs
        // sums of exactly 2^15): stop at the first symbol that overshoots
        if (kl > 32768u || kd > 32768u) return false;
        c.pos += e & 7u;
        const uint32_t got = e >> 3;
        if (got <= 15) {
            prev = got;
            put(prev);
        } else if (got == 16) {
            if (i == 0) return false;
            const uint32_t r = c.read(2) + 3;
            if (!c.ok || i + r > total) return false;
            for (uint32_t j = 0; j < r; j++) put(prev);
        } else {
            const uint32_t r = got == 17 ? c.read(3) + 3 : c.read(7) + 11;
            if (!c.ok || i + r > total) return false;
            for (uint32_t j = 0; j < r; j++) put(0);
            prev = 0;
        }
    }
    if (len256 == 0) return false;
    if (nl >= 2 && kl != 32768u) return false;
    if (nd >= 2 && kd != 32768u) return false;
    return true;
}

// Survivors are appended to A.out (order is restored on the host).
__global__ void __launch_bounds__(256) k_verify_light(VerifyArgs A) {
    __shared__ __align__(16) uint8_t s_lut[256 * 128];  // one precode table per thread
    const Src s = make_src(A.body, A.body_len);
    const uint64_t total_bits = A.body_len * 8;
    const uint32_t n = *A.n_ptr < A.cap ? *A.n_ptr : A.cap;
    const uint32_t lo = A.lo_ptr ? *A.lo_ptr : 0u;
    uint8_t* lut = s_lut + threadIdx.x * 128;
    for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t pos = A.cand[i];
        if (verify_light(s, total_bits, pos, lut)) {
            const uint32_t slot = atomicAdd(A.n_out, 1u);
            if (slot < A.out_cap) A.out[slot] = pos;
        }
    }
}

// After the verification of one input piece's candidates (host path, input
// still arriving): the next light launch starts after the candidates seen so
// far, the next heavy launch's queue after the survivors seen so far.
// counts: [0] candidates, [1] survivors, [2] heavy queue, [4] light start.
__global__ void k_verify_mark(uint32_t* counts, uint32_t cap, uint32_t cap2) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        counts[4] = counts[0] < cap ? counts[0] : cap;
        counts[2] = counts[1] < cap2 ? counts[1] : cap2;
    }
}

// One warp per light survivor: tables + 64 trial symbols (verify_heavy).
__global__ void __launch_bounds__(128) k_verify_heavy(VerifyArgs A) {
    RRG_DYN_SMEM(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    FindSmem& S = reinterpret_cast<FindSmem*>(smem_raw)[warp];
    const Src s = make_src(A.body, A.body_len);
    const uint64_t total_bits = A.body_len * 8;
    const uint32_t n = *A.n_ptr < A.cap ? *A.n_ptr : A.cap;
    for (;;) {
        uint32_t idx = 0;
        if (lane == 0) idx = atomicAdd(A.queue, 1u);
        idx = (uint32_t)bcast32((int32_t)idx);
        if (idx >= n) break;
        const bool ok = verify_heavy(S, s, total_bits, A.cand[idx], lane, true);
        if (lane == 0) A.ok[idx] = ok ? 1 : 0;
        __syncwarp();
    }
}

// ------------------------------------------------------- fixed-Huffman block starts
// A fixed-Huffman block (BTYPE=01, RFC 1951 §3.2.6) has no code-length header
// to test, so the candidate scan cannot see where one starts. The reference's
// finder looks for dynamic blocks only (block_finder.rs:60-78), and a stream of
// fixed blocks (zlib's Z_FIXED strategy, or short or low-entropy blocks at low
// levels) would decode as one sub-chunk. Instead of testing offsets, one thread
// walks the fixed code from a target bit: a prefix code resynchronises with
// the true symbol boundaries within a few symbols, so after FW_WARM symbols
// without an end-of-block or invalid code the walk is on the real symbol path
// and the next end-of-block code it meets ends a real block. The bit after it
// counts as a block start when the block there parses: a stored header with
// LEN = ~NLEN, a dynamic header that passes verify_light, or a fixed block
// whose first FW_MINSYM symbols decode without an end-of-block or invalid code
// (random bits meet one of those within about 36 symbols on average, so a walk
// over non-fixed data, where end-of-block codes are chance matches, essentially
// never passes). Any start this returns is checked again by the anchored chain.

constexpr uint32_t FW_THREADS = 128;     // four targets per block, one warp each
constexpr uint32_t FW_WARM = 256;        // symbols since the last end-of-block or invalid code before one is trusted
constexpr uint32_t FW_MINSYM = 1024;     // symbols a fixed block after the start must decode cleanly
constexpr uint32_t FW_SEG_BITS = 8192;   // bits of a round each lane starts in
constexpr uint32_t FW_OVER_BITS = 8192;  // a lane walks on this far past its segment: FW_WARM symbols of <= 32 bits

struct FixedWalkArgs {
    const uint8_t* body;
    uint64_t body_len;
    const uint64_t* from;  // bit offsets to walk from (relative to body)
    uint64_t* found;       // per target: the first block start the walk proves, or ~0
    uint32_t n;
    uint64_t limit_bits;   // how far past its target a walk may go
};

// One fixed-code symbol from `buf` (at least 32 bits buffered): 0 literal or
// length/distance pair, 1 end of block, 2 invalid code (286/287, distance
// 30/31). *used = bits taken (codes are stored MSB first, RFC 1951 §3.1.1).
// Written with selects rather than branches, so that the lanes of a warp, each
// on its own stream, stay in step; the extra-bit counts come from the codes
// (RFC 1951 §3.2.5), not from the tables in constant memory, whose divergent
// reads would be serialised.
__device__ __forceinline__ uint32_t fixed_step(uint64_t buf, uint32_t* used) {
    const uint32_t r = __brev((uint32_t)buf & 511u) >> 23;  // the next 9 code bits, MSB first
    const uint32_t t8 = r >> 1;
    const bool c7 = t8 < 0x30u;                 // 7-bit codes 0000000-0010111: symbols 256-279
    const bool c8h = t8 >= 0xc0u && t8 < 0xc8u;  // 8-bit codes 11000000-11000111: symbols 280-287
    const bool c9 = t8 >= 0xc8u;                // 9-bit codes: literals 144-255 (8-bit: literals 0-143)
    const uint32_t cl = c7 ? 7u : (c9 ? 9u : 8u);
    const uint32_t sym = c7 ? 256u + (r >> 2) : 280u + (t8 - 0xc0u);  // meaningful when c7 or c8h
    const bool eob = c7 && sym == 256u;
    const bool len_code = (c7 && sym != 256u) || (c8h && sym <= 285u);
    const bool bad_len = c8h && sym > 285u;
    const uint32_t li = sym - 257u;
    const uint32_t p = cl + (li >= 8u && li < 28u ? (li - 4u) >> 2 : 0u);
    const uint32_t dc = __brev((uint32_t)(buf >> (p & 63u)) & 31u) >> 27;  // 5-bit distance code
    const bool bad_dist = dc >= 30u;
    *used = len_code ? p + 5u + (!bad_dist && dc >= 4u ? (dc - 2u) >> 1 : 0u) : cl;
    return eob ? 1u : ((bad_len || (len_code && bad_dist)) ? 2u : 0u);
}

// Does a block start at bit e? (the tests the walk applies, see above)
__device__ bool fixed_start_ok(const Src& s, uint64_t total_bits, uint64_t e, uint8_t* lut) {
    if (e + 3 > total_bits) return false;
    const uint32_t btype = peek_at(s, e, 3) >> 1;
    if (btype == 3) return false;
    if (btype == 2) return verify_light(s, total_bits, e, lut);
    if (btype == 0) {
        const uint64_t q = (e + 3 + 7) & ~7ull;  // LEN and NLEN start at the next byte
        if (q + 32 > total_bits) return false;
        const uint32_t len = peek_at(s, q, 16), nlen = peek_at(s, q + 16, 16);
        if ((len ^ nlen) != 0xffffu) return false;
        const uint64_t nx = q + 32 + 8ull * len;  // the next block's header
        return nx + 3 <= total_bits && (peek_at(s, nx, 3) >> 1) != 3u;
    }
    BR b{s, 0, 0, 0};
    br_seek(b, e + 3);
    for (uint32_t k = 0; k < FW_MINSYM; k++) {
        br_refill(b);
        uint32_t used = 0;
        if (fixed_step(b.buf, &used) != 0) return false;
        br_consume(b, used);
        if (br_tell(b) > total_bits) return false;
    }
    return true;
}

// The lowest block start a warp proves in [p0, stop) (~0: none); uniform over
// the warp, which calls it together. A walk from p0 alone would be serial
// over the rest of its block (16,383 symbols for zlib's fixed blocks);
// instead, in each round of 32 segments, lane l walks from the start of
// segment l to FW_OVER_BITS past its end. Where lane l + 1 is still in its
// first FW_WARM symbols, lane l is already on the real symbol path, so every
// end-of-block code past the first FW_WARM symbols after p0 is tested by some
// lane. The warp keeps the lowest block start any lane proves.
__device__ uint64_t fixed_walk_warp(const Src& s, uint64_t total_bits, uint64_t p0, uint64_t stop, uint8_t* lut,
                                    int lane) {
    uint64_t found = ~0ull;
    for (uint64_t base = p0; base < stop && found == ~0ull; base += 32ull * FW_SEG_BITS) {
        const uint64_t s0 = base + (uint64_t)lane * FW_SEG_BITS;
        const uint64_t s1 = s0 + FW_SEG_BITS + FW_OVER_BITS < stop ? s0 + FW_SEG_BITS + FW_OVER_BITS : stop;
        uint64_t mine = ~0ull;
        bool walking = s0 < stop;
        BR b{s, 0, 0, 0};
        br_seek(b, walking ? s0 : p0);
        uint32_t run = 0;
        // one symbol per lane per step, the warp in step
        while (__any_sync(FULLMASK, walking)) {
            uint32_t k = 0;
            if (walking) {
                br_refill(b);
                uint32_t used = 0;
                k = fixed_step(b.buf, &used);
                br_consume(b, used);
            }
            const bool probe = walking && k == 1u && run >= FW_WARM;
            run = k == 0u ? run + 1u : 0u;
            __syncwarp();
            if (__any_sync(FULLMASK, probe)) {  // rare: the start after an end-of-block
                if (probe) {
                    const uint64_t e = br_tell(b);
                    if (e < total_bits && fixed_start_ok(s, total_bits, e, lut)) {
                        mine = e;
                        walking = false;
                    }
                }
                __syncwarp();
            }
            if (walking && br_tell(b) >= s1) walking = false;
        }
        // lowest proven start of the round (offsets from base fit 32 bits)
        const uint32_t rel = mine == ~0ull ? 0xffffffffu : (uint32_t)(mine - base);
        const uint32_t best = __reduce_min_sync(FULLMASK, rel);
        if (best != 0xffffffffu) found = base + best;
    }
    return found;
}

// One warp per target.
__global__ void __launch_bounds__(FW_THREADS) k_fixed_walk(FixedWalkArgs A) {
    __shared__ __align__(16) uint8_t s_lut[FW_THREADS * 128];  // verify_light's precode table, one per thread
    const int lane = threadIdx.x & 31;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= A.n) return;  // uniform over the warp
    const Src s = make_src(A.body, A.body_len);
    const uint64_t total_bits = A.body_len * 8;
    const uint64_t p0 = A.from[i];
    uint64_t found = ~0ull;
    if (p0 < total_bits) {
        const uint64_t stop = total_bits - p0 > A.limit_bits ? p0 + A.limit_bits : total_bits;
        found = fixed_walk_warp(s, total_bits, p0, stop, s_lut + threadIdx.x * 128, lane);
    }
    if (lane == 0) A.found[i] = found;
}

// ------------------------------------------------------- marker resolution
// A marker cell 0x8000|m of chunk k names the output byte m + 1 positions
// before chunk k's first byte (speculative.rs:12-17, :41), so every marker
// points into W_k, the 32 KiB of output before chunk k. The reference builds
// W_{k+1} from W_k one chunk after another (the tail chain,
// pipeline.rs:1045-1078) and then resolves each chunk against its window
// (resolve_markers, speculative.rs:175-213). Marker chains are long (the
// first occurrence of a frequent word may lie many chunks back), so the chain
// is restated as composition of window maps. A window map describes each of
// the 32768 bytes of a window as a literal, a position in an earlier base
// window (WM_REF | index) or an unresolvable byte (WM_BAD). Chunks form groups
// (consecutive chunks of a job), groups form supergroups. Six kernels:
//   k_win_maps    one block per group: R_k, the map of W_{k+1} relative to the
//                 group's first window, built chunk after chunk in shared
//                 memory from chunk k's last 32 KiB of cells and R_{k-1};
//   k_win_supers  one block per supergroup: each group's first window as a map
//                 relative to the supergroup's first window, group after group,
//                 and the supergroup's transfer map (the next supergroup's
//                 first window relative to this one's);
//   k_win_bases   one block per job: the supergroups' first windows as bytes,
//                 one supergroup after another (one gather per byte each);
//   k_win_expand  every group's first window as bytes, in parallel;
//   k_res_tails   the last 32 KiB of every chunk, R_k through its group's first
//                 window (staged in shared memory once per 8 chunks) straight
//                 into the output;
//   k_res_heads   every other cell with at most one gather from the 32 KiB of
//                 output before its chunk, staged in shared memory once per
//                 64 Ki-cell segment; cells read 16 bytes at a time, bytes
//                 written as aligned 8-byte words.
// The sequential steps are one 32 KiB gather each: chunks per group, groups
// per supergroup and supergroups per job, about 24 + 12 + 12 for 3,552 chunks.
// Device traffic: 2 bytes read and 1 written per cell, plus about 6 bytes per
// window byte for the maps.
constexpr int RES_THREADS = 256;
constexpr int RES_CELLS = 8;                             // cells per thread per step (one 16-byte load)
constexpr int RES_TAIL_TILE = RES_THREADS * RES_CELLS;   // window bytes per tail step
constexpr uint32_t RES_TAIL_CHUNKS = 8;                  // chunks per tail unit (one base staging)
constexpr uint64_t RES_HEAD_SEG = 65536;                 // head cells per window staging
constexpr int WM_THREADS = 1024;
constexpr uint32_t WM_REF = 0x8000u;  // | index into the base window
constexpr uint32_t WM_BAD = 0x4000u;  // the byte lies before its member (or the output)

struct ResGroup {
    uint32_t first;  // first chunk (of a group), first group (of a supergroup) or first supergroup (of a job)
    uint32_t n;      // consecutive members
};
typedef ResGroup ResJob;

struct ResolveArgs {
    uint16_t* cells;
    const ResolveChunk* chunks;
    uint32_t n_chunks;
    const ResGroup* groups;       // chunks of each group
    uint32_t n_groups;
    const ResGroup* supers;       // groups of each supergroup
    uint32_t n_supers;
    const ResJob* jobs;           // supergroups of each job
    uint32_t n_jobs;
    const uint32_t* chunk_group;  // n_chunks
    const uint32_t* group_super;  // n_groups
    const uint64_t* tail_units;   // n_groups + 1: prefix of each group's tail units (RES_TAIL_CHUNKS chunks each)
    const uint64_t* head_segs;    // n_chunks + 1: prefix of each chunk's head segments
    uint16_t* maps;               // n_chunks x WINDOW: R_k
    uint16_t* gmaps;              // n_groups x WINDOW: each group's first window relative to its supergroup's
    uint16_t* tmaps;              // n_supers x WINDOW: each supergroup's transfer map
    uint16_t* sbases;             // n_supers x WINDOW: each supergroup's first window (byte or WM_BAD)
    uint16_t* bases;              // n_groups x WINDOW: each group's first window (byte or WM_BAD)
    uint8_t* out;
    uint32_t* err;                // [0] flag, [1] chunk, [2] cell lo, [3] cell hi
    unsigned long long* markers;  // count of marker cells resolved
    const uint32_t* live;         // when set and 0, the kernels do nothing (a failed pipeline wave)
    uint32_t identity_base;       // the job's first window is unknown: maps stay relative to it
};

// Cells of a chunk that the head kernel resolves: all but the last 32 KiB.
__host__ __device__ __forceinline__ uint64_t res_head_end(uint64_t n) { return n > WINDOW ? n - WINDOW : 0; }
// First window index of R_k that lies inside chunk k.
__host__ __device__ __forceinline__ uint32_t res_tail_lo(uint64_t n) {
    return n >= WINDOW ? 0u : (uint32_t)(WINDOW - n);
}

// The chunk owning work unit t: the largest k with pre[k] <= t (pre[0] = 0,
// pre[n] > t).
__device__ __forceinline__ uint32_t res_unit_chunk(const uint64_t* pre, uint32_t n, uint64_t t) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pre[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The warp's 32 lanes hold the bytes of output positions [p, p + 256) as one
// little-endian 64-bit word each (lane l: bytes p + 8l .. p + 8l + 7); bytes
// [lo, n) of that span are written. A whole span goes out as aligned 8-byte
// words, the two words it shares with its neighbours byte by byte; anything
// else byte by byte.
__device__ __forceinline__ void warp_store8(uint8_t* dst, uint64_t v, uint32_t lo, uint32_t n, int lane) {
    const uint32_t mis = (uint32_t)((uintptr_t)dst & 7u);
    const uint64_t prev = __shfl_up_sync(FULLMASK, v, 1);
    if (lo == 0 && n == 32u * RES_CELLS) {
        if (mis == 0) {
            *reinterpret_cast<uint64_t*>(dst + 8 * lane) = v;
            return;
        }
        uint8_t* al = dst - mis;
        if (lane > 0) *reinterpret_cast<uint64_t*>(al + 8 * lane) = (v << (8 * mis)) | (prev >> (64 - 8 * mis));
        else
            for (uint32_t b = 0; b < 8 - mis; b++) dst[b] = (uint8_t)(v >> (8 * b));
        if (lane == 31)
            for (uint32_t b = 8 - mis; b < 8; b++) dst[8 * 31 + b] = (uint8_t)(v >> (8 * b));
        return;
    }
    for (uint32_t b = 0; b < 8; b++) {
        const uint32_t x = 8u * lane + b;
        if (x >= lo && x < n) dst[x] = (uint8_t)(v >> (8 * b));
    }
}

__device__ __forceinline__ void res_fail(const ResolveArgs& A, uint32_t k, uint64_t cell) {
    if (atomicCAS(A.err, 0u, 1u) == 0u) {  // the first unresolvable cell names its chunk
        A.err[1] = k;
        A.err[2] = (uint32_t)cell;
        A.err[3] = (uint32_t)(cell >> 32);
    }
}

// Dynamic shared memory: two maps (R_{k-1}, R_k) and the chunk's last 32 KiB
// of cells (staged from an 8-cell boundary, so 8 more).
constexpr size_t WM_SMEM = (size_t)(3 * WINDOW + 8) * 2;
constexpr uint32_t WM_VEC = WINDOW / (8 * WM_THREADS);  // 8-entry vectors per thread per map

__device__ __forceinline__ uint32_t u16_of(const uint4& q, int e) {
    const uint32_t w = e < 2 ? q.x : e < 4 ? q.y : e < 6 ? q.z : q.w;
    return (w >> (16 * (e & 1))) & 0xffffu;
}
__device__ __forceinline__ uint4 pack_u16x8(const uint32_t (&r)[8]) {
    return make_uint4(r[0] | (r[1] << 16), r[2] | (r[3] << 16), r[4] | (r[5] << 16), r[6] | (r[7] << 16));
}

// Cells [s0, n) of chunk k as 16-byte words, WM_VEC per thread (zeros past the end).
__device__ __forceinline__ void wm_load(const ResolveArgs& A, uint32_t k, uint4 (&v)[WM_VEC]) {
    const ResolveChunk ck = A.chunks[k];
    const uint64_t n = ck.n_cells, s0 = (n > WINDOW ? n - WINDOW : 0) & ~7ull;
    const uint4* src = reinterpret_cast<const uint4*>(A.cells + ck.slot_off + s0);
    const uint32_t nq = (uint32_t)((n - s0 + 7) / 8);
#pragma unroll
    for (uint32_t q = 0; q < WM_VEC; q++) {
        const uint32_t x = threadIdx.x + q * WM_THREADS;
        v[q] = x < nq ? src[x] : make_uint4(0, 0, 0, 0);
    }
}

__global__ void __launch_bounds__(WM_THREADS, 1) k_win_maps(ResolveArgs A) {
    if (A.live && *A.live == 0) return;
    RRG_DYN_SMEM(sm);
    uint16_t* maps2 = reinterpret_cast<uint16_t*>(sm);  // two maps, alternating by step
    uint16_t* stage = maps2 + 2 * WINDOW;               // stage[x]: cell s0 + x of the chunk
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t nmk = 0;
    for (uint32_t g = blockIdx.x; g < A.n_groups; g += gridDim.x) {
        const ResGroup G = A.groups[g];
        uint4 nxt[WM_VEC];
        wm_load(A, G.first, nxt);
        for (uint32_t t = 0; t < G.n; t++) {
            const uint32_t k = G.first + t;
            const ResolveChunk ck = A.chunks[k];
            const uint64_t n = ck.n_cells, end = ck.out_start + n;
            const uint64_t c_lo = n > WINDOW ? n - WINDOW : 0, s0 = c_lo & ~7ull;
            const uint32_t nq = (uint32_t)((n - s0 + 7) / 8);
#pragma unroll
            for (uint32_t q = 0; q < WM_VEC; q++) {
                const uint32_t x = threadIdx.x + q * WM_THREADS;
                if (x < nq) reinterpret_cast<uint4*>(stage)[x] = nxt[q];
            }
            if (nq > WM_VEC * WM_THREADS && threadIdx.x == 0)  // the 4097th word of a misaligned tail
                reinterpret_cast<uint4*>(stage)[WM_VEC * WM_THREADS] =
                    reinterpret_cast<const uint4*>(A.cells + ck.slot_off + s0)[WM_VEC * WM_THREADS];
            __syncthreads();  // also: the previous step's map is complete
            if (t + 1 < G.n) wm_load(A, k + 1, nxt);  // in flight while this step computes
            const uint16_t* prv = maps2 + ((t + 1) & 1) * WINDOW;
            uint16_t* cur = maps2 + (t & 1) * WINDOW;
            uint16_t* Rk = A.maps + (uint64_t)k * WINDOW;
            const uint64_t lim = ck.out_start - ck.member_start;  // markers m < lim stay inside the member
            const uint32_t i_lo = res_tail_lo(n);
            // stage index of window index i (for i >= i_lo)
            const uint32_t off = (uint32_t)(c_lo - s0) - i_lo;
            const bool plain = i_lo == 0 && end >= WINDOW;  // block-uniform: every entry is a cell
            // lane-consecutive entries: conflict-free shared loads, coalesced stores
            for (uint32_t sp = warp; sp < WINDOW / 256; sp += WM_THREADS / 32) {
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const uint32_t i = sp * 256 + lane + 32 * e;
                    const uint32_t si = i + off;  // wraps below i_lo of a short chunk (unused there)
                    const uint32_t v = stage[si < WINDOW + 8 ? si : 0u];
                    const uint32_t mk = v >> 15, m = v & 0x7fffu, j = WINDOW - 1 - m;
                    const uint32_t via = t ? (uint32_t)prv[j] : (WM_REF | j);
                    uint32_t r = mk ? ((uint64_t)m < lim ? via : WM_BAD) : v;
                    nmk += mk;
                    if (!plain) {
                        if (end < (uint64_t)(WINDOW - i)) {
                            r = WM_BAD;  // before the output's start
                            nmk -= mk;
                        } else if (i < i_lo) {
                            r = t ? (uint32_t)prv[(uint32_t)n + i] : (WM_REF | ((uint32_t)n + i));  // lies in W_k
                            nmk -= mk;
                        }
                    }
                    cur[i] = (uint16_t)r;
                    Rk[i] = (uint16_t)r;
                }
            }
            __syncthreads();  // the staging buffer is free again
        }
    }
    nmk = warp_sum(nmk);
    if ((threadIdx.x & 31) == 0 && nmk) atomicAdd(A.markers, (unsigned long long)nmk);
}

// One composition step of a sequential map chain held in shared memory:
// cur[i] <- R[i] through cur (a literal or WM_BAD stays, WM_REF|j becomes
// cur[j]), read first into registers so cur can be rewritten in place; the
// result also goes to `out` when set. Block-wide, WM_THREADS threads.
__device__ __forceinline__ void wm_step(uint16_t* cur, const uint16_t* R, uint16_t* out) {
    uint4 nv[WM_VEC];
#pragma unroll
    for (uint32_t v = 0; v < WM_VEC; v++) nv[v] = reinterpret_cast<const uint4*>(R)[threadIdx.x + v * WM_THREADS];
#pragma unroll
    for (uint32_t v = 0; v < WM_VEC; v++) {
        uint32_t r[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const uint32_t x = u16_of(nv[v], e);
            r[e] = (x & WM_REF) ? (uint32_t)cur[x & 0x7fffu] : x;
        }
        nv[v] = pack_u16x8(r);
    }
    __syncthreads();  // every read of cur is done
#pragma unroll
    for (uint32_t v = 0; v < WM_VEC; v++) {
        const uint32_t i0 = 8 * (threadIdx.x + v * WM_THREADS);
        *reinterpret_cast<uint4*>(cur + i0) = nv[v];
        if (out) *reinterpret_cast<uint4*>(out + i0) = nv[v];
    }
    __syncthreads();
}

// Each supergroup's groups in order: a group's first window relative to the
// supergroup's first window (the identity for the first group), then the
// transfer map after the last group.
__global__ void __launch_bounds__(WM_THREADS, 1) k_win_supers(ResolveArgs A) {
    if (A.live && *A.live == 0) return;
    RRG_DYN_SMEM(sm);
    uint16_t* cur = reinterpret_cast<uint16_t*>(sm);
    for (uint32_t sg = blockIdx.x; sg < A.n_supers; sg += gridDim.x) {
        const ResGroup SG = A.supers[sg];
        for (uint32_t i = threadIdx.x; i < WINDOW; i += blockDim.x) {
            cur[i] = (uint16_t)(WM_REF | i);
            A.gmaps[(uint64_t)SG.first * WINDOW + i] = (uint16_t)(WM_REF | i);
        }
        __syncthreads();
        for (uint32_t q = 0; q < SG.n; q++) {
            const ResGroup G = A.groups[SG.first + q];
            const uint16_t* R = A.maps + (uint64_t)(G.first + G.n - 1) * WINDOW;
            uint16_t* dst = q + 1 < SG.n ? A.gmaps + (uint64_t)(SG.first + q + 1) * WINDOW
                                         : A.tmaps + (uint64_t)sg * WINDOW;
            wm_step(cur, R, dst);
        }
    }
}

// Each job's supergroups in order: the first one's first window is the 32 KiB
// before the job (a stripe's prefix, already in the output, or WM_BAD); each
// next one applies the previous supergroup's transfer map.
__global__ void __launch_bounds__(WM_THREADS, 1) k_win_bases(ResolveArgs A) {
    if (A.live && *A.live == 0) return;
    RRG_DYN_SMEM(sm);
    uint16_t* cur = reinterpret_cast<uint16_t*>(sm);
    for (uint32_t jb = blockIdx.x; jb < A.n_jobs; jb += gridDim.x) {
        const ResJob J = A.jobs[jb];
        const ResolveChunk ck = A.chunks[A.groups[A.supers[J.first].first].first];
        for (uint32_t i = threadIdx.x; i < WINDOW; i += blockDim.x) {
            uint32_t r = WM_BAD;
            if (A.identity_base) {
                r = WM_REF | i;
            } else if (ck.out_start >= (uint64_t)(WINDOW - i)) {
                const uint64_t pos = ck.out_start - WINDOW + i;
                if (pos >= ck.member_start && pos < ck.job_out) r = A.out[pos];
            }
            cur[i] = (uint16_t)r;
            A.sbases[(uint64_t)J.first * WINDOW + i] = (uint16_t)r;
        }
        __syncthreads();
        for (uint32_t q = 0; q + 1 < J.n; q++)
            wm_step(cur, A.tmaps + (uint64_t)(J.first + q) * WINDOW, A.sbases + (uint64_t)(J.first + q + 1) * WINDOW);
    }
}

// Every group's first window as bytes: its map through its supergroup's first window.
__global__ void __launch_bounds__(RES_THREADS) k_win_expand(ResolveArgs A) {
    if (A.live && *A.live == 0) return;
    const uint64_t total = (uint64_t)A.n_groups * (WINDOW / 8);
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = (uint32_t)(x / (WINDOW / 8)), i0 = (uint32_t)(x % (WINDOW / 8)) * 8;
        const uint16_t* sb = A.sbases + (uint64_t)A.group_super[g] * WINDOW;
        const uint4 q = *reinterpret_cast<const uint4*>(A.gmaps + (uint64_t)g * WINDOW + i0);
        uint32_t r[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const uint32_t v = u16_of(q, e);
            r[e] = (v & WM_REF) ? (uint32_t)sb[v & 0x7fffu] : v;
        }
        *reinterpret_cast<uint4*>(A.bases + (uint64_t)g * WINDOW + i0) = pack_u16x8(r);
    }
}

// The window after chunk k (the last of its job) relative to the job's first
// window: R_k through its group's first window (both maps when the job's base
// is the identity).
__global__ void k_win_endmap(ResolveArgs A, uint32_t k, uint16_t* out) {
    const uint16_t* R = A.maps + (uint64_t)k * WINDOW;
    const uint16_t* B = A.bases + (uint64_t)A.chunk_group[k] * WINDOW;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < WINDOW; i += gridDim.x * blockDim.x) {
        const uint32_t r = R[i];
        out[i] = (uint16_t)((r & WM_REF) ? (uint32_t)B[r & 0x7fffu] : r);
    }
}

// Tails, one unit = up to RES_TAIL_CHUNKS chunks of one group: the group's
// first window is staged in shared memory once, then each chunk's R_k is
// read 16 bytes per lane and resolved through it.
__global__ void __launch_bounds__(RES_THREADS) k_res_tails(ResolveArgs A) {
    if (A.live && *A.live == 0) return;
    RRG_DYN_SMEM(sm);  // WINDOW u16: the group's first window
    uint16_t* base = reinterpret_cast<uint16_t*>(sm);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t n_units = A.tail_units[A.n_groups];
    for (uint64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        const uint32_t g = res_unit_chunk(A.tail_units, A.n_groups, u);
        const ResGroup G = A.groups[g];
        const uint32_t c0 = G.first + (uint32_t)(u - A.tail_units[g]) * RES_TAIL_CHUNKS;
        const uint32_t c1 = c0 + RES_TAIL_CHUNKS < G.first + G.n ? c0 + RES_TAIL_CHUNKS : G.first + G.n;
        __syncthreads();  // the previous unit's readers are done with base
        const uint4* src = reinterpret_cast<const uint4*>(A.bases + (uint64_t)g * WINDOW);
        for (uint32_t q = threadIdx.x; q < WINDOW / 8; q += blockDim.x) reinterpret_cast<uint4*>(base)[q] = src[q];
        __syncthreads();
        for (uint32_t k = c0; k < c1; k++) {
            const ResolveChunk ck = A.chunks[k];
            const uint32_t i_lo = res_tail_lo(ck.n_cells);
            const uint16_t* R = A.maps + (uint64_t)k * WINDOW;
            // window index i is output byte out_start + n - WINDOW + i
            uint8_t* dst0 = A.out + (ck.out_start + ck.n_cells - WINDOW);
            for (uint32_t i0 = (i_lo & ~(uint32_t)(32 * RES_CELLS - 1)) + warp * (32 * RES_CELLS); i0 < WINDOW;
                 i0 += RES_THREADS * RES_CELLS) {
                const uint4 q = reinterpret_cast<const uint4*>(R + i0)[lane];
                uint32_t lo32 = 0, hi32 = 0;
                bool bad = false;
#pragma unroll
                for (int e = 0; e < RES_CELLS; e++) {
                    const uint32_t i = i0 + RES_CELLS * lane + e;
                    uint32_t r = u16_of(q, e);
                    r = (r & WM_REF) ? (uint32_t)base[r & 0x7fffu] : r;
                    if (i >= i_lo) bad |= (r & WM_BAD) != 0;
                    if (e < 4) lo32 |= (r & 0xffu) << (8 * e);
                    else hi32 |= (r & 0xffu) << (8 * (e - 4));
                }
                if (bad) res_fail(A, k, i0);
                warp_store8(dst0 + i0, ((uint64_t)hi32 << 32) | lo32, i_lo > i0 ? i_lo - i0 : 0u, 32u * RES_CELLS, lane);
            }
        }
    }
}

// Four blocks per SM: 4 x 32 KiB windows in shared memory.
__global__ void __launch_bounds__(RES_THREADS, 4) k_res_heads(ResolveArgs A) {
    if (A.live && *A.live == 0) return;
    __shared__ __align__(16) uint8_t win[WINDOW + 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t n_segs = A.head_segs[A.n_chunks];
    uint32_t nmk = 0;
    for (uint64_t s = blockIdx.x; s < n_segs; s += gridDim.x) {
        const uint32_t k = res_unit_chunk(A.head_segs, A.n_chunks, s);
        const ResolveChunk ck = A.chunks[k];
        const uint64_t h_end = res_head_end(ck.n_cells);
        const uint64_t s0 = (s - A.head_segs[k]) * RES_HEAD_SEG;
        const uint64_t s1 = s0 + RES_HEAD_SEG < h_end ? s0 + RES_HEAD_SEG : h_end;
        // markers of this chunk may name positions [out_start - lim, out_start)
        const uint64_t lim = ck.out_start - ck.member_start;
        // stage the 32 KiB before the chunk: whole aligned 16-byte words inside
        // [w_lo, out_start), bytes at the edges; win[i] holds the byte at
        // address a_lo + i (addresses, not offsets from A.out: the aligned start
        // may lie before A.out itself when the window starts at the output's
        // first byte)
        const uint64_t w_lo = ck.out_start > WINDOW ? ck.out_start - WINDOW : 0;
        const uintptr_t lo_addr = (uintptr_t)(A.out + w_lo), end_addr = (uintptr_t)(A.out + ck.out_start);
        const uintptr_t a_lo = lo_addr & ~(uintptr_t)15;  // up to 15 bytes before lo_addr
        __syncthreads();  // the previous segment's readers are done with win
        for (uint64_t q = threadIdx.x; 16 * q < WINDOW + 16; q += blockDim.x) {
            const uintptr_t p = a_lo + 16 * q;  // p + 16 > lo_addr
            if (p >= end_addr) break;
            if (p >= lo_addr && p + 16 <= end_addr) {
                *reinterpret_cast<uint4*>(win + 16 * q) = *reinterpret_cast<const uint4*>(p);
            } else {
                for (int b = 0; b < 16; b++)
                    if (p + b >= lo_addr && p + b < end_addr) win[16 * q + b] = *reinterpret_cast<const uint8_t*>(p + b);
            }
        }
        __syncthreads();
        const uint64_t wbase = (uint64_t)(end_addr - 1 - a_lo);  // win index of the byte before the chunk
        const uint16_t* cells = A.cells + ck.slot_off;
        constexpr uint64_t STEP = RES_THREADS * RES_CELLS;
        // the next step's cells are loaded before this step's are processed
        uint64_t c0 = s0 + (uint64_t)warp * (32 * RES_CELLS);
        uint4 qn = make_uint4(0, 0, 0, 0);
        if (c0 + RES_CELLS * lane < s1) qn = *reinterpret_cast<const uint4*>(cells + c0 + RES_CELLS * lane);
        for (; c0 < s1; c0 += STEP) {
            const uint64_t left = s1 - c0;
            const uint32_t n = left < 32u * RES_CELLS ? (uint32_t)left : 32u * RES_CELLS;
            const uint64_t ci = c0 + (uint64_t)RES_CELLS * lane;
            const uint4 q = qn;
            qn = make_uint4(0, 0, 0, 0);
            if (ci + STEP < s1) qn = *reinterpret_cast<const uint4*>(cells + ci + STEP);
            const uint32_t w[4] = {q.x, q.y, q.z, q.w};
            bool bad = false;
            // cells past s1 belong to the tail kernel
            const uint32_t nvalid = ci < s1 ? (s1 - ci < RES_CELLS ? (uint32_t)(s1 - ci) : RES_CELLS) : 0u;
            // eight literals: their low bytes, two byte permutes
            uint32_t lo32 = __byte_perm(w[0], w[1], 0x6420), hi32 = __byte_perm(w[2], w[3], 0x6420);
            if ((w[0] | w[1] | w[2] | w[3]) & 0x80008000u) {
                lo32 = hi32 = 0;
#pragma unroll
                for (int i = 0; i < RES_CELLS; i++) {
                    const uint32_t cl = (w[i >> 1] >> (16 * (i & 1))) & 0xffffu;
                    const uint32_t mk = (cl >> 15) & ((uint32_t)i < nvalid ? 1u : 0u), m = cl & 0x7fffu;
                    // a marker m < lim reads win[wbase - m]; others read a clamped, unused byte
                    const uint32_t x = (uint32_t)wbase - m;
                    const uint32_t wb = win[x < WINDOW + 32 ? x : 0u];
                    const uint32_t b = mk ? wb : cl;
                    nmk += mk;
                    bad |= mk && (uint64_t)m >= lim;
                    if (i < 4) lo32 |= (b & 0xffu) << (8 * i);
                    else hi32 |= (b & 0xffu) << (8 * (i - 4));
                }
            }
            const uint64_t v = ((uint64_t)hi32 << 32) | lo32;
            if (bad) res_fail(A, k, ci);
            warp_store8(A.out + ck.out_start + c0, v, 0u, n, lane);
        }
    }
    nmk = warp_sum(nmk);
    if (lane == 0 && nmk) atomicAdd(A.markers, (unsigned long long)nmk);
}

// The reference-shaped entry point's scatter (speculative.rs:175-213):
// bytes[out_pos[i]] = tail[tail_len - 1 - prefix_offset[i]].
__global__ void k_resolve_list(uint8_t* bytes, uint64_t n_bytes, const uint32_t* out_pos, const uint16_t* prefix_off,
                               uint64_t n_markers, const uint8_t* tail, uint64_t tail_len, uint32_t* err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_markers;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t o = prefix_off[i], p = out_pos[i];
        if (o >= tail_len || p >= n_bytes) {
            atomicOr(err, 1u);
            continue;
        }
        bytes[p] = tail[tail_len - 1 - o];
    }
}

// ------------------------------------------------------- anchored chain on the device
// Jobs whose sub-chunks were inflated speculatively in one launch get their
// anchored chain checked on the device (pipeline.rs:758-809: each sub-chunk
// starts where the previous one stopped) and their output laid out, so resolve
// and the CRC pieces queue behind the inflate with no host round trip: the
// waves of the pipelined host path (one job per launch, carried from wave to
// wave), and the member route of a batch (every job at once). A job with any
// irregularity (a false start, a full slot, a member ending before its last
// sub-chunk, a full output range) is left empty for the host, which decodes it
// again on the checked path.
struct WaveState {         // per job, carried from wave to wave on the device
    uint64_t expected;     // body-relative bit where the next sub-chunk must start
    uint64_t out_end;      // output bytes laid out so far (absolute)
    uint32_t live;         // 0 once the job failed
    uint32_t pad;
};
struct WaveInfo {          // a job's outcome in one launch, read by the host
    uint64_t out_begin, out_len;
    uint64_t trailer_byte; // body-relative trailer offset (when its last sub-chunk is here)
    uint32_t ok;
    int32_t fail_item;     // index among the job's items of the first failing sub-chunk
    int32_t fail_status;
    uint32_t final_seen;
};
struct WaveJob {
    uint32_t first, n;     // global item indices of this launch's part of the job
    uint32_t last_item;    // global index of the job's last sub-chunk (~0u: in a later launch)
    uint32_t piece_off, piece_cap;  // the job's region of CRC pieces
    uint32_t n_all;        // items [first, first + n_all) belong to the job; those past n are unused
    uint64_t out_cap;      // the job's output may not pass this byte
    uint64_t member_start; // output byte where the job's member begins
};
struct WaveArgs {
    const ChunkItem* items;
    const ChunkResult* results;
    const WaveJob* jobs;
    uint32_t n_jobs;
    uint32_t item_base;        // chunks[] and head_segs[] are indexed by item - item_base
    uint32_t n_items;          // items of this launch; head_segs has n_items + 1 entries
    WaveState* state;          // per job
    WaveInfo* info;            // per job (may be mapped host memory)
    uint32_t* live;            // when set: 1 if job 0 passed
    ResolveChunk* chunks;      // per item (unless direct)
    uint64_t* head_segs;       // per item + 1 (unless direct): job-local, then global after k_wave_segs
    CrcPiece* pieces;
    uint32_t* n_pieces;        // per job: pieces laid out
    uint64_t* seg_total;       // per job: head segments; k_wave_segs turns it into each job's offset
    const MemberRec* mbs;
    const uint32_t* mb_count;  // records written (those past mb_cap were dropped)
    uint32_t mb_cap;
    uint32_t* exp_crc;         // per job: the member trailer
    uint32_t* exp_isize;
    uint32_t direct;           // the items decoded straight to bytes: nothing to resolve
};
constexpr int WAVE_THREADS = 1024;
constexpr uint64_t WAVE_PIECE = 256 * 1024;  // CRC piece bytes

// n status words to (mapped) host memory, so the host learns them without a
// copy queued behind the output copies.
__global__ void k_copy_words(const uint32_t* src, uint32_t* dst, uint32_t n) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Exclusive block-wide prefix of one value per thread; returns the total.
__device__ __forceinline__ uint64_t block_scan(uint64_t v, uint64_t* sh, uint64_t* excl) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int o = 1; o < WAVE_THREADS; o <<= 1) {
        const uint64_t x = t >= o ? sh[t - o] : 0;
        __syncthreads();
        sh[t] += x;
        __syncthreads();
    }
    *excl = sh[t] - v;
    const uint64_t total = sh[WAVE_THREADS - 1];
    __syncthreads();
    return total;
}

__device__ __forceinline__ uint64_t head_segs_of(uint64_t n) { return (res_head_end(n) + RES_HEAD_SEG - 1) / RES_HEAD_SEG; }

// One block per job.
__global__ void __launch_bounds__(WAVE_THREADS, 1) k_wave_chain(WaveArgs A) {
    __shared__ uint64_t sh[WAVE_THREADS];
    __shared__ int32_t s_fail;
    __shared__ uint32_t s_found, s_crc, s_isize;
    __shared__ uint64_t s_tb;
    const int t = threadIdx.x;
    for (uint32_t jb = blockIdx.x; jb < A.n_jobs; jb += gridDim.x) {
        const WaveJob J = A.jobs[jb];
        const WaveState S = A.state[jb];
        const bool has_last = J.n && J.first + J.n - 1 == J.last_item;
        __syncthreads();  // the previous job's readers of the shared words are done
        if (t == 0) {
            s_fail = S.live ? 0x7fffffff : -1;
            s_found = 0;
        }
        __syncthreads();
        // each thread checks a contiguous run of sub-chunks
        const uint32_t per = (J.n + WAVE_THREADS - 1) / WAVE_THREADS;
        const uint32_t b = t * per < J.n ? t * per : J.n, e = b + per < J.n ? b + per : J.n;
        uint64_t cells = 0, segs = 0;
        for (uint32_t q = b; q < e; q++) {
            const uint32_t k = J.first + q;
            const ChunkItem it = A.items[k];
            const ChunkResult r = A.results[k];
            const uint64_t expected = q == 0 ? S.expected : A.results[k - 1].actual_end_bit;
            // a start on a stored block's zero header byte decodes as the true start
            // in the same byte's first 6 bits, or right after an empty block
            const uint64_t d = expected - it.start_bit;
            const bool same = it.start_bit == expected ||
                              ((it.flags & ITEM_STORED_START) && expected > it.start_bit &&
                               (d <= 5 || ((it.flags & ITEM_EMPTY_STORED) && d == 40)));
            const bool last = k == J.last_item;
            bool ok = same && r.status == DS_OK;
            ok = ok && (last ? (r.final_block && r.n_members == 1) : (!r.final_block && r.n_members == 0));
            if (!ok) {
                atomicMin(reinterpret_cast<unsigned int*>(&s_fail), q);
                continue;
            }
            cells += r.n_cells;
            segs += A.direct ? 0 : head_segs_of(r.n_cells);
        }
        // the trailer of the job's only member, from the record of its last sub-chunk
        if (has_last) {
            const uint32_t id = A.items[J.last_item].id, nm = *A.mb_count < A.mb_cap ? *A.mb_count : A.mb_cap;
            for (uint32_t i = t; i < nm; i += WAVE_THREADS)
                if (A.mbs[i].item == id) {
                    s_crc = A.mbs[i].crc;
                    s_isize = A.mbs[i].isize;
                    s_tb = A.mbs[i].trailer_byte;
                    s_found = 1;
                }
        }
        __syncthreads();
        uint64_t c_ex, s_ex;
        const uint64_t total = block_scan(cells, sh, &c_ex);
        const uint64_t n_segs = block_scan(segs, sh, &s_ex);
        const uint64_t out_begin = S.out_end, out_len = total;
        const uint32_t np = (uint32_t)((out_len + WAVE_PIECE - 1) / WAVE_PIECE);
        if (t == 0 && s_fail == 0x7fffffff &&
            (out_begin + out_len > J.out_cap || np > J.piece_cap || (has_last && !s_found)))
            s_fail = (int32_t)J.n;
        __syncthreads();
        const bool failed = s_fail != 0x7fffffff;  // uniform
        // a failed job's sub-chunks are laid out empty, so resolve and the CRC
        // pieces do nothing for it; so are the unused ones past n
        if (!A.direct) {
            const uint32_t pa = (J.n_all + WAVE_THREADS - 1) / WAVE_THREADS;
            const uint32_t ua = t * pa < J.n_all ? t * pa : J.n_all, va = ua + pa < J.n_all ? ua + pa : J.n_all;
            const uint64_t empty_at = failed ? out_begin : out_begin + out_len;
            for (uint32_t q = ua; q < va; q++) {
                const uint32_t k = J.first + q;
                if (q < J.n && !failed) continue;  // written below
                A.chunks[k - A.item_base] = ResolveChunk{empty_at, A.items[k].out_off, 0, J.member_start, out_begin};
                A.head_segs[k - A.item_base] = failed ? 0 : n_segs;
            }
            for (uint32_t q = b; q < e && !failed; q++) {
                const uint32_t k = J.first + q;
                const uint64_t n = A.results[k].n_cells;
                A.chunks[k - A.item_base] =
                    ResolveChunk{out_begin + c_ex, A.items[k].out_off, n, J.member_start, out_begin};
                A.head_segs[k - A.item_base] = s_ex;
                c_ex += n;
                s_ex += head_segs_of(n);
            }
        }
        for (uint32_t p = t; p < J.piece_cap; p += WAVE_THREADS) {
            const uint64_t o = (uint64_t)p * WAVE_PIECE;
            A.pieces[J.piece_off + p] =
                (!failed && p < np) ? CrcPiece{out_begin + o, out_len - o < WAVE_PIECE ? out_len - o : WAVE_PIECE}
                                    : CrcPiece{out_begin, 0};
        }
        if (t == 0) {
            A.seg_total[jb] = failed ? 0 : n_segs;
            A.n_pieces[jb] = failed ? 0 : J.piece_cap;
            if (A.n_jobs == 1 && !A.direct) A.head_segs[A.n_items] = failed ? 0 : n_segs;
            WaveInfo& I = A.info[jb];
            I.out_begin = out_begin;
            if (failed) {
                int32_t st = 0;
                if (s_fail >= 0 && s_fail < (int32_t)J.n) st = A.results[J.first + s_fail].status;
                A.state[jb].live = 0;
                if (A.live) *A.live = 0;
                I.ok = 0;
                I.fail_item = s_fail;
                I.fail_status = st;
                I.out_len = 0;
                I.final_seen = 0;
                I.trailer_byte = 0;
            } else {
                if (has_last) {
                    A.exp_crc[jb] = s_crc;
                    A.exp_isize[jb] = s_isize;
                }
                if (J.n) A.state[jb].expected = A.results[J.first + J.n - 1].actual_end_bit;
                A.state[jb].out_end = out_begin + out_len;
                if (A.live) *A.live = 1;
                I.ok = 1;
                I.fail_item = -1;
                I.fail_status = 0;
                I.out_len = out_len;
                I.trailer_byte = has_last ? s_tb : 0;
                I.final_seen = has_last ? 1u : 0u;
            }
        }
    }
}

// Several jobs in one launch: each job's head-segment offset (one block), then
// added to the job's items (one block per job).
__global__ void __launch_bounds__(WAVE_THREADS) k_wave_segs(WaveArgs A) {
    __shared__ uint64_t sh[WAVE_THREADS];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t j0 = 0; j0 < A.n_jobs; j0 += WAVE_THREADS) {
        const uint32_t j = j0 + threadIdx.x;
        uint64_t ex;
        const uint64_t tot = block_scan(j < A.n_jobs ? A.seg_total[j] : 0, sh, &ex);
        if (j < A.n_jobs) A.seg_total[j] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) A.head_segs[A.n_items] = carry;
}
__global__ void k_wave_segs_add(WaveArgs A) {
    for (uint32_t j = blockIdx.x; j < A.n_jobs; j += gridDim.x) {
        const WaveJob J = A.jobs[j];
        const uint64_t o = A.seg_total[j];
        for (uint32_t q = threadIdx.x; q < J.n_all; q += blockDim.x) A.head_segs[J.first + q - A.item_base] += o;
    }
}

// ------------------------------------------------------- device-planned batch
// The member route of a batch with every hand-off on the device, so the whole
// decode is one captured graph: the boundary scan's verified starts pick each
// job's sub-chunk starts (the verified start nearest each ideal position,
// pipeline.rs:492-505 with the scan's starts), then the sub-chunk list with
// end hints and slot sizes is built, inflated, chain-checked, resolved and
// CRC-checked without the host.
struct BatchJob {
    uint64_t in_off;       // the body's first byte in the input buffer
    uint64_t blen;         // body bytes
    uint64_t scan_bit;     // the body's first bit relative to the scan base
    uint64_t arena;        // the job's first cell in the slot arena
    double expand;         // cells reserved per compressed byte
    uint64_t dst_off, dst_cap;
    uint32_t K;            // sub-chunks planned (ideal positions nbits*k/K, k >= 1)
    uint32_t item_first;
    uint32_t piece_off, piece_cap;
};
struct BatchArgs {
    const BatchJob* jobs;
    uint32_t n_jobs;
    const uint64_t* big_bit;   // scan_bit of the jobs with K > 1, ascending
    const uint32_t* big_job;   // their job indices
    uint32_t n_big;
    const uint64_t* surv;      // scan survivors and their verification flags
    const uint8_t* vflag;
    const uint32_t* counts;    // [1] survivors, [3] stored-block starts
    uint32_t cap2, cap3;
    const uint64_t* stored;    // stored-block starts (bit 0: an empty block)
    unsigned long long* keys;  // per item: (distance << 4 | below << 3 | kind) of the best start, ~0 none
    ChunkItem* items;
    WaveJob* wjobs;
    const uint8_t* scan_body;  // the scanned region: job J's body starts at byte J.scan_bit / 8
    uint32_t walk_kb;          // k_batch_walk: blocks per big job (4 ideals each); the grid is a multiple
};

__device__ __forceinline__ uint64_t batch_ideal(uint64_t nbits, uint32_t k, uint32_t K) { return nbits * k / K; }

// One thread per verified start (dynamic-block survivors, then stored-block
// starts): the two ideal positions around it take it if it is the nearest.
// kind: 1 a stored-block start, 3 an empty stored block.
__global__ void k_batch_select(BatchArgs A) {
    const uint32_t ns = A.counts[1] < A.cap2 ? A.counts[1] : A.cap2;
    const uint32_t nst = A.counts[3] < A.cap3 ? A.counts[3] : A.cap3;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ns + nst; i += gridDim.x * blockDim.x) {
        uint64_t v;
        uint32_t kind = 0;
        if (i < ns) {
            if (!A.vflag[i]) continue;
            v = A.surv[i];
        } else {
            const uint64_t x = A.stored[i - ns];
            v = x & ~1ull;
            kind = (x & 1) ? 3u : 1u;
        }
        // the job whose body holds v: the last big job starting at or before it
        uint32_t lo = 0, hi = A.n_big;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (A.big_bit[mid] <= v) lo = mid + 1;
            else hi = mid;
        }
        if (lo == 0) continue;
        const BatchJob J = A.jobs[A.big_job[lo - 1]];
        const uint64_t rel = v - J.scan_bit, nbits = J.blen * 8;
        if (rel == 0 || rel >= nbits) continue;
        uint32_t k = (uint32_t)(rel * J.K / nbits);  // rel < 2^36, K < 2^24
        while (k + 1 < J.K && batch_ideal(nbits, k + 1, J.K) <= rel) k++;
        while (k > 0 && batch_ideal(nbits, k, J.K) > rel) k--;
        if (k >= 1) {  // above ideal k
            const uint64_t d = rel - batch_ideal(nbits, k, J.K);
            atomicMin(A.keys + J.item_first + k, (unsigned long long)((d << 4) | kind));
        }
        if (k + 1 < J.K) {  // below ideal k + 1
            const uint64_t d = batch_ideal(nbits, k + 1, J.K) - rel;
            atomicMin(A.keys + J.item_first + k + 1, (unsigned long long)((d << 4) | 8u | kind));
        }
    }
}

// Fixed-Huffman blocks in the batch (the walk of k_fixed_walk): a job more
// than half of whose ideal starts found no candidate shows fixed blocks, and
// each of its ideals walks the fixed code up to the next ideal (at most
// 256 KiB). Block b serves big jobs b / walk_kb (striding by the
// grid) and their ideals (b % walk_kb) * 4 + warp.
__global__ void __launch_bounds__(FW_THREADS) k_batch_walk(BatchArgs A) {
    __shared__ __align__(16) uint8_t s_lut[FW_THREADS * 128];
    __shared__ uint32_t s_missing;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t kb = blockIdx.x % A.walk_kb;
    for (uint32_t m = blockIdx.x / A.walk_kb; m < A.n_big; m += gridDim.x / A.walk_kb) {
        const BatchJob J = A.jobs[A.big_job[m]];
        const uint32_t k = kb * (FW_THREADS / 32) + warp;
        __syncthreads();
        if (threadIdx.x == 0) s_missing = 0;
        __syncthreads();
        if (kb * (FW_THREADS / 32) >= J.K) continue;  // uniform over the block
        uint32_t miss = 0;
        for (uint32_t q = 1 + threadIdx.x; q < J.K; q += blockDim.x) miss += A.keys[J.item_first + q] == ~0ull;
        atomicAdd(&s_missing, miss);
        __syncthreads();
        if (2 * s_missing <= J.K - 1) continue;  // uniform: dynamic or stored blocks
        // A job of fixed blocks walks every ideal and keeps the walk's start:
        // there a dynamic-header candidate is more likely a chance match than
        // a block start (one false start sends the whole job to the checked route).
        if (k == 0 || k >= J.K) continue;  // uniform over the warp
        const uint64_t nbits = J.blen * 8, x = batch_ideal(nbits, k, J.K);
        const uint64_t nx = batch_ideal(nbits, k + 1, J.K);
        const uint64_t stop = nx - x > (256ull << 13) ? x + (256ull << 13) : nx;
        const Src s = make_src(A.scan_body + J.scan_bit / 8, J.blen);
        const uint64_t f = fixed_walk_warp(s, nbits, x, stop, s_lut + threadIdx.x * 128, lane);
        if (lane == 0 && f != ~0ull && f < nbits) A.keys[J.item_first + k] = (unsigned long long)((f - x) << 4);
    }
}

// One block per job: the chosen starts in order (repeats dropped), their end
// hints, slot sizes and offsets; unused items at the job's end are skipped.
__global__ void __launch_bounds__(WAVE_THREADS) k_batch_items(BatchArgs A) {
    __shared__ uint64_t sh[WAVE_THREADS];
    __shared__ uint64_t s_start[WAVE_THREADS + 1];
    __shared__ uint32_t s_kind[WAVE_THREADS];
    __shared__ uint64_t s_base, s_np;
    const int t = threadIdx.x;
    for (uint32_t jb = blockIdx.x; jb < A.n_jobs; jb += gridDim.x) {
        const BatchJob J = A.jobs[jb];
        const uint64_t nbits = J.blen * 8;
        __syncthreads();
        if (t == 0) {
            s_base = 0;  // cells used so far
            s_np = 0;    // items written so far
        }
        __syncthreads();
        // the job's items WAVE_THREADS at a time; the start of a tile's first
        // item after the previous tile is carried in s_start[WAVE_THREADS]
        for (uint32_t q0 = 0; q0 < J.K; q0 += WAVE_THREADS) {
            const uint32_t q = q0 + t;
            uint64_t st = ~0ull;
            uint32_t kind = 0;
            if (q < J.K) {
                if (q == 0) {
                    st = 0;
                } else {
                    const unsigned long long key = A.keys[J.item_first + q];
                    if (key != ~0ull) {
                        const uint64_t d = key >> 4, x = batch_ideal(nbits, q, J.K);
                        st = (key & 8u) ? x - d : x + d;
                        kind = (uint32_t)(key & 7u);
                        // the same start as the previous item's choice: dropped
                        const unsigned long long pk = A.keys[J.item_first + q - 1];
                        if (q > 1 && pk != ~0ull) {
                            const uint64_t px = batch_ideal(nbits, q - 1, J.K);
                            if (((pk & 8u) ? px - (pk >> 4) : px + (pk >> 4)) == st) st = ~0ull;
                        }
                    }
                }
            }
            uint64_t ex;
            const uint64_t n_here = block_scan(st != ~0ull ? 1 : 0, sh, &ex);
            // compact the present starts of this tile into s_start
            if (st != ~0ull) {
                s_start[ex] = st;
                s_kind[ex] = kind;
            }
            __syncthreads();
            // the next present start after the tile: the first of the next tile,
            // found by the next iteration; so write items one tile late, except
            // the last present one of the job, which needs the following tile
            // first. Simpler: defer each item until its successor is known.
            const uint64_t np0 = s_np;
            // items np0 .. np0 + n_here - 1 get their starts; the item before
            // them (np0 - 1, held back) now learns its end hint
            uint64_t cap = 0;
            if ((uint64_t)t < n_here) {
                const uint64_t my = s_start[t];
                const uint64_t next = (uint64_t)t + 1 < n_here ? s_start[t + 1] : ~0ull;
                ChunkItem it;
                it.in_off = J.in_off;
                it.in_len = J.blen;
                it.start_bit = my;
                it.end_hint = next;  // ~0: fixed below once the next tile is seen
                const uint64_t span = ((next == ~0ull ? nbits : next) - my + 7) / 8;
                cap = ((uint64_t)((double)span * J.expand) + 65536 + 7) & ~7ull;
                it.out_cap = cap;
                it.out_off = 0;
                it.flags = ITEM_MARKERS | (s_kind[t] == 1 ? ITEM_STORED_START
                                            : s_kind[t] == 3 ? (ITEM_STORED_START | ITEM_EMPTY_STORED) : 0u);
                it.id = J.item_first + (uint32_t)(np0 + t);
                A.items[J.item_first + np0 + t] = it;
            }
            __syncthreads();
            // the held-back last item of the previous tile ends where this tile's first begins
            if (t == 0 && np0 > 0 && n_here > 0) {
                ChunkItem& pv = A.items[J.item_first + np0 - 1];
                pv.end_hint = s_start[0];
                const uint64_t span = (s_start[0] - pv.start_bit + 7) / 8;
                pv.out_cap = ((uint64_t)((double)span * J.expand) + 65536 + 7) & ~7ull;
            }
            __syncthreads();
            if (t == 0) s_np = np0 + n_here;
            __syncthreads();
        }
        // slot offsets: a prefix of the caps over the job's present items
        const uint64_t np = s_np;
        for (uint64_t p0 = 0; p0 < np; p0 += WAVE_THREADS) {
            const uint64_t p = p0 + t;
            const uint64_t cap = p < np ? A.items[J.item_first + p].out_cap : 0;
            uint64_t ex;
            const uint64_t tot = block_scan(cap, sh, &ex);
            if (p < np) A.items[J.item_first + p].out_off = J.arena + s_base + ex;
            __syncthreads();
            if (t == 0) s_base += tot;
            __syncthreads();
        }
        for (uint32_t q = (uint32_t)np + t; q < J.K; q += WAVE_THREADS) {
            ChunkItem it{};
            it.in_off = J.in_off;
            it.in_len = J.blen;
            it.start_bit = nbits;
            it.end_hint = ~0ull;
            it.out_off = J.arena;
            it.flags = ITEM_SKIP;
            it.id = J.item_first + q;
            A.items[J.item_first + q] = it;
        }
        if (t == 0) {
            WaveJob W;
            W.first = J.item_first;
            W.n = (uint32_t)np;
            W.last_item = J.item_first + (uint32_t)np - 1;
            W.piece_off = J.piece_off;
            W.piece_cap = J.piece_cap;
            W.n_all = J.K;
            W.out_cap = J.dst_off + J.dst_cap;
            W.member_start = J.dst_off;
            A.wjobs[jb] = W;
        }
    }
}

// ------------------------------------------------------- CRC-32
// Raw CRC (register starts at 0, no final inversion) is linear:
//   raw(A||B) = raw(A) * x^(8|B|) + raw(B)   (mod P)
// and crc32(M) = raw(M) ^ (0xffffffff * x^(8|M|)) ^ 0xffffffff.
// Multiplication mod P is bit-serial in the reflected domain (bit 31 = x^0).
__device__ __forceinline__ uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
    uint32_t p = 0;
    for (int i = 0; i < 32; i++) {
        p ^= (0u - ((a >> (31 - i)) & 1u)) & b;
        b = (b >> 1) ^ ((0u - (b & 1u)) & 0xEDB88320u);
    }
    return p;
}
__device__ __forceinline__ uint32_t xpow8n(uint64_t n) {  // x^(8n) mod P
    uint32_t p = 0x80000000u;
    int k = 3;
    while (n) {
        if (n & 1) p = gf2_mulmod(c_x2k[k], p);
        n >>= 1;
        k++;
    }
    return p;
}

constexpr int CRC_THREADS = 256;

struct CrcArgs {
    const uint8_t* data;
    const CrcPiece* pieces;
    uint32_t n_pieces;
    uint32_t* piece_crc;   // raw CRC per piece
    const uint32_t* table; // 8 x 256 slice-by-8 table
    const uint32_t* n_dev; // when set, the piece count is read here
};

// One CTA per piece; each warp takes a contiguous 1/8th, each lane a
// contiguous 1/32nd of that; lanes and warps are combined with gf2_mulmod.
__global__ void __launch_bounds__(CRC_THREADS) k_crc_pieces(CrcArgs A) {
    __shared__ uint32_t T[8][256];
    __shared__ uint32_t wcrc[CRC_THREADS / 32];
    __shared__ uint64_t wlen[CRC_THREADS / 32];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) T[i >> 8][i & 255] = A.table[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t n_pieces = A.n_dev ? *A.n_dev : A.n_pieces;
    for (uint32_t pi = blockIdx.x; pi < n_pieces; pi += gridDim.x) {
        const CrcPiece pc = A.pieces[pi];
        const uint64_t per_thread = (pc.len + blockDim.x - 1) / blockDim.x;
        const uint64_t seg = (per_thread + 7) & ~7ull;
        const uint64_t t = (uint64_t)warp * 32 + lane;
        uint64_t b = t * seg;
        uint64_t e = b + seg;
        if (b > pc.len) b = pc.len;
        if (e > pc.len) e = pc.len;
        const uint8_t* p = A.data + pc.start;
        uint32_t c = 0;
        uint64_t i = b;
        for (; i < e && ((uintptr_t)(p + i) & 7); i++) c = T[0][(c ^ p[i]) & 0xff] ^ (c >> 8);
        for (; i + 8 <= e; i += 8) {
            uint2 w = *reinterpret_cast<const uint2*>(p + i);
            uint32_t lo = w.x ^ c, hi = w.y;
            c = T[7][lo & 0xff] ^ T[6][(lo >> 8) & 0xff] ^ T[5][(lo >> 16) & 0xff] ^ T[4][lo >> 24] ^
                T[3][hi & 0xff] ^ T[2][(hi >> 8) & 0xff] ^ T[1][(hi >> 16) & 0xff] ^ T[0][hi >> 24];
        }
        for (; i < e; i++) c = T[0][(c ^ p[i]) & 0xff] ^ (c >> 8);
        uint64_t len = e - b;
        // combine lanes in order: (c_a, l_a) (+) (c_b, l_b) = (c_a*x^(8 l_b) ^ c_b, l_a + l_b)
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t oc = __shfl_down_sync(FULLMASK, c, o);
            uint64_t ol = __shfl_down_sync(FULLMASK, len, o);
            if ((lane & (2 * o - 1)) == 0 && lane + o < 32) {
                c = (ol ? gf2_mulmod(c, xpow8n(ol)) : c) ^ oc;
                len += ol;
            }
        }
        if (lane == 0) {
            wcrc[warp] = c;
            wlen[warp] = len;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t cc = wcrc[0];
            for (int w = 1; w < nw; w++)
                if (wlen[w]) cc = gf2_mulmod(cc, xpow8n(wlen[w])) ^ wcrc[w];
            A.piece_crc[pi] = cc;
        }
        __syncthreads();
    }
}

// Coalesced form for the decode paths. In each 512-byte row of a piece, lane l
// of a warp takes bytes [16l, 16l + 16) with one 16-byte load, so a warp reads
// whole rows. Each lane keeps a CRC register over its own 16-byte chunks as if
// the other lanes' 496 bytes between them were zeros: before each chunk the
// register is advanced over 496 zero bytes with four lookups (Z tables, x^3968
// per byte position). Then slice-by-8 folds in the 16 bytes. Lane registers
// are shifted to their place in the last row and XORed, warps' segments are
// combined in order, and the unaligned head and the partial last row are
// folded in serially.
constexpr int CRCW_THREADS = 256;
constexpr int CRCW_ROW = 512;  // bytes per warp row (32 lanes x 16)

struct CrcWideArgs {
    const uint8_t* data;
    const CrcPiece* pieces;
    uint32_t n_pieces;
    uint32_t* piece_crc;    // raw CRC per piece
    const uint32_t* table;  // 12 x 256: slice-by-8, then the 496-zero-byte advance per byte position
    const uint32_t* n_dev;  // when set, the piece count is read here
};

__global__ void __launch_bounds__(CRCW_THREADS) k_crc_pieces_wide(CrcWideArgs A) {
    __shared__ uint32_t T[8][256];
    __shared__ uint32_t Z[4][256];
    __shared__ uint32_t wcrc[CRCW_THREADS / 32];
    __shared__ uint64_t wlen[CRCW_THREADS / 32];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) T[i >> 8][i & 255] = A.table[i];
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) Z[i >> 8][i & 255] = A.table[8 * 256 + i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = CRCW_THREADS / 32;
    const uint32_t n_pieces = A.n_dev ? *A.n_dev : A.n_pieces;
    for (uint32_t pi = blockIdx.x; pi < n_pieces; pi += gridDim.x) {
        const CrcPiece pc = A.pieces[pi];
        const uint8_t* p = A.data + pc.start;
        const uint64_t head = pc.len < ((16 - ((uintptr_t)p & 15)) & 15) ? pc.len : ((16 - ((uintptr_t)p & 15)) & 15);
        const uint64_t rows = (pc.len - head) / CRCW_ROW;
        const uint64_t r0 = (uint64_t)warp * rows / NW, r1 = (uint64_t)(warp + 1) * rows / NW;
        const uint4* q = reinterpret_cast<const uint4*>(p + head);
        uint32_t a = 0;
        for (uint64_t r = r0; r < r1; r++) {
            const uint4 w = q[r * 32 + lane];
            a = Z[0][a & 255] ^ Z[1][(a >> 8) & 255] ^ Z[2][(a >> 16) & 255] ^ Z[3][a >> 24];
            uint32_t lo = w.x ^ a, hi = w.y;
            a = T[7][lo & 0xff] ^ T[6][(lo >> 8) & 0xff] ^ T[5][(lo >> 16) & 0xff] ^ T[4][lo >> 24] ^
                T[3][hi & 0xff] ^ T[2][(hi >> 8) & 0xff] ^ T[1][(hi >> 16) & 0xff] ^ T[0][hi >> 24];
            lo = w.z ^ a;
            hi = w.w;
            a = T[7][lo & 0xff] ^ T[6][(lo >> 8) & 0xff] ^ T[5][(lo >> 16) & 0xff] ^ T[4][lo >> 24] ^
                T[3][hi & 0xff] ^ T[2][(hi >> 8) & 0xff] ^ T[1][(hi >> 16) & 0xff] ^ T[0][hi >> 24];
        }
        // bytes after this lane's last chunk in the segment's last row
        if (r1 > r0 && lane < 31) a = gf2_mulmod(a, xpow8n((uint64_t)(31 - lane) * 16));
        for (int o = 16; o; o >>= 1) a ^= __shfl_xor_sync(FULLMASK, a, o);
        if (lane == 0) {
            wcrc[warp] = a;
            wlen[warp] = (r1 - r0) * CRCW_ROW;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t cc = 0;
            for (uint64_t i = 0; i < head; i++) cc = T[0][(cc ^ p[i]) & 0xff] ^ (cc >> 8);
            for (int w = 0; w < NW; w++)
                if (wlen[w]) cc = gf2_mulmod(cc, xpow8n(wlen[w])) ^ wcrc[w];
            for (uint64_t i = head + rows * CRCW_ROW; i < pc.len; i++) cc = T[0][(cc ^ p[i]) & 0xff] ^ (cc >> 8);
            A.piece_crc[pi] = cc;
        }
        __syncthreads();
    }
}

struct CrcMemberArgs {
    const CrcPiece* pieces;
    const uint32_t* piece_crc;
    const uint32_t* member_piece_start;  // n_members + 1
    uint32_t n_members;
    const uint32_t* expected_crc;
    const uint32_t* expected_isize;
    uint32_t* got_crc;
    uint64_t* got_len;
    int32_t* status;  // DS_OK / DS_CRC / DS_ISIZE
    const uint32_t* n_dev;  // when set, the member count is read here
};

// One warp per member: fold its pieces in order, finalise, compare with the trailer.
__global__ void k_crc_members(CrcMemberArgs A) {
    const int lane = threadIdx.x & 31;
    const uint32_t n_members = A.n_dev ? *A.n_dev : A.n_members;
    for (uint32_t m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; m < n_members;
         m += (gridDim.x * blockDim.x) >> 5) {  // warp-uniform
        const uint32_t p0 = A.member_piece_start[m], p1 = A.member_piece_start[m + 1];
        const uint32_t np = p1 - p0;
        const uint32_t per = (np + 31) / 32;
        uint32_t b = p0 + lane * per, e = b + per;
        if (b > p1) b = p1;
        if (e > p1) e = p1;
        uint32_t c = 0;
        uint64_t len = 0;
        uint64_t xl = 0;          // the length whose x^(8 len) is in xp: pieces mostly share
        uint32_t xp = 0x80000000u;  // one length (256 KiB), so one multiply each
        for (uint32_t i = b; i < e; i++) {
            const uint64_t l = A.pieces[i].len;
            if (l && l != xl) {
                xp = xpow8n(l);
                xl = l;
            }
            c = (l ? gf2_mulmod(c, xp) : c) ^ A.piece_crc[i];
            len += l;
        }
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t oc = __shfl_down_sync(FULLMASK, c, o);
            uint64_t ol = __shfl_down_sync(FULLMASK, len, o);
            if ((lane & (2 * o - 1)) == 0 && lane + o < 32) {
                c = (ol ? gf2_mulmod(c, xpow8n(ol)) : c) ^ oc;
                len += ol;
            }
        }
        if (lane == 0) {
            uint32_t crc = c ^ (len ? gf2_mulmod(0xffffffffu, xpow8n(len)) : 0xffffffffu) ^ 0xffffffffu;
            A.got_crc[m] = crc;
            A.got_len[m] = len;
            int32_t st = DS_OK;
            if (crc != A.expected_crc[m]) st = DS_CRC;
            else if ((uint32_t)len != A.expected_isize[m]) st = DS_ISIZE;
            A.status[m] = st;
        }
    }
}

// ------------------------------------------------------- gzip header sniffing
// gzip.rs:311-351 parse_bgzf_block_size at byte `at` of s: the member size
// from the BC extra subfield (BSIZE + 1), or -1 (None).
__device__ int64_t dev_bgzf_size(const Src& s, uint64_t at) {
    const uint64_t n = s.hi - s.lo;
    if (at + 12 > n) return -1;
    if (src_byte(s, at) != 0x1f || src_byte(s, at + 1) != 0x8b || src_byte(s, at + 2) != 8 || !(src_byte(s, at + 3) & 4))
        return -1;
    const uint64_t xlen = src_byte(s, at + 10) | (src_byte(s, at + 11) << 8);
    if (at + 12 + xlen > n) return -1;
    uint64_t p = at + 12;
    const uint64_t end = p + xlen;
    while (p + 4 <= end) {
        const uint64_t slen = src_byte(s, p + 2) | (src_byte(s, p + 3) << 8);
        if (p + 4 + slen > end) return -1;
        if (src_byte(s, p) == 'B' && src_byte(s, p + 1) == 'C' && slen == 2)
            return (int64_t)(src_byte(s, p + 4) | (src_byte(s, p + 5) << 8)) + 1;
        p += 4 + slen;
    }
    return -1;
}

// Per file of a batch: header status and length (gzip.rs:252-300), the BGZF
// size of its first member (or -1), and the trailer's ISIZE (a size hint).
struct SniffArgs {
    const uint8_t* base;
    const uint64_t* off;
    const uint64_t* len;
    uint32_t n;
    int32_t* status;
    int32_t* msg;
    uint64_t* body_off;
    int64_t* bgzf;
    uint32_t* isize;
};

__global__ void k_sniff(SniffArgs A) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        const Src s = make_src(A.base + A.off[i], A.len[i]);
        uint64_t hl = 0;
        int msg = 0;
        A.status[i] = dev_parse_header(s, 0, &hl, &msg);
        A.msg[i] = msg;
        A.body_off[i] = hl;
        A.bgzf[i] = dev_bgzf_size(s, 0);
        A.isize[i] = A.len[i] >= 4 ? le32_at(s, A.len[i] - 4) : 0u;
    }
}

// ------------------------------------------------------- BGZF member walk
// The reference walks BGZF members one header at a time (pipeline.rs:1524-1541).
// Here every byte offset is tested for a BGZF member header in parallel, the
// hits are compacted in file order (count, prefix, collect), and one warp
// follows the chain offset -> offset + size through the sorted hits, 32 at a
// time, writing the per-member work items, CRC pieces and trailer values.
// Hits that are not on the chain (header-like bytes inside compressed data)
// are skipped. Nothing returns to the host between these kernels and the
// decode that follows, so the whole BGZF decode is one captured graph.
constexpr int BG_THREADS = 256;
constexpr int BG_SPAN = 16;                      // bytes per thread per step
constexpr int BG_STEP = BG_THREADS * BG_SPAN;    // bytes per block per step

struct BgzfScanArgs {
    const uint8_t* file;
    uint64_t len;
    uint64_t per_block;      // bytes per block (a multiple of BG_STEP)
    uint32_t* block_count;   // [gridDim.x]
    uint32_t* block_base;    // [gridDim.x + 1]
    uint64_t* cand_off;
    uint32_t* cand_size;
    uint32_t cap;
    uint32_t* n_cand;
};

// hits in this thread's BG_SPAN bytes starting at p0, as a bit mask; sizes in sz[]
__device__ __forceinline__ uint32_t bg_hits(const Src& s, uint64_t p0, uint64_t len, uint32_t* sz) {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < BG_SPAN; k++) {
        const uint64_t p = p0 + k;
        if (p < len && src_byte(s, p) == 0x1f && src_byte(s, p + 1) == 0x8b) {
            const int64_t z = dev_bgzf_size(s, p);
            if (z >= 0) {
                m |= 1u << k;
                sz[k] = (uint32_t)z;
            }
        }
    }
    return m;
}

__global__ void __launch_bounds__(BG_THREADS) k_bgzf_count(BgzfScanArgs A) {
    __shared__ uint32_t tot;
    if (threadIdx.x == 0) tot = 0;
    __syncthreads();
    const Src s = make_src(A.file, A.len);
    const uint64_t b0 = (uint64_t)blockIdx.x * A.per_block;
    const uint64_t b1 = b0 + A.per_block < A.len ? b0 + A.per_block : A.len;
    uint32_t mine = 0;
    uint32_t sz[BG_SPAN];
    for (uint64_t p = b0 + (uint64_t)threadIdx.x * BG_SPAN; p < b1; p += BG_STEP)
        mine += __popc(bg_hits(s, p, b1, sz));
    mine = warp_sum(mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&tot, mine);
    __syncthreads();
    if (threadIdx.x == 0) A.block_count[blockIdx.x] = tot;
}

// one block: exclusive prefix of the per-block counts
__global__ void __launch_bounds__(1024) k_bgzf_prefix(BgzfScanArgs A, uint32_t n_blocks) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < n_blocks; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n_blocks ? A.block_count[i] : 0u;
        uint32_t x = v;  // inclusive scan in the warp
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULLMASK, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULLMASK, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = carry + (warp ? wsum[warp - 1] : 0u) + x - v;
        if (i < n_blocks) A.block_base[i] = before;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        A.block_base[n_blocks] = carry;
        *A.n_cand = carry;
    }
}

__global__ void __launch_bounds__(BG_THREADS) k_bgzf_collect(BgzfScanArgs A) {
    __shared__ uint32_t wsum[BG_THREADS / 32];
    __shared__ uint32_t run;
    if (threadIdx.x == 0) run = A.block_base[blockIdx.x];
    __syncthreads();
    const Src s = make_src(A.file, A.len);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t b0 = (uint64_t)blockIdx.x * A.per_block;
    const uint64_t b1 = b0 + A.per_block < A.len ? b0 + A.per_block : A.len;
    uint32_t sz[BG_SPAN];
    for (uint64_t q = b0; q < b1; q += BG_STEP) {  // block-uniform trip count
        const uint64_t p = q + (uint64_t)threadIdx.x * BG_SPAN;
        const uint32_t m = p < b1 ? bg_hits(s, p, b1, sz) : 0u;
        const uint32_t v = __popc(m);
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULLMASK, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        uint32_t wb = 0, tot = 0;
        for (int w = 0; w < BG_THREADS / 32; w++) {
            if (w < warp) wb += wsum[w];
            tot += wsum[w];
        }
        uint32_t at = run + wb + x - v;
        for (uint32_t mm = m; mm; mm &= mm - 1) {
            const int k = __ffs((int)mm) - 1;
            if (at < A.cap) {
                A.cand_off[at] = p + (uint64_t)k;
                A.cand_size[at] = sz[k];
            }
            at++;
        }
        __syncthreads();
        if (threadIdx.x == 0) run += tot;
        __syncthreads();
    }
}

enum : uint32_t { BG_TRUNCATED = 1, BG_CAND_OVERFLOW = 2, BG_ITEM_OVERFLOW = 4, BG_OUT_CAPACITY = 8 };

struct BgzfChainArgs {
    const uint8_t* file;
    uint64_t len;
    const uint64_t* cand_off;
    const uint32_t* cand_size;
    const uint32_t* n_cand;
    uint32_t cap;
    ChunkItem* items;
    uint32_t item_cap;
    CrcPiece* pieces;
    uint32_t* mpiece;        // member -> first piece (one piece per member), n + 1 entries
    uint32_t* exp_crc;
    uint32_t* exp_isize;
    uint64_t out_cap;
    uint32_t* n_members;     // members to decode (0 when they do not fit)
    uint64_t* info;          // [0] end of the member chain, [1] output bytes, [2] BG_* flags, [3] members on the chain
};

// One warp. Member k+1 starts where member k ends (pipeline.rs:1524-1541).
__global__ void __launch_bounds__(32) k_bgzf_chain(BgzfChainArgs A) {
    const int lane = threadIdx.x & 31;
    const Src s = make_src(A.file, A.len);
    uint32_t flags = 0;
    uint32_t n = *A.n_cand;
    if (n > A.cap) {
        flags |= BG_CAND_OVERFLOW;
        n = A.cap;
    }
    uint64_t expected = 0, total = 0;
    uint32_t i = 0, m = 0;
    while (expected < A.len) {
        // first hit at or after `expected`
        bool found = false;
        while (i < n) {
            const uint32_t j = i + lane;
            const bool ge = j >= n || A.cand_off[j] >= expected;
            const uint32_t bal = __ballot_sync(FULLMASK, ge);
            if (bal) {
                i += __ffs((int)bal) - 1;
                found = true;
                break;
            }
            i += 32;
        }
        if (!found || i >= n || A.cand_off[i] != expected) break;  // no member here: the chain ends
        const uint32_t j = i + lane;
        const bool ok = j < n;
        const uint64_t off = ok ? A.cand_off[j] : 0;
        const uint64_t sz = ok ? A.cand_size[j] : 0;
        const uint64_t prev_end = __shfl_up_sync(FULLMASK, off + sz, 1);
        const bool link = ok && (lane == 0 ? off == expected : off == prev_end);
        const bool fits = off + sz <= A.len;
        const uint32_t acc = __ballot_sync(FULLMASK, link && fits);
        const uint32_t k = ~acc ? (uint32_t)(__ffs((int)~acc) - 1) : 32u;  // leading run of chained hits
        const uint32_t trunc = __ballot_sync(FULLMASK, link && !fits);
        const bool mine = (uint32_t)lane < k;
        uint32_t isz = 0, crc = 0;
        if (mine && sz >= 8) {
            crc = le32_at(s, off + sz - 8);
            isz = le32_at(s, off + sz - 4);
        }
        uint64_t x = isz;  // inclusive scan of member output sizes
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(FULLMASK, x, o);
            if (lane >= o) x += y;
        }
        if (mine && m + lane < A.item_cap) {
            const uint32_t idx = m + lane;
            ChunkItem it;
            it.in_off = off;
            it.in_len = sz;
            it.start_bit = 0;
            it.end_hint = ~0ull;
            it.out_off = total + x - isz;
            it.out_cap = isz;
            it.flags = ITEM_ONE_MEMBER;
            it.id = idx;
            A.items[idx] = it;
            A.pieces[idx] = CrcPiece{total + x - isz, isz};
            A.mpiece[idx] = idx;
            A.exp_crc[idx] = crc;
            A.exp_isize[idx] = isz;
        }
        if (k) {
            total += __shfl_sync(FULLMASK, x, (int)k - 1);
            expected = __shfl_sync(FULLMASK, off + sz, (int)k - 1);
            m += k;
            i += k;
        }
        // the hit right after the run sits where the chain expects a member
        // but ends past the file: truncated (the host walk's `pos + sz > len`)
        if (k < 32 && ((trunc >> k) & 1u)) {
            flags |= BG_TRUNCATED;
            break;
        }
    }
    if (m > A.item_cap) flags |= BG_ITEM_OVERFLOW;
    if (total > A.out_cap) flags |= BG_OUT_CAPACITY;
    if (lane == 0) {
        const uint32_t nm = (flags & (BG_CAND_OVERFLOW | BG_ITEM_OVERFLOW | BG_OUT_CAPACITY)) ? 0u : m;
        *A.n_members = nm;
        if (nm < A.item_cap) A.mpiece[nm] = nm;
        A.info[0] = expected;
        A.info[1] = total;
        A.info[2] = flags;
        A.info[3] = m;
    }
}

// After the decode: every member's CRC piece covers what was decoded (ISIZE
// was only its slot size) and is checked against the trailer that followed
// its deflate stream, as one-member decoding reads it.
__global__ void k_bgzf_fix(const ChunkResult* res, CrcPiece* pieces, uint32_t* exp_crc, uint32_t* exp_isize,
                           const uint32_t* n_members) {
    const uint32_t n = *n_members;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const ChunkResult r = res[i];
        pieces[i].len = r.status == DS_OK ? r.n_cells : 0;
        exp_crc[i] = (uint32_t)r.markers;
        exp_isize[i] = (uint32_t)(r.markers >> 32);
    }
}

// First member (in file order) whose decode failed -> first[0], and first
// member whose CRC32/ISIZE failed -> first[1] (both stay ~0 when none did).
__global__ void k_bgzf_first_bad(const ChunkResult* res, const int32_t* crc_status, const uint32_t* n_members,
                                 uint32_t* first) {
    const uint32_t n = *n_members;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (res[i].status != DS_OK) atomicMin(&first[0], i);
        else if (crc_status[i] != DS_OK) atomicMin(&first[1], i);
    }
}

}  // namespace rrg

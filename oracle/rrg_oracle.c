/*
 * rrg_oracle.c — CPU restatement of rusty_rapidgzip's gzip/DEFLATE decode path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); see
 * rrg_oracle.h. Written from the reference's behaviour and RFC 1951/1952, not
 * translated line by line. Reference paths are relative to the rusty_rapidgzip
 * repository, with rrg/ = crates/rusty-rapidgzip/.
 *
 * Deliberate semantic choices (documented for parity reviews):
 *  - The inflate loops use exact end-of-input semantics (an error only when a
 *    bit that is actually needed is missing), like the reference's own
 *    differential oracle rrg/src/deflate/safe_inflate.rs. The reference's fast
 *    kernels demand 48 buffered bits per symbol; inside a gzip member the
 *    8-byte trailer always supplies them, so valid files decode identically.
 *  - The block finder keeps the reference's exact peek semantics (10 bits for
 *    a LUT probe, 15 for a long code) and its 13-bit skip table, so it returns
 *    the very offsets find_next_dynamic_block returns.
 */
#define _GNU_SOURCE
#include "rrg_oracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

enum {
    ST_OK = 0,
    ST_IO = 1,
    ST_BAD_MAGIC = 2,
    ST_UNSUPPORTED_METHOD = 3,
    ST_RESERVED_FLAGS = 4,
    ST_TRUNCATED = 5,
    ST_CRC = 6,
    ST_ISIZE = 7,
    ST_EOF = 8,
    ST_INVALID = 9,
    ST_OOM = 21,
};

static void set_err(orc_error* err, int code, const char* msg) {
    if (!err) return;
    memset(err, 0, sizeof(*err));
    err->code = code;
    if (msg) snprintf(err->message, sizeof(err->message), "%s", msg);
}

void orc_free(void* p) { free(p); }

/* ------------------------------------------------------------------------ */
/* CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320).                      */
/* Table-driven update (slice-by-8) and the GF(2) combine:                    */
/*   crc(A||B) = crc(A) * x^(8|B|) + crc(B)   (mod P)                         */
/* which holds for the pre/post-inverted CRC because the inversion terms      */
/* cancel. Multiplication mod P is done bit-serially in the reflected domain. */
/* ------------------------------------------------------------------------ */
#define CRC_POLY 0xEDB88320u
static uint32_t crc_tab[8][256];
static uint32_t x2k_tab[64]; /* x^(2^k) mod P, reflected */
static pthread_once_t crc_once = PTHREAD_ONCE_INIT;

static uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
    /* reflected: bit 31 = x^0. Walk a's coefficients from x^0 upward while b
     * is multiplied by x each step. */
    uint32_t prod = 0;
    for (int i = 0; i < 32; i++) {
        if (a & (0x80000000u >> i)) prod ^= b;
        b = (b & 1u) ? (b >> 1) ^ CRC_POLY : (b >> 1);
    }
    return prod;
}

static void crc_init(void) {
    for (uint32_t n = 0; n < 256; n++) {
        uint32_t c = n;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? (c >> 1) ^ CRC_POLY : (c >> 1);
        crc_tab[0][n] = c;
    }
    for (uint32_t n = 0; n < 256; n++) {
        uint32_t c = crc_tab[0][n];
        for (int t = 1; t < 8; t++) {
            c = crc_tab[0][c & 0xff] ^ (c >> 8);
            crc_tab[t][n] = c;
        }
    }
    x2k_tab[0] = 0x40000000u; /* x^1 */
    for (int k = 1; k < 64; k++) x2k_tab[k] = gf2_mulmod(x2k_tab[k - 1], x2k_tab[k - 1]);
}

uint32_t orc_crc32(uint32_t crc, const uint8_t* p, size_t n) {
    pthread_once(&crc_once, crc_init);
    uint32_t c = ~crc;
    while (n && ((uintptr_t)p & 7)) {
        c = crc_tab[0][(c ^ *p++) & 0xff] ^ (c >> 8);
        n--;
    }
    while (n >= 8) {
        uint64_t w;
        memcpy(&w, p, 8);
        uint32_t lo = (uint32_t)w ^ c, hi = (uint32_t)(w >> 32);
        c = crc_tab[7][lo & 0xff] ^ crc_tab[6][(lo >> 8) & 0xff] ^ crc_tab[5][(lo >> 16) & 0xff] ^
            crc_tab[4][lo >> 24] ^ crc_tab[3][hi & 0xff] ^ crc_tab[2][(hi >> 8) & 0xff] ^
            crc_tab[1][(hi >> 16) & 0xff] ^ crc_tab[0][hi >> 24];
        p += 8;
        n -= 8;
    }
    while (n--) c = crc_tab[0][(c ^ *p++) & 0xff] ^ (c >> 8);
    return ~c;
}

/* x^(8*len) mod P */
static uint32_t x_pow_8n(uint64_t len) {
    pthread_once(&crc_once, crc_init);
    uint32_t p = 0x80000000u; /* x^0 */
    int k = 3;                /* 8 = 2^3 */
    while (len) {
        if (len & 1) p = gf2_mulmod(x2k_tab[k & 63], p);
        len >>= 1;
        k++;
    }
    return p;
}

uint32_t orc_crc32_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b) {
    return gf2_mulmod(x_pow_8n(len_b), crc_a) ^ crc_b;
}

/* ------------------------------------------------------------------------ */
/* Growable buffers                                                          */
/* ------------------------------------------------------------------------ */
typedef struct { uint8_t* p; size_t len, cap; } vec8;
typedef struct { uint16_t* p; size_t len, cap; } vec16;
typedef struct { uint32_t* pos; uint16_t* off; size_t len, cap; } vecm;
typedef struct { orc_member_boundary* p; size_t len, cap; } vecb;

static int vec8_reserve(vec8* v, size_t extra) {
    if (v->len + extra <= v->cap) return 0;
    size_t nc = v->cap ? v->cap : 65536;
    while (nc < v->len + extra) nc *= 2;
    uint8_t* np = (uint8_t*)realloc(v->p, nc);
    if (!np) return -1;
    v->p = np;
    v->cap = nc;
    return 0;
}
static int vec16_reserve(vec16* v, size_t extra) {
    if (v->len + extra <= v->cap) return 0;
    size_t nc = v->cap ? v->cap : 65536;
    while (nc < v->len + extra) nc *= 2;
    uint16_t* np = (uint16_t*)realloc(v->p, nc * 2);
    if (!np) return -1;
    v->p = np;
    v->cap = nc;
    return 0;
}
static int vecm_push(vecm* v, uint32_t pos, uint16_t off) {
    if (v->len == v->cap) {
        size_t nc = v->cap ? v->cap * 2 : 4096;
        uint32_t* a = (uint32_t*)realloc(v->pos, nc * 4);
        if (!a) return -1;
        v->pos = a;
        uint16_t* b = (uint16_t*)realloc(v->off, nc * 2);
        if (!b) return -1;
        v->off = b;
        v->cap = nc;
    }
    v->pos[v->len] = pos;
    v->off[v->len] = off;
    v->len++;
    return 0;
}
static int vecb_push(vecb* v, orc_member_boundary b) {
    if (v->len == v->cap) {
        size_t nc = v->cap ? v->cap * 2 : 8;
        orc_member_boundary* np = (orc_member_boundary*)realloc(v->p, nc * sizeof(*np));
        if (!np) return -1;
        v->p = np;
        v->cap = nc;
    }
    v->p[v->len++] = b;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* LSB-first bit reader (rrg/src/deflate/bitreader.rs:28-193).               */
/* ------------------------------------------------------------------------ */
typedef struct {
    const uint8_t* in;
    size_t len;
    size_t pos;   /* next unbuffered byte */
    uint64_t buf; /* low `bits` bits valid */
    uint32_t bits;
} bitrd;

static void br_init(bitrd* b, const uint8_t* in, size_t len) {
    b->in = in;
    b->len = len;
    b->pos = 0;
    b->buf = 0;
    b->bits = 0;
}
static inline uint64_t br_tell(const bitrd* b) { return (uint64_t)b->pos * 8 - b->bits; }

/* refill(n) of bitreader.rs:100-130: fast 8-byte load when possible, else
 * byte-wise until n bits are buffered; EOF when the input runs out first. */
static inline int br_refill(bitrd* b, uint32_t n) {
    if (b->bits >= n) return 0;
    if (b->pos + 8 <= b->len && b->bits <= 56) {
        uint64_t c;
        memcpy(&c, b->in + b->pos, 8);
        b->buf |= c << b->bits;
        uint32_t add = (64 - b->bits) / 8;
        b->pos += add;
        b->bits += add * 8;
        return 0;
    }
    while (b->bits < n) {
        if (b->pos >= b->len) return ST_EOF;
        b->buf |= (uint64_t)b->in[b->pos++] << b->bits;
        b->bits += 8;
    }
    return 0;
}
static inline int br_read(bitrd* b, uint32_t n, uint32_t* v) {
    if (n == 0) {
        *v = 0;
        return 0;
    }
    int r = br_refill(b, n);
    if (r) return r;
    *v = (uint32_t)(b->buf & ((1ull << n) - 1));
    b->buf >>= n;
    b->bits -= n;
    return 0;
}
static inline void br_byte_align(bitrd* b) {
    uint32_t d = b->bits & 7;
    b->buf >>= d;
    b->bits -= d;
}
static int br_seek(bitrd* b, uint64_t pos) {
    if (pos > (uint64_t)b->len * 8) return ST_EOF;
    b->pos = (size_t)(pos / 8);
    b->buf = 0;
    b->bits = 0;
    uint32_t sub = (uint32_t)(pos & 7);
    if (sub) {
        int r = br_refill(b, sub);
        if (r) return r;
        b->buf >>= sub;
        b->bits -= sub;
    }
    return 0;
}
/* Fill as many bits as fit (<= 64) without failing; used by the exact-EOF
 * inflate loops, which check availability per consumption. */
static inline void br_fill_max(bitrd* b) {
    if (b->pos + 8 <= b->len) {
        uint64_t c;
        memcpy(&c, b->in + b->pos, 8);
        b->buf |= c << b->bits;
        b->pos += (63 - b->bits) >> 3;
        b->bits |= 56;
    } else {
        while (b->bits <= 56 && b->pos < b->len) {
            b->buf |= (uint64_t)b->in[b->pos++] << b->bits;
            b->bits += 8;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* RFC 1951 tables (rrg/src/deflate/tables.rs).                              */
/* ------------------------------------------------------------------------ */
static const uint8_t CL_ORDER[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
static const uint16_t LEN_BASE[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                      31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
static const uint8_t LEN_EXTRA[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                      2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
static const uint16_t DIST_BASE[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                       33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                       1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
static const uint8_t DIST_EXTRA[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                       6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

/* ------------------------------------------------------------------------ */
/* Canonical Huffman with a 10-bit LUT + long-code list                      */
/* (rrg/src/deflate/huffman.rs:83-428; entry layouts :9-69).                 */
/* ------------------------------------------------------------------------ */
#define LUT_BITS 10
#define LUT_SIZE (1u << LUT_BITS)
#define HUFF_LITERAL (1u << 31)
#define HUFF_EXCEPTIONAL (1u << 15)
enum { ENC_SIMPLE, ENC_LITLEN, ENC_DIST };

typedef struct {
    uint32_t rev;
    uint32_t len;
    uint32_t entry;
} longcode;
typedef struct {
    uint32_t lut[LUT_SIZE];
    longcode lc[288];
    int n_lc;
} huff;

static uint32_t encode_entry(uint32_t sym, uint32_t len, int enc) {
    switch (enc) {
    case ENC_SIMPLE: return (sym << 16) | len;
    case ENC_LITLEN:
        if (sym < 256) return HUFF_LITERAL | (sym << 16) | len;
        if (sym == 256) return HUFF_EXCEPTIONAL | len;
        if (sym <= 285)
            return ((uint32_t)LEN_BASE[sym - 257] << 16) | ((uint32_t)LEN_EXTRA[sym - 257] << 8) | len;
        return HUFF_EXCEPTIONAL | (sym << 16) | len;
    default:
        if (sym <= 29) return ((uint32_t)DIST_BASE[sym] << 16) | ((uint32_t)DIST_EXTRA[sym] << 8) | len;
        return HUFF_EXCEPTIONAL | len;
    }
}

static uint32_t rev_bits(uint32_t v, uint32_t n) {
    uint32_t r = 0;
    for (uint32_t i = 0; i < n; i++) {
        r = (r << 1) | (v & 1);
        v >>= 1;
    }
    return r;
}

/* huffman.rs:215-325 build_into: rejects lengths > 15, oversubscribed trees
 * with >= 2 symbols, and (strict) incomplete trees with >= 2 symbols. Codes
 * are the RFC 1951 §3.2.2 canonical codes, keyed bit-reversed. */
static int huff_build(huff* h, const uint8_t* lengths, int n, int strict, int enc, const char** why) {
    uint32_t count[16] = {0};
    for (int i = 0; i < n; i++) {
        if (lengths[i] > 15) {
            *why = "huffman code length > 15";
            return ST_INVALID;
        }
        count[lengths[i]]++;
    }
    count[0] = 0;
    uint64_t total = 0;
    uint32_t nsym = 0;
    for (int l = 1; l <= 15; l++) {
        total += (uint64_t)count[l] << (15 - l);
        nsym += count[l];
    }
    if (nsym >= 2 && total > (1u << 15)) {
        *why = "oversubscribed huffman tree";
        return ST_INVALID;
    }
    if (strict && nsym >= 2 && total != (1u << 15)) {
        *why = "incomplete huffman tree (strict)";
        return ST_INVALID;
    }
    uint32_t next[16];
    uint32_t code = 0;
    for (int l = 1; l <= 15; l++) {
        code = (code + count[l - 1]) << 1;
        next[l] = code;
    }
    memset(h->lut, 0, sizeof(h->lut));
    h->n_lc = 0;
    for (int s = 0; s < n; s++) {
        uint32_t l = lengths[s];
        if (!l) continue;
        uint32_t r = rev_bits(next[l]++, l);
        uint32_t e = encode_entry((uint32_t)s, l, enc);
        if (l <= LUT_BITS) {
            for (uint32_t i = r; i < LUT_SIZE; i += (1u << l)) h->lut[i] = e;
        } else {
            h->lc[h->n_lc].rev = r;
            h->lc[h->n_lc].len = l;
            h->lc[h->n_lc].entry = e;
            h->n_lc++;
        }
    }
    return 0;
}

static huff g_fixed_lit, g_fixed_dist;
static pthread_once_t fixed_once = PTHREAD_ONCE_INIT;
static void fixed_init(void) {
    uint8_t l[288];
    const char* why;
    for (int i = 0; i < 144; i++) l[i] = 8;
    for (int i = 144; i < 256; i++) l[i] = 9;
    for (int i = 256; i < 280; i++) l[i] = 7;
    for (int i = 280; i < 288; i++) l[i] = 8;
    huff_build(&g_fixed_lit, l, 288, 0, ENC_LITLEN, &why);
    for (int i = 0; i < 30; i++) l[i] = 5;
    huff_build(&g_fixed_dist, l, 30, 0, ENC_DIST, &why);
}

/* Exact-EOF symbol decode: a code is accepted only if all of its bits exist. */
static inline int huff_decode_exact(bitrd* b, const huff* h, uint32_t* entry, const char** why) {
    if (b->bits < 15) br_fill_max(b);
    uint32_t e = h->lut[b->buf & (LUT_SIZE - 1)];
    uint32_t l = e & 0xff;
    if (l) {
        if (l > b->bits) return ST_EOF;
        b->buf >>= l;
        b->bits -= l;
        *entry = e;
        return 0;
    }
    for (int i = 0; i < h->n_lc; i++) {
        const longcode* c = &h->lc[i];
        if (c->len <= b->bits && (b->buf & ((1ull << c->len) - 1)) == c->rev) {
            b->buf >>= c->len;
            b->bits -= c->len;
            *entry = c->entry;
            return 0;
        }
    }
    if (b->bits < 15) return ST_EOF;
    *why = "no matching huffman code";
    return ST_INVALID;
}

/* Reference-exact symbol decode for the block finder: HuffmanDecoder::lookup
 * (huffman.rs:356-366) requires 10 buffered bits, lookup_long (:379-389) 15. */
static inline int huff_decode_ref(bitrd* b, const huff* h, uint32_t* entry) {
    if (br_refill(b, LUT_BITS)) return ST_EOF;
    uint32_t e = h->lut[b->buf & (LUT_SIZE - 1)];
    uint32_t l = e & 0xff;
    if (l == 0) {
        if (br_refill(b, 15)) return ST_EOF;
        for (int i = 0; i < h->n_lc; i++) {
            const longcode* c = &h->lc[i];
            if ((b->buf & ((1ull << c->len) - 1)) == c->rev) {
                b->buf >>= c->len;
                b->bits -= c->len;
                *entry = c->entry;
                return 0;
            }
        }
        return ST_INVALID;
    }
    b->buf >>= l;
    b->bits -= l;
    *entry = e;
    return 0;
}

/* inflate.rs:74-145 read_dynamic_header (non-strict trees), after BFINAL/BTYPE. */
static int read_dynamic_header(bitrd* b, huff* lit, huff* dist, const char** why) {
    uint32_t v;
    int r;
    if ((r = br_read(b, 5, &v))) return r;
    uint32_t hlit = v + 257;
    if ((r = br_read(b, 5, &v))) return r;
    uint32_t hdist = v + 1;
    if ((r = br_read(b, 4, &v))) return r;
    uint32_t hclen = v + 4;
    if (hlit > 286 || hdist > 30) {
        *why = "dynamic block: HLIT/HDIST out of range";
        return ST_INVALID;
    }
    uint8_t cl[19] = {0};
    for (uint32_t i = 0; i < hclen; i++) {
        if ((r = br_read(b, 3, &v))) return r;
        cl[CL_ORDER[i]] = (uint8_t)v;
    }
    huff clh;
    if ((r = huff_build(&clh, cl, 19, 0, ENC_SIMPLE, why))) return r;
    uint8_t lengths[320];
    memset(lengths, 0, sizeof(lengths));
    uint32_t total = hlit + hdist, i = 0;
    while (i < total) {
        uint32_t e;
        if ((r = huff_decode_exact(b, &clh, &e, why))) return r;
        uint32_t sym = e >> 16;
        if (sym <= 15) {
            lengths[i++] = (uint8_t)sym;
        } else if (sym == 16) {
            if (i == 0) {
                *why = "code 16 with no previous";
                return ST_INVALID;
            }
            if ((r = br_read(b, 2, &v))) return r;
            uint32_t n = v + 3;
            if (i + n > total) {
                *why = "code 16 overruns lengths";
                return ST_INVALID;
            }
            uint8_t prev = lengths[i - 1];
            for (uint32_t j = 0; j < n; j++) lengths[i + j] = prev;
            i += n;
        } else if (sym == 17) {
            if ((r = br_read(b, 3, &v))) return r;
            uint32_t n = v + 3;
            if (i + n > total) {
                *why = "code 17 overruns lengths";
                return ST_INVALID;
            }
            i += n;
        } else if (sym == 18) {
            if ((r = br_read(b, 7, &v))) return r;
            uint32_t n = v + 11;
            if (i + n > total) {
                *why = "code 18 overruns lengths";
                return ST_INVALID;
            }
            i += n;
        } else {
            *why = "bad code-length symbol";
            return ST_INVALID;
        }
    }
    if (lengths[256] == 0) {
        *why = "EOB symbol has zero length";
        return ST_INVALID;
    }
    if ((r = huff_build(lit, lengths, (int)hlit, 0, ENC_LITLEN, why))) return r;
    if ((r = huff_build(dist, lengths + hlit, (int)hdist, 0, ENC_DIST, why))) return r;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Byte-wide inflate with a real window                                      */
/* (fast_inflate.rs:186-551 decode_one_block_preload / decode_compressed;    */
/*  back-references may not reach before `floor`, the member's first byte).  */
/* ------------------------------------------------------------------------ */
#define COPY_SLACK 16

static int inflate_codes_u8(bitrd* b, vec8* out, size_t floor, const huff* lit, const huff* dist,
                            const char** why) {
    int r;
    for (;;) {
        if (out->cap - out->len < 258 + COPY_SLACK + 8) {
            if (vec8_reserve(out, 1 << 16)) return ST_OOM;
        }
        if (b->bits < 48) br_fill_max(b);
        uint32_t e = lit->lut[b->buf & (LUT_SIZE - 1)];
        uint32_t l = e & 0xff;
        if (l && l <= b->bits) {
            b->buf >>= l;
            b->bits -= l;
        } else if ((r = huff_decode_exact(b, lit, &e, why))) {
            return r;
        }
        if (e & HUFF_LITERAL) {
            out->p[out->len++] = (uint8_t)(e >> 16);
            continue;
        }
        if (e & HUFF_EXCEPTIONAL) {
            if ((e >> 16) == 0) return 0; /* end of block */
            *why = "literal/length symbol out of range";
            return ST_INVALID;
        }
        uint32_t length = (e >> 16) & 0x1ff, ex = (e >> 8) & 0x1f;
        if (ex) {
            if (ex > b->bits) return ST_EOF;
            length += (uint32_t)(b->buf & ((1u << ex) - 1));
            b->buf >>= ex;
            b->bits -= ex;
        }
        uint32_t de = dist->lut[b->buf & (LUT_SIZE - 1)];
        l = de & 0xff;
        if (l && l <= b->bits) {
            b->buf >>= l;
            b->bits -= l;
        } else if ((r = huff_decode_exact(b, dist, &de, why))) {
            return r;
        }
        if (de & HUFF_EXCEPTIONAL) {
            *why = "distance symbol out of range";
            return ST_INVALID;
        }
        uint32_t d = de >> 16, dx = (de >> 8) & 0x1f;
        if (dx) {
            if (dx > b->bits) return ST_EOF;
            d += (uint32_t)(b->buf & ((1u << dx) - 1));
            b->buf >>= dx;
            b->bits -= dx;
        }
        size_t cur = out->len;
        if (d == 0) {
            *why = "zero back-reference distance";
            return ST_INVALID;
        }
        if (d > cur - floor) {
            *why = "back-reference distance out of bounds";
            return ST_INVALID;
        }
        uint8_t* dst = out->p + cur;
        const uint8_t* src = dst - d;
        if (d >= 8) {
            for (uint32_t k = 0; k < length; k += 8) memcpy(dst + k, src + k, 8);
        } else if (d == 1) {
            memset(dst, src[0], length);
        } else {
            for (uint32_t k = 0; k < length; k++) dst[k] = src[k];
        }
        out->len = cur + length;
    }
}

static int inflate_stored_u8(bitrd* b, vec8* out, const char** why) {
    uint32_t len, nlen;
    int r;
    br_byte_align(b);
    if ((r = br_read(b, 16, &len)) || (r = br_read(b, 16, &nlen))) return r;
    if ((len ^ 0xffffu) != nlen) {
        *why = "stored block: LEN/NLEN mismatch";
        return ST_INVALID;
    }
    if (vec8_reserve(out, len + COPY_SLACK)) return ST_OOM;
    /* drain whole bytes still in the bit buffer, then copy straight from input */
    while (len && b->bits >= 8) {
        out->p[out->len++] = (uint8_t)b->buf;
        b->buf >>= 8;
        b->bits -= 8;
        len--;
    }
    if (len) {
        if (b->pos + len > b->len) return ST_EOF;
        memcpy(out->p + out->len, b->in + b->pos, len);
        out->len += len;
        b->pos += len;
        b->buf = 0;
        b->bits = 0;
    }
    return 0;
}

/* One block, byte-wide (decode_one_block_preload, fast_inflate.rs:186-206). */
static int inflate_block_u8(bitrd* b, vec8* out, size_t floor, int* bfinal, const char** why) {
    uint32_t bf, bt;
    int r;
    if ((r = br_read(b, 1, &bf)) || (r = br_read(b, 2, &bt))) return r;
    *bfinal = (int)bf;
    if (bt == 0) return inflate_stored_u8(b, out, why);
    if (bt == 1) {
        pthread_once(&fixed_once, fixed_init);
        return inflate_codes_u8(b, out, floor, &g_fixed_lit, &g_fixed_dist, why);
    }
    if (bt == 2) {
        huff lit, dist;
        if ((r = read_dynamic_header(b, &lit, &dist, why))) return r;
        return inflate_codes_u8(b, out, floor, &lit, &dist, why);
    }
    *why = "reserved block type";
    return ST_INVALID;
}

/* ------------------------------------------------------------------------ */
/* Speculative u16-cell inflate (fast_inflate.rs:1762-2234).                 */
/* A cell < 0x100 is a literal byte; 0x8000|k is an unresolved byte that     */
/* copies the k-th byte before the chunk (k = 0 is the byte just before).   */
/* Copies move whole cells, so marker-ness propagates through back-refs.     */
/* ------------------------------------------------------------------------ */
#define MARKER16 0x8000u

static int inflate_codes_u16(bitrd* b, vec16* cells, const huff* lit, const huff* dist,
                             const char** why) {
    int r;
    for (;;) {
        if (cells->cap - cells->len < 258 + COPY_SLACK) {
            if (vec16_reserve(cells, 1 << 16)) return ST_OOM;
        }
        if (b->bits < 48) br_fill_max(b);
        uint32_t e = lit->lut[b->buf & (LUT_SIZE - 1)];
        uint32_t l = e & 0xff;
        if (l && l <= b->bits) {
            b->buf >>= l;
            b->bits -= l;
        } else if ((r = huff_decode_exact(b, lit, &e, why))) {
            return r;
        }
        if (e & HUFF_LITERAL) {
            cells->p[cells->len++] = (uint16_t)((e >> 16) & 0xff);
            continue;
        }
        if (e & HUFF_EXCEPTIONAL) {
            if ((e >> 16) == 0) return 0;
            *why = "literal/length symbol out of range";
            return ST_INVALID;
        }
        uint32_t length = (e >> 16) & 0x1ff, ex = (e >> 8) & 0x1f;
        if (ex) {
            if (ex > b->bits) return ST_EOF;
            length += (uint32_t)(b->buf & ((1u << ex) - 1));
            b->buf >>= ex;
            b->bits -= ex;
        }
        uint32_t de = dist->lut[b->buf & (LUT_SIZE - 1)];
        l = de & 0xff;
        if (l && l <= b->bits) {
            b->buf >>= l;
            b->bits -= l;
        } else if ((r = huff_decode_exact(b, dist, &de, why))) {
            return r;
        }
        if (de & HUFF_EXCEPTIONAL) {
            *why = "distance symbol out of range";
            return ST_INVALID;
        }
        uint32_t d = de >> 16, dx = (de >> 8) & 0x1f;
        if (dx) {
            if (dx > b->bits) return ST_EOF;
            d += (uint32_t)(b->buf & ((1u << dx) - 1));
            b->buf >>= dx;
            b->bits -= dx;
        }
        size_t cur = cells->len;
        uint16_t* o = cells->p;
        uint32_t k = 0;
        if (d > cur) {
            /* reference into the unknown prefix: emit marker cells
             * (fast_inflate.rs:2209-2222) */
            uint32_t pre = (uint32_t)(d - cur);
            if (pre > length) pre = length;
            for (; k < pre; k++) o[cur + k] = (uint16_t)(MARKER16 | (uint32_t)(d - cur - k - 1));
        }
        for (; k < length; k++) o[cur + k] = o[cur + k - d];
        cells->len = cur + length;
    }
}

static int inflate_block_u16(bitrd* b, vec16* cells, uint32_t btype, const char** why) {
    int r;
    if (btype == 0) {
        uint32_t len, nlen, v;
        br_byte_align(b);
        if ((r = br_read(b, 16, &len)) || (r = br_read(b, 16, &nlen))) return r;
        if ((len ^ 0xffffu) != nlen) {
            *why = "stored block: LEN/NLEN mismatch";
            return ST_INVALID;
        }
        if (vec16_reserve(cells, len + COPY_SLACK)) return ST_OOM;
        for (uint32_t i = 0; i < len; i++) {
            if ((r = br_read(b, 8, &v))) return r;
            cells->p[cells->len++] = (uint16_t)v;
        }
        return 0;
    }
    if (btype == 1) {
        pthread_once(&fixed_once, fixed_init);
        return inflate_codes_u16(b, cells, &g_fixed_lit, &g_fixed_dist, why);
    }
    if (btype == 2) {
        huff lit, dist;
        if ((r = read_dynamic_header(b, &lit, &dist, why))) return r;
        return inflate_codes_u16(b, cells, &lit, &dist, why);
    }
    *why = "reserved block type";
    return ST_INVALID;
}

/* extract_from_u16 (speculative.rs:66-142): low byte of each cell, 0 for a
 * marker cell, and the marker (out_pos, prefix_offset) recorded in order. */
static int extract_cells(const vec16* cells, vec8* bytes, vecm* markers) {
    size_t base = bytes->len;
    if (vec8_reserve(bytes, cells->len + COPY_SLACK)) return ST_OOM;
    for (size_t i = 0; i < cells->len; i++) {
        uint16_t c = cells->p[i];
        if (c & MARKER16) {
            bytes->p[base + i] = 0;
            if (vecm_push(markers, (uint32_t)(base + i), (uint16_t)(c & 0x7fff))) return ST_OOM;
        } else {
            bytes->p[base + i] = (uint8_t)c;
        }
    }
    bytes->len = base + cells->len;
    return 0;
}

#define WINDOW 32768u
#define HANDOFF_AT (2u * WINDOW)

/* decode_until_u16 (fast_inflate.rs:1794-1888): phase 1 in u16 cells until the
 * chunk ends, the member ends, or >= 64 Ki cells exist with a marker-free last
 * 32 Ki; then phase 2 byte-wide against the materialised history. */
static int decode_until_u16(bitrd* b, uint64_t end_hint, vec8* bytes, vecm* markers,
                            int* hit_bfinal, const char** why) {
    vec16 cells = {0};
    int r = 0;
    *hit_bfinal = 0;
    for (;;) {
        uint32_t bf, bt;
        if ((r = br_read(b, 1, &bf)) || (r = br_read(b, 2, &bt))) goto out;
        if ((r = inflate_block_u16(b, &cells, bt, why))) goto out;
        if (bf) {
            r = extract_cells(&cells, bytes, markers);
            *hit_bfinal = 1;
            goto out;
        }
        if (br_tell(b) >= end_hint) {
            r = extract_cells(&cells, bytes, markers);
            goto out;
        }
        if (cells.len >= HANDOFF_AT) {
            int clean = 1;
            for (size_t i = cells.len - WINDOW; i < cells.len; i++)
                if (cells.p[i] & MARKER16) {
                    clean = 0;
                    break;
                }
            if (clean) break;
        }
    }
    if ((r = extract_cells(&cells, bytes, markers))) goto out;
    free(cells.p);
    cells.p = NULL;
    for (;;) {
        int bf;
        if ((r = inflate_block_u8(b, bytes, 0, &bf, why))) goto out;
        if (bf) {
            *hit_bfinal = 1;
            break;
        }
        if (br_tell(b) >= end_hint) break;
    }
out:
    free(cells.p);
    return r;
}

/* decode_member_u8 (fast_inflate.rs:117-140): a member after the first in a
 * chunk starts with an empty window at out->len. */
static int decode_member_u8(bitrd* b, uint64_t end_hint, vec8* out, int* hit_bfinal, const char** why) {
    size_t floor = out->len;
    *hit_bfinal = 0;
    for (;;) {
        int bf, r;
        if ((r = inflate_block_u8(b, out, floor, &bf, why))) return r;
        if (bf) {
            *hit_bfinal = 1;
            return 0;
        }
        if (br_tell(b) >= end_hint) return 0;
    }
}

/* ------------------------------------------------------------------------ */
/* gzip framing (gzip.rs:252-351)                                            */
/* ------------------------------------------------------------------------ */
int orc_parse_header(const uint8_t* in, size_t len, size_t* hdr_len) {
    if (len < 10) return ST_TRUNCATED;
    if (in[0] != 0x1f || in[1] != 0x8b) return ST_BAD_MAGIC;
    if (in[2] != 8) return ST_UNSUPPORTED_METHOD;
    uint8_t flg = in[3];
    if (flg & 0xe0) return ST_RESERVED_FLAGS;
    size_t pos = 10;
    if (flg & 4) {
        if (pos + 2 > len) return ST_TRUNCATED;
        size_t xlen = (size_t)in[pos] | ((size_t)in[pos + 1] << 8);
        pos += 2 + xlen;
        if (pos > len) return ST_TRUNCATED;
    }
    for (int f = 8; f <= 16; f <<= 1) { /* FNAME then FCOMMENT */
        if (flg & f) {
            if (pos > len) return ST_TRUNCATED;
            const uint8_t* z = (const uint8_t*)memchr(in + pos, 0, len - pos);
            if (!z) return ST_TRUNCATED;
            pos = (size_t)(z - in) + 1;
        }
    }
    if (flg & 2) {
        if (pos + 2 > len) return ST_TRUNCATED;
        pos += 2;
    }
    *hdr_len = pos;
    return 0;
}

static int header_error(orc_error* err, int code, const uint8_t* in, size_t len) {
    set_err(err, code, code == ST_BAD_MAGIC ? "not a gzip file (bad magic)"
                       : code == ST_UNSUPPORTED_METHOD ? "unsupported compression method"
                       : code == ST_RESERVED_FLAGS ? "reserved gzip flag bits set"
                                                   : "truncated gzip stream");
    if (err && code == ST_UNSUPPORTED_METHOD && len > 2) err->expected = in[2];
    if (err && code == ST_RESERVED_FLAGS && len > 3) err->expected = in[3];
    return code;
}

int64_t orc_bgzf_block_size(const uint8_t* in, size_t len) {
    if (len < 12 || in[0] != 0x1f || in[1] != 0x8b || in[2] != 8) return -1;
    if (!(in[3] & 4)) return -1;
    size_t xlen = (size_t)in[10] | ((size_t)in[11] << 8);
    if (12 + xlen > len) return -1;
    size_t p = 12, end = 12 + xlen;
    while (p + 4 <= end) {
        size_t slen = (size_t)in[p + 2] | ((size_t)in[p + 3] << 8);
        if (p + 4 + slen > end) return -1;
        if (in[p] == 'B' && in[p + 1] == 'C' && slen == 2)
            return (int64_t)((uint32_t)in[p + 4] | ((uint32_t)in[p + 5] << 8)) + 1;
        p += 4 + slen;
    }
    return -1;
}

static inline uint32_t le32(const uint8_t* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

static int deflate_error(orc_error* err, int code, const char* why) {
    if (code == ST_EOF) set_err(err, code, "unexpected end of input");
    else if (code == ST_OOM) set_err(err, code, "out of memory");
    else set_err(err, code, why ? why : "invalid deflate stream");
    return code;
}

int orc_inflate_raw(const uint8_t* in, size_t len, uint8_t** out, size_t* out_len, uint64_t* end_bit,
                    orc_error* err) {
    bitrd b;
    br_init(&b, in, len);
    vec8 o = {0};
    const char* why = NULL;
    for (;;) {
        int bf, r = inflate_block_u8(&b, &o, 0, &bf, &why);
        if (r) {
            free(o.p);
            return deflate_error(err, r, why);
        }
        if (bf) break;
    }
    *out = o.p;
    *out_len = o.len;
    if (end_bit) *end_bit = br_tell(&b);
    return 0;
}

/* gzip.rs:87-141 decode_one_indexed over in[0..len): returns consumed bytes. */
static int decode_member_checked(const uint8_t* in, size_t len, vec8* out, uint32_t member,
                                 uint64_t file_off, size_t* consumed, orc_error* err) {
    size_t hl;
    int r = orc_parse_header(in, len, &hl);
    if (r) return header_error(err, r, in, len);
    size_t start = out->len;
    bitrd b;
    br_init(&b, in + hl, len - hl);
    const char* why = NULL;
    for (;;) {
        int bf;
        r = inflate_block_u8(&b, out, start, &bf, &why);
        if (r) return deflate_error(err, r, why);
        if (bf) break;
    }
    br_byte_align(&b);
    size_t trailer = hl + (size_t)(br_tell(&b) / 8);
    if (trailer + 8 > len) {
        set_err(err, ST_TRUNCATED, "truncated gzip stream");
        return ST_TRUNCATED;
    }
    uint32_t crc_exp = le32(in + trailer), isz_exp = le32(in + trailer + 4);
    uint64_t n = out->len - start;
    uint32_t crc = orc_crc32(0, out->p + start, n);
    if (crc != crc_exp) {
        set_err(err, ST_CRC, "CRC32 mismatch");
        err->member = member;
        err->expected = crc_exp;
        err->got_crc = crc;
        err->uncompressed = n;
        err->trailer_byte = file_off + trailer;
        return ST_CRC;
    }
    if ((uint32_t)n != isz_exp) {
        set_err(err, ST_ISIZE, "ISIZE mismatch");
        err->member = member;
        err->expected = isz_exp;
        err->got = n;
        err->uncompressed = n;
        err->trailer_byte = file_off + trailer;
        return ST_ISIZE;
    }
    *consumed = trailer + 8;
    return 0;
}

int orc_decode_all(const uint8_t* in, size_t len, uint8_t** out, size_t* out_len, orc_error* err) {
    vec8 o = {0};
    size_t pos = 0;
    uint32_t member = 0;
    while (pos < len) {
        size_t used;
        int r = decode_member_checked(in + pos, len - pos, &o, member, pos, &used, err);
        if (r) {
            free(o.p);
            return r;
        }
        pos += used;
        member++;
    }
    *out = o.p;
    *out_len = o.len;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Block finder (rrg/src/deflate/block_finder.rs:55-301)                     */
/* ------------------------------------------------------------------------ */
static uint8_t next_lut[1 << 13];
static pthread_once_t finder_once = PTHREAD_ONCE_INIT;

static int is_dynamic_candidate(uint32_t bits) {
    if (bits & 1) return 0;                   /* BFINAL = 0 */
    if (((bits >> 1) & 3) != 2) return 0;     /* BTYPE = 0b10 */
    if (((bits >> 3) & 31) > 29) return 0;    /* HLIT <= 29 */
    if (((bits >> 8) & 31) > 29) return 0;    /* HDIST <= 29 */
    return 1;
}
static void finder_init(void) {
    for (uint32_t i = 0; i < (1u << 13); i++) {
        uint32_t step = 0, v = i;
        while (step < 13 && !is_dynamic_candidate(v)) {
            v >>= 1;
            step++;
        }
        next_lut[i] = (uint8_t)step;
    }
}

int orc_verify_candidate(const uint8_t* data, size_t len, uint64_t pos) {
    bitrd b;
    br_init(&b, data, len);
    uint32_t v, e;
    if (br_seek(&b, pos) || br_read(&b, 3, &v)) return 0;
    /* read_dynamic_header_strict_into (block_finder.rs:196-262) */
    if (br_read(&b, 5, &v)) return 0;
    uint32_t hlit = v + 257;
    if (br_read(&b, 5, &v)) return 0;
    uint32_t hdist = v + 1;
    if (br_read(&b, 4, &v)) return 0;
    uint32_t hclen = v + 4;
    if (hlit > 286 || hdist > 30) return 0;
    uint8_t cl[19] = {0};
    for (uint32_t i = 0; i < hclen; i++) {
        if (br_read(&b, 3, &v)) return 0;
        cl[CL_ORDER[i]] = (uint8_t)v;
    }
    huff clh, lit, dist;
    const char* why;
    if (huff_build(&clh, cl, 19, 1, ENC_SIMPLE, &why)) return 0;
    uint8_t lengths[320];
    memset(lengths, 0, sizeof(lengths));
    uint32_t total = hlit + hdist, i = 0;
    while (i < total) {
        if (huff_decode_ref(&b, &clh, &e)) return 0;
        uint32_t sym = e >> 16;
        if (sym <= 15) {
            lengths[i++] = (uint8_t)sym;
        } else if (sym == 16) {
            if (i == 0 || br_read(&b, 2, &v)) return 0;
            uint32_t n = v + 3;
            if (i + n > total) return 0;
            for (uint32_t j = 0; j < n; j++) lengths[i + j] = lengths[i - 1];
            i += n;
        } else if (sym == 17) {
            if (br_read(&b, 3, &v)) return 0;
            if (i + v + 3 > total) return 0;
            i += v + 3;
        } else if (sym == 18) {
            if (br_read(&b, 7, &v)) return 0;
            if (i + v + 11 > total) return 0;
            i += v + 11;
        } else {
            return 0;
        }
    }
    if (lengths[256] == 0) return 0;
    if (huff_build(&lit, lengths, (int)hlit, 1, ENC_SIMPLE, &why)) return 0;
    if (huff_build(&dist, lengths + hlit, (int)hdist, 1, ENC_SIMPLE, &why)) return 0;
    /* trial_decode (block_finder.rs:268-301), 64 symbols */
    for (int s = 0; s < 64; s++) {
        if (huff_decode_ref(&b, &lit, &e)) return 0;
        uint32_t sym = e >> 16;
        if (sym < 256) continue;
        if (sym == 256) return 1;
        if (sym > 285) return 0;
        if (LEN_EXTRA[sym - 257] && br_read(&b, LEN_EXTRA[sym - 257], &v)) return 0;
        if (huff_decode_ref(&b, &dist, &e)) return 0;
        uint32_t ds = e >> 16;
        if (ds >= 30) return 0;
        if (DIST_EXTRA[ds] && br_read(&b, DIST_EXTRA[ds], &v)) return 0;
    }
    return 1;
}

int orc_find_next_dynamic_block(const uint8_t* data, size_t len, uint64_t from_bit, uint64_t until_bit,
                                uint64_t* found) {
    pthread_once(&finder_once, finder_init);
    uint64_t total = (uint64_t)len * 8;
    uint64_t limit = until_bit < total ? until_bit : total;
    if (from_bit >= limit) return 0;
    uint64_t pos = from_bit;
    while (pos + 13 <= limit) {
        /* 13-bit window at pos (pos + 13 <= total) */
        uint64_t byte = pos >> 3;
        uint32_t sh = (uint32_t)(pos & 7);
        uint32_t w = 0;
        for (int k = 0; k < 3 && byte + k < len; k++) w |= (uint32_t)data[byte + k] << (8 * k);
        w = (w >> sh) & 0x1fff;
        uint32_t step = next_lut[w];
        if (step == 0) {
            if (orc_verify_candidate(data, len, pos)) {
                *found = pos;
                return 1;
            }
            pos += 1;
        } else {
            pos += step;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* One speculative chunk (pipeline.rs:1080-1185 decode_one_chunk)            */
/* ------------------------------------------------------------------------ */
void orc_chunk_free(orc_chunk* c) {
    if (!c) return;
    free(c->bytes);
    free(c->marker_pos);
    free(c->marker_off);
    free(c->mbs);
    c->bytes = NULL;
    c->marker_pos = NULL;
    c->marker_off = NULL;
    c->mbs = NULL;
    c->n_bytes = c->n_markers = c->n_mbs = 0;
}

int orc_decode_chunk(const uint8_t* body, size_t body_len, uint64_t start_bit, uint64_t end_bit_hint,
                     orc_chunk* out, orc_error* err) {
    memset(out, 0, sizeof(*out));
    out->start_bit = start_bit;
    out->end_bit_hint = end_bit_hint;
    bitrd b;
    br_init(&b, body, body_len);
    vec8 bytes = {0};
    vecm markers = {0};
    vecb mbs = {0};
    const char* why = NULL;
    int r = br_seek(&b, start_bit);
    if (r) {
        deflate_error(err, r, why);
        goto fail;
    }
    int first = 1;
    for (;;) {
        if (br_tell(&b) >= end_bit_hint) break;
        int hit;
        if (first) r = decode_until_u16(&b, end_bit_hint, &bytes, &markers, &hit, &why);
        else r = decode_member_u8(&b, end_bit_hint, &bytes, &hit, &why);
        if (r) {
            deflate_error(err, r, why);
            goto fail;
        }
        first = 0;
        if (!hit) break;
        br_byte_align(&b);
        uint64_t trailer = br_tell(&b) / 8;
        if (trailer + 8 > body_len) {
            r = ST_TRUNCATED;
            set_err(err, r, "truncated gzip stream");
            goto fail;
        }
        orc_member_boundary mb = {bytes.len, le32(body + trailer), le32(body + trailer + 4), trailer};
        if (vecb_push(&mbs, mb)) {
            r = ST_OOM;
            set_err(err, r, "out of memory");
            goto fail;
        }
        uint64_t after = trailer + 8;
        if (after >= body_len) {
            out->final_block = 1;
            br_seek(&b, after * 8);
            break;
        }
        size_t hl;
        r = orc_parse_header(body + after, body_len - after, &hl);
        if (r) {
            header_error(err, r, body + after, body_len - after);
            goto fail;
        }
        if ((r = br_seek(&b, (after + hl) * 8))) {
            deflate_error(err, r, why);
            goto fail;
        }
    }
    out->actual_end_bit = br_tell(&b);
    out->bytes = bytes.p;
    out->n_bytes = bytes.len;
    out->marker_pos = markers.pos;
    out->marker_off = markers.off;
    out->n_markers = markers.len;
    out->mbs = mbs.p;
    out->n_mbs = mbs.len;
    out->status = 0;
    return 0;
fail:
    free(bytes.p);
    free(markers.pos);
    free(markers.off);
    free(mbs.p);
    out->status = r;
    return r;
}

int orc_resolve_markers(orc_chunk* c, const uint8_t* tail, size_t tail_len, orc_error* err) {
    for (uint64_t i = 0; i < c->n_markers; i++) {
        size_t off = c->marker_off[i];
        if (off >= tail_len) {
            set_err(err, ST_INVALID, "marker references bytes outside the available prefix window");
            return ST_INVALID;
        }
        c->bytes[c->marker_pos[i]] = tail[tail_len - 1 - off];
    }
    c->n_markers = 0;
    return 0;
}

size_t orc_build_prev_tail(const orc_chunk* c, const uint8_t* prev, size_t prev_len, uint8_t* out) {
    size_t len = (size_t)c->n_bytes;
    size_t ts = len > WINDOW ? len - WINDOW : 0;
    size_t n = len - ts;
    size_t carry = 0;
    if (len < WINDOW && prev_len) {
        size_t need = WINDOW - len;
        carry = prev_len < need ? prev_len : need;
        memcpy(out, prev + prev_len - carry, carry);
    }
    memcpy(out + carry, c->bytes + ts, n);
    /* markers landing in the tail, patched from the previous window */
    size_t lo = 0, hi = (size_t)c->n_markers;
    while (lo < hi) {
        size_t mid = (lo + hi) / 2;
        if (c->marker_pos[mid] < ts) lo = mid + 1;
        else hi = mid;
    }
    for (size_t i = lo; i < c->n_markers; i++) {
        size_t off = c->marker_off[i];
        if (off < prev_len) out[carry + (c->marker_pos[i] - ts)] = prev[prev_len - 1 - off];
    }
    return carry + n;
}

/* ------------------------------------------------------------------------ */
/* Threaded member pipeline (pipeline.rs:468-1041)                           */
/* Decode pool -> serial anchored chain + tail chain (stage A) -> resolve    */
/* pool (markers + per-member CRC pieces) -> ordered output with CRC combine.*/
/* ------------------------------------------------------------------------ */
enum { CS_PENDING = 0, CS_DECODED, CS_READY, CS_RESOLVED };

typedef struct {
    uint32_t crc;
    uint64_t len;
} crcpiece;

typedef struct {
    orc_chunk c;
    uint8_t* prev_tail;
    size_t prev_len;
    crcpiece* pieces; /* one per member boundary, then the trailing piece */
    int state;
    int rstatus;
} slot;

typedef struct {
    const uint8_t* body;
    size_t body_len;
    uint64_t body_off;
    size_t n;
    uint64_t* starts;
    uint64_t* hints;
    slot* s;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    size_t next_decode;
    size_t next_resolve;
    size_t out_done;
    size_t cap;
    size_t final_id; /* n if not yet known */
    int abort;
    int err_code;
    orc_error err;
    uint64_t spec_failures;
} mpipe;

static void mp_fail(mpipe* m, int code, const orc_error* e) {
    pthread_mutex_lock(&m->mu);
    if (!m->err_code) {
        m->err_code = code;
        if (e) m->err = *e;
    }
    m->abort = 1;
    pthread_cond_broadcast(&m->cv);
    pthread_mutex_unlock(&m->mu);
}

static void* mp_decode_worker(void* arg) {
    mpipe* m = (mpipe*)arg;
    for (;;) {
        pthread_mutex_lock(&m->mu);
        while (!m->abort && m->next_decode < m->n && m->next_decode < m->final_id &&
               m->next_decode - m->out_done >= m->cap)
            pthread_cond_wait(&m->cv, &m->mu);
        if (m->abort || m->next_decode >= m->n || m->next_decode >= m->final_id) {
            pthread_mutex_unlock(&m->mu);
            return NULL;
        }
        size_t i = m->next_decode++;
        pthread_mutex_unlock(&m->mu);
        orc_error e;
        orc_decode_chunk(m->body, m->body_len, m->starts[i], m->hints[i], &m->s[i].c, &e);
        pthread_mutex_lock(&m->mu);
        m->s[i].state = CS_DECODED;
        pthread_cond_broadcast(&m->cv);
        pthread_mutex_unlock(&m->mu);
    }
}

static void* mp_stage_a(void* arg) {
    mpipe* m = (mpipe*)arg;
    uint64_t expected = 0;
    uint8_t* prev = NULL;
    size_t prev_len = 0;
    for (size_t i = 0; i < m->n; i++) {
        pthread_mutex_lock(&m->mu);
        while (!m->abort && m->s[i].state < CS_DECODED) pthread_cond_wait(&m->cv, &m->mu);
        int ab = m->abort;
        pthread_mutex_unlock(&m->mu);
        if (ab) break;
        slot* s = &m->s[i];
        if (s->c.status != 0 || s->c.start_bit != expected) {
            /* false boundary or failed speculative decode: re-decode from the
             * anchored offset (pipeline.rs:788-809) */
            orc_chunk_free(&s->c);
            m->spec_failures++;
            orc_error e;
            int r = orc_decode_chunk(m->body, m->body_len, expected, m->hints[i], &s->c, &e);
            if (r) {
                mp_fail(m, r, &e);
                break;
            }
        }
        expected = s->c.actual_end_bit;
        uint8_t* nt = (uint8_t*)malloc(WINDOW);
        if (!nt) {
            orc_error e;
            set_err(&e, ST_OOM, "out of memory");
            mp_fail(m, ST_OOM, &e);
            break;
        }
        size_t nl = orc_build_prev_tail(&s->c, prev, prev_len, nt);
        s->prev_tail = prev;
        s->prev_len = prev_len;
        prev = nt;
        prev_len = nl;
        pthread_mutex_lock(&m->mu);
        s->state = CS_READY;
        if (s->c.final_block) m->final_id = i + 1;
        pthread_cond_broadcast(&m->cv);
        pthread_mutex_unlock(&m->mu);
        if (s->c.final_block) break;
    }
    free(prev);
    return NULL;
}

static void* mp_resolve_worker(void* arg) {
    mpipe* m = (mpipe*)arg;
    for (;;) {
        pthread_mutex_lock(&m->mu);
        while (!m->abort && m->next_resolve < m->final_id && m->next_resolve < m->n &&
               m->s[m->next_resolve].state < CS_READY)
            pthread_cond_wait(&m->cv, &m->mu);
        if (m->abort || m->next_resolve >= m->final_id || m->next_resolve >= m->n) {
            pthread_mutex_unlock(&m->mu);
            return NULL;
        }
        size_t i = m->next_resolve++;
        pthread_mutex_unlock(&m->mu);
        slot* s = &m->s[i];
        orc_error e;
        int r = orc_resolve_markers(&s->c, s->prev_tail, s->prev_len, &e);
        if (!r) {
            s->pieces = (crcpiece*)malloc((s->c.n_mbs + 1) * sizeof(crcpiece));
            if (!s->pieces) {
                r = ST_OOM;
                set_err(&e, r, "out of memory");
            } else {
                uint64_t cursor = 0;
                for (uint64_t k = 0; k < s->c.n_mbs; k++) {
                    uint64_t end = s->c.mbs[k].byte_offset_in_chunk;
                    s->pieces[k].crc = orc_crc32(0, s->c.bytes + cursor, end - cursor);
                    s->pieces[k].len = end - cursor;
                    cursor = end;
                }
                s->pieces[s->c.n_mbs].crc = orc_crc32(0, s->c.bytes + cursor, s->c.n_bytes - cursor);
                s->pieces[s->c.n_mbs].len = s->c.n_bytes - cursor;
            }
        }
        if (r) {
            mp_fail(m, r, &e);
            return NULL;
        }
        pthread_mutex_lock(&m->mu);
        s->state = CS_RESOLVED;
        pthread_cond_broadcast(&m->cv);
        pthread_mutex_unlock(&m->mu);
    }
}

static size_t effective_threads(uint32_t n) {
    if (n) return n;
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (size_t)c : 1;
}

/* serial_decode_member (pipeline.rs:1211-1345): one thread, real window, no
 * markers; emits ~chunk_target pieces, CRC/ISIZE checked inline. */
static int serial_member(const uint8_t* file, size_t flen, size_t body_off, uint64_t chunk_target,
                         orc_sink_fn sink, void* user, orc_stats* st, orc_error* err) {
    const uint8_t* body = file + body_off;
    size_t blen = flen - body_off;
    bitrd b;
    br_init(&b, body, blen);
    vec8 out = {0};
    uint32_t member = 0;
    uint32_t mcrc = 0;
    uint64_t mlen = 0;
    size_t floor = 0;
    const char* why = NULL;
    int r = 0;
    for (;;) {
        int bf;
        r = inflate_block_u8(&b, &out, floor, &bf, &why);
        if (r) {
            deflate_error(err, r, why);
            goto done;
        }
        if (!bf) {
            while (out.len >= chunk_target + WINDOW) {
                size_t emit = out.len - WINDOW;
                mcrc = orc_crc32(mcrc, out.p, emit);
                mlen += emit;
                st->uncompressed_bytes += emit;
                if (sink && sink(user, out.p, emit)) goto done;
                st->chunks_decoded++;
                memmove(out.p, out.p + emit, WINDOW);
                out.len = WINDOW;
                floor = 0;
            }
            continue;
        }
        mcrc = orc_crc32(mcrc, out.p + floor, out.len - floor);
        mlen += out.len - floor;
        if (out.len > floor) {
            st->uncompressed_bytes += out.len - floor;
            if (sink && sink(user, out.p + floor, out.len - floor)) goto done;
            st->chunks_decoded++;
        }
        br_byte_align(&b);
        uint64_t trailer = br_tell(&b) / 8;
        if (trailer + 8 > blen) {
            r = ST_TRUNCATED;
            set_err(err, r, "truncated gzip stream");
            goto done;
        }
        uint32_t ce = le32(body + trailer), ie = le32(body + trailer + 4);
        if (mcrc != ce) {
            r = ST_CRC;
            set_err(err, r, "CRC32 mismatch");
            err->member = member;
            err->expected = ce;
            err->got_crc = mcrc;
            err->uncompressed = mlen;
            err->trailer_byte = body_off + trailer;
            goto done;
        }
        if ((uint32_t)mlen != ie) {
            r = ST_ISIZE;
            set_err(err, r, "ISIZE mismatch");
            err->member = member;
            err->expected = ie;
            err->got = mlen;
            err->uncompressed = mlen;
            err->trailer_byte = body_off + trailer;
            goto done;
        }
        member++;
        uint64_t after = trailer + 8;
        if (after >= blen) goto done;
        size_t hl;
        r = orc_parse_header(body + after, blen - after, &hl);
        if (r) {
            header_error(err, r, body + after, blen - after);
            goto done;
        }
        if ((r = br_seek(&b, (after + hl) * 8))) {
            deflate_error(err, r, why);
            goto done;
        }
        out.len = 0;
        floor = 0;
        mcrc = 0;
        mlen = 0;
    }
done:
    free(out.p);
    return r;
}

typedef struct {
    const uint8_t* body;
    size_t blen;
    uint64_t chunk_bits, total_bits;
    uint64_t* found;
    size_t n;
    atomic_size_t next;
} scan_job;

static void* scan_worker(void* arg) {
    scan_job* j = (scan_job*)arg;
    for (;;) {
        size_t i = atomic_fetch_add(&j->next, 1);
        if (i >= j->n) return NULL;
        uint64_t f;
        j->found[i] = orc_find_next_dynamic_block(j->body, j->blen, (i + 1) * j->chunk_bits, j->total_bits, &f)
                          ? f
                          : UINT64_MAX;
    }
}

static int member_pipeline(const uint8_t* file, size_t flen, size_t body_off, uint32_t num_threads,
                           uint64_t chunk_size, orc_sink_fn sink, void* user, orc_stats* st,
                           orc_error* err) {
    size_t nt = effective_threads(num_threads);
    if (nt == 1) return serial_member(file, flen, body_off, chunk_size < 65536 ? 65536 : chunk_size, sink, user, st, err);
    const uint8_t* body = file + body_off;
    size_t blen = flen - body_off;
    uint64_t total_bits = (uint64_t)blen * 8;
    uint64_t chunk_bits = (chunk_size < 65536 ? 65536 : chunk_size) * 8;
    size_t ntargets = 0;
    for (uint64_t c = chunk_bits; c < total_bits; c += chunk_bits) ntargets++;
    uint64_t* found = (uint64_t*)malloc((ntargets + 1) * sizeof(uint64_t));
    uint64_t* starts = (uint64_t*)malloc((ntargets + 2) * sizeof(uint64_t));
    uint64_t* hints = (uint64_t*)malloc((ntargets + 2) * sizeof(uint64_t));
    if (!found || !starts || !hints) {
        free(found);
        free(starts);
        free(hints);
        set_err(err, ST_OOM, "out of memory");
        return ST_OOM;
    }
    /* boundary scan, parallel over targets (pipeline.rs:492-543) */
    scan_job sj = {body, blen, chunk_bits, total_bits, found, ntargets, 0};
    size_t nscan = nt < ntargets ? nt : ntargets;
    pthread_t* sth = (pthread_t*)malloc((nscan ? nscan : 1) * sizeof(pthread_t));
    for (size_t i = 0; i < nscan; i++) pthread_create(&sth[i], NULL, scan_worker, &sj);
    for (size_t i = 0; i < nscan; i++) pthread_join(sth[i], NULL);
    free(sth);
    size_t n = 0;
    starts[n++] = 0;
    for (size_t i = 0; i < ntargets; i++)
        if (found[i] != UINT64_MAX && found[i] > starts[n - 1]) starts[n++] = found[i];
    for (size_t i = 0; i < n; i++) hints[i] = i + 1 < n ? starts[i + 1] : UINT64_MAX;
    free(found);

    mpipe m;
    memset(&m, 0, sizeof(m));
    m.body = body;
    m.body_len = blen;
    m.body_off = body_off;
    m.n = n;
    m.starts = starts;
    m.hints = hints;
    m.s = (slot*)calloc(n, sizeof(slot));
    m.cap = 2 * nt > 16 ? 2 * nt : 16; /* InflightCap: max(2N, 16) (pipeline.rs:348-373) */
    m.final_id = n;
    pthread_mutex_init(&m.mu, NULL);
    pthread_cond_init(&m.cv, NULL);
    size_t nres = nt < 4 ? nt : 4;
    pthread_t* dec = (pthread_t*)malloc(nt * sizeof(pthread_t));
    pthread_t* res = (pthread_t*)malloc(nres * sizeof(pthread_t));
    pthread_t sa;
    for (size_t i = 0; i < nt; i++) pthread_create(&dec[i], NULL, mp_decode_worker, &m);
    pthread_create(&sa, NULL, mp_stage_a, &m);
    for (size_t i = 0; i < nres; i++) pthread_create(&res[i], NULL, mp_resolve_worker, &m);

    /* ordered output + CRC combine (pipeline.rs:873-935) */
    uint32_t cur_crc = 0;
    uint64_t cur_len = 0;
    uint32_t member = 0;
    int sink_closed = 0, saw_final = 0;
    for (size_t i = 0; i < n; i++) {
        pthread_mutex_lock(&m.mu);
        while (!m.abort && m.s[i].state < CS_RESOLVED) pthread_cond_wait(&m.cv, &m.mu);
        int ab = m.abort;
        pthread_mutex_unlock(&m.mu);
        if (ab) break;
        slot* s = &m.s[i];
        int bad = 0;
        for (uint64_t k = 0; k < s->c.n_mbs && !bad; k++) {
            cur_crc = orc_crc32_combine(cur_crc, s->pieces[k].crc, s->pieces[k].len);
            cur_len += s->pieces[k].len;
            const orc_member_boundary* mb = &s->c.mbs[k];
            orc_error e;
            memset(&e, 0, sizeof(e));
            if (cur_crc != mb->crc_expected) {
                set_err(&e, ST_CRC, "CRC32 mismatch");
                e.member = member;
                e.expected = mb->crc_expected;
                e.got_crc = cur_crc;
                e.uncompressed = cur_len;
                e.trailer_byte = body_off + mb->trailer_input_byte;
                mp_fail(&m, ST_CRC, &e);
                bad = 1;
            } else if ((uint32_t)cur_len != mb->isize_expected) {
                set_err(&e, ST_ISIZE, "ISIZE mismatch");
                e.member = member;
                e.expected = mb->isize_expected;
                e.got = cur_len;
                e.uncompressed = cur_len;
                e.trailer_byte = body_off + mb->trailer_input_byte;
                mp_fail(&m, ST_ISIZE, &e);
                bad = 1;
            }
            member++;
            cur_crc = 0;
            cur_len = 0;
        }
        if (bad) break;
        cur_crc = orc_crc32_combine(cur_crc, s->pieces[s->c.n_mbs].crc, s->pieces[s->c.n_mbs].len);
        cur_len += s->pieces[s->c.n_mbs].len;
        st->uncompressed_bytes += s->c.n_bytes;
        int closed = sink ? sink(user, s->c.bytes, (size_t)s->c.n_bytes) : 0;
        int fin = s->c.final_block;
        orc_chunk_free(&s->c);
        free(s->prev_tail);
        s->prev_tail = NULL;
        free(s->pieces);
        s->pieces = NULL;
        pthread_mutex_lock(&m.mu);
        m.out_done = i + 1;
        if (closed || fin) m.abort = m.abort || closed;
        pthread_cond_broadcast(&m.cv);
        pthread_mutex_unlock(&m.mu);
        if (closed) {
            sink_closed = 1;
            break;
        }
        st->chunks_decoded++;
        if (fin) {
            saw_final = 1;
            break;
        }
    }
    pthread_mutex_lock(&m.mu);
    m.abort = 1;
    pthread_cond_broadcast(&m.cv);
    pthread_mutex_unlock(&m.mu);
    for (size_t i = 0; i < nt; i++) pthread_join(dec[i], NULL);
    pthread_join(sa, NULL);
    for (size_t i = 0; i < nres; i++) pthread_join(res[i], NULL);
    int rc = 0;
    if (!sink_closed && m.err_code) {
        rc = m.err_code;
        if (err) *err = m.err;
    } else if (!sink_closed && !saw_final) {
        rc = ST_IO;
        set_err(err, rc, "parallel decode produced no final block");
    }
    st->speculation_failures += m.spec_failures;
    st->n_chunks += n;
    for (size_t i = 0; i < n; i++) {
        orc_chunk_free(&m.s[i].c);
        free(m.s[i].prev_tail);
        free(m.s[i].pieces);
    }
    free(m.s);
    free(dec);
    free(res);
    free(starts);
    free(hints);
    pthread_mutex_destroy(&m.mu);
    pthread_cond_destroy(&m.cv);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* BGZF route (pipeline.rs:1357-1636)                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
    size_t first, count; /* member index range */
    vec8 out;
    int status;
    orc_error err;
    int done;
} bgzf_batch;

typedef struct {
    const uint8_t* file;
    uint64_t* mstart;
    uint64_t* mend;
    bgzf_batch* batches;
    size_t nb;
    atomic_size_t next;
    pthread_mutex_t mu;
    pthread_cond_t cv;
} bgzf_pool;

static void* bgzf_worker(void* arg) {
    bgzf_pool* p = (bgzf_pool*)arg;
    for (;;) {
        size_t i = atomic_fetch_add(&p->next, 1);
        if (i >= p->nb) return NULL;
        bgzf_batch* bt = &p->batches[i];
        for (size_t k = 0; k < bt->count; k++) {
            size_t mi = bt->first + k, used;
            int r = decode_member_checked(p->file + p->mstart[mi], p->mend[mi] - p->mstart[mi], &bt->out,
                                          (uint32_t)mi, p->mstart[mi], &used, &bt->err);
            if (r) {
                bt->status = r;
                break;
            }
        }
        pthread_mutex_lock(&p->mu);
        bt->done = 1;
        pthread_cond_broadcast(&p->cv);
        pthread_mutex_unlock(&p->mu);
    }
}

static int bgzf_route(const uint8_t* file, size_t len, uint32_t num_threads, uint64_t chunk_size,
                      orc_sink_fn sink, void* user, orc_stats* st, orc_error* err) {
    size_t nt = effective_threads(num_threads);
    size_t cap = 1024, nm = 0;
    uint64_t* ms = (uint64_t*)malloc(cap * 8);
    uint64_t* me = (uint64_t*)malloc(cap * 8);
    size_t pos = 0;
    int walk_err = 0;
    while (pos < len) {
        int64_t sz = orc_bgzf_block_size(file + pos, len - pos);
        if (sz < 0) break;
        if (pos + (size_t)sz > len) {
            walk_err = ST_TRUNCATED;
            break;
        }
        if (nm == cap) {
            cap *= 2;
            ms = (uint64_t*)realloc(ms, cap * 8);
            me = (uint64_t*)realloc(me, cap * 8);
        }
        ms[nm] = pos;
        me[nm] = pos + (size_t)sz;
        nm++;
        pos += (size_t)sz;
    }
    /* batches ramp from 64 KiB to chunk_size (pipeline.rs:1501-1541) */
    uint64_t target = 65536, chunk_target = chunk_size < 65536 ? 65536 : chunk_size;
    size_t nbcap = 64, nb = 0;
    bgzf_batch* bs = (bgzf_batch*)calloc(nbcap, sizeof(bgzf_batch));
    size_t first = 0;
    uint64_t bytes = 0;
    for (size_t i = 0; i < nm; i++) {
        bytes += me[i] - ms[i];
        if (bytes >= target || i + 1 == nm) {
            if (nb == nbcap) {
                nbcap *= 2;
                bs = (bgzf_batch*)realloc(bs, nbcap * sizeof(bgzf_batch));
                memset(bs + nb, 0, (nbcap - nb) * sizeof(bgzf_batch));
            }
            bs[nb].first = first;
            bs[nb].count = i + 1 - first;
            nb++;
            first = i + 1;
            if (bytes >= target) target = target * 2 < chunk_target ? target * 2 : chunk_target;
            bytes = 0;
        }
    }
    bgzf_pool p;
    memset(&p, 0, sizeof(p));
    p.file = file;
    p.mstart = ms;
    p.mend = me;
    p.batches = bs;
    p.nb = nb;
    atomic_init(&p.next, 0);
    pthread_mutex_init(&p.mu, NULL);
    pthread_cond_init(&p.cv, NULL);
    pthread_t* th = (pthread_t*)malloc(nt * sizeof(pthread_t));
    for (size_t i = 0; i < nt; i++) pthread_create(&th[i], NULL, bgzf_worker, &p);
    int rc = 0, closed = 0;
    for (size_t i = 0; i < nb; i++) {
        pthread_mutex_lock(&p.mu);
        while (!bs[i].done) pthread_cond_wait(&p.cv, &p.mu);
        pthread_mutex_unlock(&p.mu);
        if (bs[i].status) {
            rc = bs[i].status;
            if (err) *err = bs[i].err;
            atomic_store(&p.next, nb);
            break;
        }
        st->uncompressed_bytes += bs[i].out.len;
        if (sink && sink(user, bs[i].out.p, bs[i].out.len)) {
            closed = 1;
            rc = ST_IO;
            set_err(err, rc, "sink closed");
            atomic_store(&p.next, nb);
            break;
        }
        st->chunks_decoded++;
        free(bs[i].out.p);
        bs[i].out.p = NULL;
    }
    for (size_t i = 0; i < nt; i++) pthread_join(th[i], NULL);
    for (size_t i = 0; i < nb; i++) free(bs[i].out.p);
    free(bs);
    free(th);
    free(ms);
    free(me);
    pthread_mutex_destroy(&p.mu);
    pthread_cond_destroy(&p.cv);
    (void)closed;
    if (rc) return rc;
    if (walk_err) {
        set_err(err, walk_err, "truncated gzip stream");
        return walk_err;
    }
    if (pos < len) {
        /* non-BGZF remainder goes through the member route (pipeline.rs:1622-1633) */
        size_t hl;
        int r = orc_parse_header(file + pos, len - pos, &hl);
        if (r) return header_error(err, r, file + pos, len - pos);
        return member_pipeline(file, len, pos + hl, num_threads, chunk_size, sink, user, st, err);
    }
    return 0;
}

int orc_read_gz_buffer(const uint8_t* file, size_t len, uint32_t num_threads, uint64_t chunk_size,
                       orc_sink_fn sink, void* user, orc_stats* stats, orc_error* err) {
    orc_stats st;
    memset(&st, 0, sizeof(st));
    orc_error e;
    memset(&e, 0, sizeof(e));
    if (!chunk_size) chunk_size = 4u << 20;
    st.compressed_bytes = len;
    int r;
    if (len == 0) {
        r = ST_TRUNCATED; /* zero-byte file (pipeline.rs:2066-2077) */
        set_err(&e, r, "truncated gzip stream");
    } else if (orc_bgzf_block_size(file, len) >= 0) {
        r = bgzf_route(file, len, num_threads, chunk_size, sink, user, &st, &e);
    } else {
        size_t hl;
        r = orc_parse_header(file, len, &hl);
        if (r) header_error(&e, r, file, len);
        else r = member_pipeline(file, len, hl, num_threads, chunk_size, sink, user, &st, &e);
    }
    if (stats) *stats = st;
    if (err) *err = e;
    return r;
}

typedef struct {
    vec8 v;
    int oom;
} collect_ctx;
static int collect_sink(void* user, const uint8_t* p, size_t n) {
    collect_ctx* c = (collect_ctx*)user;
    if (vec8_reserve(&c->v, n + 1)) {
        c->oom = 1;
        return 1;
    }
    memcpy(c->v.p + c->v.len, p, n);
    c->v.len += n;
    return 0;
}

int orc_read_gz_to_buffer(const uint8_t* file, size_t len, uint32_t num_threads, uint64_t chunk_size,
                          uint8_t** out, size_t* out_len, orc_stats* stats, orc_error* err) {
    collect_ctx c;
    memset(&c, 0, sizeof(c));
    int r = orc_read_gz_buffer(file, len, num_threads, chunk_size, collect_sink, &c, stats, err);
    if (!r && c.oom) {
        r = ST_OOM;
        set_err(err, r, "out of memory");
    }
    if (r) {
        free(c.v.p);
        return r;
    }
    *out = c.v.p ? c.v.p : (uint8_t*)malloc(1);
    *out_len = c.v.len;
    return 0;
}

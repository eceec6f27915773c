// rrg_gpu.cu — host orchestration and C ABI (include/rrg_gpu.h) of the B200
// gzip/DEFLATE decoder.
//
// Member route (rrg/src/pipeline.rs:468-1041, parallel_decode_member):
//   k_find_blocks  -> sub-chunk boundaries every `gpu_chunk_bytes` of compressed input
//   k_inflate<u16> -> every sub-chunk decoded at once, one warp each, unknown-window
//                     back-references emitted as 16-bit marker cells
//   host chain     -> anchored verification (pipeline.rs:758-809): chunk k is kept iff
//                     it starts where chunk k-1 stopped; otherwise it is re-decoded
//   k_win_maps, k_win_bases -> the tail chain as composed window maps: every chunk's
//                     window relative to its group's first window, then those windows
//   k_res_tails    -> every chunk's last 32 KiB of cells to bytes through its map
//   k_res_heads    -> the other cells to bytes, markers gathered from the 32 KiB of
//                     output before the chunk
//   k_crc_*        -> CRC32/ISIZE of every member from per-piece CRCs + GF(2) combine
// BGZF route (pipeline.rs:1357-1636): members found by a header walk, one warp
// per member through the persistent k_inflate<u8> work queue, CRC as above.
#ifndef RRG_EMU
#include <cuda_runtime.h>
#endif

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <unordered_map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rrg_gpu.h"
#include "rrg_common.h"
#include "rrg_kernels.cuh"

#ifdef RRG_EMU
#define RRG_LAUNCH(kern, grid, block, smem, strm, ...) emu::launch((grid), (block), (smem), [&] { kern(__VA_ARGS__); })
#else
#define RRG_LAUNCH(kern, grid, block, smem, strm, ...) kern<<<(grid), (block), (smem), (strm)>>>(__VA_ARGS__)
#endif

using namespace rrg;

namespace {

std::atomic<uint64_t> g_launches{0};

const char* msg_text(int m) {
    switch (m) {
    case MSG_RESERVED_BTYPE: return "reserved block type";
    case MSG_STORED_NLEN: return "stored block: LEN/NLEN mismatch";
    case MSG_LITLEN_RANGE: return "literal/length symbol out of range";
    case MSG_DIST_RANGE: return "distance symbol out of range";
    case MSG_NO_CODE: return "no matching huffman code";
    case MSG_OVERSUB: return "oversubscribed huffman tree";
    case MSG_HLIT_HDIST: return "dynamic block: HLIT/HDIST out of range";
    case MSG_CODE16_FIRST: return "code 16 with no previous";
    case MSG_CODE16_OVER: return "code 16 overruns lengths";
    case MSG_CODE17_OVER: return "code 17 overruns lengths";
    case MSG_CODE18_OVER: return "code 18 overruns lengths";
    case MSG_BAD_CL_SYM: return "bad code-length symbol";
    case MSG_EOB_ZERO: return "EOB symbol has zero length";
    case MSG_DIST_FAR: return "back-reference distance out of bounds";
    case MSG_MARKER_WINDOW: return "marker references bytes outside the available prefix window";
    default: return "invalid deflate stream";
    }
}

void set_err(rrg_error* e, int code, const char* fmt, ...) {
    if (!e) return;
    std::memset(e, 0, sizeof(*e));
    e->code = code;
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(e->message, sizeof(e->message), fmt, ap);
    va_end(ap);
}

int status_err(rrg_error* e, int st, int msg, uint64_t where) {
    switch (st) {
    case DS_EOF: set_err(e, RRG_ERR_DEFLATE_EOF, "unexpected end of input"); break;
    case DS_INVALID: set_err(e, RRG_ERR_DEFLATE_INVALID, "%s", msg_text(msg)); break;
    case DS_TRUNCATED: set_err(e, RRG_ERR_TRUNCATED, "truncated gzip stream"); break;
    case DS_BAD_MAGIC: set_err(e, RRG_ERR_BAD_MAGIC, "not a gzip file (bad magic)"); break;
    case DS_METHOD:
        set_err(e, RRG_ERR_UNSUPPORTED_METHOD, "unsupported compression method: %d", msg);
        if (e) e->expected = (uint32_t)msg;
        break;
    case DS_FLAGS:
        set_err(e, RRG_ERR_RESERVED_FLAGS, "reserved gzip flag bits set: %#x", msg);
        if (e) e->expected = (uint32_t)msg;
        break;
    default: set_err(e, RRG_ERR_DEFLATE_INVALID, "decode status %d", st); break;
    }
    if (e) e->trailer_byte = where;
    return e ? e->code : RRG_ERR_DEFLATE_INVALID;
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------- host CRC
uint32_t g_crc_tab[8][256];
uint32_t g_crc_z496[4][256];  // register advanced over 496 zero bytes, per byte position
uint32_t g_x2k[67];
std::once_flag g_tab_once;

uint32_t host_mulmod(uint32_t a, uint32_t b) {
    uint32_t p = 0;
    for (int i = 0; i < 32; i++) {
        if (a & (0x80000000u >> i)) p ^= b;
        b = (b & 1u) ? (b >> 1) ^ 0xEDB88320u : (b >> 1);
    }
    return p;
}

void init_tables() {
    for (uint32_t n = 0; n < 256; n++) {
        uint32_t c = n;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? (c >> 1) ^ 0xEDB88320u : (c >> 1);
        g_crc_tab[0][n] = c;
    }
    for (uint32_t n = 0; n < 256; n++) {
        uint32_t c = g_crc_tab[0][n];
        for (int t = 1; t < 8; t++) {
            c = g_crc_tab[0][c & 0xff] ^ (c >> 8);
            g_crc_tab[t][n] = c;
        }
    }
    for (int j = 0; j < 4; j++)
        for (uint32_t b = 0; b < 256; b++) {
            uint32_t v = b << (8 * j);
            for (int i = 0; i < 496; i++) v = g_crc_tab[0][v & 0xff] ^ (v >> 8);
            g_crc_z496[j][b] = v;
        }
    g_x2k[0] = 0x40000000u;
    for (int k = 1; k < 67; k++) g_x2k[k] = host_mulmod(g_x2k[k - 1], g_x2k[k - 1]);
}

// 13-bit prefilter skip table (block_finder.rs:60-101).
uint8_t g_next_lut[8192];
std::once_flag g_lut_once;
void init_next_lut() {
    auto cand = [](uint32_t b) {
        return !(b & 1) && ((b >> 1) & 3) == 2 && ((b >> 3) & 31) <= 29 && ((b >> 8) & 31) <= 29;
    };
    for (uint32_t i = 0; i < 8192; i++) {
        uint32_t s = 0, v = i;
        while (s < 13 && !cand(v)) {
            v >>= 1;
            s++;
        }
        g_next_lut[i] = (uint8_t)s;
    }
}

// gzip.rs:252-300
int host_parse_header(const uint8_t* in, size_t len, size_t* hl, int* detail) {
    *detail = 0;
    if (len < 10) return DS_TRUNCATED;
    if (in[0] != 0x1f || in[1] != 0x8b) return DS_BAD_MAGIC;
    if (in[2] != 8) {
        *detail = in[2];
        return DS_METHOD;
    }
    uint8_t flg = in[3];
    if (flg & 0xe0) {
        *detail = flg;
        return DS_FLAGS;
    }
    size_t pos = 10;
    if (flg & 4) {
        if (pos + 2 > len) return DS_TRUNCATED;
        pos += 2 + ((size_t)in[pos] | ((size_t)in[pos + 1] << 8));
        if (pos > len) return DS_TRUNCATED;
    }
    for (int f = 8; f <= 16; f <<= 1) {
        if (flg & f) {
            const void* z = pos < len ? std::memchr(in + pos, 0, len - pos) : nullptr;
            if (!z) return DS_TRUNCATED;
            pos = (size_t)((const uint8_t*)z - in) + 1;
        }
    }
    if (flg & 2) {
        if (pos + 2 > len) return DS_TRUNCATED;
        pos += 2;
    }
    *hl = pos;
    return DS_OK;
}

// gzip.rs:311-351 parse_bgzf_block_size; -1 = None.
int64_t host_bgzf_size(const uint8_t* in, size_t len) {
    if (len < 12 || in[0] != 0x1f || in[1] != 0x8b || in[2] != 8 || !(in[3] & 4)) return -1;
    size_t xlen = (size_t)in[10] | ((size_t)in[11] << 8);
    if (12 + xlen > len) return -1;
    size_t p = 12, end = 12 + xlen;
    while (p + 4 <= end) {
        size_t slen = (size_t)in[p + 2] | ((size_t)in[p + 3] << 8);
        if (p + 4 + slen > end) return -1;
        if (in[p] == 'B' && in[p + 1] == 'C' && slen == 2) return (int64_t)(in[p + 4] | (in[p + 5] << 8)) + 1;
        p += 4 + slen;
    }
    return -1;
}

uint64_t le32h(const uint8_t* p) {
    return (uint64_t)p[0] | ((uint64_t)p[1] << 8) | ((uint64_t)p[2] << 16) | ((uint64_t)p[3] << 24);
}

struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
};

}  // namespace

// buffers and shapes a captured BGZF decode graph refers to
struct BgzfKey {
    const void* p[24];
    uint64_t v[6];
};
// ... and a captured device-planned member batch
struct BatchKey {
    const void* p[20];
    uint64_t v[21];
};
constexpr int BATCH_MARKS = 5;  // events between the stages: plan | inflate | chain + resolve | CRC

#ifndef RRG_EMU
// Captured graphs by shape. A shape is captured the second time it runs (a
// one-off shape, such as one small file, runs its launches directly: an
// instantiation costs more than it saves), and the most recent few stay
// instantiated, so the waves of a repeated multi-wave batch all replay.
template <class Key>
struct GraphCache {
    struct Ent {
        Key k;
        cudaGraphExec_t e;
        uint32_t kernels;
    };
    static constexpr size_t CAP = 8, SEEN = 32;
    std::vector<Ent> ents;  // most recent first
    std::vector<Key> seen;  // shapes run once without a graph, most recent first
    static bool same(const Key& a, const Key& b) { return std::memcmp(&a, &b, sizeof(Key)) == 0; }
    Ent* find(const Key& k) {
        for (size_t i = 0; i < ents.size(); i++)
            if (same(ents[i].k, k)) {
                std::rotate(ents.begin(), ents.begin() + i, ents.begin() + i + 1);
                return &ents[0];
            }
        return nullptr;
    }
    // true when the shape ran before (capture it now); else remembers it
    bool repeat(const Key& k) {
        for (size_t i = 0; i < seen.size(); i++)
            if (same(seen[i], k)) {
                seen.erase(seen.begin() + i);
                return true;
            }
        seen.insert(seen.begin(), k);
        if (seen.size() > SEEN) seen.pop_back();
        return false;
    }
    Ent* add(const Key& k, cudaGraphExec_t e, uint32_t kernels) {
        if (ents.size() >= CAP) {
            cudaGraphExecDestroy(ents.back().e);
            ents.pop_back();
        }
        ents.insert(ents.begin(), Ent{k, e, kernels});
        return &ents[0];
    }
    void clear() {
        for (Ent& x : ents) cudaGraphExecDestroy(x.e);
        ents.clear();
        seen.clear();
    }
};
#endif

// One range of a member split across GPUs, between its two phases: the
// decoded cells stay in the context's slot arena, laid out from out + WINDOW.
struct SplitState {
    bool ready = false;
    std::vector<ResolveChunk> rchunks;
    uint64_t dst_off = 0, total = 0, end_bit = 0;
    bool has_trailer = false;          // the member's trailer lies in this range
    uint32_t crc = 0, isize = 0;       // that trailer
    uint64_t trailer_byte = 0;
    std::vector<uint16_t> end_map;     // WINDOW entries
};

// ====================================================================== ctx
struct rrg_ctx {
    rrg_config cfg{};
    int device = 0;
    int n_sm = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    bool tables_uploaded = false;

    // device buffers (grow-only)
    DBuf items, results, order, queue, mbs, mbcount, cells, out, targets, limits, found, next_lut, chunks,
        tiles, rerr, markers, win, cand, ncand, vflag, lane_scratch, crc_table, pieces, piece_crc, mpiece, exp_crc, exp_isize, got_crc, got_len,
        mstatus, comp, comp2, pfx;
    // pinned host staging
    uint8_t* h_stage[2] = {nullptr, nullptr};
    size_t h_stage_cap = 0;
    uint8_t* h_in = nullptr;
    size_t h_in_cap = 0;
    uint8_t* h_file = nullptr;  // page-locked copy of a file read by rrg_gpu_read_gz
    size_t h_file_cap = 0;

    // tunables
    uint64_t gpu_chunk = 0;
    bool lanes = false;        // lane-per-chunk inflate (default: one chunk per warp)
    bool scan_bounds = true;   // full-stream boundary scan (boundary_mode 1: one finder search per target)
    uint32_t inflate_warps = 4;
    uint32_t finder_tile = 1024;
    uint32_t scan_threads = 256;  // boundary scan tile = scan_threads x 16 bytes
    uint32_t warps_per_member = 1; // BGZF: 1 = a member per warp; 2-4 = sub-chunks per member
    double expand = 6.0;
    uint64_t slots = 0;        // resident decoders of one inflate wave (lazy)
    // host path: the input's H2D copy in pieces (end byte, event), so the
    // boundary scan can start on the pieces that have arrived
    const uint8_t* arr_base = nullptr;
    std::vector<std::pair<uint64_t, cudaEvent_t>> arr_pieces;
    cudaEvent_t arr_events[8] = {};
    cudaStream_t copy_stream = nullptr;
    // pipelined host path: waves decode, resolve and checksum in order on the
    // context stream while earlier waves' output copies run on copy_stream
    DBuf pipe;                       // wave tables, states, CRC pieces
    uint8_t* h_ring = nullptr;       // pinned result pieces
    size_t h_ring_cap = 0;           // bytes per piece buffer
    uint8_t* h_wave = nullptr;       // pinned wave outcomes
    size_t h_wave_cap = 0;
    bool pipeline = true;            // take the pipelined path where it applies
    SplitState* split = nullptr;     // a range of a split member between its phases
    // destination provider of the current *_into call (null: library staging)
    rrg_buffer_fn get_buf = nullptr;
    void* get_user = nullptr;
    DBuf sniff;                // per-file header results of a batch
        // BGZF route: device member table and the captured decode graph
    DBuf bg_bcount, bg_bbase, bg_coff, bg_csize, bg_small;
    uint64_t* h_bg = nullptr;  // pinned: the 64 result bytes of one BGZF decode
    uint32_t bg_cap = 0;
    bool use_graphs = true;
#ifndef RRG_EMU
    GraphCache<BgzfKey> bg_graphs;
#endif
    // device-planned member batch: plan and state, and its captured graph
    DBuf bplan;
    cudaEvent_t bt_marks[BATCH_MARKS] = {};  // stage boundaries, recorded by the graph
#ifndef RRG_EMU
    GraphCache<BatchKey> bt_graphs;
#endif

    rrg_stats st{};
    uint64_t launches = 0;

    // serving loop (created on first use)
    struct Server* srv = nullptr;
    std::mutex srv_create_mu;
};

// Serving loop. Each engine is a sub-context with its own stream and
// device scratch, resident across requests, and its own host thread. An idle
// engine takes the oldest waiting requests that fit the HBM budget together
// (continuous batching: requests that arrive while other batches are on the
// GPU join the next batch an engine takes) and decodes them as one batch;
// engines overlap on the device. Finished requests wait in a bounded
// completion queue: engines stop taking work while it is full.
struct Server {
    struct Req {
        int64_t id;
        std::vector<uint8_t> copy;   // the request's bytes when submit copied them
        const uint8_t* bytes = nullptr;  // the bytes (the copy, or the caller's buffer)
        uint64_t len = 0;
        double t_submit;
        uint64_t out_need = 0;  // exact output size once known (a retry after RRG_ERR_CAPACITY)
    };
    struct Done {
        int64_t id;
        uint8_t* out;
        size_t len;
        int32_t status;
        double t_submit;
        double latency_ms;
        rrg_error err;  // the failure's detail (code 0 when it succeeded)
    };
    std::vector<rrg_ctx*> engines;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req> waiting;
    std::deque<Done> done;
    uint64_t budget = 0, in_use = 0;
    uint32_t max_ready = 64, max_batch = 64;
    bool stop = false;
    int64_t next_id = 0;
    int64_t outstanding = 0;  // submitted and not yet polled
    rrg_serve_stats stats{};
};

namespace {

uint64_t round8(uint64_t v) { return (v + 7) & ~7ull; }

cudaError_t dgrow(DBuf& b, size_t n) {
    if (n == 0) n = 16;
    if (n <= b.cap) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
#ifdef RRG_STRICT_ALLOC
    size_t c = n;  // exact sizes, so an address checker sees any overrun
#else
    size_t c = n + n / 8 + 256;
#endif
    cudaError_t e = cudaMalloc(&b.p, c);
    if (e == cudaSuccess) b.cap = c;
    return e;
}

int cuda_fail(rrg_error* err, cudaError_t e, const char* what) {
    set_err(err, e == cudaErrorMemoryAllocation ? RRG_ERR_OUT_OF_MEMORY : RRG_ERR_CUDA, "%s: %s", what,
            cudaGetErrorString(e));
    return err ? err->code : RRG_ERR_CUDA;
}

#define CK(call)                                                 \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail(err, e_, #call); \
    } while (0)

#define LAUNCHED(ctx)                                                               \
    do {                                                                            \
        g_launches.fetch_add(1);                                                    \
        (ctx)->launches++;                                                          \
        cudaError_t e_ = cudaGetLastError();                                        \
        if (e_ != cudaSuccess) return cuda_fail(err, e_, "kernel launch");         \
    } while (0)

// Device time of one kernel launch, measured with events on the launch stream.
struct KTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit KTimer(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    void stop() { cudaEventRecord(b, s); }
    // call after the stream has been synchronised
    double ms() {
        float f = 0;
        cudaEventElapsedTime(&f, a, b);
        return (double)f;
    }
    ~KTimer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

int upload_tables(rrg_ctx* c, rrg_error* err) {
    if (c->tables_uploaded) return 0;
    std::call_once(g_tab_once, init_tables);
    std::call_once(g_lut_once, init_next_lut);
    CK(cudaMemcpyToSymbol(c_x2k, g_x2k, sizeof(g_x2k)));
    CK(dgrow(c->crc_table, sizeof(g_crc_tab) + sizeof(g_crc_z496)));
    CK(cudaMemcpy(c->crc_table.p, g_crc_tab, sizeof(g_crc_tab), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((uint8_t*)c->crc_table.p + sizeof(g_crc_tab), g_crc_z496, sizeof(g_crc_z496),
                  cudaMemcpyHostToDevice));
    CK(dgrow(c->next_lut, sizeof(g_next_lut)));
    CK(cudaMemcpy(c->next_lut.p, g_next_lut, sizeof(g_next_lut), cudaMemcpyHostToDevice));
    c->tables_uploaded = true;
    return 0;
}

uint32_t persistent_blocks(rrg_ctx* c, uint32_t per_sm, uint64_t work_units, uint32_t units_per_block) {
    uint64_t need = (work_units + units_per_block - 1) / units_per_block;
    uint64_t cap = (uint64_t)c->n_sm * per_sm;
    return (uint32_t)std::max<uint64_t>(1, std::min(need, cap));
}

// The host path's input pieces: make the decode stream wait for all of them.
int wait_arrival(rrg_ctx* c, rrg_error* err) {
    if (!c->arr_base) return 0;
    if (!c->arr_pieces.empty()) CK(cudaStreamWaitEvent(c->stream, c->arr_pieces.back().second, 0));
    c->arr_base = nullptr;
    c->arr_pieces.clear();
    return 0;
}

// ------------------------------------------------------------ inflate launch
int launch_inflate(rrg_ctx* c, const uint8_t* d_in, const std::vector<ChunkItem>& items, bool bytes_out,
                   void* d_out_cells, std::vector<ChunkResult>& res, std::vector<MemberRec>* mrecs,
                   rrg_error* err) {
    if (int rw = wait_arrival(c, err)) return rw;
    const uint32_t n = (uint32_t)items.size();
    res.assign(n, ChunkResult{});
    if (!n) return 0;
    // largest spans first: long chunks start early, short ones fill the tail
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    auto span = [&](uint32_t i) {
        uint64_t e = items[i].end_hint == ~0ull ? items[i].in_len * 8 : items[i].end_hint;
        return e > items[i].start_bit ? e - items[i].start_bit : 0;
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return span(a) > span(b); });
    uint32_t mb_cap = mrecs ? (uint32_t)std::max<size_t>(4096, mrecs->capacity()) : 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        CK(dgrow(c->items, n * sizeof(ChunkItem)));
        CK(dgrow(c->results, n * sizeof(ChunkResult)));
        CK(dgrow(c->order, n * sizeof(uint32_t)));
        CK(dgrow(c->queue, 16));
        CK(dgrow(c->mbs, (size_t)std::max<uint32_t>(mb_cap, 1) * sizeof(MemberRec)));
        CK(dgrow(c->mbcount, 16));
        CK(cudaMemcpyAsync(c->items.p, items.data(), n * sizeof(ChunkItem), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->order.p, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemsetAsync(c->queue.p, 0, 16, c->stream));
        CK(cudaMemsetAsync(c->mbcount.p, 0, 16, c->stream));
        InflateArgs A{};
        A.in = d_in;
        A.items = (const ChunkItem*)c->items.p;
        A.results = (ChunkResult*)c->results.p;
        A.n_items = n;
        A.order = (const uint32_t*)c->order.p;
        A.queue = (uint32_t*)c->queue.p;
        A.out = d_out_cells;
        A.mbs = (MemberRec*)c->mbs.p;
        A.mb_count = (uint32_t*)c->mbcount.p;
        A.mb_cap = mb_cap;
        const uint32_t W = c->inflate_warps;
        const size_t smem = W * sizeof(WarpSmem);
        // as many resident blocks per SM as registers and shared memory allow
        int occ = 0;
        if (bytes_out) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint8_t>, W * 32, smem);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint16_t>, W * 32, smem);
        const uint32_t per_sm = std::max<uint32_t>(1, (uint32_t)occ);
        const uint32_t grid = persistent_blocks(c, per_sm, n, W);
        KTimer kt(c->stream);
        if (c->lanes) {
            const size_t lsmem = LANE_THREADS * sizeof(LaneTab);
            int locc = 0;
            if (bytes_out) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&locc, k_inflate_lanes<uint8_t>, LANE_THREADS, lsmem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&locc, k_inflate_lanes<uint16_t>, LANE_THREADS, lsmem);
            const uint32_t lgrid = persistent_blocks(c, std::max(1, locc), n, LANE_THREADS);
            CK(dgrow(c->lane_scratch, (size_t)lgrid * LANE_THREADS * sizeof(LaneScratch)));
            if (bytes_out) {
                RRG_LAUNCH(k_inflate_lanes<uint8_t>, lgrid, LANE_THREADS, lsmem, c->stream, A,
                           (LaneScratch*)c->lane_scratch.p);
            } else {
                RRG_LAUNCH(k_inflate_lanes<uint16_t>, lgrid, LANE_THREADS, lsmem, c->stream, A,
                           (LaneScratch*)c->lane_scratch.p);
            }
        } else if (bytes_out) {
            RRG_LAUNCH(k_inflate<uint8_t>, grid, W * 32, smem, c->stream, A);
        } else {
            RRG_LAUNCH(k_inflate<uint16_t>, grid, W * 32, smem, c->stream, A);
        }
        kt.stop();
        LAUNCHED(c);
        CK(cudaMemcpyAsync(res.data(), c->results.p, n * sizeof(ChunkResult), cudaMemcpyDeviceToHost, c->stream));
        uint32_t cnt = 0;
        CK(cudaMemcpyAsync(&cnt, c->mbcount.p, 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->st.inflate_ms += kt.ms();
        if (!mrecs) return 0;
        if (cnt <= mb_cap) {
            mrecs->resize(cnt);
            if (cnt)
                CK(cudaMemcpy(mrecs->data(), c->mbs.p, cnt * sizeof(MemberRec), cudaMemcpyDeviceToHost));
            return 0;
        }
        mb_cap = cnt + 1024;  // member records overflowed: once more with room for all
    }
    set_err(err, RRG_ERR_OUT_OF_MEMORY, "member record buffer overflow");
    return RRG_ERR_OUT_OF_MEMORY;
}

// ------------------------------------------------------------ CRC check
struct MemberSpan {
    uint64_t out_start, len;
    uint32_t crc, isize;
    uint64_t trailer_byte;
};

// CRC32/ISIZE of every span on the device; per-span status (DS_OK, DS_CRC,
// DS_ISIZE), computed CRC and length come back in stv/got/glen.
int crc_spans(rrg_ctx* c, const uint8_t* d_out, const std::vector<MemberSpan>& ms, std::vector<int32_t>& stv,
              std::vector<uint32_t>& got, std::vector<uint64_t>& glen, rrg_error* err) {
    const uint32_t nm = (uint32_t)ms.size();
    stv.assign(nm, 0);
    got.assign(nm, 0);
    glen.assign(nm, 0);
    if (!nm) return 0;
    const uint64_t PIECE = 256 * 1024;
    std::vector<CrcPiece> pieces;
    std::vector<uint32_t> mstart(nm + 1);
    std::vector<uint32_t> ecrc(nm), eisz(nm);
    for (uint32_t m = 0; m < nm; m++) {
        mstart[m] = (uint32_t)pieces.size();
        for (uint64_t o = 0; o < ms[m].len; o += PIECE)
            pieces.push_back(CrcPiece{ms[m].out_start + o, std::min(PIECE, ms[m].len - o)});
        ecrc[m] = ms[m].crc;
        eisz[m] = ms[m].isize;
    }
    mstart[nm] = (uint32_t)pieces.size();
    const uint32_t np = (uint32_t)pieces.size();
    CK(dgrow(c->pieces, std::max<size_t>(np, 1) * sizeof(CrcPiece)));
    CK(dgrow(c->piece_crc, std::max<size_t>(np, 1) * 4));
    CK(dgrow(c->mpiece, (nm + 1) * 4));
    CK(dgrow(c->exp_crc, nm * 4));
    CK(dgrow(c->exp_isize, nm * 4));
    CK(dgrow(c->got_crc, nm * 4));
    CK(dgrow(c->got_len, nm * 8));
    CK(dgrow(c->mstatus, nm * 4));
    if (np) CK(cudaMemcpyAsync(c->pieces.p, pieces.data(), np * sizeof(CrcPiece), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->mpiece.p, mstart.data(), (nm + 1) * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->exp_crc.p, ecrc.data(), nm * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->exp_isize.p, eisz.data(), nm * 4, cudaMemcpyHostToDevice, c->stream));
    KTimer kt(c->stream);
    if (np) {
        CrcWideArgs A{d_out, (const CrcPiece*)c->pieces.p, np, (uint32_t*)c->piece_crc.p,
                      (const uint32_t*)c->crc_table.p, nullptr};
        uint32_t grid = persistent_blocks(c, 8, np, 1);
        RRG_LAUNCH(k_crc_pieces_wide, grid, CRCW_THREADS, 0, c->stream, A);
        LAUNCHED(c);
    }
    CrcMemberArgs B{(const CrcPiece*)c->pieces.p, (const uint32_t*)c->piece_crc.p, (const uint32_t*)c->mpiece.p, nm,
                    (const uint32_t*)c->exp_crc.p, (const uint32_t*)c->exp_isize.p, (uint32_t*)c->got_crc.p,
                    (uint64_t*)c->got_len.p, (int32_t*)c->mstatus.p};
    RRG_LAUNCH(k_crc_members, (nm * 32 + 255) / 256, 256, 0, c->stream, B);
    kt.stop();
    LAUNCHED(c);
    CK(cudaMemcpyAsync(stv.data(), c->mstatus.p, nm * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(got.data(), c->got_crc.p, nm * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(glen.data(), c->got_len.p, nm * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->st.crc_ms += kt.ms();
    c->st.members += nm;
    return 0;
}

// GzipError::{CrcMismatch, IsizeMismatch} for one member (gzip.rs:26-60).
int member_error(rrg_error* err, const MemberSpan& m, uint32_t member, int32_t st, uint32_t got, uint64_t glen) {
    if (st == DS_CRC) {
        set_err(err, RRG_ERR_CRC_MISMATCH,
                "CRC32 mismatch in member #%u (uncompressed bytes: %llu, trailer at byte %llu): expected "
                "%#010x, got %#010x",
                member, (unsigned long long)glen, (unsigned long long)m.trailer_byte, m.crc, got);
        err->member = member;
        err->expected = m.crc;
        err->got_crc = got;
        err->uncompressed = glen;
        err->trailer_byte = m.trailer_byte;
        return RRG_ERR_CRC_MISMATCH;
    }
    set_err(err, RRG_ERR_ISIZE_MISMATCH, "ISIZE mismatch in member #%u (trailer at byte %llu): expected %u, got %llu",
            member, (unsigned long long)m.trailer_byte, m.isize, (unsigned long long)glen);
    err->member = member;
    err->expected = m.isize;
    err->got = glen;
    err->uncompressed = glen;
    err->trailer_byte = m.trailer_byte;
    return RRG_ERR_ISIZE_MISMATCH;
}

// All spans of one stream: the first failing member is the error.
int check_members(rrg_ctx* c, const uint8_t* d_out, const std::vector<MemberSpan>& ms, uint32_t member_base,
                  rrg_error* err) {
    std::vector<int32_t> stv;
    std::vector<uint32_t> got;
    std::vector<uint64_t> glen;
    int rc = crc_spans(c, d_out, ms, stv, got, glen, err);
    if (rc) return rc;
    for (size_t m = 0; m < ms.size(); m++)
        if (stv[m] == DS_CRC || stv[m] == DS_ISIZE)
            return member_error(err, ms[m], member_base + (uint32_t)m, stv[m], got[m], glen[m]);
    return 0;
}

// ------------------------------------------------------------ output target
// Where decoded bytes go: a caller buffer of fixed capacity, or the context's
// own buffer, which grows on demand keeping the bytes already written.
struct OutTarget {
    uint8_t* p;
    uint64_t cap;
    bool grow;
};

int ensure_out(rrg_ctx* c, OutTarget& t, uint64_t need, uint64_t keep, rrg_error* err) {
    if (need <= t.cap) return 0;
    if (!t.grow) {
        set_err(err, RRG_ERR_CAPACITY, "output buffer too small: need %llu bytes", (unsigned long long)need);
        return RRG_ERR_CAPACITY;
    }
    void* np = nullptr;
    size_t nc = need + need / 8 + 4096;
    CK(cudaMalloc(&np, nc));
    if (keep && t.p) {
        CK(cudaMemcpyAsync(np, t.p, keep, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    if (c->out.p) cudaFree(c->out.p);
    c->out.p = np;
    c->out.cap = nc;
    t.p = (uint8_t*)np;
    t.cap = nc;
    return 0;
}

// ------------------------------------------------------------ resolve
// The resolve kernels' grouping of a run of jobs' chunks (consecutive in the
// chunk table): groups of consecutive chunks sized so one job's groups fill
// the SMs (k_win_maps runs one block per group, chunk after chunk),
// supergroups of about sqrt(groups) groups, and the tail units.
struct ResTables {
    std::vector<ResGroup> groups, supers;
    std::vector<ResJob> jobs;
    std::vector<uint32_t> chunk_group, group_super;
    std::vector<uint64_t> tail_units;  // groups + 1
    // one device blob: groups | supers | jobs | chunk_group | group_super | tail_units
    size_t o_sup = 0, o_job = 0, o_cg = 0, o_gs = 0, o_tu = 0, bytes = 0;
    void layout() {
        o_sup = round8(groups.size() * sizeof(ResGroup));
        o_job = o_sup + round8(supers.size() * sizeof(ResGroup));
        o_cg = o_job + round8(jobs.size() * sizeof(ResJob));
        o_gs = o_cg + round8(chunk_group.size() * 4);
        o_tu = o_gs + round8(group_super.size() * 4);
        bytes = o_tu + tail_units.size() * 8;
    }
    void write(uint8_t* dst) const {
        std::memcpy(dst, groups.data(), groups.size() * sizeof(ResGroup));
        std::memcpy(dst + o_sup, supers.data(), supers.size() * sizeof(ResGroup));
        std::memcpy(dst + o_job, jobs.data(), jobs.size() * sizeof(ResJob));
        std::memcpy(dst + o_cg, chunk_group.data(), chunk_group.size() * 4);
        std::memcpy(dst + o_gs, group_super.data(), group_super.size() * 4);
        std::memcpy(dst + o_tu, tail_units.data(), tail_units.size() * 8);
    }
};

void build_res_tables(const std::vector<uint32_t>& job_chunks, uint32_t n_sm, ResTables& T) {
    T = ResTables{};
    uint32_t c0 = 0;
    for (uint32_t cj : job_chunks) {
        const uint32_t S = std::max<uint32_t>(1, (cj + n_sm - 1) / n_sm);
        const uint32_t g0 = (uint32_t)T.groups.size();
        for (uint32_t f = c0; f < c0 + cj; f += S) {
            const uint32_t n = std::min(S, c0 + cj - f);
            for (uint32_t k = 0; k < n; k++) T.chunk_group.push_back((uint32_t)T.groups.size());
            T.groups.push_back(ResGroup{f, n});
        }
        const uint32_t ng = (uint32_t)T.groups.size() - g0;
        const uint32_t SG = std::max<uint32_t>(1, (uint32_t)std::ceil(std::sqrt((double)ng)));
        const uint32_t s0 = (uint32_t)T.supers.size();
        for (uint32_t g = g0; g < g0 + ng; g += SG) {
            const uint32_t n = std::min(SG, g0 + ng - g);
            for (uint32_t q = 0; q < n; q++) T.group_super.push_back((uint32_t)T.supers.size());
            T.supers.push_back(ResGroup{g, n});
        }
        T.jobs.push_back(ResJob{s0, (uint32_t)T.supers.size() - s0});
        c0 += cj;
    }
    T.tail_units.assign(T.groups.size() + 1, 0);
    for (size_t g = 0; g < T.groups.size(); g++)
        T.tail_units[g + 1] = T.tail_units[g] + (T.groups[g].n + RES_TAIL_CHUNKS - 1) / RES_TAIL_CHUNKS;
    T.layout();
}

// Device pointers of a tables blob at `dev`, and the map arrays at `win`.
void res_args(ResolveArgs& R, const ResTables& T, const uint8_t* dev, uint16_t* win, uint32_t n_chunks) {
    R.n_chunks = n_chunks;
    R.groups = (const ResGroup*)dev;
    R.n_groups = (uint32_t)T.groups.size();
    R.supers = (const ResGroup*)(dev + T.o_sup);
    R.n_supers = (uint32_t)T.supers.size();
    R.jobs = (const ResJob*)(dev + T.o_job);
    R.n_jobs = (uint32_t)T.jobs.size();
    R.chunk_group = (const uint32_t*)(dev + T.o_cg);
    R.group_super = (const uint32_t*)(dev + T.o_gs);
    R.tail_units = (const uint64_t*)(dev + T.o_tu);
    const size_t W = WINDOW;
    R.maps = win;
    R.gmaps = R.maps + (size_t)n_chunks * W;
    R.bases = R.gmaps + (size_t)R.n_groups * W;
    R.tmaps = R.bases + (size_t)R.n_groups * W;
    R.sbases = R.tmaps + (size_t)R.n_supers * W;
}
size_t res_win_bytes(const ResTables& T, uint32_t n_chunks) {
    return ((size_t)n_chunks + 2 * T.groups.size() + 2 * T.supers.size()) * WINDOW * 2;
}

// The six resolve launches on `s` (tables and head segments already on the device).
int launch_resolve(rrg_ctx* c, const ResolveArgs& R, cudaStream_t s, rrg_error* err) {
    const uint32_t nsm = c->n_sm;
    RRG_LAUNCH(k_win_maps, std::min<uint32_t>(R.n_groups, nsm), WM_THREADS, WM_SMEM, s, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_win_supers, std::min<uint32_t>(R.n_supers, nsm), WM_THREADS, WINDOW * 2, s, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_win_bases, std::min<uint32_t>(R.n_jobs, nsm), WM_THREADS, WINDOW * 2, s, R);
    LAUNCHED(c);
    const uint64_t ex = (uint64_t)R.n_groups * (WINDOW / 8);
    RRG_LAUNCH(k_win_expand, (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((ex + 255) / 256, nsm * 8ull)),
               RES_THREADS, 0, s, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_res_tails, nsm * 3, RES_THREADS, WINDOW * 2, s, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_res_heads, nsm * 4, RES_THREADS, 0, s, R);
    LAUNCHED(c);
    return 0;
}

// Window maps, bases, chunk tails, then the rest of every chunk, into d_dst.
// Chunks of one job are consecutive in `rchunks` with rising out_start; the
// job's first chunk has out_start == job_out. Returns 0 or an error code; a
// failure names its chunk in *bad_chunk.
int run_resolve(rrg_ctx* c, const std::vector<ResolveChunk>& rchunks, uint8_t* d_dst, rrg_error* err,
                int64_t* bad_chunk = nullptr) {
    const uint32_t nc = (uint32_t)rchunks.size();
    if (!nc) return 0;
    std::vector<uint32_t> job_chunks;
    for (uint32_t a = 0; a < nc;) {
        uint32_t b = a + 1;
        while (b < nc && rchunks[b].job_out == rchunks[a].job_out && rchunks[b].out_start > rchunks[b - 1].out_start)
            b++;
        job_chunks.push_back(b - a);
        a = b;
    }
    ResTables T;
    build_res_tables(job_chunks, c->n_sm, T);
    std::vector<uint64_t> hs(nc + 1, 0);
    for (uint32_t k = 0; k < nc; k++)
        hs[k + 1] = hs[k] + (res_head_end(rchunks[k].n_cells) + RES_HEAD_SEG - 1) / RES_HEAD_SEG;
    // one upload: chunks | head segments | tables
    const size_t o_hs = round8(nc * sizeof(ResolveChunk)), o_t = o_hs + round8((nc + 1) * 8), total = o_t + T.bytes;
    std::vector<uint8_t> blob(total);
    std::memcpy(blob.data(), rchunks.data(), nc * sizeof(ResolveChunk));
    std::memcpy(blob.data() + o_hs, hs.data(), (nc + 1) * 8);
    T.write(blob.data() + o_t);
    CK(dgrow(c->chunks, total));
    CK(dgrow(c->win, res_win_bytes(T, nc)));
    CK(dgrow(c->rerr, 16));
    CK(dgrow(c->markers, 8));
    CK(cudaMemcpyAsync(c->chunks.p, blob.data(), total, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->rerr.p, 0, 16, c->stream));
    CK(cudaMemsetAsync(c->markers.p, 0, 8, c->stream));
    uint8_t* dev = (uint8_t*)c->chunks.p;
    ResolveArgs R{};
    R.cells = (uint16_t*)c->cells.p;
    R.chunks = (const ResolveChunk*)dev;
    R.head_segs = (const uint64_t*)(dev + o_hs);
    res_args(R, T, dev + o_t, (uint16_t*)c->win.p, nc);
    R.out = d_dst;
    R.err = (uint32_t*)c->rerr.p;
    R.markers = (unsigned long long*)c->markers.p;
    KTimer kt(c->stream);
    if (int rc = launch_resolve(c, R, c->stream, err)) return rc;
    kt.stop();
    uint32_t e4[4];
    unsigned long long nmk = 0;
    CK(cudaMemcpyAsync(e4, c->rerr.p, 16, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&nmk, c->markers.p, 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->st.resolve_ms += kt.ms();
    c->st.markers += nmk;
    if (e4[0]) {
        if (bad_chunk) *bad_chunk = e4[1];
        set_err(err, RRG_ERR_DEFLATE_INVALID, "%s", msg_text(MSG_MARKER_WINDOW));
        return RRG_ERR_DEFLATE_INVALID;
    }
    return 0;
}

// The window after the last chunk of `rchunks` (one job) as a map relative to
// the job's first window, which is not known yet: the window kernels run with
// an identity first window, and the map comes back to the host (WINDOW u16).
int run_resolve_map(rrg_ctx* c, const std::vector<ResolveChunk>& rchunks, std::vector<uint16_t>& map,
                    rrg_error* err) {
    const uint32_t nc = (uint32_t)rchunks.size();
    map.assign(WINDOW, 0);
    if (!nc) {  // nothing decoded: the window is unchanged
        for (uint32_t i = 0; i < WINDOW; i++) map[i] = (uint16_t)(WM_REF | i);
        return 0;
    }
    ResTables T;
    build_res_tables({nc}, c->n_sm, T);
    const size_t o_t = round8(nc * sizeof(ResolveChunk)), total = o_t + T.bytes;
    std::vector<uint8_t> blob(total);
    std::memcpy(blob.data(), rchunks.data(), nc * sizeof(ResolveChunk));
    T.write(blob.data() + o_t);
    CK(dgrow(c->chunks, total));
    CK(dgrow(c->win, res_win_bytes(T, nc) + WINDOW * 2));
    CK(dgrow(c->markers, 8));
    CK(cudaMemcpyAsync(c->chunks.p, blob.data(), total, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->markers.p, 0, 8, c->stream));
    uint8_t* dev = (uint8_t*)c->chunks.p;
    ResolveArgs R{};
    R.cells = (uint16_t*)c->cells.p;
    R.chunks = (const ResolveChunk*)dev;
    res_args(R, T, dev + o_t, (uint16_t*)c->win.p, nc);
    R.markers = (unsigned long long*)c->markers.p;
    R.identity_base = 1;
    uint16_t* d_map = (uint16_t*)((uint8_t*)c->win.p + res_win_bytes(T, nc));
    const uint32_t nsm = c->n_sm;
    RRG_LAUNCH(k_win_maps, std::min<uint32_t>(R.n_groups, nsm), WM_THREADS, WM_SMEM, c->stream, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_win_supers, std::min<uint32_t>(R.n_supers, nsm), WM_THREADS, WINDOW * 2, c->stream, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_win_bases, 1, WM_THREADS, WINDOW * 2, c->stream, R);
    LAUNCHED(c);
    const uint64_t ex = (uint64_t)R.n_groups * (WINDOW / 8);
    RRG_LAUNCH(k_win_expand, (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((ex + 255) / 256, nsm * 8ull)),
               RES_THREADS, 0, c->stream, R);
    LAUNCHED(c);
    RRG_LAUNCH(k_win_endmap, 32, 256, 0, c->stream, R, nc - 1, d_map);
    LAUNCHED(c);
    CK(cudaMemcpyAsync(map.data(), d_map, WINDOW * 2, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// ------------------------------------------------------------ boundary scan
// Every bit offset of the body tested on the device; returns the sorted
// offsets that pass the block finder's full strict verification.
// With `tiles` (sorted indices of scan tiles, each scan_threads x 16 bytes
// from the body's 16-byte-aligned start), only those tiles are tested.
int scan_boundaries(rrg_ctx* c, const uint8_t* body, uint64_t blen, std::vector<uint64_t>& verified,
                    std::vector<uint64_t>* stored_out, rrg_error* err,
                    const std::vector<uint32_t>* tiles = nullptr) {
    verified.clear();
    if (stored_out) stored_out->clear();
    if (blen < 4) return 0;
    KTimer kt(c->stream);
    // candidates (prefilter + precode), then light-verify survivors, then the
    // heavy check; counts stay on the device between the three kernels
    const uint32_t cap = (uint32_t)std::min<uint64_t>(blen / 64 + 65536, 1ull << 28);
    const uint32_t cap2 = std::max<uint32_t>(cap / 16, 65536);
    const uint32_t cap3 = (uint32_t)std::min<uint64_t>(blen / 1024 + 4096, 1ull << 26);
    CK(dgrow(c->cand, (size_t)cap * 8 + (size_t)cap2 * 8 + (size_t)cap3 * 8));
    CK(dgrow(c->ncand, 64));
    CK(dgrow(c->vflag, cap2));
    CK(cudaMemsetAsync(c->ncand.p, 0, 64, c->stream));
    uint64_t* cand = (uint64_t*)c->cand.p;
    uint64_t* surv = cand + cap;
    uint64_t* stored = surv + cap2;
    uint32_t* counts = (uint32_t*)c->ncand.p;  // [0] candidates, [1] survivors, [2] heavy queue, [3] stored
    ScanArgs S{body, blen, cand, counts, cap, stored, counts + 3, cap3, 0, ~0ull, nullptr, 0};
    // tile width: scan_threads x 16 bytes per block step (64, 128 or 256 threads)
    const uint32_t st = c->scan_threads;
    const uint64_t tb = (uint64_t)st * 16;
    const uint64_t n_tiles = ((uint64_t)((uintptr_t)body & 15) + blen + tb - 1) / tb;
    if (tiles && !tiles->empty()) {
        CK(dgrow(c->tiles, tiles->size() * 4));
        CK(cudaMemcpyAsync(c->tiles.p, tiles->data(), tiles->size() * 4, cudaMemcpyHostToDevice, c->stream));
    }
    auto scan = [&](uint64_t t_lo, uint64_t t_hi) -> int {
        if (t_hi <= t_lo) return 0;
        S.tile_lo = t_lo;
        S.tile_hi = t_hi;
        uint64_t work = t_hi - t_lo;
        if (tiles) {  // the listed tiles in [t_lo, t_hi)
            const size_t a = std::lower_bound(tiles->begin(), tiles->end(), (uint32_t)t_lo) - tiles->begin();
            const size_t b = std::lower_bound(tiles->begin(), tiles->end(), (uint32_t)std::min<uint64_t>(t_hi, ~0u)) -
                             tiles->begin();
            if (b <= a) return 0;
            S.tile_list = (const uint32_t*)c->tiles.p + a;
            S.n_list = (uint32_t)(b - a);
            work = b - a;
        }
        const uint32_t sgrid =
            (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(work, (uint64_t)c->n_sm * (2048 / st)));
        if (st == 64) RRG_LAUNCH(k_scan_candidates<64>, sgrid, 64, 0, c->stream, S);
        else if (st == 128) RRG_LAUNCH(k_scan_candidates<128>, sgrid, 128, 0, c->stream, S);
        else RRG_LAUNCH(k_scan_candidates<256>, sgrid, 256, 0, c->stream, S);
        LAUNCHED(c);
        return 0;
    };
    // both verifications of the candidates found so far; the light one starts
    // after the candidates it has seen (counts[4]), the heavy one's queue
    // after the survivors it has seen (counts[2])
    VerifyArgs V{body, blen, cand, counts, cap, surv, counts + 1, cap2, nullptr, nullptr, counts + 4};
    VerifyArgs H{body, blen, surv, counts + 1, cap2, nullptr, nullptr, 0, (uint8_t*)c->vflag.p, counts + 2, nullptr};
    const uint32_t W = 4;
    auto verify = [&]() -> int {
        RRG_LAUNCH(k_verify_light, c->n_sm * 8, 256, 0, c->stream, V);
        LAUNCHED(c);
        RRG_LAUNCH(k_verify_heavy, c->n_sm * 4, W * 32, W * sizeof(FindSmem), c->stream, H);
        LAUNCHED(c);
        return 0;
    };
    // Input still arriving (host path): scan each tile as soon as its bytes,
    // and the 64 KiB past them that the stored-block check may read, are here,
    // and verify its candidates (their reads stay inside that margin).
    uint64_t t_done = 0;
    if (c->arr_base && !c->arr_pieces.empty()) {
        const uint8_t* tile0 = (const uint8_t*)((uintptr_t)body & ~(uintptr_t)15);
        const uint64_t skip = (uint64_t)(tile0 - c->arr_base);
#ifdef RRG_EMU
        const uint64_t piece_min = 0;  // the CPU emulation exercises per-piece verification on small inputs
#else
        const uint64_t piece_min = 16ull << 20;
#endif
        const bool per_piece = c->arr_pieces.size() > 1 && c->arr_pieces[0].first >= piece_min;
        for (const auto& pc : c->arr_pieces) {
            CK(cudaStreamWaitEvent(c->stream, pc.second, 0));
            const uint64_t have = pc.first > skip ? pc.first - skip : 0;
            const uint64_t t_hi = have > 65600 ? std::min(n_tiles, (have - 65600) / tb) : 0;
            if (t_hi <= t_done) continue;
            int rc0 = scan(t_done, t_hi);
            if (rc0) return rc0;
            t_done = t_hi;
            // verification per piece pays only when a piece's copy outlasts
            // the launches (pieces of at least 16 MiB); smaller inputs verify once
            if (per_piece) {
                if (int rv = verify()) return rv;
                RRG_LAUNCH(k_verify_mark, 1, 32, 0, c->stream, counts, cap, cap2);
                LAUNCHED(c);
            }
        }
        c->arr_base = nullptr;  // everything has arrived for the kernels that follow
        c->arr_pieces.clear();
    }
    int rcs = scan(t_done, n_tiles);
    if (rcs) return rcs;
    if (int rv = verify()) return rv;
    kt.stop();
    uint32_t cnt[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(cnt, counts, 16, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->cfg.verbose >= 2)
        std::fprintf(stderr, "[rrg-gpu] boundary scan of %llu bytes: %u candidates, %u after the code-length check, "
                     "%u stored-block starts\n", (unsigned long long)blen, cnt[0], cnt[1], cnt[3]);
    if (cnt[3]) {  // stored-block starts need no verification (the anchored chain checks them)
        const uint32_t ns = std::min(cnt[3], cap3);
        std::vector<uint64_t> st(ns);
        CK(cudaMemcpyAsync(st.data(), stored, (size_t)ns * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (uint64_t v : st) verified.push_back(v & ~1ull);  // bit 0: empty block
        if (stored_out) {
            *stored_out = st;
            std::sort(stored_out->begin(), stored_out->end());
        }
    }
    if (cnt[0] > cap || cnt[1] > cap2) {
        set_err(err, RRG_ERR_OUT_OF_MEMORY, "boundary scan: %u candidates exceed the list", cnt[0]);
        return RRG_ERR_OUT_OF_MEMORY;
    }
    const uint32_t m = cnt[1];
    std::vector<uint64_t> sv(m);
    std::vector<uint8_t> ok(m);
    if (m) {
        CK(cudaMemcpyAsync(sv.data(), surv, (size_t)m * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(ok.data(), c->vflag.p, m, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    for (uint32_t i = 0; i < m; i++)
        if (ok[i]) verified.push_back(sv[i]);
    std::sort(verified.begin(), verified.end());
    c->st.finder_ms += kt.ms();
    return 0;
}

// Targets (bits from `body`) that have no start in `verified` within `half`
// bits on either side.
std::vector<uint64_t> lone_targets(const std::vector<uint64_t>& targets, const std::vector<uint64_t>& verified,
                                   uint64_t half) {
    std::vector<uint64_t> lone;
    for (uint64_t x : targets) {
        auto it = std::lower_bound(verified.begin(), verified.end(), x > half ? x - half : 0);
        if (it == verified.end() || *it > x + half) lone.push_back(x);
    }
    return lone;
}

// Targets for the fixed-code walk. A target with no start within 256 KiB shows
// fixed-Huffman blocks nearby (zlib's dynamic and stored blocks are at most a
// few tens of KiB apart); then every target with no start within 16 KiB is
// walked, so that one false dynamic-header match among fixed blocks does not
// leave a wide span to a single sub-chunk. A stream without such a target
// walks nothing.
std::vector<uint64_t> walk_targets(const std::vector<uint64_t>& targets, const std::vector<uint64_t>& verified) {
    if (lone_targets(targets, verified, (256ull << 10) * 8).empty()) return {};
    return lone_targets(targets, verified, (16ull << 10) * 8);
}

// Block starts found by walking the fixed Huffman code forward from each
// target (k_fixed_walk), for targets the candidate scan left without a start,
// as in a stream of fixed-Huffman blocks. They join `verified`, which stays
// sorted and free of duplicates. A walk gives up 256 KiB past its target.
int fixed_walk_starts(rrg_ctx* c, const uint8_t* body, uint64_t blen, const std::vector<uint64_t>& from,
                      std::vector<uint64_t>& verified, rrg_error* err) {
    if (from.empty() || blen < 8) return 0;
    const uint32_t n = (uint32_t)from.size();
    KTimer kt(c->stream);
    CK(dgrow(c->targets, (size_t)n * 8));
    CK(dgrow(c->found, (size_t)n * 8));
    CK(cudaMemcpyAsync(c->targets.p, from.data(), (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    FixedWalkArgs F{body, blen, (const uint64_t*)c->targets.p, (uint64_t*)c->found.p, n, (256ull << 10) * 8};
    RRG_LAUNCH(k_fixed_walk, (n + FW_THREADS / 32 - 1) / (FW_THREADS / 32), FW_THREADS, 0, c->stream, F);
    LAUNCHED(c);
    kt.stop();
    std::vector<uint64_t> found(n);
    CK(cudaMemcpyAsync(found.data(), c->found.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->st.finder_ms += kt.ms();
    size_t added = 0;
    for (uint64_t f : found)
        if (f != ~0ull) {
            verified.push_back(f);
            added++;
        }
    if (c->cfg.verbose >= 2)
        std::fprintf(stderr, "[rrg-gpu] fixed-code walk from %u targets: %zu block starts\n", n, added);
    if (added) {
        std::sort(verified.begin(), verified.end());
        verified.erase(std::unique(verified.begin(), verified.end()), verified.end());
    }
    return 0;
}

// ------------------------------------------------------------ member route
// Decoders resident at once on the device: warps (or lanes) of one full wave
// of the inflate kernel.
uint64_t inflate_slots(rrg_ctx* c) {
    if (!c->slots) {
        int occ = 0;
        if (c->lanes) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate_lanes<uint16_t>, LANE_THREADS,
                                                          LANE_THREADS * sizeof(LaneTab));
            c->slots = (uint64_t)c->n_sm * std::max(occ, 1) * LANE_THREADS;
        } else {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint16_t>, c->inflate_warps * 32,
                                                          c->inflate_warps * sizeof(WarpSmem));
            c->slots = (uint64_t)c->n_sm * std::max(occ, 1) * c->inflate_warps;
        }
    }
    return c->slots;
}

struct Decoded {
    uint64_t total = 0;  // bytes written at the job's destination
    uint64_t consumed = 0;
    uint32_t members = 0;
};

// One gzip member stream (a file, or what follows a BGZF prefix) for the
// member route. Several jobs share every kernel launch.
struct MemberJob {
    uint64_t file_off = 0;    // the file's first byte in the base buffer
    uint64_t len = 0;         // file bytes from file_off
    uint64_t body_off = 0;    // first member's deflate body, relative to file_off
    uint64_t dst_off = 0;     // first output byte in the target
    uint64_t dst_cap = ~0ull; // output bytes available at dst_off (~0: the target grows)
    uint32_t member_base = 0; // index of the first member, for error reports
    double expand = 0;        // output cells per compressed byte to reserve (0: the context's estimate)
    uint64_t isize_hint = 0;  // the trailer's ISIZE (0: unknown), for balancing sub-chunks
    // A stripe of a non-seekable stream: decoding starts at start_bit (relative
    // to body_off) inside a member whose earlier bytes have been delivered,
    // and stops at the first block edge at or after stop_bit. The last
    // prefix_len of those bytes sit in the target just before dst_off (for
    // back-references); crc_prev/len_prev are their CRC32 and count.
    uint64_t start_bit = 0;
    uint64_t stop_bit = ~0ull;  // ~0: decode to the end of the input
    uint64_t report_off = 0;    // added to input offsets in error reports (the stripe's place in the stream)
    bool check_crc = true;      // false: a range read from a seek point (members are only partly decoded)
    // when set: every sub-chunk start the chain kept, as (bit relative to
    // body_off, output offset relative to dst_off), for a seek index
    std::vector<std::pair<uint64_t, uint64_t>>* capture = nullptr;
    // when set: decode and lay out only, save what resolving needs here and
    // compute the map of the job's last window relative to its first window
    // (one range of a member split across GPUs)
    struct SplitState* split = nullptr;
    uint64_t prefix_len = 0;
    uint32_t crc_prev = 0;
    uint64_t len_prev = 0;
    // results
    int rc = 0;
    rrg_error err{};
    Decoded out;
    uint64_t end_bit = 0;       // where decoding stopped, relative to body_off
    bool open_member = false;   // stopped inside a member (stripe jobs)
    uint64_t open_start = 0;    // output offset (from dst_off) where that member's bytes in this stripe begin
    uint32_t open_crc = 0;      // CRC32 and length of that member so far, earlier stripes included
    uint64_t open_len = 0;
};

// CRC32 of A||B from CRC32(A), CRC32(B) and |B| (GF(2) polynomial product
// with x^(8|B|) from the x^(2^k) table).
uint32_t host_crc_combine(uint32_t a, uint32_t b, uint64_t len_b) {
    uint32_t p = 0x80000000u;  // x^0
    const uint64_t n = len_b;
    for (int k = 0; k < 61; k++)
        if ((n >> k) & 1u) p = host_mulmod(p, g_x2k[k + 3]);
    return host_mulmod(a, p) ^ b;
}

namespace mr {
struct Acc {
    ChunkItem it;
    ChunkResult r;
    std::vector<MemberRec> m;
};
struct JobState {
    size_t first = 0, n = 0;  // the job's initial items
    size_t k = 0;             // next initial item to chain
    uint64_t expected = 0;
    bool final_seen = false, done = false;
    std::vector<Acc> acc;
    std::vector<size_t> overflow;  // indices into acc
    int64_t pending = -1;          // index into the current re-decode list
};
}  // namespace mr

// Decodes every job's member stream (pipeline.rs:468-1041 per job) with one
// boundary search, one inflate launch (plus rare re-decode launches), one
// resolve and one CRC pass for all of them. A failing job gets its own
// rc/err and leaves the others untouched; the return value is non-zero only
// for failures of the whole batch (device errors, allocation).
int members_route(rrg_ctx* c, const uint8_t* d_base, std::vector<MemberJob>& jobs, OutTarget& tgt, rrg_error* err) {
    using namespace mr;
    const size_t nj = jobs.size();
    // Sub-chunk spacing. A fixed gpu_chunk_bytes takes the first boundary at
    // least that far from the previous one. Otherwise the compressed bytes of
    // all jobs are spread over one wave of the inflate kernel's resident
    // decoders: each job gets chunks in proportion to its size, and each
    // boundary is the verified block start nearest its ideal position.
    uint64_t total_c = 0;
    for (const MemberJob& j : jobs) total_c += j.len - j.body_off;
    const bool fixed_g = c->gpu_chunk != 0;
    const uint64_t g_min = c->lanes ? (8ull << 10) : (16ull << 10);
    const uint64_t slots = inflate_slots(c);
    const uint64_t G = fixed_g ? std::max<uint64_t>(c->gpu_chunk, 4096)
                               : std::max<uint64_t>(g_min, (total_c + slots - 1) / slots);
    std::vector<std::vector<uint64_t>> starts(nj);
    for (size_t i = 0; i < nj; i++) starts[i].push_back(jobs[i].start_bit);
    std::vector<std::vector<uint64_t>> stored_starts(nj);  // sorted, relative to each body
    auto fail = [&](MemberJob& j, int st, int msg, uint64_t where) { j.rc = status_err(&j.err, st, msg, where); };
    // ---- sub-chunk boundaries
    if (c->scan_bounds) {
        // verified dynamic-block starts; the bodies are scanned in clusters of
        // nearby ranges, one scan per cluster
        std::vector<size_t> big;
        for (size_t i = 0; i < nj; i++)
            if (jobs[i].len - jobs[i].body_off > G) big.push_back(i);
        std::sort(big.begin(), big.end(), [&](size_t a, size_t b) { return jobs[a].file_off < jobs[b].file_off; });
        for (size_t a = 0; a < big.size();) {
            uint64_t lo = jobs[big[a]].file_off + jobs[big[a]].body_off, hi = jobs[big[a]].file_off + jobs[big[a]].len;
            size_t b = a + 1;
            while (b < big.size() && jobs[big[b]].file_off + jobs[big[b]].body_off <= hi + (1u << 20)) {
                hi = std::max(hi, jobs[big[b]].file_off + jobs[big[b]].len);
                b++;
            }
            std::vector<uint64_t> verified, stored;
            // With automatic spacing only the bytes around each ideal start are
            // scanned (a window of +-16 KiB holds one or more block starts of
            // ordinary deflate output); targets whose window held none are
            // scanned again +-256 KiB wide. Fixed spacing scans everything.
            std::vector<uint64_t> ideal;  // bits from lo
            for (size_t q = a; q < b && !fixed_g; q++) {
                const MemberJob& j = jobs[big[q]];
                const uint64_t b0 = (j.file_off + j.body_off - lo) * 8, b1 = (j.file_off + j.len - lo) * 8;
                const uint64_t s0 = b0 + j.start_bit, s1 = j.stop_bit == ~0ull ? b1 : std::min(b1, b0 + j.stop_bit);
                const uint64_t nbits = s1 > s0 ? s1 - s0 : 0;
                const uint64_t K = std::max<uint64_t>(1, (nbits / 8 + G / 2) / G);
                for (uint64_t k = 1; k < K; k++) ideal.push_back(s0 + nbits * k / K);
            }
            const uint64_t tb = (uint64_t)c->scan_threads * 16, mis = (uintptr_t)(d_base + lo) & 15;
            const uint64_t n_tiles = (mis + (hi - lo) + tb - 1) / tb;
            auto windows = [&](const std::vector<uint64_t>& at, uint64_t half, const std::vector<uint32_t>* skip) {
                std::vector<uint32_t> t;
                for (uint64_t x : at) {
                    const uint64_t byte = x / 8;
                    const uint64_t t0 = (mis + (byte > half ? byte - half : 0)) / tb;
                    const uint64_t t1 = std::min(n_tiles - 1, (mis + byte + half) / tb);
                    for (uint64_t k = t0; k <= t1; k++)
                        if (!skip || !std::binary_search(skip->begin(), skip->end(), (uint32_t)k)) t.push_back((uint32_t)k);
                }
                std::sort(t.begin(), t.end());
                t.erase(std::unique(t.begin(), t.end()), t.end());
                return t;
            };
            constexpr uint64_t NEAR = 16 << 10, WIDE = 256 << 10;
            std::vector<uint32_t> tiles;
            const bool windowed = !fixed_g && !ideal.empty() && n_tiles <= 0xffffffffull &&
                                  (tiles = windows(ideal, NEAR, nullptr)).size() * 2 < n_tiles;
            int rc0 = scan_boundaries(c, d_base + lo, hi - lo, verified, &stored, err, windowed ? &tiles : nullptr);
            if (rc0) return rc0;
            if (windowed) {
                std::vector<uint64_t> missing;
                for (uint64_t x : ideal) {
                    auto it = std::lower_bound(verified.begin(), verified.end(), x > NEAR * 8 ? x - NEAR * 8 : 0);
                    if (it == verified.end() || *it > x + NEAR * 8) missing.push_back(x);
                }
                if (!missing.empty()) {
                    const std::vector<uint32_t> more = windows(missing, WIDE, &tiles);
                    std::vector<uint64_t> v2, s2;
                    if (!more.empty()) {
                        rc0 = scan_boundaries(c, d_base + lo, hi - lo, v2, &s2, err, &more);
                        if (rc0) return rc0;
                        verified.insert(verified.end(), v2.begin(), v2.end());
                        std::sort(verified.begin(), verified.end());
                        stored.insert(stored.end(), s2.begin(), s2.end());
                        std::sort(stored.begin(), stored.end());
                    }
                }
            }
            // fixed-Huffman blocks: starts found by walking the fixed code
            if (int rf = fixed_walk_starts(c, d_base + lo, hi - lo, walk_targets(ideal, verified), verified,
                                           err))
                return rf;
            // verified offsets are sorted bit offsets from `lo`
            for (size_t q = a; q < b; q++) {
                MemberJob& j = jobs[big[q]];
                const uint64_t b0 = (j.file_off + j.body_off - lo) * 8, b1 = (j.file_off + j.len - lo) * 8;
                auto& st = starts[big[q]];
                for (auto it = std::lower_bound(stored.begin(), stored.end(), b0); it != stored.end() && *it < b1; ++it)
                    stored_starts[big[q]].push_back(*it - b0);  // keeps the empty-block bit
                // a stripe job splits only its own bit range
                const uint64_t s0 = b0 + j.start_bit;
                const uint64_t s1 = j.stop_bit == ~0ull ? b1 : std::min(b1, b0 + j.stop_bit);
                auto lo_it = std::lower_bound(verified.begin(), verified.end(), s0);
                auto hi_it = std::lower_bound(lo_it, verified.end(), std::max(s0, s1));
                if (fixed_g) {
                    for (auto it = lo_it; it != hi_it; ++it)
                        if (*it - b0 >= st.back() + G * 8) st.push_back(*it - b0);
                } else {
                    const uint64_t nbits = s1 > s0 ? s1 - s0 : 0;
                    const uint64_t K = std::max<uint64_t>(1, (nbits / 8 + G / 2) / G);
                    for (uint64_t k = 1; k < K; k++) {
                        const uint64_t ideal = s0 + nbits * k / K;
                        auto it = std::lower_bound(lo_it, hi_it, ideal);
                        uint64_t best = ~0ull;
                        if (it != hi_it) best = *it;
                        if (it != lo_it && (best == ~0ull || ideal - *(it - 1) < best - ideal)) best = *(it - 1);
                        if (best != ~0ull && best - b0 > st.back()) st.push_back(best - b0);
                    }
                }
            }
            a = b;
        }
    } else {
        // first dynamic block at/after every G bytes (find_next_dynamic_block per target)
        std::vector<uint64_t> targets, limits;
        std::vector<size_t> owner;
        for (size_t i = 0; i < nj; i++) {
            const uint64_t base_bit = (jobs[i].file_off + jobs[i].body_off) * 8;
            const uint64_t total_bits = std::min((jobs[i].len - jobs[i].body_off) * 8, jobs[i].stop_bit);
            const size_t t0 = targets.size();
            for (uint64_t t = jobs[i].start_bit + G * 8; t < total_bits; t += G * 8) {
                targets.push_back(base_bit + t);
                owner.push_back(i);
            }
            for (size_t q = t0; q < targets.size(); q++)
                limits.push_back(q + 1 < targets.size() ? targets[q + 1] : base_bit + total_bits);
        }
        if (int rw = wait_arrival(c, err)) return rw;
        if (!targets.empty()) {
            const uint32_t n = (uint32_t)targets.size();
            std::vector<uint64_t> found(n, ~0ull);
            uint64_t span_hi = 0;
            for (const MemberJob& j : jobs) span_hi = std::max(span_hi, j.file_off + j.len);
            CK(dgrow(c->targets, n * 8));
            CK(dgrow(c->limits, n * 8));
            CK(dgrow(c->found, n * 8));
            CK(dgrow(c->queue, 16));
            CK(cudaMemcpyAsync(c->targets.p, targets.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(c->limits.p, limits.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemsetAsync(c->queue.p, 0, 16, c->stream));
            FindArgs F{d_base, span_hi, (const uint64_t*)c->targets.p, (const uint64_t*)c->limits.p,
                       (uint64_t*)c->found.p, n, (uint32_t*)c->queue.p, (const uint8_t*)c->next_lut.p, c->finder_tile};
            const uint32_t W = 4;
            uint32_t grid = persistent_blocks(c, 4, n, W);
            KTimer kt(c->stream);
            RRG_LAUNCH(k_find_blocks, grid, W * 32, W * sizeof(FindSmem), c->stream, F);
            kt.stop();
            LAUNCHED(c);
            CK(cudaMemcpyAsync(found.data(), c->found.p, n * 8, cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            c->st.finder_ms += kt.ms();
            for (uint32_t q = 0; q < n; q++) {
                const size_t i = owner[q];
                const uint64_t base_bit = (jobs[i].file_off + jobs[i].body_off) * 8;
                if (found[q] != ~0ull && found[q] - base_bit > starts[i].back()) starts[i].push_back(found[q] - base_bit);
            }
        }
    }
    std::vector<JobState> js(nj);
    for (size_t i = 0; i < nj; i++) js[i].expected = jobs[i].start_bit;
    uint32_t next_id = 0;
    std::unordered_map<uint32_t, std::vector<MemberRec>> by_item;
    auto bucket = [&](const std::vector<MemberRec>& all) {
        for (const MemberRec& m : all) by_item[m.item].push_back(m);
    };
    auto take_recs = [&](uint32_t id) {
        std::vector<MemberRec> v;
        auto f = by_item.find(id);
        if (f != by_item.end()) {
            v.swap(f->second);
            std::sort(v.begin(), v.end(), [](const MemberRec& a, const MemberRec& b) { return a.seq < b.seq; });
        }
        return v;
    };
    // ---- a stream of one chunk with a fixed destination decodes straight to
    // its bytes: it cannot hold markers, so there is nothing to resolve
    // (only when no stream is split: otherwise they join the one speculative
    // launch, so that a single persistent wave covers every stream)
    std::vector<char> direct(nj, 0);
    std::vector<std::vector<MemberRec>> direct_recs(nj);
    bool any_split = false;
    for (size_t i = 0; i < nj; i++) any_split |= starts[i].size() > 1;
    {
        std::vector<ChunkItem> ditems;
        std::vector<size_t> djob;
        for (size_t i = 0; i < nj && !tgt.grow && !any_split; i++) {
            if (starts[i].size() != 1 || jobs[i].start_bit || jobs[i].stop_bit != ~0ull) continue;
            const MemberJob& j = jobs[i];
            direct[i] = 1;
            ChunkItem it{};
            it.in_off = j.file_off + j.body_off;
            it.in_len = j.len - j.body_off;
            it.start_bit = 0;
            it.end_hint = ~0ull;
            it.out_off = j.dst_off;
            it.out_cap = j.dst_cap;
            it.flags = 0;
            it.id = next_id++;
            ditems.push_back(it);
            djob.push_back(i);
        }
        if (!ditems.empty()) {
            std::vector<ChunkResult> dres;
            std::vector<MemberRec> dm;
            dm.reserve(4096);
            int rc0 = launch_inflate(c, d_base, ditems, true, tgt.p, dres, &dm, err);
            if (rc0) return rc0;
            c->st.gpu_chunks += ditems.size();
            bucket(dm);
            for (size_t q = 0; q < ditems.size(); q++) {
                MemberJob& j = jobs[djob[q]];
                const ChunkResult& r = dres[q];
                js[djob[q]].done = true;
                j.out.total = r.n_cells;
                j.out.consumed = j.file_off + j.body_off + r.actual_end_bit / 8;
                if (r.status == DS_OVERFLOW) {
                    set_err(&j.err, RRG_ERR_CAPACITY, "output buffer too small: need %llu bytes",
                            (unsigned long long)r.n_cells);
                    j.rc = RRG_ERR_CAPACITY;
                } else if (r.status != DS_OK) {
                    fail(j, r.status, r.msg, j.report_off + j.file_off + j.body_off + r.err_bit / 8);
                } else if (!r.final_block) {
                    set_err(&j.err, RRG_ERR_IO, "parallel decode produced no final block");
                    j.rc = RRG_ERR_IO;
                }
                direct_recs[djob[q]] = take_recs(ditems[q].id);
            }
        }
    }
    // ---- items and the slot arena: every chunk gets expand x its compressed span
    std::vector<ChunkItem> items;
    uint64_t arena = 0;
    for (size_t i = 0; i < nj; i++) {
        if (direct[i]) continue;
        const MemberJob& j = jobs[i];
        const uint64_t blen = j.len - j.body_off, total_bits = blen * 8;
        const auto& st = starts[i];
        js[i].first = items.size();
        js[i].n = st.size();
        for (size_t k = 0; k < st.size(); k++) {
            ChunkItem it;
            it.in_off = j.file_off + j.body_off;
            it.in_len = blen;
            it.start_bit = st[k];
            it.end_hint = k + 1 < st.size() ? st[k + 1] : j.stop_bit;
            const uint64_t span = ((k + 1 < st.size() ? st[k + 1] : total_bits) - st[k] + 7) / 8;
            it.out_cap = round8((uint64_t)(span * (j.expand > 0 ? j.expand : c->expand)) + 65536);
            it.out_off = arena;
            // the first chunk too, as in the reference: a reference before the
            // stream's start becomes a marker that fails to resolve
            it.flags = ITEM_MARKERS;
            if (k) {
                if (std::binary_search(stored_starts[i].begin(), stored_starts[i].end(), st[k]))
                    it.flags |= ITEM_STORED_START;
                else if (std::binary_search(stored_starts[i].begin(), stored_starts[i].end(), st[k] | 1))
                    it.flags |= ITEM_STORED_START | ITEM_EMPTY_STORED;
            }
            it.id = next_id++;
            arena += it.out_cap;
            items.push_back(it);
        }
    }
    const uint64_t arena_cap = arena + arena / 4 + (1u << 20);
    CK(dgrow(c->cells, arena_cap * 2));
    std::vector<ChunkResult> res;
    std::vector<MemberRec> mrecs;
    mrecs.reserve(4096);
    int rc = launch_inflate(c, d_base, items, false, c->cells.p, res, &mrecs, err);
    if (rc) return rc;
    c->st.gpu_chunks += items.size();

    bucket(mrecs);
    // ---- anchored chain (pipeline.rs:758-809), in rounds: every job walks its
    // chunks until one needs a re-decode from the true anchor; the re-decodes
    // of all jobs share one launch
    for (;;) {
        std::vector<ChunkItem> redo;
        std::vector<size_t> redo_job;
        for (size_t i = 0; i < nj; i++) {
            JobState& s = js[i];
            MemberJob& j = jobs[i];
            while (!s.done && s.pending < 0) {
                if (s.final_seen || s.k >= s.n) {
                    s.done = true;
                    // a stripe job ends at the block edge past its stop bit
                    if (!s.final_seen && !(j.stop_bit != ~0ull && s.expected >= j.stop_bit)) {
                        set_err(&j.err, RRG_ERR_IO, "parallel decode produced no final block");
                        j.rc = RRG_ERR_IO;
                    }
                    break;
                }
                ChunkItem it = items[s.first + s.k];
                const ChunkResult r = res[s.first + s.k];
                // A start on a zero header byte of a stored block decodes exactly as
                // the true start does when that lies in the same byte's first 6 bits
                // (BFINAL=0 and BTYPE=00 are read from zeros, and the padding ends at
                // the same byte boundary), or, for an empty block, when the true start
                // is right after it (the block adds nothing to the output).
                const uint64_t d = s.expected - it.start_bit;
                const bool same_start =
                    it.start_bit == s.expected ||
                    ((it.flags & ITEM_STORED_START) && s.expected > it.start_bit &&
                     (d <= 5 || ((it.flags & ITEM_EMPTY_STORED) && d == 40)));
                if (same_start && (r.status == DS_OK || r.status == DS_OVERFLOW)) {
                    s.acc.push_back(Acc{it, r, take_recs(it.id)});
                } else {
                    // false boundary or failed speculative decode: re-decode from the anchor
                    c->st.speculation_failures++;
                    if (c->cfg.verbose >= 2)
                        std::fprintf(stderr, "[rrg-gpu] re-decode: chunk at bit %llu (flags %u) status %d, anchor %llu\n",
                                     (unsigned long long)it.start_bit, it.flags, r.status,
                                     (unsigned long long)s.expected);
                    if (it.end_hint != ~0ull && s.expected >= it.end_hint) {  // empty chunk
                        s.k++;
                        continue;
                    }
                    // the anchor lies at or after the guessed start (the previous chunk
                    // stops on a block edge at/after its end hint), so the re-decode
                    // spans no more input than the guess did and reuses its slot
                    it.start_bit = s.expected;
                    it.id = next_id++;
                    s.pending = (int64_t)redo.size();
                    redo.push_back(it);
                    redo_job.push_back(i);
                    break;
                }
                if (s.acc.back().r.status == DS_OVERFLOW) s.overflow.push_back(s.acc.size() - 1);
                s.expected = s.acc.back().r.actual_end_bit;
                s.final_seen = s.acc.back().r.final_block != 0;
                s.k++;
            }
        }
        if (redo.empty()) break;
        std::vector<ChunkResult> r1;
        std::vector<MemberRec> m1;
        m1.reserve(4096);
        rc = launch_inflate(c, d_base, redo, false, c->cells.p, r1, &m1, err);
        if (rc) return rc;
        bucket(m1);
        for (size_t q = 0; q < redo.size(); q++) {
            JobState& s = js[redo_job[q]];
            MemberJob& j = jobs[redo_job[q]];
            s.pending = -1;
            const ChunkResult& r = r1[q];
            if (r.status != DS_OK && r.status != DS_OVERFLOW) {
                fail(j, r.status, r.msg, j.report_off + j.file_off + j.body_off + r.err_bit / 8);
                s.done = true;
                continue;
            }
            s.acc.push_back(Acc{redo[q], r, take_recs(redo[q].id)});
            if (r.status == DS_OVERFLOW) s.overflow.push_back(s.acc.size() - 1);
            s.expected = r.actual_end_bit;
            s.final_seen = r.final_block != 0;
            s.k++;
        }
    }
    // ---- overflowed slots: decode again with the exact size now known
    {
        std::vector<ChunkItem> redo;
        std::vector<std::pair<size_t, size_t>> where;  // (job, acc index)
        uint64_t need = 0;
        for (size_t i = 0; i < nj; i++) {
            if (jobs[i].rc) continue;
            for (size_t a : js[i].overflow) {
                ChunkItem it = js[i].acc[a].it;
                it.out_cap = round8(js[i].acc[a].r.n_cells + 8);
                it.id = next_id++;
                need += it.out_cap;
                redo.push_back(it);
                where.push_back({i, a});
            }
        }
        if (!redo.empty()) {
            if (arena + need > arena_cap) {
                // the slots were far too small for this data: decode everything
                // again with a larger expansion estimate (DEFLATE expands <= 1032x)
                // (size hints from the trailers are dropped first)
                bool hinted = false;
                for (const MemberJob& j : jobs) hinted |= j.expand > 0;
                if (!hinted && c->expand >= 1100.0) {
                    set_err(err, RRG_ERR_OUT_OF_MEMORY, "output slot arena exhausted");
                    return RRG_ERR_OUT_OF_MEMORY;
                }
                if (!hinted) c->expand = std::min(1100.0, c->expand * 8);
                for (MemberJob& j : jobs) {
                    j.rc = 0;
                    j.err = rrg_error{};
                    j.out = Decoded{};
                    j.expand = 0;
                }
                return members_route(c, d_base, jobs, tgt, err);
            }
            for (auto& it : redo) {
                it.out_off = arena;
                arena += it.out_cap;
            }
            std::vector<ChunkResult> r2;
            std::vector<MemberRec> m2;
            m2.reserve(4096);
            rc = launch_inflate(c, d_base, redo, false, c->cells.p, r2, &m2, err);
            if (rc) return rc;
            bucket(m2);
            for (size_t q = 0; q < redo.size(); q++) {
                MemberJob& j = jobs[where[q].first];
                if (j.rc) continue;
                if (r2[q].status != DS_OK) {
                    fail(j, r2[q].status, r2[q].msg, j.report_off + j.file_off + j.body_off + r2[q].err_bit / 8);
                    continue;
                }
                Acc& a = js[where[q].first].acc[where[q].second];
                a.it = redo[q];
                a.r = r2[q];
                a.m = take_recs(redo[q].id);
            }
        }
    }
    // ---- output layout and member spans
    uint64_t grow_need = 0;
    for (size_t i = 0; i < nj; i++) {
        MemberJob& j = jobs[i];
        if (j.rc || direct[i]) continue;
        uint64_t pos = 0;
        for (const Acc& a : js[i].acc) pos += a.r.n_cells;
        j.out.total = pos;
        j.out.consumed = j.file_off + j.body_off + js[i].expected / 8;
        j.end_bit = js[i].expected;
        if (j.dst_cap != ~0ull && pos > j.dst_cap) {
            set_err(&j.err, RRG_ERR_CAPACITY, "output buffer too small: need %llu bytes", (unsigned long long)pos);
            j.rc = RRG_ERR_CAPACITY;
            continue;
        }
        grow_need = std::max(grow_need, j.dst_off + pos);
    }
    if (tgt.grow) {
        uint64_t keep = ~0ull;
        for (const MemberJob& j : jobs) keep = std::min(keep, j.dst_off);
        rc = ensure_out(c, tgt, grow_need, keep == ~0ull ? 0 : keep, err);
        if (rc) return rc;
    }
    for (size_t i = 0; i < nj; i++) {
        MemberJob& j = jobs[i];
        if (j.rc || !j.capture) continue;
        j.capture->clear();
        if (direct[i]) {
            j.capture->push_back({j.start_bit, 0});
            continue;
        }
        uint64_t pos = 0;
        for (const Acc& a : js[i].acc) {
            j.capture->push_back({a.it.start_bit, pos});
            pos += a.r.n_cells;
        }
    }
    std::vector<ResolveChunk> rchunks;
    std::vector<size_t> chunk_job;
    std::vector<MemberSpan> spans;
    std::vector<size_t> span_job;
    std::vector<uint32_t> span_member;
    // 0: a whole member; 1: a member continued from earlier stripes, ended
    // here; 2: the member a stripe stops in (no trailer yet)
    std::vector<uint8_t> span_kind;
    for (size_t i = 0; i < nj; i++) {
        MemberJob& j = jobs[i];
        if (j.rc) continue;
        uint64_t pos = 0, mstart = 0;
        uint32_t nm = 0;
        const bool continued = j.start_bit != 0 || j.len_prev != 0;
        if (direct[i]) {
            for (const MemberRec& m : direct_recs[i]) {
                spans.push_back(MemberSpan{j.dst_off + mstart, m.cell_off - mstart, m.crc, m.isize,
                                           j.report_off + j.file_off + j.body_off + m.trailer_byte});
                span_job.push_back(i);
                span_member.push_back(j.member_base + nm++);
                span_kind.push_back(0);
                mstart = m.cell_off;
            }
            j.out.members = nm;
            continue;
        }
        for (const Acc& a : js[i].acc) {
            if (a.r.n_cells) {
                // the first member of a stripe began before dst_off: its last
                // prefix_len bytes there serve the chunk windows
                const uint64_t ms = (nm == 0 && continued) ? j.dst_off - j.prefix_len : j.dst_off + mstart;
                rchunks.push_back(ResolveChunk{j.dst_off + pos, a.it.out_off, a.r.n_cells, ms, j.dst_off});
                chunk_job.push_back(i);
            }
            for (const MemberRec& m : a.m) {
                const uint64_t end = pos + m.cell_off;
                spans.push_back(MemberSpan{j.dst_off + mstart, end - mstart, m.crc, m.isize,
                                           j.report_off + j.file_off + j.body_off + m.trailer_byte});
                span_job.push_back(i);
                span_member.push_back(j.member_base + nm);
                span_kind.push_back(nm == 0 && continued ? 1 : 0);
                nm++;
                mstart = end;
            }
            pos += a.r.n_cells;
        }
        j.out.members = nm;
        if (j.stop_bit != ~0ull && !js[i].final_seen) {
            spans.push_back(MemberSpan{j.dst_off + mstart, pos - mstart, 0, 0, 0});
            span_job.push_back(i);
            span_member.push_back(j.member_base + nm);
            span_kind.push_back(nm == 0 && continued ? 3 : 2);  // 3: also the continued first member
        }
    }
    // ---- one range of a split member: stop before resolving
    if (nj == 1 && jobs[0].split) {
        MemberJob& j = jobs[0];
        if (j.rc) return 0;
        SplitState& S = *j.split;
        size_t ends = 0, last = 0;
        for (size_t m = 0; m < spans.size(); m++)
            if (span_kind[m] <= 1) {
                ends++;
                last = m;
            }
        if (ends > 1 || (ends == 1 && !js[0].final_seen)) {
            set_err(&j.err, RRG_ERR_INVALID_ARGUMENT, "a split decode takes a single-member stream");
            j.rc = RRG_ERR_INVALID_ARGUMENT;
            return 0;
        }
        S.rchunks = rchunks;
        S.dst_off = j.dst_off;
        S.total = j.out.total;
        S.end_bit = js[0].expected;
        S.has_trailer = ends == 1;
        if (ends) {
            S.crc = spans[last].crc;
            S.isize = spans[last].isize;
            S.trailer_byte = spans[last].trailer_byte;
        }
        S.ready = false;
        if (int rm = run_resolve_map(c, rchunks, S.end_map, err)) return rm;
        S.ready = true;
        return 0;
    }
    // ---- resolve markers + compact; a failing chunk fails its job only
    int64_t bad = -1;
    rrg_error rerr{};
    rc = run_resolve(c, rchunks, tgt.p, &rerr, &bad);
    if (rc && (rc != RRG_ERR_DEFLATE_INVALID || bad < 0 || (uint64_t)bad >= chunk_job.size())) {
        if (err) *err = rerr;
        return rc;
    }
    if (rc) {
        jobs[chunk_job[bad]].rc = rc;
        jobs[chunk_job[bad]].err = rerr;
    }
    // ---- CRC32/ISIZE of every member (spans are positions in the target)
    std::vector<int32_t> stv;
    std::vector<uint32_t> got;
    std::vector<uint64_t> glen;
    rc = crc_spans(c, tgt.p, spans, stv, got, glen, err);
    if (rc) return rc;
    for (size_t m = 0; m < spans.size(); m++) {
        MemberJob& j = jobs[span_job[m]];
        if (j.rc || !j.check_crc) continue;
        if (span_kind[m] >= 2) {  // the member continues in the next stripe
            j.open_member = true;
            j.open_start = spans[m].out_start - j.dst_off;
            j.open_crc = span_kind[m] == 3 ? host_crc_combine(j.crc_prev, got[m], glen[m]) : got[m];
            j.open_len = (span_kind[m] == 3 ? j.len_prev : 0) + glen[m];
            continue;
        }
        if (span_kind[m] == 1) {  // whole-member check with the earlier stripes' bytes
            got[m] = host_crc_combine(j.crc_prev, got[m], glen[m]);
            glen[m] += j.len_prev;
            stv[m] = got[m] != spans[m].crc ? DS_CRC : (uint32_t)glen[m] != spans[m].isize ? DS_ISIZE : DS_OK;
        }
        if (stv[m] != DS_CRC && stv[m] != DS_ISIZE) continue;
        j.rc = member_error(&j.err, spans[m], span_member[m], stv[m], got[m], glen[m]);
    }
    return 0;
}

// One member stream at d_file (its first header already parsed) into
// tgt.p[dst_off ..]. On RRG_ERR_CAPACITY `out->total` holds the size required.
int member_route(rrg_ctx* c, const uint8_t* d_file, uint64_t len, uint64_t body_off, OutTarget& tgt, uint64_t dst_off,
                 uint32_t member_base, Decoded* out, rrg_error* err) {
    std::vector<MemberJob> jobs(1);
    jobs[0].len = len;
    jobs[0].body_off = body_off;
    jobs[0].dst_off = dst_off;
    jobs[0].dst_cap = tgt.grow ? ~0ull : (tgt.cap > dst_off ? tgt.cap - dst_off : 0);
    jobs[0].member_base = member_base;
    int rc = members_route(c, d_file, jobs, tgt, err);
    *out = jobs[0].out;
    if (rc) return rc;
    if (jobs[0].rc && err) *err = jobs[0].err;
    return jobs[0].rc;
}

// ------------------------------------------------------------ BGZF route
// The whole BGZF decode is enqueued without a host round trip: member scan,
// chain walk, one persistent k_inflate<u8> launch over every member, CRC
// pieces and combine, and a first-failure reduction; the host reads 64 bytes
// of results at the end. The sequence is captured into a CUDA graph and
// replayed while the buffers it names stay the same.
constexpr int BGK_KERNELS = 9;  // kernels in one BGZF decode

int bgzf_enqueue(rrg_ctx* c, const uint8_t* d_file, uint64_t len, uint8_t* d_out, uint64_t out_cap, uint32_t sgrid,
                 uint64_t per_block, uint32_t cap, rrg_error* err) {
    uint64_t* small = (uint64_t*)c->bg_small.p;
    uint32_t* nmem = (uint32_t*)(small + 4);
    uint32_t* first = (uint32_t*)(small + 5);
    uint32_t* ncand = (uint32_t*)(small + 6);
    BgzfScanArgs S{d_file, len, per_block, (uint32_t*)c->bg_bcount.p, (uint32_t*)c->bg_bbase.p,
                   (uint64_t*)c->bg_coff.p, (uint32_t*)c->bg_csize.p, cap, ncand};
    RRG_LAUNCH(k_bgzf_count, sgrid, BG_THREADS, 0, c->stream, S);
    LAUNCHED(c);
    RRG_LAUNCH(k_bgzf_prefix, 1, 1024, 0, c->stream, S, sgrid);
    LAUNCHED(c);
    RRG_LAUNCH(k_bgzf_collect, sgrid, BG_THREADS, 0, c->stream, S);
    LAUNCHED(c);
    BgzfChainArgs C{d_file, len, (const uint64_t*)c->bg_coff.p, (const uint32_t*)c->bg_csize.p, ncand, cap,
                    (ChunkItem*)c->items.p, cap, (CrcPiece*)c->pieces.p, (uint32_t*)c->mpiece.p,
                    (uint32_t*)c->exp_crc.p, (uint32_t*)c->exp_isize.p, out_cap, nmem, small};
    RRG_LAUNCH(k_bgzf_chain, 1, 32, 0, c->stream, C);
    LAUNCHED(c);
    CK(cudaMemsetAsync(c->queue.p, 0, 16, c->stream));
    CK(cudaMemsetAsync(first, 0xff, 8, c->stream));
    InflateArgs A{};
    A.in = d_file;
    A.items = (const ChunkItem*)c->items.p;
    A.results = (ChunkResult*)c->results.p;
    A.n_items = cap;
    A.n_items_dev = nmem;
    A.order = nullptr;
    A.queue = (uint32_t*)c->queue.p;
    A.out = d_out;
    A.mbs = (MemberRec*)c->mbs.p;
    A.mb_count = (uint32_t*)c->mbcount.p;
    A.mb_cap = 0;
    if (c->lanes) {
        int locc = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&locc, k_inflate_lanes<uint8_t>, LANE_THREADS,
                                                      LANE_THREADS * sizeof(LaneTab));
        const uint32_t lgrid = (uint32_t)c->n_sm * std::max(1, locc);
        RRG_LAUNCH(k_inflate_lanes<uint8_t>, lgrid, LANE_THREADS, LANE_THREADS * sizeof(LaneTab), c->stream, A,
                   (LaneScratch*)c->lane_scratch.p);
    } else {
        const uint32_t W = c->inflate_warps;
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint8_t>, W * 32, W * sizeof(WarpSmem));
        RRG_LAUNCH(k_inflate<uint8_t>, (uint32_t)c->n_sm * std::max(1, occ), W * 32, W * sizeof(WarpSmem), c->stream,
                   A);
    }
    LAUNCHED(c);
    RRG_LAUNCH(k_bgzf_fix, c->n_sm * 4, 256, 0, c->stream, (const ChunkResult*)c->results.p, (CrcPiece*)c->pieces.p,
               (uint32_t*)c->exp_crc.p, (uint32_t*)c->exp_isize.p, (const uint32_t*)nmem);
    LAUNCHED(c);
    CrcWideArgs P{d_out, (const CrcPiece*)c->pieces.p, 0, (uint32_t*)c->piece_crc.p, (const uint32_t*)c->crc_table.p,
                  nmem};
    RRG_LAUNCH(k_crc_pieces_wide, c->n_sm * 8, CRCW_THREADS, 0, c->stream, P);
    LAUNCHED(c);
    CrcMemberArgs M{(const CrcPiece*)c->pieces.p, (const uint32_t*)c->piece_crc.p, (const uint32_t*)c->mpiece.p, 0,
                    (const uint32_t*)c->exp_crc.p, (const uint32_t*)c->exp_isize.p, (uint32_t*)c->got_crc.p,
                    (uint64_t*)c->got_len.p, (int32_t*)c->mstatus.p, nmem};
    RRG_LAUNCH(k_crc_members, c->n_sm * 4, 256, 0, c->stream, M);
    LAUNCHED(c);
    RRG_LAUNCH(k_bgzf_first_bad, c->n_sm * 4, 256, 0, c->stream, (const ChunkResult*)c->results.p,
               (const int32_t*)c->mstatus.p, (const uint32_t*)nmem, first);
    LAUNCHED(c);
    CK(cudaMemcpyAsync(c->h_bg, small, 64, cudaMemcpyDeviceToHost, c->stream));
    return 0;
}

// Decodes the BGZF members from byte 0 of d_file into tgt; *rem = where the
// member chain ended, *truncated = the member there runs past the file.
int bgzf_route(rrg_ctx* c, const uint8_t* d_file, uint64_t len, OutTarget& tgt, Decoded* out, uint64_t* rem,
               bool* truncated, rrg_error* err) {
    *out = Decoded{};
    if (int rw = wait_arrival(c, err)) return rw;
    if (!c->h_bg) CK(cudaMallocHost((void**)&c->h_bg, 64));
    uint32_t cap = std::max<uint32_t>(c->bg_cap, (uint32_t)std::min<uint64_t>(len / 2048 + 4096, 1u << 30));
    const uint32_t sgrid =
        (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)c->n_sm * 8, (len + BG_STEP - 1) / BG_STEP));
    const uint64_t per_block = ((len + sgrid - 1) / sgrid + BG_STEP - 1) / BG_STEP * BG_STEP;
    const uint64_t* hb = c->h_bg;
    for (int attempt = 0;; attempt++) {
        if (attempt > 4) {
            set_err(err, RRG_ERR_OUT_OF_MEMORY, "BGZF member table does not converge");
            return RRG_ERR_OUT_OF_MEMORY;
        }
        c->bg_cap = cap;
        CK(dgrow(c->bg_bcount, (size_t)sgrid * 4));
        CK(dgrow(c->bg_bbase, (size_t)(sgrid + 1) * 4));
        CK(dgrow(c->bg_coff, (size_t)cap * 8));
        CK(dgrow(c->bg_csize, (size_t)cap * 4));
        CK(dgrow(c->bg_small, 64));
        CK(dgrow(c->items, (size_t)cap * sizeof(ChunkItem)));
        CK(dgrow(c->results, (size_t)cap * sizeof(ChunkResult)));
        CK(dgrow(c->pieces, (size_t)cap * sizeof(CrcPiece)));
        CK(dgrow(c->piece_crc, (size_t)cap * 4));
        CK(dgrow(c->mpiece, (size_t)(cap + 1) * 4));
        CK(dgrow(c->exp_crc, (size_t)cap * 4));
        CK(dgrow(c->exp_isize, (size_t)cap * 4));
        CK(dgrow(c->got_crc, (size_t)cap * 4));
        CK(dgrow(c->got_len, (size_t)cap * 8));
        CK(dgrow(c->mstatus, (size_t)cap * 4));
        CK(dgrow(c->queue, 16));
        CK(dgrow(c->mbs, sizeof(MemberRec)));
        CK(dgrow(c->mbcount, 16));
        if (c->lanes) {
            int locc = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&locc, k_inflate_lanes<uint8_t>, LANE_THREADS,
                                                          LANE_THREADS * sizeof(LaneTab));
            CK(dgrow(c->lane_scratch, (size_t)c->n_sm * std::max(1, locc) * LANE_THREADS * sizeof(LaneScratch)));
        }
        KTimer kt(c->stream);
        bool ran = false;
#ifndef RRG_EMU
        BgzfKey key{};
        const DBuf* bs[] = {&c->bg_bcount, &c->bg_bbase, &c->bg_coff, &c->bg_csize, &c->bg_small, &c->items,
                            &c->results,   &c->pieces,   &c->piece_crc, &c->mpiece, &c->exp_crc,  &c->exp_isize,
                            &c->got_crc,   &c->got_len,  &c->mstatus, &c->queue,  &c->mbs,      &c->mbcount,
                            &c->lane_scratch, &c->crc_table};
        for (size_t i = 0; i < sizeof(bs) / sizeof(bs[0]); i++) key.p[i] = bs[i]->p;
        key.p[20] = d_file;
        key.p[21] = tgt.p;
        key.p[22] = c->stream;
        key.p[23] = c->h_bg;
        key.v[0] = len;
        key.v[1] = tgt.cap;
        key.v[2] = cap;
        key.v[3] = sgrid;
        key.v[4] = c->lanes;
        key.v[5] = c->inflate_warps;
        if (c->use_graphs) {
            auto* ent = c->bg_graphs.find(key);
            if (!ent && c->bg_graphs.repeat(key)) {
                cudaGraph_t g = nullptr;
                cudaGraphExec_t ex = nullptr;
                if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                    const uint64_t l0 = c->launches;
                    int rc = bgzf_enqueue(c, d_file, len, tgt.p, tgt.cap, sgrid, per_block, cap, err);
                    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
                    // kernels recorded into the graph are counted when it runs
                    g_launches.fetch_sub(c->launches - l0);
                    c->launches = l0;
                    if (rc == 0 && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess)
                        ent = c->bg_graphs.add(key, ex, BGK_KERNELS);
                    if (g) cudaGraphDestroy(g);
                }
                cudaGetLastError();  // a failed capture leaves no sticky error; run directly below
            }
            if (ent) {
                CK(cudaGraphLaunch(ent->e, c->stream));
                g_launches.fetch_add(ent->kernels);
                c->launches += ent->kernels;
                c->st.graph_launches++;
                ran = true;
            }
        }
#endif
        if (!ran) {
            int rc = bgzf_enqueue(c, d_file, len, tgt.p, tgt.cap, sgrid, per_block, cap, err);
            if (rc) return rc;
        }
        kt.stop();
        CK(cudaStreamSynchronize(c->stream));
        c->st.inflate_ms += kt.ms();
        const uint64_t flags = hb[2];
        const uint32_t n_cand = ((const uint32_t*)(hb + 6))[0];
        if (flags & (BG_CAND_OVERFLOW | BG_ITEM_OVERFLOW)) {
            cap = std::max<uint32_t>(n_cand, (uint32_t)hb[3]) + 4096;
            continue;
        }
        if (flags & BG_OUT_CAPACITY) {
            if (tgt.grow) {
                int rc = ensure_out(c, tgt, hb[1], 0, err);
                if (rc) return rc;
                continue;
            }
            out->total = hb[1];
            set_err(err, RRG_ERR_CAPACITY, "output buffer too small: need %llu bytes", (unsigned long long)hb[1]);
            return RRG_ERR_CAPACITY;
        }
        break;
    }
    const uint32_t nm = (uint32_t)hb[3];
    out->total = hb[1];
    out->members = nm;
    out->consumed = hb[0];
    *rem = hb[0];
    *truncated = (hb[2] & BG_TRUNCATED) != 0;
    c->st.gpu_chunks += nm;
    c->st.members += nm;
    const uint32_t* first = (const uint32_t*)(hb + 5);
    if (first[0] != ~0u) {  // a member failed to decode
        const uint32_t i = first[0];
        ChunkResult r;
        ChunkItem it;
        CK(cudaMemcpy(&r, (const ChunkResult*)c->results.p + i, sizeof(r), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&it, (const ChunkItem*)c->items.p + i, sizeof(it), cudaMemcpyDeviceToHost));
        const uint64_t trailer = it.in_off + it.in_len - 8;
        if (r.status == DS_OVERFLOW) {
            set_err(err, RRG_ERR_ISIZE_MISMATCH, "ISIZE mismatch in member #%u (trailer at byte %llu): expected %u, got %llu",
                    i, (unsigned long long)trailer, (uint32_t)it.out_cap, (unsigned long long)r.n_cells);
            err->member = i;
            err->expected = (uint32_t)it.out_cap;
            err->got = r.n_cells;
            err->trailer_byte = trailer;
            return RRG_ERR_ISIZE_MISMATCH;
        }
        return status_err(err, r.status, r.msg, it.in_off + r.err_bit / 8);
    }
    if (first[1] != ~0u) {  // a member's CRC32 or ISIZE did not match its trailer
        const uint32_t i = first[1];
        ChunkItem it;
        int32_t st = 0;
        uint32_t got = 0, ecrc = 0, eisz = 0;
        uint64_t glen = 0;
        CK(cudaMemcpy(&it, (const ChunkItem*)c->items.p + i, sizeof(it), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&st, (const int32_t*)c->mstatus.p + i, 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&got, (const uint32_t*)c->got_crc.p + i, 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&glen, (const uint64_t*)c->got_len.p + i, 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&ecrc, (const uint32_t*)c->exp_crc.p + i, 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&eisz, (const uint32_t*)c->exp_isize.p + i, 4, cudaMemcpyDeviceToHost));
        MemberSpan m{it.out_off, glen, ecrc, eisz, it.in_off + it.in_len - 8};
        return member_error(err, m, i, st, got, glen);
    }
    return 0;
}

// ------------------------------------------------------------ whole file
// Decode a whole gzip file at d_file (device) into d_dst. `h_file` (optional)
// is the same bytes in host memory, used for header parsing.
int batch_device(rrg_ctx* c, const uint8_t* d_in, std::vector<MemberJob>& jobs, OutTarget& tgt, bool* taken,
                 rrg_error* err);

int decode_file(rrg_ctx* c, const uint8_t* d_file, uint64_t len, const uint8_t* h_file, OutTarget& tgt, Decoded* out,
                rrg_error* err) {
    *out = Decoded{};
    if (len == 0) {
        set_err(err, RRG_ERR_TRUNCATED, "truncated gzip stream");
        return RRG_ERR_TRUNCATED;
    }
    int rc = upload_tables(c, err);
    if (rc) return rc;
    // first bytes to the host for header parsing / BGZF sniff
    std::vector<uint8_t> head;
    const uint8_t* hp = h_file;
    uint64_t hlen = len;
    if (!hp) {
        hlen = std::min<uint64_t>(len, 1 << 16);
        head.resize(hlen);
        CK(cudaMemcpy(head.data(), d_file, hlen, cudaMemcpyDeviceToHost));
        hp = head.data();
    }
    if (host_bgzf_size(hp, hlen) >= 0 && c->warps_per_member > 1) {
        // W warps per member: the file as one member stream, split at verified
        // block starts every (first member's size / W) compressed bytes
        size_t hl = 0;
        int detail = 0;
        if (host_parse_header(hp, hlen, &hl, &detail) == DS_OK) {
            const uint64_t g_save = c->gpu_chunk;
            c->gpu_chunk = std::max<uint64_t>(4096, (uint64_t)host_bgzf_size(hp, hlen) / c->warps_per_member);
            rc = member_route(c, d_file, len, hl, tgt, 0, 0, out, err);
            c->gpu_chunk = g_save;
            return rc;
        }
    }
    if (host_bgzf_size(hp, hlen) >= 0) {
        Decoded d1;
        uint64_t rem = 0;
        bool trunc = false;
        rc = bgzf_route(c, d_file, len, tgt, &d1, &rem, &trunc, err);
        out->total = d1.total;
        if (rc) return rc;
        if (trunc) {
            set_err(err, RRG_ERR_TRUNCATED, "truncated gzip stream");
            return RRG_ERR_TRUNCATED;
        }
        out->members = d1.members;
        if (rem < len) {
            // what follows the BGZF members is an ordinary member stream
            std::vector<uint8_t> rh;
            const uint8_t* rp = h_file ? h_file + rem : nullptr;
            uint64_t rl = len - rem;
            if (!rp) {
                rl = std::min<uint64_t>(rl, 1 << 16);
                rh.resize(rl);
                CK(cudaMemcpy(rh.data(), d_file + rem, rl, cudaMemcpyDeviceToHost));
                rp = rh.data();
            }
            size_t hl;
            int detail;
            int st = host_parse_header(rp, rl, &hl, &detail);
            if (st == DS_TRUNCATED && rl < len - rem) {
                rh.resize(len - rem);
                CK(cudaMemcpy(rh.data(), d_file + rem, len - rem, cudaMemcpyDeviceToHost));
                st = host_parse_header(rh.data(), len - rem, &hl, &detail);
            }
            if (st) return status_err(err, st, detail, rem);
            Decoded d2;
            rc = member_route(c, d_file, len, rem + hl, tgt, d1.total, d1.members, &d2, err);
            out->total = d1.total + d2.total;
            out->members += d2.members;
            if (rc) return rc;
        }
        return 0;
    }
    size_t hl = 0;
    int detail = 0;
    int st = host_parse_header(hp, hlen, &hl, &detail);
    if (st == DS_TRUNCATED && hlen < len) {
        head.resize(len);
        CK(cudaMemcpy(head.data(), d_file, len, cudaMemcpyDeviceToHost));
        st = host_parse_header(head.data(), len, &hl, &detail);
    }
    if (st) return status_err(err, st, detail, 0);
    // A large member stream into a fixed destination takes the device-planned
    // route of the batch path: sub-chunk starts, the anchored chain, resolve
    // and CRC are planned and checked on the device with no host round trip,
    // and a repeated shape replays as one captured graph. What that route
    // cannot finish (more than one member, trailing bytes, a false start) is
    // decoded on the checked member route.
#ifdef RRG_EMU
    constexpr uint64_t PLANNED_MIN = 256u << 10;  // small inputs exercise the route in the CPU emulation
#else
    constexpr uint64_t PLANNED_MIN = 16ull << 20;
#endif
    if (!tgt.grow && len - hl >= PLANNED_MIN) {
        std::vector<MemberJob> jobs(1);
        jobs[0].len = len;
        jobs[0].body_off = hl;
        jobs[0].dst_cap = tgt.cap;
        bool taken = false;
        if (int rc0 = batch_device(c, d_file, jobs, tgt, &taken, err)) return rc0;
        if (taken) {
            *out = jobs[0].out;
            if (jobs[0].rc && err) *err = jobs[0].err;
            return jobs[0].rc;
        }
    }
    return member_route(c, d_file, len, hl, tgt, 0, 0, out, err);
}

int ensure_stage(rrg_ctx* c, size_t n, rrg_error* err) {
    if (c->h_stage_cap >= n) return 0;
    for (auto& p : c->h_stage)
        if (p) cudaFreeHost(p);
    c->h_stage[0] = c->h_stage[1] = nullptr;
    c->h_stage_cap = 0;
    CK(cudaMallocHost((void**)&c->h_stage[0], n));
    CK(cudaMallocHost((void**)&c->h_stage[1], n));
    c->h_stage_cap = n;
    return 0;
}

// Stream d_src[0..n) to the sink in order through two pinned buffers.
int deliver(rrg_ctx* c, const uint8_t* d_src, uint64_t n, rrg_sink_fn sink, void* user, bool* closed, rrg_error* err) {
    *closed = false;
    if (!n || !sink) return 0;
    const uint64_t P = std::max<uint64_t>(1 << 20, std::min<uint64_t>(c->cfg.chunk_size_bytes * 2, 16ull << 20));
    int rc = ensure_stage(c, P, err);
    if (rc) return rc;
    double t0 = now_ms();
    uint64_t npieces = (n + P - 1) / P;
    cudaEvent_t ev[2];
    CK(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    uint8_t* dst[2] = {c->h_stage[0], c->h_stage[1]};  // the consumer's buffer, or the staging buffer
    auto issue = [&](uint64_t i) -> cudaError_t {
        uint64_t o = i * P, l = std::min(P, n - o);
        dst[i & 1] = c->h_stage[i & 1];
        if (c->get_buf) {
            size_t cap = 0;
            uint8_t* b = c->get_buf(c->get_user, (size_t)l, &cap);
            if (b && cap >= l) dst[i & 1] = b;
        }
        cudaError_t e = cudaMemcpyAsync(dst[i & 1], d_src + o, l, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[i & 1], c->stream);
        return e;
    };
    cudaError_t e = issue(0);
    for (uint64_t i = 0; e == cudaSuccess && i < npieces; i++) {
        e = cudaEventSynchronize(ev[i & 1]);
        if (e != cudaSuccess) break;
        if (i + 1 < npieces) {
            e = issue(i + 1);
            if (e != cudaSuccess) break;
        }
        uint64_t o = i * P, l = std::min(P, n - o);
        c->st.chunks_decoded++;
        if (sink(user, dst[i & 1], (size_t)l)) {
            *closed = true;
            break;
        }
    }
    cudaStreamSynchronize(c->stream);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    c->st.d2h_ms += now_ms() - t0;
    if (e != cudaSuccess) return cuda_fail(err, e, "deliver");
    return 0;
}

}  // namespace

// ------------------------------------------------------------ pipelined host path
// One large member stream from host memory to the sink, with the copy of the
// output to the host overlapping the decode. The sub-chunks are decoded in
// W waves (each one resident set of decoders, in stream order); each wave's
// anchored chain is checked and its output laid out on the device
// (k_wave_chain), so its resolve, CRC pieces and device-to-host copy queue
// behind its inflate while the next wave decodes. The reference's output stage
// likewise sends chunks while later chunks decode (pipeline.rs:873-935): bytes
// of the member go out as they are resolved, and the member's CRC32/ISIZE is
// checked before its last piece is delivered. Any irregularity stops the
// pipeline at that wave; the rest is decoded on the checked path from the
// last verified bit.
namespace {

struct PipeWave {
    uint32_t first = 0, n = 0;       // items
    uint32_t piece_off = 0, piece_cap = 0;
    size_t tab_off = 0;              // offset of this wave's resolve tables in the blob
    ResTables tab;
};

int ensure_ring(rrg_ctx* c, size_t piece, uint32_t waves, rrg_error* err) {
    constexpr int RING = 4;
    if (c->h_ring_cap < piece) {
        if (c->h_ring) cudaFreeHost(c->h_ring);
        c->h_ring = nullptr;
        c->h_ring_cap = 0;
        CK(cudaMallocHost((void**)&c->h_ring, piece * RING));
        c->h_ring_cap = piece;
    }
    const size_t need = (size_t)waves * (sizeof(WaveInfo) + 16) + 64;
    if (c->h_wave_cap < need) {
        if (c->h_wave) cudaFreeHost(c->h_wave);
        c->h_wave = nullptr;
        c->h_wave_cap = 0;
        CK(cudaMallocHost((void**)&c->h_wave, need));
        c->h_wave_cap = need;
    }
    return 0;
}

// Waves the pipelined path would use for a body of `blen` compressed bytes:
// each wave needs one sub-chunk of at least 32 KiB per resident decoder (at
// most 4 waves), or the configured count, as long as each sub-chunk keeps at
// least 8 KiB.
uint32_t pipeline_waves(rrg_ctx* c, uint64_t blen) {
    if (!c->pipeline || !c->scan_bounds || c->lanes || c->gpu_chunk) return 0;
    const uint64_t slots = inflate_slots(c);
    if (c->cfg.host_pipeline >= 2)
        return (uint32_t)std::min<uint64_t>(c->cfg.host_pipeline, blen / (slots * (8ull << 10)));
    return (uint32_t)std::min<uint64_t>(4, blen / (slots * (32ull << 10)));
}

// Returns 0 with *taken = false when the file does not suit the pipeline
// (nothing has been decoded or delivered then).
int pipelined_host(rrg_ctx* c, const uint8_t* d_file, uint64_t len, const uint8_t* h_file, uint64_t hl,
                   rrg_sink_fn sink, void* user, bool* closed, uint64_t* total_out, bool* taken, rrg_error* err) {
    *taken = false;
    *closed = false;
    const uint64_t blen = len - hl;
    const uint32_t W = pipeline_waves(c, blen);
    if (W < 2 || len < 8) return 0;
    *taken = true;
    c->st.pipeline_waves = W;
    const uint8_t* body = d_file + hl;
    const double t_enter = now_ms();
    double t_mark[4] = {0, 0, 0, 0};  // host timeline (verbose)
    const uint64_t slots = inflate_slots(c);
    const uint64_t nbits = blen * 8;
    // Wave shares of the input. The last wave's output copy is the one that
    // nothing overlaps, so it gets 0.4 of the others' share (measured on a
    // 1 GiB level-9 member with three waves: 48.6 -> 43.0 ms end to end).
    std::vector<double> cum(W + 1, 0.0);
    for (uint32_t w = 0; w < W; w++) cum[w + 1] = cum[w] + (w + 1 == W && W <= 4 ? 0.4 : 1.0);
    auto wave_ideal = [&](uint32_t w) { return (uint64_t)((double)nbits * cum[w] / cum[W]); };
    // sub-chunk targets (one per resident decoder and wave), for the fixed-code walk
    const uint64_t K = slots * W;
    auto targets_in = [&](uint64_t lo, uint64_t hi) {
        std::vector<uint64_t> t;
        for (uint64_t k = 1; k < K; k++) {
            const uint64_t x = nbits * k / K;
            if (x >= lo && x < hi) t.push_back(x);
        }
        return t;
    };
    // ---- planning state of both phases
    std::vector<uint64_t> cand{0};  // block starts a sub-chunk may begin at
    std::vector<uint64_t> st;       // sub-chunk starts
    std::vector<uint32_t> wfirst;   // first sub-chunk of each wave
    std::vector<ChunkItem> items;
    std::vector<PipeWave> waves;
    std::vector<uint32_t> order;
    std::vector<uint8_t> tabs;  // ResGroup[], ResJob[1], chunk_group[] per wave, 8-byte aligned
    uint64_t arena = 0;
    uint32_t total_pieces = 0;
    auto set_cand = [&](const std::vector<uint64_t>& v) {
        cand.assign(1, 0);
        for (uint64_t x : v)
            if (x > cand.back() && x < nbits) cand.push_back(x);
    };
    auto end_of = [&](size_t i) { return i < cand.size() ? cand[i] : nbits; };
    auto nearest = [&](uint64_t x, size_t i_lo) {  // index of the candidate nearest x, at or after i_lo
        size_t i = (size_t)(std::lower_bound(cand.begin() + i_lo, cand.end(), x) - cand.begin());
        if (i == cand.size() || (i > i_lo && x - cand[i - 1] < cand[i] - x)) i--;
        return i;
    };
    // Waves [w_from, w_to) over the candidates [i_from, i_end): wave edges are
    // the block starts nearest each wave's share; within a wave (one item per
    // resident decoder), runs of consecutive blocks whose largest span is as
    // small as possible (the wave ends with its largest sub-chunk, and a block
    // is the finest unit a sub-chunk can take).
    auto plan_starts = [&](uint32_t w_from, uint32_t w_to, size_t i_from, size_t i_end) {
        std::vector<size_t> wedge{i_from};
        for (uint32_t w = w_from + 1; w < w_to; w++) {
            const size_t i = std::min(nearest(wave_ideal(w), i_from), i_end);
            if (i > wedge.back() && i < i_end) wedge.push_back(i);
        }
        wedge.push_back(i_end);
        for (size_t w = 0; w + 1 < wedge.size(); w++) {
            const size_t a = wedge[w], b = wedge[w + 1];
            auto runs = [&](uint64_t B, std::vector<uint64_t>* out) {
                uint64_t cnt = 0;
                for (size_t i = a; i < b;) {
                    size_t j = i + 1;
                    while (j < b && end_of(j + 1) - cand[i] <= B) j++;
                    if (out) out->push_back(cand[i]);
                    cnt++;
                    i = j;
                }
                return cnt;
            };
            // the answer lies between an even split and an even split plus the widest block
            uint64_t gap = 0;
            for (size_t i = a; i < b; i++) gap = std::max(gap, end_of(i + 1) - cand[i]);
            const uint64_t range = end_of(b) - cand[a];
            uint64_t lo = std::max<uint64_t>(1, range / slots), hi = std::min(range, range / slots + gap);
            while (lo < hi) {  // the smallest largest span that fits one wave
                const uint64_t mid = lo + (hi - lo) / 2;
                if (runs(mid, nullptr) <= slots) hi = mid;
                else lo = mid + 1;
            }
            wfirst.push_back((uint32_t)st.size());
            runs(lo, &st);
        }
    };
    // items [k_from, st.size()): the last one ends at next_start (~0: the member's end)
    auto make_items = [&](uint32_t k_from, uint64_t next_start, const std::vector<uint64_t>& stored) {
        const uint32_t k_to = (uint32_t)st.size();
        for (uint32_t k = k_from; k < k_to; k++) {
            ChunkItem it{};
            it.in_off = hl;
            it.in_len = blen;
            it.start_bit = st[k];
            it.end_hint = k + 1 < k_to ? st[k + 1] : next_start;
            const uint64_t span = ((it.end_hint == ~0ull ? nbits : it.end_hint) - st[k] + 7) / 8;
            it.out_cap = round8((uint64_t)(span * c->expand) + 65536);
            it.out_off = arena;
            it.flags = ITEM_MARKERS;
            if (k) {
                if (std::binary_search(stored.begin(), stored.end(), st[k])) it.flags |= ITEM_STORED_START;
                else if (std::binary_search(stored.begin(), stored.end(), st[k] | 1))
                    it.flags |= ITEM_STORED_START | ITEM_EMPTY_STORED;
            }
            it.id = k;
            arena += it.out_cap;
            items.push_back(it);
        }
    };
    // waves [waves.size(), wfirst.size()) (the last one ends at the last item):
    // each wave's resolve tables and a CRC piece region large enough for any
    // output its slots can hold
    auto make_waves = [&]() {
        order.resize(items.size());
        for (uint32_t w = (uint32_t)waves.size(); w < wfirst.size(); w++) {
            PipeWave pw;
            pw.first = wfirst[w];
            pw.n = (w + 1 < wfirst.size() ? wfirst[w + 1] : (uint32_t)st.size()) - wfirst[w];
            uint64_t cap = 0;
            for (uint32_t q = 0; q < pw.n; q++) cap += items[pw.first + q].out_cap;
            pw.piece_off = total_pieces;
            pw.piece_cap = (uint32_t)(cap / WAVE_PIECE + 2);
            total_pieces += pw.piece_cap;
            // largest spans first within the wave
            for (uint32_t q = 0; q < pw.n; q++) order[pw.first + q] = pw.first + q;
            std::stable_sort(order.begin() + pw.first, order.begin() + pw.first + pw.n,
                             [&](uint32_t a, uint32_t b) { return items[a].out_cap > items[b].out_cap; });
            build_res_tables({pw.n}, c->n_sm, pw.tab);
            pw.tab_off = tabs.size();
            tabs.resize(pw.tab_off + round8(pw.tab.bytes));
            pw.tab.write(tabs.data() + pw.tab_off);
            waves.push_back(std::move(pw));
        }
    };
    // ---- boundaries (the scan overlaps the input's arrival) and sub-chunk starts
    std::vector<uint64_t> verified, stored;
    if (int rc = scan_boundaries(c, body, blen, verified, &stored, err)) return rc;
    if (int rf = fixed_walk_starts(c, body, blen, walk_targets(targets_in(0, nbits), verified), verified,
                                   err))
        return rf;
    const double t_scanned = now_ms();
    set_cand(verified);
    plan_starts(0, W, 0, cand.size());
    make_items(0, ~0ull, stored);
    make_waves();
    t_mark[0] = now_ms();
    // ---- device memory, sized for every wave (nothing is allocated once the first wave runs)
    const uint64_t n_max = slots * W;
    const uint64_t arena_max = (uint64_t)((double)(blen + n_max) * c->expand) + n_max * (65536 + 8) + 64;
    const uint32_t pieces_max = (uint32_t)(arena_max / WAVE_PIECE + 2 * W);
    ResTables full;
    build_res_tables({(uint32_t)slots}, c->n_sm, full);
    const size_t tabs_max = (size_t)W * round8(full.bytes);
    const size_t max_win = res_win_bytes(full, (uint32_t)slots);
    const uint32_t max_n = (uint32_t)slots;
    // pipe layout: state | infos | live | n_pieces[W] | fin (exp/got/status/mpiece) | seg total |
    //              wave jobs[W] | chunks[max_n] | head_segs[max_n+1] | pieces | piece_crc | tabs
    const size_t o_info = 64, o_live = o_info + round8(W * sizeof(WaveInfo)), o_np = o_live + 8,
                 o_fin = o_np + round8(W * 4), o_seg = o_fin + 64, o_wj = o_seg + 8,
                 o_chunks = o_wj + round8(W * sizeof(WaveJob)),
                 o_hs = o_chunks + round8((size_t)max_n * sizeof(ResolveChunk)),
                 o_pc = o_hs + ((size_t)max_n + 1) * 8, o_pcrc = o_pc + (size_t)pieces_max * sizeof(CrcPiece),
                 o_tabs = o_pcrc + round8((size_t)pieces_max * 4), p_total = o_tabs + tabs_max;
    const uint64_t isize_hint = le32h(h_file + len - 4);
    OutTarget tgt{(uint8_t*)c->out.p, c->out.cap, true};
    const uint64_t out_cap = std::min<uint64_t>(arena_max, std::max<uint64_t>(isize_hint, 2 * len) + (1u << 20));
    if (int rc = ensure_out(c, tgt, out_cap, 0, err)) return rc;
    CK(dgrow(c->pipe, p_total));
    CK(dgrow(c->items, (size_t)n_max * sizeof(ChunkItem)));
    CK(dgrow(c->results, (size_t)n_max * sizeof(ChunkResult)));
    CK(dgrow(c->order, (size_t)n_max * 4));
    CK(dgrow(c->queue, (size_t)W * 16));
    CK(dgrow(c->mbs, 4096 * sizeof(MemberRec)));
    CK(dgrow(c->mbcount, 16));
    CK(dgrow(c->cells, (arena_max + 8) * 2));
    CK(dgrow(c->win, max_win));
    CK(dgrow(c->rerr, 16));
    CK(dgrow(c->markers, 8));
    CK(dgrow(c->crc_table, sizeof(g_crc_tab) + sizeof(g_crc_z496)));
    if (int rc = ensure_ring(c, 16u << 20, W, err)) return rc;
    if (!c->copy_stream) CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    t_mark[1] = now_ms();
    uint8_t* P = (uint8_t*)c->pipe.p;
    const uint32_t Wn = (uint32_t)waves.size();
    const uint32_t n = (uint32_t)items.size();
    WaveState st0{0, 0, 1, 0};
    CK(cudaMemcpyAsync(P, &st0, sizeof(st0), cudaMemcpyHostToDevice, c->stream));
    std::vector<WaveJob> wj(Wn);
    for (uint32_t w = 0; w < Wn; w++)
        wj[w] = WaveJob{waves[w].first, waves[w].n, n - 1, waves[w].piece_off, waves[w].piece_cap, waves[w].n,
                        tgt.cap, 0};
    CK(cudaMemcpyAsync(P + o_wj, wj.data(), Wn * sizeof(WaveJob), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(P + o_tabs, tabs.data(), tabs.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->items.p, items.data(), (size_t)n * sizeof(ChunkItem), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->order.p, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->queue.p, 0, (size_t)W * 16, c->stream));
    CK(cudaMemsetAsync(c->mbcount.p, 0, 16, c->stream));
    CK(cudaMemsetAsync(c->rerr.p, 0, 16, c->stream));
    CK(cudaMemsetAsync(c->markers.p, 0, 8, c->stream));
    // the final member check: one member over every wave's piece region
    const uint32_t mps[2] = {0, total_pieces};
    CK(cudaMemcpyAsync(P + o_fin + 48, mps, 8, cudaMemcpyHostToDevice, c->stream));
    t_mark[2] = now_ms();
    // every stream starts after the input, the scan and these uploads
    cudaEvent_t ev0 = nullptr;
    std::vector<cudaEvent_t> evs;  // destroyed on every return
    struct EvGuard {
        std::vector<cudaEvent_t>& v;
        ~EvGuard() {
            for (cudaEvent_t e : v) cudaEventDestroy(e);
        }
    } guard{evs};
    auto mkev = [&](cudaEvent_t* e, bool timing) -> cudaError_t {
        cudaError_t r = timing ? cudaEventCreate(e) : cudaEventCreateWithFlags(e, cudaEventDisableTiming);
        if (r == cudaSuccess) evs.push_back(*e);
        return r;
    };
    CK(mkev(&ev0, true));
    CK(cudaEventRecord(ev0, c->stream));
    CK(cudaStreamWaitEvent(c->copy_stream, ev0, 0));
    // ---- per wave: inflate | chain check, resolve, CRC pieces
    const uint32_t IW = c->inflate_warps;
    const size_t ismem = IW * sizeof(WarpSmem);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint16_t>, IW * 32, ismem);
    std::vector<cudaEvent_t> e_chain(W), e_res(W), e_inf(W);
    WaveInfo* h_info = (WaveInfo*)c->h_wave;
    uint32_t* h_err = (uint32_t*)(c->h_wave + W * sizeof(WaveInfo));  // resolve error word per wave
    uint32_t* h_fin = h_err + W + 1;                                    // status, got_crc, got_len lo/hi
    auto enqueue_inflate = [&](uint32_t w) -> int {
        const PipeWave& pw = waves[w];
        InflateArgs A{};
        A.in = d_file;
        A.items = (const ChunkItem*)c->items.p;
        A.results = (ChunkResult*)c->results.p;
        A.n_items = pw.n;
        A.order = (const uint32_t*)c->order.p + pw.first;
        A.queue = (uint32_t*)c->queue.p + 4 * w;
        A.out = c->cells.p;
        A.mbs = (MemberRec*)c->mbs.p;
        A.mb_count = (uint32_t*)c->mbcount.p;
        A.mb_cap = 4096;
        RRG_LAUNCH(k_inflate<uint16_t>, persistent_blocks(c, std::max(1, occ), pw.n, IW), IW * 32, ismem, c->stream,
                   A);
        LAUNCHED(c);
        CK(mkev(&e_inf[w], true));
        CK(cudaEventRecord(e_inf[w], c->stream));
        return 0;
    };
    auto enqueue_rest = [&](uint32_t w) -> int {
        const PipeWave& pw = waves[w];
        cudaStream_t rs = c->stream;
        WaveArgs WA{};
        WA.items = (const ChunkItem*)c->items.p;
        WA.results = (const ChunkResult*)c->results.p;
        WA.jobs = (const WaveJob*)(P + o_wj) + w;
        WA.n_jobs = 1;
        WA.item_base = pw.first;
        WA.n_items = pw.n;
        WA.state = (WaveState*)P;
        WA.info = h_info + w;  // mapped pinned memory: no copy queued behind the output
        WA.live = (uint32_t*)(P + o_live);
        WA.chunks = (ResolveChunk*)(P + o_chunks);
        WA.head_segs = (uint64_t*)(P + o_hs);
        WA.pieces = (CrcPiece*)(P + o_pc);
        WA.n_pieces = (uint32_t*)(P + o_np) + w;
        WA.seg_total = (uint64_t*)(P + o_seg);
        WA.mbs = (const MemberRec*)c->mbs.p;
        WA.mb_count = (const uint32_t*)c->mbcount.p;
        WA.mb_cap = 4096;
        WA.exp_crc = (uint32_t*)(P + o_fin);
        WA.exp_isize = (uint32_t*)(P + o_fin) + 1;
        RRG_LAUNCH(k_wave_chain, 1, WAVE_THREADS, 0, rs, WA);
        LAUNCHED(c);
        CK(mkev(&e_chain[w], true));
        CK(cudaEventRecord(e_chain[w], rs));
        ResolveArgs RA{};
        RA.cells = (uint16_t*)c->cells.p;
        RA.chunks = WA.chunks;
        RA.head_segs = WA.head_segs;
        res_args(RA, pw.tab, P + o_tabs + pw.tab_off, (uint16_t*)c->win.p, pw.n);
        RA.out = tgt.p;
        RA.err = (uint32_t*)c->rerr.p;
        RA.markers = (unsigned long long*)c->markers.p;
        RA.live = WA.live;
        if (int rc = launch_resolve(c, RA, rs, err)) return rc;
        CrcWideArgs CA{tgt.p, WA.pieces + pw.piece_off, pw.piece_cap, (uint32_t*)(P + o_pcrc) + pw.piece_off,
                       (const uint32_t*)c->crc_table.p, WA.n_pieces};
        RRG_LAUNCH(k_crc_pieces_wide, persistent_blocks(c, 8, pw.piece_cap, 1), CRCW_THREADS, 0, rs, CA);
        LAUNCHED(c);
        RRG_LAUNCH(k_copy_words, 1, 32, 0, rs, (const uint32_t*)c->rerr.p, h_err + w, 1u);
        LAUNCHED(c);
        CK(mkev(&e_res[w], true));
        CK(cudaEventRecord(e_res[w], rs));
        return 0;
    };
    for (uint32_t w = 0; w < (uint32_t)waves.size(); w++) {
        if (int rc = enqueue_inflate(w)) return rc;
        if (int rc = enqueue_rest(w)) return rc;
    }
    t_mark[3] = now_ms();
    if (c->cfg.verbose >= 2)
        std::fprintf(stderr, "[rrg-gpu] host: scan results %.3f ms, plan %.3f, memory %.3f, uploads %.3f, "
                     "waves enqueued %.3f ms after the call\n", t_scanned - t_enter, t_mark[0] - t_enter,
                     t_mark[1] - t_enter, t_mark[2] - t_enter, t_mark[3] - t_enter);
    // the member's CRC32/ISIZE over all pieces (meaningful when every wave passed)
    {
        uint32_t* fin = (uint32_t*)(P + o_fin);
        CrcMemberArgs B{(const CrcPiece*)(P + o_pc), (const uint32_t*)(P + o_pcrc), fin + 12, 1, fin, fin + 1,
                        fin + 2, (uint64_t*)(fin + 4), (int32_t*)(fin + 6)};
        RRG_LAUNCH(k_crc_members, 1, 32, 0, c->stream, B);
        LAUNCHED(c);
        RRG_LAUNCH(k_copy_words, 1, 32, 0, c->stream, (const uint32_t*)fin, h_fin, 8u);
        LAUNCHED(c);
    }
    cudaEvent_t e_fin = nullptr;
    CK(mkev(&e_fin, true));
    CK(cudaEventRecord(e_fin, c->stream));
    auto drain = [&]() {
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->copy_stream);
    };
    // ---- deliver: pieces of each wave's output through a ring of pinned buffers
    constexpr uint32_t RING = 4;
    const uint64_t PS = c->h_ring_cap;
    cudaEvent_t ring_ev[RING];
    for (auto& e : ring_ev) CK(mkev(&e, false));
    struct Piece {
        uint64_t off, len;
        uint32_t wave;
    };
    std::vector<Piece> pcs;
    uint64_t total = 0;
    uint32_t known = 0;  // waves whose pieces are listed
    size_t issued = 0, delivered = 0;
    int failed_wave = -1;
    const double t_start = now_ms();
    uint8_t* slot_dst[RING];  // per ring slot: the consumer's buffer or the library's piece buffer
    auto issue = [&](size_t i) -> cudaError_t {
        const Piece& pc = pcs[i];
        slot_dst[i % RING] = c->h_ring + (i % RING) * PS;
        if (c->get_buf) {
            size_t cap = 0;
            uint8_t* b = c->get_buf(c->get_user, (size_t)pc.len, &cap);
            if (b && cap >= pc.len) slot_dst[i % RING] = b;
        }
        cudaError_t e = cudaStreamWaitEvent(c->copy_stream, e_res[pc.wave], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(slot_dst[i % RING], tgt.p + pc.off, pc.len, cudaMemcpyDeviceToHost,
                                c->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(ring_ev[i % RING], c->copy_stream);
        return e;
    };
    for (;;) {
        // learn the next wave's outcome when its pieces are needed
        if (issued == pcs.size() && known < Wn && failed_wave < 0) {
            CK(cudaEventSynchronize(e_chain[known]));
            const WaveInfo wi = h_info[known];
            if (c->cfg.verbose >= 3)
                std::fprintf(stderr, "[rrg-gpu] wave %u of %u: ok %u, output [%llu, +%llu), trailer %llu, items %u\n",
                             known, Wn, wi.ok, (unsigned long long)wi.out_begin, (unsigned long long)wi.out_len,
                             (unsigned long long)wi.trailer_byte, waves[known].n);
            if (!wi.ok) {
                failed_wave = (int)known;
            } else {
                for (uint64_t o = 0; o < wi.out_len; o += PS)
                    pcs.push_back(Piece{wi.out_begin + o, std::min(PS, wi.out_len - o), known});
                total = wi.out_begin + wi.out_len;
                known++;
            }
            continue;
        }
        while (issued < pcs.size() && issued < delivered + RING) CK(issue(issued++));
        if (delivered == issued) break;  // nothing in flight: all waves done, or stopped at a failed wave
        const Piece& pc = pcs[delivered];
        CK(cudaEventSynchronize(ring_ev[delivered % RING]));
        if (h_err[pc.wave]) {
            drain();
            set_err(err, RRG_ERR_DEFLATE_INVALID, "%s", msg_text(MSG_MARKER_WINDOW));
            return RRG_ERR_DEFLATE_INVALID;
        }
        const bool very_last = failed_wave < 0 && known == Wn && delivered + 1 == pcs.size();
        if (very_last) {  // the member's trailer is checked before its last piece goes out
            CK(cudaEventSynchronize(e_fin));
            if (h_fin[6] == DS_CRC || h_fin[6] == DS_ISIZE) {
                drain();
                const WaveInfo& li = h_info[Wn - 1];
                const MemberSpan ms{0, total, h_fin[0], h_fin[1], hl + li.trailer_byte};
                return member_error(err, ms, 0, (int32_t)h_fin[6], h_fin[2],
                                    (uint64_t)h_fin[4] | ((uint64_t)h_fin[5] << 32));
            }
        }
        c->st.chunks_decoded++;
        if (sink && sink(user, slot_dst[delivered % RING], (size_t)pc.len)) {
            *closed = true;
            drain();
            *total_out = total;
            return 0;
        }
        delivered++;
    }
    drain();
    {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ev0, e_inf[Wn - 1]) == cudaSuccess) c->st.inflate_ms += ms;
        if (c->cfg.verbose >= 2) {  // the device timeline of every wave, from the end of the scan
            for (uint32_t w = 0; w < Wn && (failed_wave < 0 || (int)w <= failed_wave); w++) {
                float a = 0, b = 0, r = 0;
                cudaEventElapsedTime(&a, ev0, e_inf[w]);
                cudaEventElapsedTime(&b, ev0, e_chain[w]);
                cudaEventElapsedTime(&r, ev0, e_res[w]);
                std::fprintf(stderr, "[rrg-gpu] wave %u: %u sub-chunks, inflate done %.3f ms, chain %.3f ms, "
                             "resolve+crc done %.3f ms\n", w, waves[w].n, a, b, r);
            }
            float f = 0;
            cudaEventElapsedTime(&f, ev0, e_fin);
            std::fprintf(stderr, "[rrg-gpu] member check %.3f ms; delivery loop %.3f ms on the host\n", f,
                         now_ms() - t_start);
        }
    }
    c->st.gpu_chunks += n;
    c->st.d2h_ms += now_ms() - t_start;
    unsigned long long nmk = 0;
    CK(cudaMemcpy(&nmk, c->markers.p, 8, cudaMemcpyDeviceToHost));
    c->st.markers += nmk;
    if (failed_wave < 0) {
        c->st.members += 1;
        *total_out = total;
        return 0;
    }
    // ---- the rest on the checked path, from the last verified bit
    c->st.pipeline_fallbacks = 1;
    WaveState S{};
    CK(cudaMemcpy(&S, P, sizeof(S), cudaMemcpyDeviceToHost));
    if (c->cfg.verbose >= 2)
        std::fprintf(stderr, "[rrg-gpu] pipeline stopped at wave %d (sub-chunk %d, status %d): checked path from bit %llu\n",
                     failed_wave, h_info[failed_wave].fail_item, h_info[failed_wave].fail_status,
                     (unsigned long long)S.expected);
    std::vector<MemberJob> jobs(1);
    MemberJob& j = jobs[0];
    j.len = len;
    j.body_off = hl;
    j.start_bit = S.expected;
    j.dst_off = S.out_end;
    j.prefix_len = std::min<uint64_t>(WINDOW, S.out_end);
    if (S.out_end) {
        std::vector<int32_t> stv;
        std::vector<uint32_t> got;
        std::vector<uint64_t> glen;
        const uint64_t members = c->st.members;  // the prefix's CRC32 checks no member
        if (int rc = crc_spans(c, tgt.p, {MemberSpan{0, S.out_end, 0, 0, 0}}, stv, got, glen, err)) return rc;
        c->st.members = members;
        j.crc_prev = got[0];
        j.len_prev = glen[0];
    }
    tgt.cap = c->out.cap;
    if (int rc = members_route(c, d_file, jobs, tgt, err)) return rc;
    if (j.rc) {
        if (err) *err = j.err;
        return j.rc;
    }
    *total_out = S.out_end + j.out.total;
    return deliver(c, tgt.p + S.out_end, j.out.total, sink, user, closed, err);
}

}  // namespace

namespace {

int decode_host_impl(rrg_ctx* c, const uint8_t* data, size_t len, rrg_sink_fn sink, void* user, rrg_stats* stats,
                     rrg_error* err) {
    double t_all = now_ms();
    c->st = rrg_stats{};
    c->launches = 0;
    c->st.compressed_bytes = len;
    if (len == 0) {
        set_err(err, RRG_ERR_TRUNCATED, "truncated gzip stream");
        if (stats) *stats = c->st;
        return RRG_ERR_TRUNCATED;
    }
    double t0 = now_ms();
    CK(dgrow(c->comp, len + 16));
#ifdef RRG_EMU
    const size_t pipe_min = 256u << 10;  // the CPU emulation exercises the piecewise path on small inputs
#else
    const size_t pipe_min = 16u << 20;
#endif
    if (len >= pipe_min && host_bgzf_size(data, len) < 0) {
        // a member stream: copy in 8 pieces on the copy stream; the boundary
        // scan starts on each piece as it lands (and everything else waits
        // for the last one)
        if (!c->copy_stream) CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        const uint64_t P = (len + 7) / 8;
        c->arr_pieces.clear();
        for (int i = 0; i < 8; i++) {
            const uint64_t o = (uint64_t)i * P;
            if (o >= len) break;
            const uint64_t l = std::min<uint64_t>(P, len - o);
            if (!c->arr_events[i]) CK(cudaEventCreateWithFlags(&c->arr_events[i], cudaEventDisableTiming));
            CK(cudaMemcpyAsync((uint8_t*)c->comp.p + o, data + o, l, cudaMemcpyHostToDevice, c->copy_stream));
            CK(cudaEventRecord(c->arr_events[i], c->copy_stream));
            c->arr_pieces.push_back({o + l, c->arr_events[i]});
        }
        c->arr_base = (const uint8_t*)c->comp.p;
    } else {
        CK(cudaMemcpyAsync(c->comp.p, data, len, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    c->st.h2d_ms = now_ms() - t0;
    int rc = upload_tables(c, err);
    bool closed = false, taken = false;
    if (!rc && host_bgzf_size(data, len) < 0) {
        // a large member stream: decode in waves with the copy-out overlapped
        size_t hl = 0;
        int detail = 0;
        if (host_parse_header(data, len, &hl, &detail) == DS_OK) {
            uint64_t total = 0;
            rc = pipelined_host(c, (const uint8_t*)c->comp.p, len, data, hl, sink, user, &closed, &total, &taken,
                                err);
            if (taken) c->st.uncompressed_bytes = total;
        }
    }
    if (!rc && !taken) {
        // output size is only known after the chain; decode into the context buffer
        Decoded d;
        OutTarget tgt{(uint8_t*)c->out.p, c->out.cap, true};
        rc = decode_file(c, (const uint8_t*)c->comp.p, len, data, tgt, &d, err);
        if (!rc) {
            c->st.uncompressed_bytes = d.total;
            rc = deliver(c, tgt.p, d.total, sink, user, &closed, err);
        }
    }
    if (c->arr_base) {  // a path that launched nothing (an early error): drain the copies
        c->arr_base = nullptr;
        c->arr_pieces.clear();
        cudaStreamSynchronize(c->copy_stream);
    }
    c->st.kernel_launches = c->launches;
    c->st.total_ms = now_ms() - t_all;
    if (stats) *stats = c->st;
    if (c->cfg.verbose)
        std::fprintf(stderr,
                     "[rrg-gpu] %zu -> %llu bytes, %llu sub-chunks, %llu speculation failures, %llu markers, "
                     "finder %.3f ms, inflate %.3f ms, resolve %.3f ms, crc %.3f ms, total %.3f ms\n",
                     len, (unsigned long long)c->st.uncompressed_bytes, (unsigned long long)c->st.gpu_chunks,
                     (unsigned long long)c->st.speculation_failures, (unsigned long long)c->st.markers, c->st.finder_ms,
                     c->st.inflate_ms, c->st.resolve_ms, c->st.crc_ms, c->st.total_ms);
    return rc;
}

// ------------------------------------------------------------ non-seekable input
// A stream read forward in stripes (streaming.rs:389-614 keeps a sliding read
// buffer for the same reason). Each stripe is a job of the member route that
// starts at the exact bit where the previous one stopped and stops at the
// first block edge past its stop bit, leaving a lookahead of input unread so
// that the last sub-chunk can finish its block. Between stripes only the open
// member's last 32 KiB of output (for back-references), its running CRC32 and
// length, and the unread input survive, so memory stays a few stripes whatever
// the stream's length.
//
// Reading overlaps decoding: a reader thread fills one of two pinned buffers
// with the next stripe's bytes while the device decodes the current stripe.
// A stripe is assembled on the device: the previous stripe's unread bytes
// (moved there device to device) followed by the newly read ones.

// One background read at a time into a caller's buffer.
struct StreamReader {
    rrg_read_fn rd;
    void* user;
    std::mutex m;
    std::condition_variable cv;
    std::thread th;
    uint8_t* buf = nullptr;
    uint64_t want = 0, got = 0;
    bool busy = false, quit = false, eof = false, failed = false;
    StreamReader(rrg_read_fn r, void* u) : rd(r), user(u) {
        th = std::thread([this] {
            std::unique_lock<std::mutex> lk(m);
            for (;;) {
                cv.wait(lk, [this] { return busy || quit; });
                if (quit) return;
                uint8_t* b = buf;
                const uint64_t w = want;
                lk.unlock();
                uint64_t n = 0;
                bool e = false, f = false;
                while (n < w) {
                    const int64_t r = rd(user, b + n, (size_t)(w - n));
                    if (r < 0) {
                        f = true;
                        break;
                    }
                    if (r == 0) {
                        e = true;
                        break;
                    }
                    n += (uint64_t)r;
                }
                lk.lock();
                got = n;
                eof = eof || e;
                failed = failed || f;
                busy = false;
                cv.notify_all();
            }
        });
    }
    ~StreamReader() {
        {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [this] { return !busy; });
            quit = true;
        }
        cv.notify_all();
        th.join();
    }
    void start(uint8_t* b, uint64_t w) {  // no read may be in flight
        std::lock_guard<std::mutex> lk(m);
        buf = b;
        want = w;
        got = 0;
        busy = !eof && w > 0;
        cv.notify_all();
    }
    uint64_t wait(bool* at_eof, bool* fail) {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [this] { return !busy; });
        *at_eof = eof;
        *fail = failed;
        const uint64_t n = got;
        got = 0;
        return n;
    }
};

int stream_impl(rrg_ctx* c, rrg_read_fn rd, void* ruser, rrg_sink_fn sink, void* suser, uint64_t stripe_bytes,
                rrg_stats* stats, rrg_error* err) {
    double t_all = now_ms();
    c->st = rrg_stats{};
    c->launches = 0;
    int rc = upload_tables(c, err);
    if (rc) return rc;
    const uint64_t S = stripe_bytes ? std::max<uint64_t>(stripe_bytes, 1 << 16) : (256ull << 20);
    uint64_t L = std::max<uint64_t>(1ull << 16, S / 8);  // lookahead; doubled when a block outruns it
    constexpr uint64_t PRE = 32768;  // the prefix region in front of every stripe's output
    // two pinned read buffers of S + L bytes each (c->h_in)
    const uint64_t PB = S + L;
    if (c->h_in_cap < 2 * PB) {
        if (c->h_in) cudaFreeHost(c->h_in);
        c->h_in = nullptr;
        c->h_in_cap = 0;
        CK(cudaMallocHost((void**)&c->h_in, (size_t)(2 * PB)));
        c->h_in_cap = (size_t)(2 * PB);
    }
    uint8_t* pb[2] = {c->h_in, c->h_in + PB};
    // the stripe on the device: comp[0..have); comp2 takes the unread tail
    uint64_t dcap = 2 * PB + 16;
    CK(dgrow(c->comp, dcap));
    CK(dgrow(c->comp2, dcap));
    CK(dgrow(c->pfx, PRE));
    OutTarget tgt{(uint8_t*)c->out.p, c->out.cap, true};
    rc = ensure_out(c, tgt, PRE + 4096, 0, err);
    if (rc) return rc;
    StreamReader reader(rd, ruser);
    int cur = 0;
    reader.start(pb[cur], PB);
    uint64_t have = 0, in_base = 0;  // comp[0..have) = stream bytes [in_base, in_base + have)
    bool eof = false;
    // append the read in flight (buffer pb[cur]) to the device stripe and start
    // the next read into the other buffer
    auto take = [&](uint64_t next_want) -> int {
        bool fail = false;
        const uint64_t n = reader.wait(&eof, &fail);
        if (fail) {
            set_err(err, RRG_ERR_IO, "io: stream read failed");
            return RRG_ERR_IO;
        }
        if (have + n + 16 > dcap) {  // a stripe grown by retries: keep its bytes
            const uint64_t ncap = 2 * (have + n) + 16;
            CK(dgrow(c->comp2, ncap));
            if (have) CK(cudaMemcpyAsync(c->comp2.p, c->comp.p, have, cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            std::swap(c->comp, c->comp2);
            CK(dgrow(c->comp2, ncap));
            dcap = ncap;
        }
        if (n) CK(cudaMemcpyAsync((uint8_t*)c->comp.p + have, pb[cur], n, cudaMemcpyHostToDevice, c->stream));
        have += n;
        CK(cudaStreamSynchronize(c->stream));  // pb[cur] may be refilled from here on
        cur ^= 1;
        if (!eof) reader.start(pb[cur], std::min(next_want, PB));
        return 0;
    };
    if ((rc = take(S))) return rc;
    bool in_member = false, any = false;
    uint64_t start_bit = 0, len_prev = 0, prefix_len = 0;
    uint32_t crc_prev = 0, members = 0;
    uint64_t total_out = 0;
    std::vector<uint8_t> head;
    for (;;) {
        uint64_t body_off = 0;
        if (!in_member) {
            if (have == 0 && eof) break;  // end of the stream between members
            head.resize((size_t)std::min<uint64_t>(have, 1 << 16));
            if (!head.empty()) {
                CK(cudaMemcpyAsync(head.data(), c->comp.p, head.size(), cudaMemcpyDeviceToHost, c->stream));
                CK(cudaStreamSynchronize(c->stream));
            }
            size_t hl = 0;
            int detail = 0;
            int st = host_parse_header(head.data(), head.size(), &hl, &detail);
            if (st) {
                if (st == DS_TRUNCATED && !eof) {
                    if ((rc = take(S))) return rc;
                    continue;
                }
                return status_err(err, st, detail, in_base);
            }
            body_off = hl;
            start_bit = 0;
            crc_prev = 0;
            len_prev = 0;
            prefix_len = 0;
            in_member = true;
        }
        // the stop bit: a lookahead's worth before the end of what has been read
        uint64_t stop = ~0ull;
        if (!eof) {
            const uint64_t lim = have > L ? have - L : 0;
            if (lim * 8 <= body_off * 8 + start_bit + 8) {  // too little read for a stripe
                if ((rc = take(S))) return rc;
                continue;
            }
            stop = lim * 8 - body_off * 8;
        }
        if (prefix_len)
            CK(cudaMemcpyAsync(tgt.p + PRE - prefix_len, (const uint8_t*)c->pfx.p + PRE - prefix_len, prefix_len,
                               cudaMemcpyDeviceToDevice, c->stream));
        std::vector<MemberJob> jobs(1);
        MemberJob& j = jobs[0];
        j.len = have;
        j.body_off = body_off;
        j.dst_off = PRE;
        j.member_base = members;
        j.start_bit = start_bit;
        j.stop_bit = stop;
        j.report_off = in_base;
        j.prefix_len = prefix_len;
        j.crc_prev = crc_prev;
        j.len_prev = len_prev;
        c->st.compressed_bytes = in_base + have;
        rc = members_route(c, (const uint8_t*)c->comp.p, jobs, tgt, err);
        if (rc) return rc;
        if (j.rc) {
            // a block that runs past the read input: read more and redo the stripe
            if (!eof && (j.rc == RRG_ERR_DEFLATE_EOF || j.rc == RRG_ERR_TRUNCATED)) {
                L *= 2;
                if ((rc = take(S))) return rc;
                continue;
            }
            if (err) *err = j.err;
            return j.rc;
        }
        any = true;
        if (c->cfg.verbose >= 2)
            std::fprintf(stderr, "[rrg-gpu] stripe at stream byte %llu: %llu bytes read, start bit %llu, stop bit %llu, "
                         "%llu bytes out, %s\n", (unsigned long long)in_base, (unsigned long long)have,
                         (unsigned long long)start_bit, (unsigned long long)stop, (unsigned long long)j.out.total,
                         j.open_member ? "member open" : "members closed");
        bool closed = false;
        rc = deliver(c, tgt.p + PRE, j.out.total, sink, suser, &closed, err);
        if (rc) return rc;
        total_out += j.out.total;
        members += j.out.members;
        if (closed) break;  // the sink stopped taking bytes (pipeline.rs:1028-1030)
        uint64_t used;
        if (j.open_member) {
            const uint64_t end_bit = body_off * 8 + j.end_bit;
            used = end_bit / 8;
            start_bit = end_bit % 8;
            crc_prev = j.open_crc;
            len_prev = j.open_len;
            // the open member's last bytes: this stripe's output from its start,
            // after the previous prefix when the member continues it
            const uint64_t p = std::min<uint64_t>(PRE, len_prev);
            if (p)
                CK(cudaMemcpyAsync((uint8_t*)c->pfx.p + PRE - p, tgt.p + PRE + j.out.total - p, p,
                                   cudaMemcpyDeviceToDevice, c->stream));
            prefix_len = p;
        } else {
            used = j.out.consumed;  // the members ended inside the read input
            in_member = false;
        }
        // the unread bytes move to the front of the other device buffer
        if (have > used)
            CK(cudaMemcpyAsync(c->comp2.p, (const uint8_t*)c->comp.p + used, have - used, cudaMemcpyDeviceToDevice,
                               c->stream));
        std::swap(c->comp, c->comp2);
        have -= used;
        in_base += used;
        if (!eof) {  // a read is in flight until the stream ends
            if ((rc = take(used ? used : S))) return rc;
        }
        if (!in_member && have == 0 && eof) break;
    }
    CK(cudaStreamSynchronize(c->stream));
    if (!any) {
        set_err(err, RRG_ERR_TRUNCATED, "truncated gzip stream");
        if (stats) *stats = c->st;
        return RRG_ERR_TRUNCATED;
    }
    c->st.compressed_bytes = in_base + have;
    c->st.uncompressed_bytes = total_out;
    c->st.members = members;
    c->st.kernel_launches = c->launches;
    c->st.total_ms = now_ms() - t_all;
    if (stats) *stats = c->st;
    return 0;
}

// ------------------------------------------------------------ seek index
// Random access into a member stream (the reference has none: README.md:45).
// A full, CRC-checked decode records the sub-chunk starts the anchored chain
// kept: each is a block start with its exact bit and output offset. Kept at
// least `spacing` output bytes apart, each checkpoint stores the 32 KiB of
// output before it. A range read is then a stripe job (the same machinery as
// the stream route) from the checkpoint at or before the range, with that
// window as its prefix, to the first checkpoint at or past the range's end.
}  // namespace

struct rrg_index {
    uint64_t file_len = 0, body_off = 0, total_out = 0;
    std::vector<uint64_t> in_bit;    // relative to body_off
    std::vector<uint64_t> out_off;   // output offset of the checkpoint
    std::vector<uint32_t> win_len;   // bytes of window before it (<= 32768)
    std::vector<uint8_t> win;        // 32768 bytes per checkpoint, right-aligned
};

namespace {
int index_build_impl(rrg_ctx* c, const uint8_t* data, size_t len, uint64_t spacing, rrg_index** out,
                     rrg_stats* stats, rrg_error* err) {
    double t_all = now_ms();
    c->st = rrg_stats{};
    c->launches = 0;
    c->st.compressed_bytes = len;
    int rc = upload_tables(c, err);
    if (rc) return rc;
    size_t hl = 0;
    int detail = 0;
    int st = host_parse_header(data, len, &hl, &detail);
    if (st) return status_err(err, st, detail, 0);
    if (host_bgzf_size(data, len) >= 0) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "BGZF: every member already starts a seekable block");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    CK(dgrow(c->comp, len + 16));
    CK(cudaMemcpyAsync(c->comp.p, data, len, cudaMemcpyHostToDevice, c->stream));
    std::vector<std::pair<uint64_t, uint64_t>> cps;
    std::vector<MemberJob> jobs(1);
    jobs[0].len = len;
    jobs[0].body_off = hl;
    jobs[0].capture = &cps;
    OutTarget tgt{(uint8_t*)c->out.p, c->out.cap, true};
    rc = members_route(c, (const uint8_t*)c->comp.p, jobs, tgt, err);
    if (rc) return rc;
    if (jobs[0].rc) {
        if (err) *err = jobs[0].err;
        return jobs[0].rc;
    }
    auto* idx = new rrg_index;
    idx->file_len = len;
    idx->body_off = hl;
    idx->total_out = jobs[0].out.total;
    constexpr uint64_t W = 32768;
    for (const auto& cp : cps) {
        if (!idx->out_off.empty() && cp.second < idx->out_off.back() + spacing) continue;
        idx->in_bit.push_back(cp.first);
        idx->out_off.push_back(cp.second);
        idx->win_len.push_back((uint32_t)std::min(W, cp.second));
    }
    idx->win.assign(idx->out_off.size() * W, 0);
    for (size_t k = 0; k < idx->out_off.size(); k++) {
        const uint64_t wl = idx->win_len[k];
        if (wl) {
            cudaError_t e = cudaMemcpyAsync(idx->win.data() + k * W + (W - wl), tgt.p + idx->out_off[k] - wl, wl,
                                            cudaMemcpyDeviceToHost, c->stream);
            if (e != cudaSuccess) {
                delete idx;
                return cuda_fail(err, e, "index windows");
            }
        }
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        delete idx;
        return cuda_fail(err, e, "index windows");
    }
    c->st.uncompressed_bytes = idx->total_out;
    c->st.kernel_launches = c->launches;
    c->st.total_ms = now_ms() - t_all;
    if (stats) *stats = c->st;
    *out = idx;
    return 0;
}

int read_range_impl(rrg_ctx* c, const uint8_t* data, size_t len, const rrg_index* idx, uint64_t off, uint64_t n,
                    uint8_t* dst, rrg_error* err) {
    if (len != idx->file_len || off > idx->total_out || n > idx->total_out - off || idx->out_off.empty()) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "range or file does not match the index");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (!n) return 0;
    int rc = upload_tables(c, err);
    if (rc) return rc;
    // checkpoints around [off, off + n)
    const auto& oo = idx->out_off;
    const size_t lo = (size_t)(std::upper_bound(oo.begin(), oo.end(), off) - oo.begin()) - 1;
    const size_t hi = (size_t)(std::lower_bound(oo.begin(), oo.end(), off + n) - oo.begin());
    const uint64_t bit0 = idx->body_off * 8 + idx->in_bit[lo];
    const uint64_t byte0 = bit0 / 8;
    // input from the first checkpoint's byte to the last one's, plus room for
    // the bit reader's read-ahead (or to the end of the file)
    const uint64_t end_byte =
        hi < oo.size() ? std::min<uint64_t>(len, (idx->body_off * 8 + idx->in_bit[hi]) / 8 + (64u << 10)) : len;
    if (byte0 >= len || end_byte <= byte0 || (hi < oo.size() && idx->in_bit[hi] <= idx->in_bit[lo])) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "seek index checkpoints lie outside the file");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    const uint64_t clen = end_byte - byte0;
    CK(dgrow(c->comp, clen + 16));
    CK(cudaMemcpyAsync(c->comp.p, data + byte0, clen, cudaMemcpyHostToDevice, c->stream));
    constexpr uint64_t W = 32768;
    const uint64_t wl = idx->win_len[lo];
    OutTarget tgt{(uint8_t*)c->out.p, c->out.cap, true};
    rc = ensure_out(c, tgt, W + 4096, 0, err);
    if (rc) return rc;
    if (wl)
        CK(cudaMemcpyAsync(tgt.p + W - wl, idx->win.data() + lo * W + (W - wl), wl, cudaMemcpyHostToDevice,
                           c->stream));
    std::vector<MemberJob> jobs(1);
    MemberJob& j = jobs[0];
    j.len = clen;
    j.body_off = 0;
    j.start_bit = bit0 - byte0 * 8;
    j.stop_bit = hi < oo.size() ? idx->body_off * 8 + idx->in_bit[hi] - byte0 * 8 : ~0ull;
    j.dst_off = W;
    j.prefix_len = wl;
    j.len_prev = wl;  // decoding continues a member (its CRC is not checked)
    j.check_crc = false;
    j.report_off = byte0;
    rc = members_route(c, (const uint8_t*)c->comp.p, jobs, tgt, err);
    if (rc) return rc;
    if (j.rc) {
        if (err) *err = j.err;
        return j.rc;
    }
    const uint64_t skip = off - oo[lo];
    if (skip + n > j.out.total) {
        set_err(err, RRG_ERR_DEFLATE_INVALID, "seek point decode ended early");
        return RRG_ERR_DEFLATE_INVALID;
    }
    CK(cudaMemcpyAsync(dst, tgt.p + W + skip, n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// ------------------------------------------------------------ batches
// Independent gzip files (or members) already on the device, each with its
// own output range. Headers are parsed on the device; BGZF files take the
// BGZF route one by one; every other file is a job of the member route, in
// waves whose reserved output cells fit the device budget.
// ------------------------------------------------------------ device-planned member batch
// The member route of a batch with every stage hand-off on the device (sub-
// chunk starts from the scan's verified starts, the item list, the anchored
// chain, resolve and CRC), so the decode after the header sniff is one
// sequence of launches with no host round trip, captured once as a CUDA graph
// and replayed while the batch's shape (sizes and buffers) stays the same. The
// plan's contents (jobs, orders, tables) are uploaded before each launch, so a
// new batch of the same shape replays the same graph. Jobs the device could not
// take through (a false start, a full slot, a CRC piece region too small) come
// back unfinished and go through the checked member route.
struct BatchLaunch {
    bool direct = false;           // no job split: every file decodes straight to its bytes
    uint32_t nj = 0, n_items = 0, n_big = 0, total_pieces = 0, mb_cap = 0;
    const uint8_t* scan_body = nullptr;
    uint64_t scan_len = 0, n_tiles = 0;
    uint32_t cap = 0, cap2 = 0, cap3 = 0, n_list = 0, sgrid = 0, igrid = 0;
    uint32_t walk_kb = 1;          // k_batch_walk: blocks per big job (4 ideals each)
    ResTables tab;
    // c->bplan layout: uploaded | device-written
    size_t o_jobs = 0, o_bigbit = 0, o_bigjob = 0, o_order = 0, o_mp = 0, o_tabs = 0, o_state = 0, o_wj = 0,
           up_end = 0;
    size_t o_info = 0, o_ecrc = 0, o_eisz = 0, o_gcrc = 0, o_glen = 0, o_mst = 0, down_end = 0;
    size_t o_np = 0, o_seg = 0, o_chunks = 0, o_hs = 0, o_pc = 0, o_pcrc = 0, o_keys = 0, total = 0;
};

int batch_enqueue(rrg_ctx* c, const uint8_t* d_in, uint8_t* d_out, const BatchLaunch& L, cudaEvent_t* marks,
                  rrg_error* err) {
    uint8_t* P = (uint8_t*)c->bplan.p;
    cudaStream_t s = c->stream;
    // under stream capture the records are external, so they become
    // event-record nodes of the graph (a plain record would only order the
    // captured work); outside a capture they are plain records
    cudaStreamCaptureStatus cap_st = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &cap_st));
    const bool capturing = cap_st == cudaStreamCaptureStatusActive;
    auto mark = [&](int i) -> int {
        if (!marks) return 0;
        if (capturing) CK(cudaEventRecordWithFlags(marks[i], s, cudaEventRecordExternal));
        else CK(cudaEventRecord(marks[i], s));
        return 0;
    };
    if (int r = mark(0)) return r;
    CK(cudaMemsetAsync(c->queue.p, 0, 16, s));
    CK(cudaMemsetAsync(c->mbcount.p, 0, 16, s));
    CK(cudaMemsetAsync(c->rerr.p, 0, 16, s));
    CK(cudaMemsetAsync(c->markers.p, 0, 8, s));
    if (!L.direct) {
        // ---- scan, verification, start selection and the item list
        CK(cudaMemsetAsync(c->ncand.p, 0, 64, s));
        CK(cudaMemsetAsync(P + L.o_keys, 0xff, (size_t)L.n_items * 8, s));
        uint64_t* cand = (uint64_t*)c->cand.p;
        uint64_t* surv = cand + L.cap;
        uint64_t* stored = surv + L.cap2;
        uint32_t* counts = (uint32_t*)c->ncand.p;
        ScanArgs S{L.scan_body, L.scan_len, cand, counts, L.cap, stored, counts + 3, L.cap3, 0, L.n_tiles,
                   L.n_list ? (const uint32_t*)c->tiles.p : nullptr, L.n_list};
        const uint32_t st = c->scan_threads;
        if (st == 64) RRG_LAUNCH(k_scan_candidates<64>, L.sgrid, 64, 0, s, S);
        else if (st == 128) RRG_LAUNCH(k_scan_candidates<128>, L.sgrid, 128, 0, s, S);
        else RRG_LAUNCH(k_scan_candidates<256>, L.sgrid, 256, 0, s, S);
        LAUNCHED(c);
        VerifyArgs V{L.scan_body, L.scan_len, cand, counts, L.cap, surv, counts + 1, L.cap2, nullptr, nullptr, counts + 4};
        VerifyArgs H{L.scan_body, L.scan_len, surv, counts + 1, L.cap2, nullptr, nullptr, 0, (uint8_t*)c->vflag.p,
                     counts + 2, nullptr};
        RRG_LAUNCH(k_verify_light, c->n_sm * 8, 256, 0, s, V);
        LAUNCHED(c);
        RRG_LAUNCH(k_verify_heavy, c->n_sm * 4, 4 * 32, 4 * sizeof(FindSmem), s, H);
        LAUNCHED(c);
        BatchArgs B{};
        B.jobs = (const BatchJob*)(P + L.o_jobs);
        B.n_jobs = L.nj;
        B.big_bit = (const uint64_t*)(P + L.o_bigbit);
        B.big_job = (const uint32_t*)(P + L.o_bigjob);
        B.n_big = L.n_big;
        B.surv = surv;
        B.vflag = (const uint8_t*)c->vflag.p;
        B.counts = counts;
        B.cap2 = L.cap2;
        B.cap3 = L.cap3;
        B.stored = stored;
        B.keys = (unsigned long long*)(P + L.o_keys);
        B.items = (ChunkItem*)c->items.p;
        B.wjobs = (WaveJob*)(P + L.o_wj);
        B.scan_body = L.scan_body;
        B.walk_kb = L.walk_kb;
        RRG_LAUNCH(k_batch_select, c->n_sm * 4, 256, 0, s, B);
        LAUNCHED(c);
        if (L.n_big) {  // ideal starts with no candidate in jobs of fixed-Huffman blocks
            RRG_LAUNCH(k_batch_walk, L.walk_kb * std::min<uint32_t>(L.n_big, 4096), FW_THREADS, 0, s, B);
            LAUNCHED(c);
        }
        RRG_LAUNCH(k_batch_items, std::min<uint32_t>(L.nj, c->n_sm * 2), WAVE_THREADS, 0, s, B);
        LAUNCHED(c);
    }
    if (int r = mark(1)) return r;
    // ---- inflate
    InflateArgs A{};
    A.in = d_in;
    A.items = (const ChunkItem*)c->items.p;
    A.results = (ChunkResult*)c->results.p;
    A.n_items = L.n_items;
    A.order = (const uint32_t*)(P + L.o_order);
    A.queue = (uint32_t*)c->queue.p;
    A.out = L.direct ? (void*)d_out : c->cells.p;
    A.mbs = (MemberRec*)c->mbs.p;
    A.mb_count = (uint32_t*)c->mbcount.p;
    A.mb_cap = L.mb_cap;
    const uint32_t IW = c->inflate_warps;
    if (L.direct) RRG_LAUNCH(k_inflate<uint8_t>, L.igrid, IW * 32, IW * sizeof(WarpSmem), s, A);
    else RRG_LAUNCH(k_inflate<uint16_t>, L.igrid, IW * 32, IW * sizeof(WarpSmem), s, A);
    LAUNCHED(c);
    if (int r = mark(2)) return r;
    // ---- anchored chains and layout, then resolve
    WaveArgs WA{};
    WA.items = (const ChunkItem*)c->items.p;
    WA.results = (const ChunkResult*)c->results.p;
    WA.jobs = (const WaveJob*)(P + L.o_wj);
    WA.n_jobs = L.nj;
    WA.item_base = 0;
    WA.n_items = L.n_items;
    WA.state = (WaveState*)(P + L.o_state);
    WA.info = (WaveInfo*)(P + L.o_info);
    WA.live = nullptr;
    WA.chunks = (ResolveChunk*)(P + L.o_chunks);
    WA.head_segs = (uint64_t*)(P + L.o_hs);
    WA.pieces = (CrcPiece*)(P + L.o_pc);
    WA.n_pieces = (uint32_t*)(P + L.o_np);
    WA.seg_total = (uint64_t*)(P + L.o_seg);
    WA.mbs = (const MemberRec*)c->mbs.p;
    WA.mb_count = (const uint32_t*)c->mbcount.p;
    WA.mb_cap = L.mb_cap;
    WA.exp_crc = (uint32_t*)(P + L.o_ecrc);
    WA.exp_isize = (uint32_t*)(P + L.o_eisz);
    WA.direct = L.direct ? 1u : 0u;
    RRG_LAUNCH(k_wave_chain, std::min<uint32_t>(L.nj, c->n_sm * 2), WAVE_THREADS, 0, s, WA);
    LAUNCHED(c);
    if (!L.direct) {
        if (L.nj > 1) {
            RRG_LAUNCH(k_wave_segs, 1, WAVE_THREADS, 0, s, WA);
            LAUNCHED(c);
            RRG_LAUNCH(k_wave_segs_add, std::min<uint32_t>(L.nj, c->n_sm * 4), 256, 0, s, WA);
            LAUNCHED(c);
        }
        ResolveArgs R{};
        R.cells = (uint16_t*)c->cells.p;
        R.chunks = WA.chunks;
        R.head_segs = WA.head_segs;
        res_args(R, L.tab, P + L.o_tabs, (uint16_t*)c->win.p, L.n_items);
        R.out = d_out;
        R.err = (uint32_t*)c->rerr.p;
        R.markers = (unsigned long long*)c->markers.p;
        if (int rc = launch_resolve(c, R, s, err)) return rc;
    }
    if (int r = mark(3)) return r;
    // ---- CRC32 and ISIZE of every member
    CrcWideArgs CA{d_out, (const CrcPiece*)(P + L.o_pc), L.total_pieces, (uint32_t*)(P + L.o_pcrc),
                   (const uint32_t*)c->crc_table.p, nullptr};
    RRG_LAUNCH(k_crc_pieces_wide, persistent_blocks(c, 8, L.total_pieces, 1), CRCW_THREADS, 0, s, CA);
    LAUNCHED(c);
    CrcMemberArgs CB{(const CrcPiece*)(P + L.o_pc), (const uint32_t*)(P + L.o_pcrc), (const uint32_t*)(P + L.o_mp),
                     L.nj, (const uint32_t*)(P + L.o_ecrc), (const uint32_t*)(P + L.o_eisz),
                     (uint32_t*)(P + L.o_gcrc), (uint64_t*)(P + L.o_glen), (int32_t*)(P + L.o_mst), nullptr};
    RRG_LAUNCH(k_crc_members, (L.nj * 32 + 255) / 256, 256, 0, s, CB);
    LAUNCHED(c);
    if (int r = mark(4)) return r;
    return 0;
}

// Decodes the jobs (whole single-member streams with fixed destinations) on the
// device-planned route. *taken is false when the route does not apply (the
// caller then uses members_route); jobs it could not finish are decoded by
// members_route here.
int batch_device(rrg_ctx* c, const uint8_t* d_in, std::vector<MemberJob>& jobs, OutTarget& tgt, bool* taken,
                 rrg_error* err) {
    *taken = false;
    const size_t nj = jobs.size();
    if (!nj || tgt.grow || !c->scan_bounds || c->lanes || c->cfg.batch_plan < 0 || nj > (1u << 24)) return 0;
    for (const MemberJob& j : jobs)
        if (j.start_bit || j.stop_bit != ~0ull || j.dst_cap == ~0ull || j.capture || j.split || !j.check_crc) return 0;
    if (int rc = upload_tables(c, err)) return rc;
    // ---- plan: sub-chunks per job. A sub-chunk's decode time grows with its
    // compressed bytes (symbols) and its output bytes (cells written), so with
    // automatic spacing every job gets sub-chunks in proportion to
    // C + U/3 (U from the trailer's ISIZE), spreading one wave of resident
    // decoders evenly over text, low-entropy and stored content alike; none is
    // smaller than 16 KiB of input. A fixed gpu_chunk_bytes spaces by input.
    const uint64_t slots = inflate_slots(c);
    auto cost_of = [&](const MemberJob& j) -> uint64_t {
        const uint64_t blen = j.len - j.body_off;
        const uint64_t u = j.isize_hint >= blen / 4 ? j.isize_hint : blen * 3;  // a wrapped or absent ISIZE
        return blen + u / 3;
    };
    uint64_t total_cost = 0;
    for (const MemberJob& j : jobs) total_cost += cost_of(j);
    const uint64_t G = c->gpu_chunk ? std::max<uint64_t>(c->gpu_chunk, 4096) : 0;
    const uint64_t Gc = std::max<uint64_t>(16ull << 10, (total_cost + slots - 1) / slots);
    BatchLaunch L;
    L.nj = (uint32_t)nj;
    std::vector<BatchJob> bj(nj);
    uint64_t n_items = 0, arena = 0, pieces = 0;
    bool any_split = false;
    for (size_t i = 0; i < nj; i++) {
        const MemberJob& j = jobs[i];
        const uint64_t blen = j.len - j.body_off;
        uint64_t K = 1;
        if (G) {
            K = blen > G ? std::max<uint64_t>(1, (blen + G / 2) / G) : 1;
        } else {
            const uint64_t cj = cost_of(j);
            K = cj > Gc ? std::max<uint64_t>(1, (cj + Gc / 2) / Gc) : 1;
            K = std::min<uint64_t>(K, std::max<uint64_t>(1, blen / (16ull << 10)));
        }
        any_split |= K > 1;
        BatchJob& b = bj[i];
        b.in_off = j.file_off + j.body_off;
        b.blen = blen;
        b.expand = j.expand > 0 ? j.expand : c->expand;
        b.dst_off = j.dst_off;
        b.dst_cap = j.dst_cap;
        b.K = (uint32_t)K;
        b.item_first = (uint32_t)n_items;
        b.arena = arena;
        // every slot holds span x expand + 64 KiB (rounded to 8): the spans of
        // the job's items add up to at most blen + K bytes
        // (a multiple of 8 cells, so every slot starts 16-byte aligned)
        const uint64_t slots_bound = round8((uint64_t)std::ceil((double)(blen + K) * b.expand) + K * (65536 + 16));
        arena += slots_bound;
        b.piece_off = (uint32_t)pieces;
        b.piece_cap = (uint32_t)(std::min<uint64_t>(j.dst_cap, slots_bound) / WAVE_PIECE + 2);
        pieces += b.piece_cap;
        n_items += K;
        if (n_items > (1u << 30) || pieces > (1u << 30)) return 0;
    }
    L.direct = !any_split;
    L.n_items = (uint32_t)n_items;
    L.total_pieces = (uint32_t)pieces;
    L.mb_cap = L.n_items + 4096;
    std::vector<ChunkItem> ditems;
    std::vector<WaveJob> wj(nj);
    if (L.direct) {  // one item per job, straight into its destination
        ditems.resize(nj);
        for (size_t i = 0; i < nj; i++) {
            ChunkItem& it = ditems[i];
            it = ChunkItem{};
            it.in_off = bj[i].in_off;
            it.in_len = bj[i].blen;
            it.end_hint = ~0ull;
            it.out_off = bj[i].dst_off;
            it.out_cap = bj[i].dst_cap;
            it.id = (uint32_t)i;
            wj[i] = WaveJob{(uint32_t)i, 1, (uint32_t)i, bj[i].piece_off, bj[i].piece_cap, 1,
                            bj[i].dst_off + bj[i].dst_cap, bj[i].dst_off};
        }
    }
    // ---- scan region (every split job) and the tiles around the ideal starts
    std::vector<uint64_t> big_bit;
    std::vector<uint32_t> big_job, tiles;
    if (!L.direct) {
        std::vector<uint32_t> bigs;
        for (size_t i = 0; i < nj; i++)
            if (bj[i].K > 1) bigs.push_back((uint32_t)i);
        std::sort(bigs.begin(), bigs.end(), [&](uint32_t a, uint32_t b) { return bj[a].in_off < bj[b].in_off; });
        uint64_t lo = ~0ull, hi = 0;
        for (uint32_t i : bigs) {
            lo = std::min(lo, bj[i].in_off);
            hi = std::max(hi, bj[i].in_off + bj[i].blen);
        }
        uint32_t max_k = 0;
        for (uint32_t i : bigs) {
            bj[i].scan_bit = (bj[i].in_off - lo) * 8;
            big_bit.push_back(bj[i].scan_bit);
            big_job.push_back(i);
            max_k = std::max(max_k, bj[i].K);
        }
        L.walk_kb = std::max<uint32_t>(1, (max_k + FW_THREADS / 32 - 1) / (FW_THREADS / 32));
        L.n_big = (uint32_t)bigs.size();
        L.scan_body = d_in + lo;
        L.scan_len = hi - lo;
        const uint64_t tb = (uint64_t)c->scan_threads * 16, mis = (uintptr_t)(d_in + lo) & 15;
        L.n_tiles = (mis + L.scan_len + tb - 1) / tb;
        constexpr uint64_t NEAR = 16 << 10;
        for (uint32_t i : bigs) {
            const uint64_t nbits = bj[i].blen * 8;
            for (uint32_t k = 1; k < bj[i].K; k++) {
                const uint64_t byte = (bj[i].scan_bit + nbits * k / bj[i].K) / 8;
                const uint64_t t0 = (mis + (byte > NEAR ? byte - NEAR : 0)) / tb;
                const uint64_t t1 = std::min(L.n_tiles - 1, (mis + byte + NEAR) / tb);
                for (uint64_t t = t0; t <= t1; t++) tiles.push_back((uint32_t)t);
            }
        }
        std::sort(tiles.begin(), tiles.end());
        tiles.erase(std::unique(tiles.begin(), tiles.end()), tiles.end());
        if (L.n_tiles > 0xffffffffull || tiles.size() * 2 >= L.n_tiles) tiles.clear();  // scan everything
        L.n_list = (uint32_t)tiles.size();
        L.cap = (uint32_t)std::min<uint64_t>(L.scan_len / 64 + 65536, 1ull << 28);
        L.cap2 = std::max<uint32_t>(L.cap / 16, 65536);
        L.cap3 = (uint32_t)std::min<uint64_t>(L.scan_len / 1024 + 4096, 1ull << 26);
        const uint64_t work = L.n_list ? L.n_list : L.n_tiles;
        L.sgrid = (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(work, (uint64_t)c->n_sm * (2048 / c->scan_threads)));
        std::vector<uint32_t> jc(nj);
        for (size_t i = 0; i < nj; i++) jc[i] = bj[i].K;
        build_res_tables(jc, c->n_sm, L.tab);
    }
    // the costliest sub-chunks first
    std::vector<uint32_t> jorder(nj), order(L.n_items);
    std::vector<uint64_t> per(nj);
    for (uint32_t i = 0; i < nj; i++) {
        jorder[i] = i;
        per[i] = cost_of(jobs[i]) / bj[i].K;
    }
    std::stable_sort(jorder.begin(), jorder.end(), [&](uint32_t a, uint32_t b) { return per[a] > per[b]; });
    {
        size_t q = 0;
        for (uint32_t i : jorder)
            for (uint32_t k = 0; k < bj[i].K; k++) order[q++] = bj[i].item_first + k;
    }
    std::vector<uint32_t> mp(nj + 1);
    for (size_t i = 0; i < nj; i++) mp[i] = bj[i].piece_off;
    mp[nj] = L.total_pieces;
    std::vector<WaveState> st0(nj);
    for (size_t i = 0; i < nj; i++) st0[i] = WaveState{0, bj[i].dst_off, 1, 0};
    // ---- layout of c->bplan
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = round8(o + bytes);
        return at;
    };
    L.o_jobs = take(nj * sizeof(BatchJob));
    L.o_bigbit = take(big_bit.size() * 8);
    L.o_bigjob = take(big_job.size() * 4);
    L.o_order = take((size_t)L.n_items * 4);
    L.o_mp = take((nj + 1) * 4);
    L.o_tabs = take(L.direct ? 0 : L.tab.bytes);
    L.o_state = take(nj * sizeof(WaveState));
    L.o_wj = take(nj * sizeof(WaveJob));
    L.up_end = o;
    L.o_info = take(nj * sizeof(WaveInfo));
    L.o_ecrc = take(nj * 4);
    L.o_eisz = take(nj * 4);
    L.o_gcrc = take(nj * 4);
    L.o_glen = take(nj * 8);
    L.o_mst = take(nj * 4);
    L.down_end = o;
    L.o_np = take(nj * 4);
    L.o_seg = take(nj * 8);
    L.o_chunks = take(L.direct ? 0 : (size_t)L.n_items * sizeof(ResolveChunk));
    L.o_hs = take(L.direct ? 0 : ((size_t)L.n_items + 1) * 8);
    L.o_pc = take((size_t)L.total_pieces * sizeof(CrcPiece));
    L.o_pcrc = take((size_t)L.total_pieces * 4);
    L.o_keys = take(L.direct ? 0 : (size_t)L.n_items * 8);
    L.total = o;
    std::vector<uint8_t> up(L.up_end);
    std::memcpy(up.data() + L.o_jobs, bj.data(), nj * sizeof(BatchJob));
    if (!big_bit.empty()) std::memcpy(up.data() + L.o_bigbit, big_bit.data(), big_bit.size() * 8);
    if (!big_job.empty()) std::memcpy(up.data() + L.o_bigjob, big_job.data(), big_job.size() * 4);
    std::memcpy(up.data() + L.o_order, order.data(), (size_t)L.n_items * 4);
    std::memcpy(up.data() + L.o_mp, mp.data(), (nj + 1) * 4);
    if (!L.direct) L.tab.write(up.data() + L.o_tabs);
    std::memcpy(up.data() + L.o_state, st0.data(), nj * sizeof(WaveState));
    std::memcpy(up.data() + L.o_wj, wj.data(), nj * sizeof(WaveJob));
    // ---- device memory
    CK(dgrow(c->bplan, L.total));
    CK(dgrow(c->items, (size_t)L.n_items * sizeof(ChunkItem)));
    CK(dgrow(c->results, (size_t)L.n_items * sizeof(ChunkResult)));
    CK(dgrow(c->queue, 16));
    CK(dgrow(c->mbs, (size_t)L.mb_cap * sizeof(MemberRec)));
    CK(dgrow(c->mbcount, 16));
    CK(dgrow(c->rerr, 16));
    CK(dgrow(c->markers, 8));
    if (!L.direct) {
        CK(dgrow(c->cells, (arena + 8) * 2));
        CK(dgrow(c->win, res_win_bytes(L.tab, L.n_items)));
        CK(dgrow(c->cand, (size_t)L.cap * 8 + (size_t)L.cap2 * 8 + (size_t)L.cap3 * 8));
        CK(dgrow(c->ncand, 64));
        CK(dgrow(c->vflag, L.cap2));
        if (L.n_list) CK(dgrow(c->tiles, (size_t)L.n_list * 4));
    }
    {
        const uint32_t IW = c->inflate_warps;
        int occ = 0;
        if (L.direct) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint8_t>, IW * 32, IW * sizeof(WarpSmem));
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_inflate<uint16_t>, IW * 32, IW * sizeof(WarpSmem));
        L.igrid = persistent_blocks(c, std::max(1, occ), L.n_items, IW);
    }
    if (int rw = wait_arrival(c, err)) return rw;
    *taken = true;
    // ---- uploads (outside the graph: the graph reads them from fixed buffers)
    CK(cudaMemcpyAsync(c->bplan.p, up.data(), L.up_end, cudaMemcpyHostToDevice, c->stream));
    if (L.direct)
        CK(cudaMemcpyAsync(c->items.p, ditems.data(), nj * sizeof(ChunkItem), cudaMemcpyHostToDevice, c->stream));
    if (L.n_list) CK(cudaMemcpyAsync(c->tiles.p, tiles.data(), (size_t)L.n_list * 4, cudaMemcpyHostToDevice, c->stream));
    cudaEvent_t* marks = c->bt_marks;
    bool timed = true;
    for (int i = 0; i < BATCH_MARKS; i++)
        if (!marks[i] && cudaEventCreate(&marks[i]) != cudaSuccess) {
            marks[i] = nullptr;
            timed = false;
        }
    cudaGetLastError();
    bool ran = false;
#ifndef RRG_EMU
    if (c->use_graphs) {
        BatchKey key{};
        const DBuf* bs[] = {&c->bplan, &c->items, &c->results, &c->queue, &c->mbs,   &c->mbcount, &c->rerr,
                            &c->markers, &c->cells, &c->win,   &c->cand,  &c->ncand, &c->vflag,   &c->tiles,
                            &c->crc_table};
        for (size_t i = 0; i < sizeof(bs) / sizeof(bs[0]); i++) key.p[i] = bs[i]->p;
        key.p[15] = d_in;
        key.p[16] = tgt.p;
        key.p[17] = c->stream;
        key.p[18] = L.scan_body;
        key.p[19] = timed ? marks[0] : nullptr;
        const uint64_t vals[] = {L.direct, L.nj, L.n_items, L.n_big, L.total_pieces, L.mb_cap, L.scan_len, L.n_tiles,
                                 L.cap, L.cap2, L.cap3, L.n_list, L.sgrid, L.igrid, L.tab.groups.size(),
                                 L.tab.supers.size(), L.tab.jobs.size(), L.total,
                                 ((uint64_t)c->scan_threads << 32) | c->inflate_warps, L.o_tabs, L.walk_kb};
        for (size_t i = 0; i < sizeof(vals) / sizeof(vals[0]); i++) key.v[i] = vals[i];
        auto* ent = c->bt_graphs.find(key);
        if (!ent && c->bt_graphs.repeat(key)) {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ex = nullptr;
            if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const uint64_t l0 = c->launches;
                int rc = batch_enqueue(c, d_in, tgt.p, L, timed ? marks : nullptr, err);
                const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
                const uint32_t kernels = (uint32_t)(c->launches - l0);
                g_launches.fetch_sub(c->launches - l0);  // counted when the graph runs
                c->launches = l0;
                if (rc == 0 && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess)
                    ent = c->bt_graphs.add(key, ex, kernels);
                if (g) cudaGraphDestroy(g);
            }
            cudaGetLastError();  // a failed capture leaves no sticky error; run directly below
        }
        if (ent) {
            CK(cudaGraphLaunch(ent->e, c->stream));
            g_launches.fetch_add(ent->kernels);
            c->launches += ent->kernels;
            c->st.graph_launches++;
            ran = true;
        }
    }
#endif
    if (!ran) {
        if (int rc = batch_enqueue(c, d_in, tgt.p, L, timed ? marks : nullptr, err)) return rc;
    }
    // ---- outcomes: one copy of the per-job words, one synchronisation
    std::vector<uint8_t> down(L.down_end - L.o_info);
    std::vector<WaveJob> wout(nj);
    uint32_t e4[4] = {0, 0, 0, 0};
    unsigned long long nmk = 0;
    uint8_t* P = (uint8_t*)c->bplan.p;
    CK(cudaMemcpyAsync(down.data(), P + L.o_info, down.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(wout.data(), P + L.o_wj, nj * sizeof(WaveJob), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(e4, c->rerr.p, 16, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&nmk, c->markers.p, 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (timed) {
        float f[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; i++)
            if (cudaEventElapsedTime(&f[i], marks[i], marks[i + 1]) != cudaSuccess) f[i] = 0;
        cudaGetLastError();
        c->st.finder_ms += f[0];
        c->st.inflate_ms += f[1];
        c->st.resolve_ms += f[2];
        c->st.crc_ms += f[3];
    }
    c->st.markers += nmk;
    auto at = [&](size_t off) { return down.data() + (off - L.o_info); };
    const WaveInfo* info = (const WaveInfo*)at(L.o_info);
    const uint32_t* ecrc = (const uint32_t*)at(L.o_ecrc);
    const uint32_t* eisz = (const uint32_t*)at(L.o_eisz);
    const uint32_t* gcrc = (const uint32_t*)at(L.o_gcrc);
    const uint64_t* glen = (const uint64_t*)at(L.o_glen);
    const int32_t* mst = (const int32_t*)at(L.o_mst);
    int64_t bad_job = -1;
    if (e4[0] && !L.direct) {  // the first chunk whose markers did not resolve
        for (size_t i = 0; i < nj; i++)
            if (e4[1] >= bj[i].item_first && e4[1] < bj[i].item_first + bj[i].K) bad_job = (int64_t)i;
    }
    std::vector<size_t> redo;
    for (size_t i = 0; i < nj; i++) {
        MemberJob& j = jobs[i];
        c->st.gpu_chunks += wout[i].n;
        if (!info[i].ok) {
            redo.push_back(i);
            continue;
        }
        j.out.total = info[i].out_len;
        j.out.members = 1;
        j.out.consumed = j.file_off + j.len;
        c->st.members++;
        if ((int64_t)i == bad_job) {
            set_err(&j.err, RRG_ERR_DEFLATE_INVALID, "%s", msg_text(MSG_MARKER_WINDOW));
            j.rc = RRG_ERR_DEFLATE_INVALID;
            continue;
        }
        if (mst[i] == DS_CRC || mst[i] == DS_ISIZE) {
            const MemberSpan m{j.dst_off, glen[i], ecrc[i], eisz[i],
                               j.report_off + j.file_off + j.body_off + info[i].trailer_byte};
            j.rc = member_error(&j.err, m, j.member_base, mst[i], gcrc[i], glen[i]);
        }
    }
    // ---- jobs the device route did not finish: the checked route
    if (!redo.empty()) {
        std::vector<MemberJob> rj;
        for (size_t i : redo) {
            MemberJob j = jobs[i];
            j.rc = 0;
            j.err = rrg_error{};
            j.out = Decoded{};
            rj.push_back(j);
        }
        if (int rc = members_route(c, d_in, rj, tgt, err)) return rc;
        for (size_t q = 0; q < redo.size(); q++) jobs[redo[q]] = rj[q];
    }
    return 0;
}

int batch_impl(rrg_ctx* c, const uint8_t* d_in, const uint64_t* in_off, const uint64_t* in_len, uint8_t* d_out,
               const uint64_t* out_off, const uint64_t* out_cap, uint64_t* out_len, int32_t* status, size_t n,
               rrg_error* err) {
    int rc = upload_tables(c, err);
    if (rc || !n) return rc;
    // ---- headers, BGZF sniff and the trailers' size hints, one thread per file
    // 4 x 8-byte and 3 x 4-byte values per file
    CK(dgrow(c->sniff, n * 44));
    uint8_t* sb = (uint8_t*)c->sniff.p;
    uint64_t* d_off = (uint64_t*)sb;
    uint64_t* d_len = d_off + n;
    uint64_t* d_body = d_len + n;
    int64_t* d_bgzf = (int64_t*)(d_body + n);
    int32_t* d_st = (int32_t*)(d_bgzf + n);
    int32_t* d_msg = d_st + n;
    uint32_t* d_isz = (uint32_t*)(d_msg + n);
    CK(cudaMemcpyAsync(d_off, in_off, n * 8, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_len, in_len, n * 8, cudaMemcpyHostToDevice, c->stream));
    SniffArgs SA{d_in, d_off, d_len, (uint32_t)n, d_st, d_msg, d_body, d_bgzf, d_isz};
    RRG_LAUNCH(k_sniff, (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)c->n_sm * 4), 256, 0, c->stream, SA);
    LAUNCHED(c);
    std::vector<uint64_t> body(n);
    std::vector<int64_t> bg(n);
    std::vector<int32_t> hst(n), hmsg(n);
    std::vector<uint32_t> isz(n);
    CK(cudaMemcpyAsync(body.data(), d_body, n * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(bg.data(), d_bgzf, n * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hst.data(), d_st, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hmsg.data(), d_msg, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(isz.data(), d_isz, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<MemberJob> jobs;
    std::vector<size_t> job_item;
    for (size_t i = 0; i < n; i++) {
        out_len[i] = 0;
        status[i] = RRG_OK;
        if (in_len[i] == 0) {
            status[i] = RRG_ERR_TRUNCATED;
            continue;
        }
        if (bg[i] >= 0) {  // BGZF file: its own device walk and decode
            rrg_error e{};
            OutTarget t{d_out + out_off[i], out_cap[i], false};
            Decoded d;
            int r = decode_file(c, d_in + in_off[i], in_len[i], nullptr, t, &d, &e);
            if (r == RRG_ERR_CUDA || r == RRG_ERR_OUT_OF_MEMORY) {
                if (err) *err = e;
                return r;
            }
            status[i] = r;
            out_len[i] = d.total;
            continue;
        }
        if (hst[i]) {
            rrg_error e{};
            status[i] = status_err(&e, hst[i], hmsg[i], 0);
            continue;
        }
        MemberJob j;
        j.file_off = in_off[i];
        j.len = in_len[i];
        j.body_off = body[i];
        j.dst_off = out_off[i];
        j.dst_cap = out_cap[i];
        const uint64_t blen = j.len - j.body_off;
        // ISIZE of the (last) member: a size hint for the reserved cells
        if (isz[i] && blen)
            j.expand = std::min(1100.0, std::max(1.05, 1.25 * (double)isz[i] / (double)blen + 0.05));
        j.isize_hint = isz[i];
        jobs.push_back(j);
        job_item.push_back(i);
    }
    // ---- waves: reserved cells (2 bytes each) within the budget and free memory
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const uint64_t budget = std::max<uint64_t>(
        8ull << 20, std::min<uint64_t>(c->cfg.hbm_budget_bytes, (uint64_t)((free_b + c->cells.cap) * 0.6)));
    OutTarget tgt{d_out, ~0ull, false};
    for (size_t a = 0; a < jobs.size();) {
        size_t b = a;
        uint64_t need = 0;
        while (b < jobs.size()) {
            const MemberJob& j = jobs[b];
            const uint64_t blen = j.len - j.body_off;
            const uint64_t cells = (uint64_t)((double)blen * (j.expand > 0 ? j.expand : c->expand) * 1.6) + (1u << 20);
            if (b > a && need + 2 * cells > budget) break;
            need += 2 * cells;
            b++;
        }
        std::vector<MemberJob> wave(jobs.begin() + a, jobs.begin() + b);
        bool taken = false;
        rc = batch_device(c, d_in, wave, tgt, &taken, err);
        if (!rc && !taken) rc = members_route(c, d_in, wave, tgt, err);
        if (rc) return rc;
        for (size_t q = 0; q < wave.size(); q++) {
            const size_t i = job_item[a + q];
            status[i] = wave[q].rc;
            out_len[i] = wave[q].out.total;
        }
        a = b;
    }
    return 0;
}

// ------------------------------------------------------------ autotuner
// Times the batch path on the caller's sample under a coordinate sweep of the
// tunables (sub-chunk size, boundary search and scan tile, warps per BGZF
// member) and keeps the fastest setting in the context.
struct Tunables {
    uint64_t gpu_chunk;
    bool scan_bounds;
    uint32_t scan_threads, warps_per_member;
};
Tunables get_tun(const rrg_ctx* c) { return Tunables{c->gpu_chunk, c->scan_bounds, c->scan_threads, c->warps_per_member}; }
void set_tun(rrg_ctx* c, const Tunables& t) {
    c->gpu_chunk = t.gpu_chunk;
    c->scan_bounds = t.scan_bounds;
    c->scan_threads = t.scan_threads;
    c->warps_per_member = t.warps_per_member;
}

int autotune_impl(rrg_ctx* c, const uint8_t* d_in, const uint64_t* in_off, const uint64_t* in_len, uint8_t* d_out,
                  const uint64_t* out_off, const uint64_t* out_cap, size_t n, rrg_tuning* res, rrg_error* err) {
    std::vector<uint64_t> olen(n);
    std::vector<int32_t> stv(n);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    uint32_t trials = 0;
    // best of 2 timed runs after one untimed run; infinity if any item fails
    auto measure = [&](const Tunables& t, double* ms) -> int {
        set_tun(c, t);
        double best = 1e30;
#ifdef RRG_EMU
        const int reps = 1;  // the CPU emulation checks the sweep, not the timings
#else
        const int reps = 3;
#endif
        for (int r = 0; r < reps; r++) {
            CK(cudaEventRecord(e0, c->stream));
            int rc = batch_impl(c, d_in, in_off, in_len, d_out, out_off, out_cap, olen.data(), stv.data(), n, err);
            if (rc) return rc;
            CK(cudaEventRecord(e1, c->stream));
            CK(cudaEventSynchronize(e1));
            float f = 0;
            cudaEventElapsedTime(&f, e0, e1);
            for (size_t i = 0; i < n; i++)
                if (stv[i] != RRG_OK) f = 1e30f;
            if (r || reps == 1) best = std::min(best, (double)f);
        }
        trials++;
        *ms = best;
        return 0;
    };
    bool any_bgzf = false;
    for (size_t i = 0; i < n; i++) {
        uint8_t h[64] = {0};
        const size_t k = (size_t)std::min<uint64_t>(in_len[i], sizeof(h));
        CK(cudaMemcpy(h, d_in + in_off[i], k, cudaMemcpyDeviceToHost));
        any_bgzf |= host_bgzf_size(h, k) >= 0;
    }
    Tunables best = get_tun(c), t = best;
    double best_ms = 0, ms = 0;
    int rc = measure(best, &best_ms);
    if (rc) return rc;
    const double default_ms = best_ms;
    // 1. sub-chunk size (0 = one wave of resident decoders)
    for (uint64_t g : {0ull, 32ull << 10, 64ull << 10, 128ull << 10, 256ull << 10, 1ull << 20}) {
        t = best;
        t.gpu_chunk = g;
        if (g == best.gpu_chunk) continue;
        if ((rc = measure(t, &ms))) return rc;
        if (ms < best_ms) best = t, best_ms = ms;
    }
    // 2. boundary search: the scan with each tile width, or one search per target
    for (uint32_t st : {64u, 128u, 256u, 0u}) {
        t = best;
        t.scan_bounds = st != 0;
        if (st) t.scan_threads = st;
        if (t.scan_bounds == best.scan_bounds && t.scan_threads == best.scan_threads) continue;
        if ((rc = measure(t, &ms))) return rc;
        if (ms < best_ms) best = t, best_ms = ms;
    }
    // 3. warps per BGZF member
    if (any_bgzf)
        for (uint32_t w = 1; w <= 4; w++) {
            t = best;
            t.warps_per_member = w;
            if (w == best.warps_per_member) continue;
            if ((rc = measure(t, &ms))) return rc;
            if (ms < best_ms) best = t, best_ms = ms;
        }
    set_tun(c, best);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (res) {
        res->gpu_chunk_bytes = best.gpu_chunk;
        res->boundary_mode = best.scan_bounds ? 0 : 1;
        res->finder_tile_bits = (uint64_t)best.scan_threads * 16 * 8;
        res->warps_per_member = (int32_t)best.warps_per_member;
        res->best_ms = best_ms;
        res->default_ms = default_ms;
        res->trials = trials;
    }
    return 0;
}

// Frees every device buffer of the context (they grow again on demand).
void release_scratch(rrg_ctx* c) {
    DBuf* bufs[] = {&c->cand, &c->ncand, &c->vflag, &c->lane_scratch, &c->win, &c->items,  &c->results, &c->order,     &c->queue,    &c->mbs,      &c->mbcount,   &c->cells,
                    &c->out,    &c->targets, &c->limits,    &c->found,    &c->next_lut, &c->chunks,    &c->tiles,
                    &c->rerr,   &c->markers, &c->crc_table, &c->pieces,   &c->piece_crc, &c->mpiece,   &c->exp_crc,
                    &c->exp_isize, &c->got_crc, &c->got_len, &c->mstatus, &c->comp, &c->comp2, &c->pfx, &c->bg_bcount, &c->bg_bbase,
                    &c->bg_coff, &c->bg_csize, &c->bg_small, &c->sniff, &c->pipe, &c->bplan};
#ifndef RRG_EMU
    c->bg_graphs.clear();
    c->bt_graphs.clear();
#endif
    for (cudaEvent_t& e : c->bt_marks) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    for (DBuf* b : bufs) {
        if (b->p) cudaFree(b->p);
        b->p = nullptr;
        b->cap = 0;
    }
    c->tables_uploaded = false;
}

// ------------------------------------------------------------ result buffers
// Serving results are host buffers the caller releases with rrg_gpu_free.
// Buffers of 1 MiB and more are page-locked (the engines copy results into
// them straight from the device at the link's rate) and, once freed, kept by
// size class (powers of two, at most 32 GiB in all) and handed out again, so a
// steady request stream neither pins nor faults in fresh memory.
struct ResultPool {
    std::mutex mu;
    std::unordered_map<void*, int> cls;           // every pooled block ever handed out -> class
    std::vector<std::vector<void*>> free_by_cls;  // class -> idle blocks
    uint64_t idle_bytes = 0;
};
ResultPool& result_pool() {
    static ResultPool* p = new ResultPool;
    return *p;
}
constexpr uint64_t POOL_MIN = 1ull << 20, POOL_MAX_IDLE = 32ull << 30;

void* result_alloc(uint64_t n) {
    if (n < POOL_MIN) return std::malloc(std::max<uint64_t>(n, 1));
    int k = 20;
    while ((1ull << k) < n) k++;
    ResultPool& P = result_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        if ((int)P.free_by_cls.size() > k && !P.free_by_cls[k].empty()) {
            void* b = P.free_by_cls[k].back();
            P.free_by_cls[k].pop_back();
            P.idle_bytes -= 1ull << k;
            return b;
        }
    }
    void* b = nullptr;
    if (cudaMallocHost(&b, 1ull << k) != cudaSuccess) {
        cudaGetLastError();  // not sticky: fall back to pageable memory
        b = nullptr;
    }
    if (!b) return std::malloc(1ull << k);
    {
        std::lock_guard<std::mutex> g(P.mu);
        P.cls[b] = k;
    }
    return b;
}

void result_free(void* b) {
    if (!b) return;
    ResultPool& P = result_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.cls.find(b);
        if (it != P.cls.end()) {
            const int k = it->second;
            if (P.idle_bytes + (1ull << k) <= POOL_MAX_IDLE) {
                if ((int)P.free_by_cls.size() <= k) P.free_by_cls.resize(k + 1);
                P.free_by_cls[k].push_back(b);
                P.idle_bytes += 1ull << k;
                return;
            }
            P.cls.erase(it);
            cudaFreeHost(b);
            return;
        }
    }
    std::free(b);
}

// ------------------------------------------------------------ serving engines
// Device bytes a request holds while admitted: its input, its output and
// the speculative-decode scratch (u16 cells plus slack), from the trailer's
// ISIZE as the size hint.
uint64_t serve_reserve(const Server::Req& r, double expand_cap) {
    const uint64_t c = r.len;
    const uint64_t isz = c >= 4 ? le32h(r.bytes + c - 4) : 0;
    const uint64_t out = r.out_need ? r.out_need : std::max<uint64_t>(isz, c);
    const double ex = c ? std::min(expand_cap, std::max(1.05, 1.25 * (double)out / (double)c + 0.05)) : 1.0;
    return c + out + (uint64_t)(2.0 * 1.6 * ex * (double)c) + (2ull << 20);
}

void engine_loop(Server* S, rrg_ctx* E) {
    if (E->cfg.device >= 0) cudaSetDevice(E->cfg.device);
    else cudaSetDevice(E->device);
    for (;;) {
        std::vector<Server::Req> batch;
        uint64_t reserved = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] {
                if (S->stop) return true;
                if (S->waiting.empty() || S->done.size() >= S->max_ready) return false;
                return S->in_use == 0 || S->in_use + serve_reserve(S->waiting.front(), E->expand) <= S->budget;
            });
            if (S->stop) return;
            // the oldest waiting requests that fit together (at least one). A
            // batch stays within this engine's share of the budget, so the
            // engines' resident scratch stays within the budget as a whole.
            const uint64_t slice = S->budget / S->engines.size();
            while (!S->waiting.empty() && batch.size() < S->max_batch) {
                const uint64_t r = serve_reserve(S->waiting.front(), E->expand);
                if (!batch.empty() && reserved + r > slice) break;
                if (!batch.empty() || S->in_use) {
                    if (S->in_use + reserved + r > S->budget) break;
                }
                reserved += r;
                batch.push_back(std::move(S->waiting.front()));
                S->waiting.pop_front();
                if (S->in_use + reserved > S->budget) break;  // a lone request above the budget
            }
            S->in_use += reserved;
            S->stats.batches++;
            S->stats.max_batch = std::max<uint64_t>(S->stats.max_batch, batch.size());
            S->stats.engines_busy++;
            S->stats.max_engines_busy = std::max(S->stats.max_engines_busy, S->stats.engines_busy);
            S->stats.peak_in_use_bytes = std::max(S->stats.peak_in_use_bytes, S->in_use);
        }
        // ---- one batch on this engine's stream
        const size_t n = batch.size();
        std::vector<uint64_t> in_off(n), in_len(n), out_off(n), out_cap(n), out_len(n, 0);
        std::vector<int32_t> status(n, RRG_OK);
        uint64_t ti = 0, to = 0;
        for (size_t i = 0; i < n; i++) {
            const Server::Req& r = batch[i];
            const uint64_t c = r.len;
            const uint64_t isz = c >= 4 ? le32h(r.bytes + c - 4) : 0;
            in_off[i] = ti;
            in_len[i] = c;
            ti += (c + 255) & ~255ull;
            out_off[i] = to;
            out_cap[i] = r.out_need ? r.out_need : std::max<uint64_t>(isz, c);
            to += (out_cap[i] + 255) & ~255ull;
        }
        rrg_error err{};
        int rc = 0;
        auto fail_all = [&](int code) {
            for (size_t i = 0; i < n; i++) status[i] = code;
        };
        double t_h2d = 0, t_dec = 0;
        for (int attempt = 0; attempt < 2; attempt++) {
            rc = 0;
            std::fill(status.begin(), status.end(), RRG_OK);
            const double ta = now_ms();
            if (dgrow(E->comp, ti + 64) != cudaSuccess || dgrow(E->out, to + 64) != cudaSuccess) {
                cudaGetLastError();
                rc = RRG_ERR_OUT_OF_MEMORY;
            }
            for (size_t i = 0; i < n && !rc; i++)
                if (in_len[i] && cudaMemcpyAsync((uint8_t*)E->comp.p + in_off[i], batch[i].bytes, in_len[i],
                                                 cudaMemcpyHostToDevice, E->stream) != cudaSuccess)
                    rc = RRG_ERR_CUDA;
            const double tb = now_ms();
            if (!rc) {
                E->st = rrg_stats{};
                rc = batch_impl(E, (const uint8_t*)E->comp.p, in_off.data(), in_len.data(), (uint8_t*)E->out.p,
                                out_off.data(), out_cap.data(), out_len.data(), status.data(), n, &err);
            }
            t_h2d += tb - ta;
            t_dec += now_ms() - tb;
            if (rc != RRG_ERR_OUT_OF_MEMORY) break;
            // device memory ran out: drop this engine's resident scratch, once more
            cudaGetLastError();
            release_scratch(E);
        }
        if (rc) fail_all(rc);
        std::vector<Server::Done> fin;
        std::vector<Server::Req> retry;
        const double t_out = now_ms();
        for (size_t i = 0; i < n; i++) {
            Server::Req& r = batch[i];
            if (status[i] == RRG_ERR_CAPACITY && !r.out_need && out_len[i] > out_cap[i]) {
                r.out_need = out_len[i];  // the ISIZE hint was short (several members): again, exact
                retry.push_back(std::move(r));
                continue;
            }
            Server::Done d{r.id, nullptr, 0, status[i], r.t_submit, 0.0, rrg_error{}};
            if (status[i] != RRG_OK) {
                if (rc && err.code) d.err = err;  // the whole batch failed: its error
                else set_err(&d.err, status[i], "request failed with status %d", status[i]);
            }
            if (status[i] == RRG_OK) {
                d.out = (uint8_t*)result_alloc(out_len[i]);
                d.len = out_len[i];
                if (!d.out) {
                    d.status = RRG_ERR_OUT_OF_MEMORY;
                    d.len = 0;
                } else if (out_len[i] &&
                           cudaMemcpyAsync(d.out, (const uint8_t*)E->out.p + out_off[i], out_len[i],
                                           cudaMemcpyDeviceToHost, E->stream) != cudaSuccess) {
                    // one copy per result, straight into its (page-locked) buffer
                    d.status = RRG_ERR_CUDA;
                }
            }
            fin.push_back(d);
        }
        cudaStreamSynchronize(E->stream);
        const double t_fin = now_ms();
        // a lone request above this engine's share grew its scratch past it: give it back
        if (reserved > S->budget / S->engines.size()) release_scratch(E);
        {
            std::lock_guard<std::mutex> g(S->mu);
            S->stats.h2d_ms += t_h2d;
            S->stats.decode_ms += t_dec;
            S->stats.d2h_ms += t_fin - t_out;
            S->in_use -= reserved;
            S->stats.engines_busy--;
            for (auto& r : retry) S->waiting.push_front(std::move(r));
            for (auto& d : fin) {
                if (d.status != RRG_OK && d.out) {
                    result_free(d.out);
                    d.out = nullptr;
                    d.len = 0;
                }
                if (d.status != RRG_OK && !d.err.code) set_err(&d.err, d.status, "result copy failed");
                d.latency_ms = t_fin - d.t_submit;
                S->done.push_back(d);
                S->stats.completed++;
                S->stats.bytes_out += d.len;
            }
            S->cv_done.notify_all();
            S->cv_work.notify_all();
        }
    }
}

int serve_start(rrg_ctx* c, uint32_t engines, uint32_t max_ready, rrg_error* err) {
    std::lock_guard<std::mutex> g(c->srv_create_mu);
    if (c->srv) return 0;
    Server* S = new Server();
    S->budget = c->cfg.hbm_budget_bytes;
    if (max_ready) S->max_ready = max_ready;
    const uint32_t ne = engines ? std::min<uint32_t>(engines, 8) : 2;
    for (uint32_t i = 0; i < ne; i++) {
        rrg_config cfg = c->cfg;
        cfg.device = c->device;
        rrg_ctx* E = rrg_gpu_create(&cfg, err);
        if (!E) {
            for (rrg_ctx* x : S->engines) rrg_gpu_destroy(x);
            delete S;
            return err ? err->code : RRG_ERR_CUDA;
        }
        // the owner's tuned settings
        E->gpu_chunk = c->gpu_chunk;
        E->scan_bounds = c->scan_bounds;
        E->scan_threads = c->scan_threads;
        E->warps_per_member = c->warps_per_member;
        E->lanes = c->lanes;
        S->engines.push_back(E);
    }
    for (rrg_ctx* E : S->engines) S->threads.emplace_back(engine_loop, S, E);
    c->srv = S;
    return 0;
}

void serve_stop(rrg_ctx* c) {
    std::lock_guard<std::mutex> g(c->srv_create_mu);
    Server* S = c->srv;
    if (!S) return;
    {
        std::lock_guard<std::mutex> l(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
    }
    for (auto& t : S->threads) t.join();
    for (rrg_ctx* E : S->engines) rrg_gpu_destroy(E);
    for (auto& d : S->done)
        if (d.out) result_free(d.out);
    delete S;
    c->srv = nullptr;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

rrg_ctx* rrg_gpu_create(const rrg_config* cfg, rrg_error* err) {
    rrg_ctx* c = new rrg_ctx();
    if (cfg) c->cfg = *cfg;
    if (!c->cfg.chunk_size_bytes) c->cfg.chunk_size_bytes = 4ull << 20;
    if (!c->cfg.hbm_budget_bytes) c->cfg.hbm_budget_bytes = 120ull * 1000 * 1000 * 1000;
    c->pipeline = c->cfg.host_pipeline >= 0;
    c->gpu_chunk = c->cfg.gpu_chunk_bytes;
    if (c->cfg.finder_tile_bits) {
        c->finder_tile = (uint32_t)std::min<uint64_t>(FIND_TILE, (c->cfg.finder_tile_bits + 31) & ~31ull);
        // the boundary scan's tile: 8192, 16384 or 32768 bits (1, 2 or 4 KiB)
        c->scan_threads = c->cfg.finder_tile_bits <= 8192 ? 64 : c->cfg.finder_tile_bits <= 16384 ? 128 : 256;
    }
    if (c->cfg.warps_per_stream > 1) c->warps_per_member = (uint32_t)std::min(4, c->cfg.warps_per_stream);
    cudaError_t e;
    if (c->cfg.device >= 0) {
        e = cudaSetDevice(c->cfg.device);
        if (e != cudaSuccess) {
            cuda_fail(err, e, "cudaSetDevice");
            delete c;
            return nullptr;
        }
    }
    cudaGetDevice(&c->device);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) == cudaSuccess && sms > 0) c->n_sm = sms;
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cuda_fail(err, e, "cudaStreamCreate");
        delete c;
        return nullptr;
    }
    c->stream = c->own_stream;
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    size_t want = (size_t)c->inflate_warps * sizeof(WarpSmem);
    cudaFuncSetAttribute(k_find_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * sizeof(FindSmem)));
    cudaFuncSetAttribute(k_win_maps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WM_SMEM);
    cudaFuncSetAttribute(k_win_bases, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(WINDOW * 2));
    cudaFuncSetAttribute(k_win_supers, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(WINDOW * 2));
    cudaFuncSetAttribute(k_res_tails, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(WINDOW * 2));
    cudaFuncSetAttribute(k_verify_heavy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * sizeof(FindSmem)));
    cudaFuncSetAttribute(k_inflate_lanes<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(LANE_THREADS * sizeof(LaneTab)));
    cudaFuncSetAttribute(k_inflate_lanes<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(LANE_THREADS * sizeof(LaneTab)));
    if (c->cfg.warps_per_stream < 0) c->lanes = true;  // -1: one decoder per lane (32 chunks per warp)
    if (c->cfg.boundary_mode == 1) c->scan_bounds = false;
    if (smem_optin > 0 && want > 48 * 1024) {
        cudaFuncSetAttribute(k_inflate<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
        cudaFuncSetAttribute(k_inflate<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
    }
    if (err) std::memset(err, 0, sizeof(*err));
    return c;
}

void rrg_gpu_destroy(rrg_ctx* c) {
    if (!c) return;
    serve_stop(c);
    release_scratch(c);
    for (auto& p : c->h_stage)
        if (p) cudaFreeHost(p);
    if (c->h_bg) cudaFreeHost(c->h_bg);
    if (c->h_in) cudaFreeHost(c->h_in);
    if (c->h_file) cudaFreeHost(c->h_file);
    for (cudaEvent_t e : c->arr_events)
        if (e) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->h_ring) cudaFreeHost(c->h_ring);
    if (c->h_wave) cudaFreeHost(c->h_wave);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c->split;
    delete c;
}

int rrg_gpu_decode_host(rrg_ctx* c, const uint8_t* data, size_t len, rrg_sink_fn sink, void* user, rrg_stats* stats,
                        rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || (!data && len)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context or data");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    return decode_host_impl(c, data, len, sink, user, stats, err);
}

int rrg_gpu_read_gz(rrg_ctx* c, const char* path, rrg_sink_fn sink, void* user, rrg_stats* stats, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || !path) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context or path");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    int fd = open(path, O_RDONLY);
    if (fd < 0) {
        set_err(err, RRG_ERR_IO, "io: cannot open %s: %s", path, std::strerror(errno));
        return RRG_ERR_IO;
    }
    struct stat sb;
    if (fstat(fd, &sb) != 0) {
        set_err(err, RRG_ERR_IO, "io: stat %s: %s", path, std::strerror(errno));
        close(fd);
        return RRG_ERR_IO;
    }
    if (!S_ISREG(sb.st_mode)) {
        // pipes, sockets, character devices: decoded stripe by stripe as they
        // are read (lib.rs:378-431 streams these)
        if (err) std::memset(err, 0, sizeof(*err));
        auto rd = [](void* u, uint8_t* buf, size_t cap) -> int64_t {
            for (;;) {
                const ssize_t r = read(*(int*)u, buf, cap);
                if (r >= 0 || errno != EINTR) return (int64_t)r;
            }
        };
        const int rc = stream_impl(c, rd, &fd, sink, user, 0, stats, err);
        close(fd);
        return rc;
    }
    // The file goes into page-locked memory (so the copy to the device runs at
    // the link's rate), read by num_threads threads in parallel (0: one per
    // core, at most 16), each a run of at least 8 MiB.
    const size_t size = (size_t)sb.st_size;
    std::vector<uint8_t> fallback;
    uint8_t* buf = nullptr;
    if (size <= (16ull << 30)) {
        if (c->h_file_cap < size) {
            if (c->h_file) cudaFreeHost(c->h_file);
            c->h_file = nullptr;
            c->h_file_cap = 0;
            if (cudaMallocHost((void**)&c->h_file, std::max<size_t>(size, 1)) == cudaSuccess) c->h_file_cap = size;
            else cudaGetLastError();
        }
        if (c->h_file_cap >= size) buf = c->h_file;
    }
    if (!buf) {
        fallback.resize(size);
        buf = fallback.data();
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t want = c->cfg.num_threads ? c->cfg.num_threads : std::min(hw, 16u);
    const size_t T = std::max<size_t>(1, std::min(want, size / (8u << 20)));
    std::vector<size_t> got(T, 0);
    auto reader = [&](size_t t) {
        const size_t a = size * t / T, b = size * (t + 1) / T;
        size_t at = a;
        while (at < b) {
            const ssize_t r = pread(fd, buf + at, b - at, (off_t)at);
            if (r < 0 && errno == EINTR) continue;
            if (r <= 0) break;
            at += (size_t)r;
        }
        got[t] = at - a;
    };
    if (T == 1) {
        reader(0);
    } else {
        std::vector<std::thread> th;
        for (size_t t = 0; t < T; t++) th.emplace_back(reader, t);
        for (auto& x : th) x.join();
    }
    close(fd);
    size_t n = 0;
    for (size_t t = 0; t < T && got[t] == size * (t + 1) / T - size * t / T; t++) n = size * (t + 1) / T;
    if (err) std::memset(err, 0, sizeof(*err));
    return decode_host_impl(c, buf, n, sink, user, stats, err);
}

// The destination provider is the context's for the duration of one call.
struct ProviderScope {
    rrg_ctx* c;
    ProviderScope(rrg_ctx* ctx, rrg_buffer_fn get, void* user) : c(ctx) {
        if (c) {
            c->get_buf = get;
            c->get_user = user;
        }
    }
    ~ProviderScope() {
        if (c) {
            c->get_buf = nullptr;
            c->get_user = nullptr;
        }
    }
};

int rrg_gpu_decode_host_into(rrg_ctx* c, const uint8_t* data, size_t len, rrg_buffer_fn get, rrg_sink_fn sink,
                             void* user, rrg_stats* stats, rrg_error* err) {
    ProviderScope scope(c, get, user);
    return rrg_gpu_decode_host(c, data, len, sink, user, stats, err);
}

int rrg_gpu_read_gz_into(rrg_ctx* c, const char* path, rrg_buffer_fn get, rrg_sink_fn sink, void* user,
                         rrg_stats* stats, rrg_error* err) {
    ProviderScope scope(c, get, user);
    return rrg_gpu_read_gz(c, path, sink, user, stats, err);
}

int rrg_gpu_index_build(rrg_ctx* c, const uint8_t* data, size_t len, uint64_t spacing, rrg_index** out,
                        rrg_stats* stats, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    if (!c || !data || !out) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context, data or index pointer");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (len == 0) {
        set_err(err, RRG_ERR_TRUNCATED, "truncated gzip stream");
        return RRG_ERR_TRUNCATED;
    }
    return index_build_impl(c, data, len, spacing ? spacing : (4ull << 20), out, stats, err);
}

int rrg_gpu_read_range(rrg_ctx* c, const uint8_t* data, size_t len, const rrg_index* idx, uint64_t off, uint64_t n,
                       uint8_t* dst, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    if (!c || !data || !idx || (!dst && n)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context, data, index or destination");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    return read_range_impl(c, data, len, idx, off, n, dst, err);
}

uint64_t rrg_index_total_out(const rrg_index* idx) { return idx ? idx->total_out : 0; }

size_t rrg_index_count(const rrg_index* idx) { return idx ? idx->out_off.size() : 0; }

int rrg_index_point(const rrg_index* idx, size_t k, uint64_t* out_off, uint64_t* in_bit) {
    if (!idx || k >= idx->out_off.size()) return RRG_ERR_INVALID_ARGUMENT;
    if (out_off) *out_off = idx->out_off[k];
    if (in_bit) *in_bit = idx->body_off * 8 + idx->in_bit[k];
    return 0;
}

// "RRGI", version 1, file_len, body_off, total_out, count, then per checkpoint
// in_bit, out_off, win_len and the window's bytes (all little-endian).
size_t rrg_index_serialize(const rrg_index* idx, uint8_t* buf, size_t cap) {
    if (!idx) return 0;
    size_t need = 8 + 4 * 8;
    for (size_t k = 0; k < idx->out_off.size(); k++) need += 20 + idx->win_len[k];
    if (!buf || cap < need) return need;
    uint8_t* p = buf;
    auto put = [&](uint64_t v, int nb) {
        for (int i = 0; i < nb; i++) *p++ = (uint8_t)(v >> (8 * i));
    };
    std::memcpy(p, "RRGI", 4);
    p += 4;
    put(1, 4);
    put(idx->file_len, 8);
    put(idx->body_off, 8);
    put(idx->total_out, 8);
    put(idx->out_off.size(), 8);
    for (size_t k = 0; k < idx->out_off.size(); k++) {
        put(idx->in_bit[k], 8);
        put(idx->out_off[k], 8);
        put(idx->win_len[k], 4);
        std::memcpy(p, idx->win.data() + k * 32768 + (32768 - idx->win_len[k]), idx->win_len[k]);
        p += idx->win_len[k];
    }
    return need;
}

rrg_index* rrg_index_deserialize(const uint8_t* buf, size_t n, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    const uint8_t* p = buf;
    const uint8_t* end = buf ? buf + n : nullptr;
    auto get = [&](int nb, uint64_t* v) {
        if (!p || end - p < nb) return false;
        *v = 0;
        for (int i = 0; i < nb; i++) *v |= (uint64_t)p[i] << (8 * i);
        p += nb;
        return true;
    };
    uint64_t ver = 0, cnt = 0;
    auto* idx = new rrg_index;
    bool ok = buf && n >= 8 && std::memcmp(buf, "RRGI", 4) == 0;
    if (ok) {
        p += 4;
        ok = get(4, &ver) && ver == 1 && get(8, &idx->file_len) && get(8, &idx->body_off) &&
             get(8, &idx->total_out) && get(8, &cnt) && cnt <= n / 20;
    }
    for (uint64_t k = 0; ok && k < cnt; k++) {
        uint64_t ib = 0, oo = 0, wl = 0;
        // checkpoints lie inside the file's body, in increasing bit and output
        // order, and carry at most one window of history
        ok = get(8, &ib) && get(8, &oo) && get(4, &wl) && wl <= 32768 && wl <= oo && (uint64_t)(end - p) >= wl &&
             (idx->out_off.empty() || (oo > idx->out_off.back() && ib > idx->in_bit.back())) &&
             oo <= idx->total_out && idx->body_off < idx->file_len &&
             ib < (idx->file_len - idx->body_off) * 8;
        if (!ok) break;
        idx->in_bit.push_back(ib);
        idx->out_off.push_back(oo);
        idx->win_len.push_back((uint32_t)wl);
        idx->win.resize(idx->out_off.size() * 32768, 0);
        std::memcpy(idx->win.data() + k * 32768 + (32768 - wl), p, wl);
        p += wl;
    }
    if (!ok || idx->out_off.empty() || idx->out_off[0] != 0 || idx->file_len > (1ull << 61)) {
        delete idx;
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "not a seek index");
        return nullptr;
    }
    return idx;
}

void rrg_index_free(rrg_index* idx) { delete idx; }

int rrg_gpu_read_stream(rrg_ctx* c, rrg_read_fn read_fn, void* read_user, rrg_sink_fn sink, void* user,
                        uint64_t stripe_bytes, rrg_stats* stats, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    if (!c || !read_fn) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context or read callback");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    return stream_impl(c, read_fn, read_user, sink, user, stripe_bytes, stats, err);
}

int rrg_gpu_decode_device(rrg_ctx* c, const uint8_t* d_in, size_t len, uint8_t* d_out, size_t out_cap, size_t* out_len,
                          void* stream, rrg_stats* stats, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || (!d_in && len)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context or input");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    double t_all = now_ms();
    c->st = rrg_stats{};
    c->launches = 0;
    c->st.compressed_bytes = len;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    Decoded d;
    OutTarget tgt{d_out, out_cap, false};
    int rc = decode_file(c, d_in, len, nullptr, tgt, &d, err);
    c->stream = c->own_stream;
    if (out_len) *out_len = (size_t)d.total;
    c->st.uncompressed_bytes = rc ? 0 : d.total;
    c->st.kernel_launches = c->launches;
    c->st.total_ms = now_ms() - t_all;
    if (stats) *stats = c->st;
    return rc;
}

int rrg_gpu_decode_batch(rrg_ctx* c, const uint8_t* d_in, const uint64_t* in_off, const uint64_t* in_len, uint8_t* d_out,
                         const uint64_t* out_off, const uint64_t* out_cap, uint64_t* out_len, int32_t* status, size_t n,
                         void* stream, rrg_stats* stats, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || (n && (!d_in || !in_off || !in_len || !d_out || !out_off || !out_cap || !out_len || !status))) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    double t_all = now_ms();
    c->st = rrg_stats{};
    c->launches = 0;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    int rc = batch_impl(c, d_in, in_off, in_len, d_out, out_off, out_cap, out_len, status, n, err);
    int first_bad = RRG_OK;
    if (!rc) {
        for (size_t i = 0; i < n; i++) {
            c->st.compressed_bytes += in_len[i];
            if (status[i] == RRG_OK) c->st.uncompressed_bytes += out_len[i];
            else if (first_bad == RRG_OK) {
                first_bad = status[i];
                set_err(err, status[i], "batch item %zu failed with status %d", i, status[i]);
            }
        }
    }
    c->stream = c->own_stream;
    c->st.kernel_launches = c->launches;
    c->st.total_ms = now_ms() - t_all;
    if (stats) *stats = c->st;
    return rc ? rc : first_bad;
}

int rrg_gpu_autotune(rrg_ctx* c, const uint8_t* d_in, const uint64_t* in_off, const uint64_t* in_len, uint8_t* d_out,
                     const uint64_t* out_off, const uint64_t* out_cap, size_t n, void* stream, rrg_tuning* result,
                     rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || !n || !d_in || !in_off || !in_len || !d_out || !out_off || !out_cap) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument or empty sample");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    std::memset(err, 0, sizeof(*err));
    c->st = rrg_stats{};
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    int rc = autotune_impl(c, d_in, in_off, in_len, d_out, out_off, out_cap, n, result, err);
    c->stream = c->own_stream;
    return rc;
}

uint32_t rrg_crc32_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b) {
    std::call_once(g_tab_once, init_tables);
    return host_crc_combine(crc_a, crc_b, len_b);
}

int rrg_gpu_split_begin(rrg_ctx* c, const uint8_t* data, size_t len, uint64_t body_off, uint64_t start_target,
                        uint64_t stop_target, uint32_t flags, uint16_t* end_map, rrg_split_info* info,
                        rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    if (!c || !data || !end_map || !info || body_off + 8 > len || start_target >= (len - body_off) * 8 ||
        (stop_target != ~0ull && stop_target <= start_target)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "split range outside the member body");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    int rc = upload_tables(c, err);
    if (rc) return rc;
    if (!c->split) c->split = new SplitState;
    SplitState& S = *c->split;
    S.ready = false;
    // the compressed bytes from the start target's byte to 16 MiB past the stop target
    const uint64_t byte0 = body_off + start_target / 8;
    const uint64_t end_byte =
        stop_target == ~0ull ? len : std::min<uint64_t>(len, body_off + stop_target / 8 + (16u << 20));
    const uint64_t clen = end_byte - byte0;
    CK(dgrow(c->comp, clen + 16));
    CK(cudaMemcpyAsync(c->comp.p, data + byte0, clen, cudaMemcpyHostToDevice, c->stream));
    const uint8_t* d_span = (const uint8_t*)c->comp.p;
    auto rel = [&](uint64_t body_bit) { return body_off * 8 + body_bit - byte0 * 8; };
    // block starts from the targets (find_next_dynamic_block, block_finder.rs:109-141)
    std::vector<uint64_t> targets, limits;
    const bool search_start = start_target != 0 && !(flags & RRG_SPLIT_EXACT_START);
    if (search_start) targets.push_back(rel(start_target));
    if (stop_target != ~0ull) targets.push_back(rel(stop_target));
    limits.assign(targets.size(), clen * 8);
    std::vector<uint64_t> found(targets.size(), ~0ull);
    if (!targets.empty()) {
        const size_t n = targets.size();
        CK(dgrow(c->targets, n * 8));
        CK(dgrow(c->limits, n * 8));
        CK(dgrow(c->found, n * 8));
        CK(dgrow(c->queue, 16));
        CK(cudaMemcpyAsync(c->targets.p, targets.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->limits.p, limits.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemsetAsync(c->queue.p, 0, 16, c->stream));
        FindArgs F{d_span, clen, (const uint64_t*)c->targets.p, (const uint64_t*)c->limits.p,
                   (uint64_t*)c->found.p, (uint32_t)n, (uint32_t*)c->queue.p, (const uint8_t*)c->next_lut.p,
                   c->finder_tile};
        RRG_LAUNCH(k_find_blocks, persistent_blocks(c, 4, n, 4), 128, 4 * sizeof(FindSmem), c->stream, F);
        LAUNCHED(c);
        CK(cudaMemcpyAsync(found.data(), c->found.p, n * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    const uint64_t start_rel = search_start ? found[0] : rel(start_target);
    const uint64_t stop_rel = stop_target == ~0ull ? ~0ull : found.back();
    if (start_rel == ~0ull) {
        // no dynamic block after the target: an empty range (the previous one,
        // whose stop search meets the same nothing, decodes to the member's end)
        S.rchunks.clear();
        S.dst_off = WINDOW;
        S.total = 0;
        S.has_trailer = false;
        S.end_map.resize(WINDOW);
        for (uint32_t i = 0; i < WINDOW; i++) S.end_map[i] = (uint16_t)(WM_REF | i);
        std::memset(info, 0, sizeof(*info));
        info->start_bit = info->end_bit = ~0ull;
        std::memcpy(end_map, S.end_map.data(), WINDOW * 2);
        S.ready = true;
        return 0;
    }
    OutTarget tgt{(uint8_t*)c->out.p, c->out.cap, true};
    if ((rc = ensure_out(c, tgt, WINDOW + 4096, 0, err))) return rc;
    const bool continued = byte0 * 8 + start_rel > body_off * 8;
    std::vector<MemberJob> jobs(1);
    MemberJob& j = jobs[0];
    j.len = clen;
    j.body_off = 0;
    j.start_bit = start_rel;
    j.stop_bit = stop_rel;
    j.dst_off = WINDOW;
    j.prefix_len = continued ? WINDOW : 0;  // the window is not known yet: all of it may be referenced
    j.len_prev = continued ? 1 : 0;         // marks the first member as continued from earlier ranges
    j.check_crc = false;
    j.report_off = byte0;
    j.split = &S;
    if ((rc = members_route(c, d_span, jobs, tgt, err))) return rc;
    if (j.rc) {
        *err = j.err;
        return j.rc;
    }
    const auto body_bit = [&](uint64_t r) { return r + byte0 * 8 - body_off * 8; };
    info->start_bit = body_bit(start_rel);
    info->end_bit = body_bit(S.end_bit);
    info->out_len = S.total;
    info->has_trailer = S.has_trailer ? 1u : 0u;
    info->crc = S.crc;
    info->isize = S.isize;
    info->trailer_byte = S.trailer_byte;
    std::memcpy(end_map, S.end_map.data(), WINDOW * 2);
    return 0;
}

int rrg_gpu_split_finish(rrg_ctx* c, const uint8_t* window, size_t window_len, rrg_sink_fn sink, void* user,
                         uint32_t* crc_out, uint64_t* len_out, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    if (!c || !c->split || !c->split->ready || window_len > WINDOW || (window_len && !window)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "no split range awaits its window");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    SplitState& S = *c->split;
    S.ready = false;
    uint8_t* out = (uint8_t*)c->out.p;
    if (window_len)
        CK(cudaMemcpyAsync(out + S.dst_off - window_len, window, window_len, cudaMemcpyHostToDevice, c->stream));
    // the continued first member now starts window_len bytes before the range
    for (ResolveChunk& rc : S.rchunks)
        if (rc.member_start == S.dst_off - WINDOW) rc.member_start = S.dst_off - window_len;
    if (!S.total) {
        if (crc_out) *crc_out = 0;
        if (len_out) *len_out = 0;
        return 0;
    }
    int rc = run_resolve(c, S.rchunks, out, err);
    if (rc) return rc;
    std::vector<int32_t> stv;
    std::vector<uint32_t> got;
    std::vector<uint64_t> glen;
    const uint64_t members = c->st.members;
    if ((rc = crc_spans(c, out, {MemberSpan{S.dst_off, S.total, 0, 0, 0}}, stv, got, glen, err))) return rc;
    c->st.members = members;
    if (crc_out) *crc_out = got.empty() ? 0u : got[0];
    if (len_out) *len_out = S.total;
    bool closed = false;
    return deliver(c, out + S.dst_off, S.total, sink, user, &closed, err);
}

int rrg_gpu_find_blocks(rrg_ctx* c, const uint8_t* d_body, size_t body_len, const uint64_t* targets,
                        const uint64_t* limits, uint64_t* found, size_t n, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || (n && (!targets || !limits || !found))) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    int rc = upload_tables(c, err);
    if (rc || !n) return rc;
    CK(dgrow(c->targets, n * 8));
    CK(dgrow(c->limits, n * 8));
    CK(dgrow(c->found, n * 8));
    CK(dgrow(c->queue, 16));
    CK(cudaMemcpyAsync(c->targets.p, targets, n * 8, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->limits.p, limits, n * 8, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->queue.p, 0, 16, c->stream));
    FindArgs F{d_body, body_len, (const uint64_t*)c->targets.p, (const uint64_t*)c->limits.p, (uint64_t*)c->found.p,
               (uint32_t)n, (uint32_t*)c->queue.p, (const uint8_t*)c->next_lut.p, c->finder_tile};
    const uint32_t W = 4;
    RRG_LAUNCH(k_find_blocks, persistent_blocks(c, 4, n, W), W * 32, W * sizeof(FindSmem), c->stream, F);
    LAUNCHED(c);
    CK(cudaMemcpyAsync(found, c->found.p, n * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int rrg_gpu_crc32(rrg_ctx* c, const uint8_t* d_data, size_t len, uint32_t* crc_out, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || !crc_out || (len && !d_data)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    int rc = upload_tables(c, err);
    if (rc) return rc;
    // a single member spanning the buffer, checked against a dummy trailer:
    // the computed CRC is reported back through got_crc
    std::vector<MemberSpan> one{MemberSpan{0, len, 0, (uint32_t)len, 0}};
    rrg_error tmp;
    rc = check_members(c, d_data, one, 0, &tmp);
    if (rc && rc != RRG_ERR_CRC_MISMATCH && rc != RRG_ERR_ISIZE_MISMATCH) {
        if (err) *err = tmp;
        return rc;
    }
    CK(cudaMemcpy(crc_out, c->got_crc.p, 4, cudaMemcpyDeviceToHost));
    return 0;
}

int rrg_gpu_resolve_markers(rrg_ctx* c, uint8_t* d_bytes, size_t n_bytes, const uint32_t* d_out_pos,
                            const uint16_t* d_prefix_offset, size_t n_markers, const uint8_t* d_tail, size_t tail_len,
                            rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || (n_markers && (!d_bytes || !d_out_pos || !d_prefix_offset))) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    if (!n_markers) return 0;
    // resolve_markers (speculative.rs:175-213) on the device: one thread per
    // marker writes its byte from the tail; an offset past the tail or a
    // position past the bytes fails the call
    CK(dgrow(c->rerr, 16));
    CK(cudaMemsetAsync(c->rerr.p, 0, 16, c->stream));
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n_markers + 255) / 256, c->n_sm * 16ull));
    RRG_LAUNCH(k_resolve_list, grid, 256, 0, c->stream, d_bytes, (uint64_t)n_bytes, d_out_pos, d_prefix_offset,
               (uint64_t)n_markers, d_tail, (uint64_t)tail_len, (uint32_t*)c->rerr.p);
    LAUNCHED(c);
    uint32_t bad = 0;
    CK(cudaMemcpyAsync(&bad, c->rerr.p, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (bad) {
        set_err(err, RRG_ERR_DEFLATE_INVALID, "%s", msg_text(MSG_MARKER_WINDOW));
        return RRG_ERR_DEFLATE_INVALID;
    }
    return 0;
}

int rrg_gpu_decode_chunk(rrg_ctx* c, const uint8_t* d_body, size_t body_len, uint64_t start_bit, uint64_t end_bit_hint,
                         uint8_t* bytes, size_t* n_bytes, uint32_t* marker_pos, uint16_t* marker_off, size_t* n_markers,
                         uint64_t* actual_end_bit, int32_t* final_block, rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    if (!c || !d_body || !n_bytes || !n_markers) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (err) std::memset(err, 0, sizeof(*err));
    int rc = upload_tables(c, err);
    if (rc) return rc;
    const uint64_t cap_b = *n_bytes, cap_m = *n_markers;
    uint64_t cap = round8(std::max<uint64_t>(cap_b, 64));
    CK(dgrow(c->cells, cap * 2 + 64));
    std::vector<ChunkItem> items{ChunkItem{0, body_len, start_bit, end_bit_hint, 0, cap, ITEM_MARKERS, 0}};
    std::vector<ChunkResult> res;
    std::vector<MemberRec> mr;
    mr.reserve(4096);
    rc = launch_inflate(c, d_body, items, false, c->cells.p, res, &mr, err);
    if (rc) return rc;
    const ChunkResult& r = res[0];
    if (r.status == DS_OVERFLOW) {
        *n_bytes = r.n_cells;
        set_err(err, RRG_ERR_CAPACITY, "chunk needs %llu bytes", (unsigned long long)r.n_cells);
        return RRG_ERR_CAPACITY;
    }
    if (r.status) return status_err(err, r.status, r.msg, r.err_bit / 8);
    std::vector<uint16_t> cells(r.n_cells);
    if (r.n_cells) CK(cudaMemcpy(cells.data(), c->cells.p, r.n_cells * 2, cudaMemcpyDeviceToHost));
    uint64_t nm = 0;
    for (uint64_t i = 0; i < r.n_cells; i++) {
        uint16_t v = cells[i];
        if (v & MARKER16) {
            if (nm < cap_m) {
                if (marker_pos) marker_pos[nm] = (uint32_t)i;
                if (marker_off) marker_off[nm] = (uint16_t)(v & 0x7fff);
            }
            nm++;
            if (bytes && i < cap_b) bytes[i] = 0;
        } else if (bytes && i < cap_b) {
            bytes[i] = (uint8_t)v;
        }
    }
    *n_bytes = r.n_cells;
    *n_markers = nm;
    if (actual_end_bit) *actual_end_bit = r.actual_end_bit;
    if (final_block) *final_block = r.final_block;
    if (nm > cap_m) {
        set_err(err, RRG_ERR_CAPACITY, "chunk has %llu markers", (unsigned long long)nm);
        return RRG_ERR_CAPACITY;
    }
    return 0;
}

int rrg_gpu_serve_start(rrg_ctx* c, uint32_t engines, uint32_t max_ready, rrg_error* err) {
    if (!c) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null context");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    return serve_start(c, engines, max_ready, err);
}

void rrg_gpu_serve_stop(rrg_ctx* c) {
    if (c) serve_stop(c);
}

int rrg_gpu_serve_stats(rrg_ctx* c, rrg_serve_stats* out) {
    if (!c || !out) return RRG_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (!c->srv) return 0;
    std::lock_guard<std::mutex> g(c->srv->mu);
    *out = c->srv->stats;
    out->in_use_bytes = c->srv->in_use;
    out->budget_bytes = c->srv->budget;
    out->waiting = c->srv->waiting.size();
    return 0;
}

static int64_t submit_impl(rrg_ctx* c, const uint8_t* data, size_t len, bool copy, rrg_error* err) {
    if (!c || (!data && len)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return -1;
    }
    const double t0 = now_ms();
    if (!c->srv) {
        int rc = serve_start(c, 0, 0, err);
        if (rc) return -1;
    }
    Server* S = c->srv;
    Server::Req r;
    r.t_submit = t0;
    r.len = len;
    if (copy) {
        r.copy.assign(data, data + len);
        r.bytes = r.copy.data();
    } else {
        r.bytes = data;
    }
    std::lock_guard<std::mutex> g(S->mu);
    r.id = S->next_id++;
    const int64_t id = r.id;
    S->waiting.push_back(std::move(r));
    S->outstanding++;
    S->stats.submitted++;
    S->cv_work.notify_all();
    return id;
}

int64_t rrg_gpu_submit(rrg_ctx* c, const uint8_t* data, size_t len, rrg_error* err) {
    return submit_impl(c, data, len, true, err);
}

int64_t rrg_gpu_submit_nocopy(rrg_ctx* c, const uint8_t* data, size_t len, rrg_error* err) {
    return submit_impl(c, data, len, false, err);
}

int rrg_gpu_poll(rrg_ctx* c, int64_t* request_id, uint8_t** out, size_t* out_len, int32_t* status, double* latency_ms,
                 int32_t timeout_ms, rrg_error* err) {
    if (!c || !request_id || !out || !out_len || !status) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return -RRG_ERR_INVALID_ARGUMENT;
    }
    if (!c->srv) return 0;
    Server* S = c->srv;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->done.empty() && timeout_ms > 0)
        S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !S->done.empty(); });
    if (S->done.empty()) return 0;
    Server::Done d = S->done.front();
    S->done.pop_front();
    S->outstanding--;
    S->cv_work.notify_all();  // room in the completion queue
    lk.unlock();
    *request_id = d.id;
    *out = d.out;
    *out_len = d.len;
    *status = d.status;
    if (latency_ms) *latency_ms = d.latency_ms;
    if (err) *err = d.err;
    return 1;
}

int64_t rrg_gpu_pending(rrg_ctx* c) {
    if (!c) return -1;
    if (!c->srv) return 0;
    std::lock_guard<std::mutex> g(c->srv->mu);
    return c->srv->outstanding;
}

void rrg_gpu_free(void* p) { result_free(p); }

const char* rrg_gpu_version(void) { return "rrg-gpu 0.1 (sm_100a)"; }

uint64_t rrg_gpu_kernel_launch_count(void) { return g_launches.load(); }

}  // extern "C"

// ====================================================================== allocation-free CRC32
// For callers that cannot let a library allocate device memory: code that
// owns all of the GPU's memory through its own pool allocator (a cudaMalloc
// behind its back can fail once the pool has reserved the device, and the
// matching cudaFree synchronises the whole device), or a latency-critical
// serving path that must not stall on allocation. Everything this entry point
// needs beyond the caller's input and output lives in one fixed, file-scope
// device array, so a call allocates nothing.
namespace {

constexpr uint64_t NA_PIECE = 256 * 1024;             // bytes per CRC piece
constexpr uint32_t NA_MAX_PIECES = 16384;             // => at most 4 GiB per call
constexpr uint64_t NA_MAX_BYTES = NA_PIECE * NA_MAX_PIECES;

struct NoAllocScratch {
    uint32_t table[8 * 256];                  // slice-by-8 CRC table
    CrcPiece pieces[NA_MAX_PIECES];
    uint32_t piece_crc[NA_MAX_PIECES];
    uint32_t member_piece_start[2];
    uint32_t expected_crc, expected_isize, got_crc;
    int32_t status;
    uint64_t got_len;
};

}  // namespace

// The scratch every call shares (about 336 KB, held by every GPU that loads
// this library until the process exits).
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {

std::mutex g_noalloc_mu;
// Per device ordinal: the scratch's device address and the id of the CUDA
// context it was set up in. A new context on that device (after
// cudaDeviceReset, for example) holds a fresh copy of the array without the
// tables, so the set-up runs again there.
struct NoAllocDev {
    NoAllocScratch* p = nullptr;
    unsigned long long ctx_id = 0;
};
NoAllocDev g_noalloc_dev[64];

// Unique id of the calling thread's current context (cuCtxGetCurrent and
// cuCtxGetId, reached through the runtime's driver entry points); 0 when no
// context is current or the driver does not provide them.
unsigned long long current_ctx_id() {
#ifdef RRG_EMU
    return 1;
#else
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)f;
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
#endif
}

// Piece descriptors for one buffer; also resets the fields k_crc_members reads.
__global__ void k_noalloc_pieces(NoAllocScratch* S, uint64_t len, uint32_t n_pieces) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pieces; i += gridDim.x * blockDim.x) {
        const uint64_t o = (uint64_t)i * NA_PIECE;
        S->pieces[i] = CrcPiece{o, len - o < NA_PIECE ? len - o : NA_PIECE};
        S->piece_crc[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->member_piece_start[0] = 0;
        S->member_piece_start[1] = n_pieces;
        S->expected_crc = 0;
        S->expected_isize = (uint32_t)len;
        S->got_crc = 0;
        S->got_len = 0;
        S->status = 0;
    }
}

// First call on the current device (or in a new context on it): find the
// scratch's device address and load the CRC tables into it and into constant
// memory.
int noalloc_setup(int dev, NoAllocScratch** out, rrg_error* err) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (dev < 0 || dev >= 64) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "device ordinal %d out of range", dev);
        return RRG_ERR_INVALID_ARGUMENT;
    }
    NoAllocDev& D = g_noalloc_dev[dev];
    // before the runtime's first call on this device no context is current
    // (id 0); the set-up below creates it
    const unsigned long long id = current_ctx_id();
    if (!D.p || (id != 0 && id != D.ctx_id)) {
        std::call_once(g_tab_once, init_tables);
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        CK(cudaMemcpy(p, g_crc_tab, sizeof(g_crc_tab), cudaMemcpyHostToDevice));
        CK(cudaMemcpyToSymbol(c_x2k, g_x2k, sizeof(g_x2k)));
        D.p = (NoAllocScratch*)p;
        D.ctx_id = current_ctx_id();
    }
    *out = D.p;
    return 0;
}

}  // namespace

extern "C" int rrg_gpu_crc32_noalloc(const uint8_t* d_data, size_t len, uint32_t* crc_out, void* stream,
                                     rrg_error* err) {
    rrg_error local_err;
    if (!err) err = &local_err;
    std::memset(err, 0, sizeof(*err));
    if (!crc_out || (len && !d_data)) {
        set_err(err, RRG_ERR_INVALID_ARGUMENT, "null argument");
        return RRG_ERR_INVALID_ARGUMENT;
    }
    if (len > NA_MAX_BYTES) {
        set_err(err, RRG_ERR_CAPACITY, "rrg_gpu_crc32_noalloc handles at most %llu bytes per call, got %llu",
                (unsigned long long)NA_MAX_BYTES, (unsigned long long)len);
        return RRG_ERR_CAPACITY;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    NoAllocScratch* S = nullptr;
    int rc = noalloc_setup(dev, &S, err);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t np = (uint32_t)((len + NA_PIECE - 1) / NA_PIECE);
    RRG_LAUNCH(k_noalloc_pieces, (np + 255) / 256 + 1, 256, 0, st, S, (uint64_t)len, np);
    g_launches.fetch_add(1);
    CK(cudaGetLastError());
    if (np) {
        CrcArgs A{d_data, S->pieces, np, S->piece_crc, S->table};
        RRG_LAUNCH(k_crc_pieces, std::min<uint32_t>(np, 148u * 8u), CRC_THREADS, 0, st, A);
        g_launches.fetch_add(1);
        CK(cudaGetLastError());
    }
    CrcMemberArgs B{S->pieces, S->piece_crc, S->member_piece_start, 1, &S->expected_crc, &S->expected_isize,
                    &S->got_crc, &S->got_len, &S->status};
    RRG_LAUNCH(k_crc_members, 1, 32, 0, st, B);
    g_launches.fetch_add(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(crc_out, &S->got_crc, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

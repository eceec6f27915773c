// cuda_emu.h — CPU emulation of the CUDA subset used by rusty_rapidgzip_b200/csrc.
//
// TEST INFRASTRUCTURE ONLY. Lets the unit tests compile the product's kernel
// and host sources with g++ (-DRRG_EMU -include cuda_emu.h) and run them on
// the CPU: every thread of a block is a user-level fiber on the launching
// thread; warp shuffles, ballots, matches and __syncwarp go through a per-warp
// exchange with a 32-party barrier; __syncthreads is a block barrier; blocks
// of a launch run one after another. Device memory is host memory. The resulting library is used only by
// `-m "not gpu"` tests and never stands in for the GPU build.
#pragma once
#include <ucontext.h>

#include <cstdio>
#include <deque>
#include <mutex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __constant__
#define __shared__ static
#define __launch_bounds__(...)
#define __align__(n) __attribute__((aligned(n)))

struct dim3 {
    unsigned x = 1, y = 1, z = 1;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct __attribute__((aligned(8))) uint2 {
    unsigned x, y;
};
struct __attribute__((aligned(16))) uint4 {
    unsigned x, y, z, w;
};
inline uint2 make_uint2(unsigned x, unsigned y) { return uint2{x, y}; }
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }

typedef int cudaError_t;
typedef void* cudaStream_t;
typedef struct emu_event* cudaEvent_t;
enum : int { cudaSuccess = 0, cudaErrorMemoryAllocation = 2, cudaErrorInvalidValue = 1 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice, cudaMemcpyDefault };
enum cudaDeviceAttr { cudaDevAttrMultiProcessorCount = 16, cudaDevAttrMaxSharedMemoryPerBlockOptin = 97 };
enum cudaFuncAttribute { cudaFuncAttributeMaxDynamicSharedMemorySize = 8 };
#define cudaStreamNonBlocking 1u
#define cudaEventDisableTiming 2u

namespace emu {

// ---- fibers. The threads of a block run as user-level contexts on the
// launching thread, one at a time; a barrier parks the calling fiber until the
// last one arrives, which releases them all. No OS threads, no futexes.
struct Fiber {
    ucontext_t ctx;
    char* stack = nullptr;
    unsigned tid = 0;
    bool parked = false;
};
struct Sched {
    ucontext_t main;
    Fiber* cur = nullptr;
    std::deque<Fiber*> ready;
    std::function<void(unsigned)> enter;  // sets the fiber's identity, then runs the kernel body
};
inline thread_local Sched* t_sched = nullptr;

struct Barrier {
    unsigned needed, count = 0;
    std::vector<Fiber*> parked;
    explicit Barrier(unsigned n) : needed(n) {}
    void arrive_and_wait() {
        Sched* s = t_sched;
        if (++count == needed) {  // the last arrival releases the others and continues
            count = 0;
            for (Fiber* f : parked) {
                f->parked = false;
                s->ready.push_back(f);
            }
            parked.clear();
            return;
        }
        Fiber* me = s->cur;
        me->parked = true;
        parked.push_back(me);
        swapcontext(&me->ctx, &s->main);
    }
};

struct Warp {
    Barrier bar{32};
    uint64_t slot[32];
};
struct Block {
    std::unique_ptr<Barrier> bar;
    std::vector<std::unique_ptr<Warp>> warps;
};
inline thread_local Block* t_block = nullptr;
inline thread_local Warp* t_warp = nullptr;
inline thread_local dim3 t_tid, t_bid, t_bdim, t_gdim;
inline std::vector<unsigned char>& dyn_buf() {
    static std::vector<unsigned char> b;
    return b;
}
inline unsigned char* dyn_smem() { return dyn_buf().data(); }
inline std::mutex& launch_mutex() {
    static std::mutex m;
    return m;
}

constexpr size_t FIBER_STACK = 256 << 10;

inline void fiber_main() {
    Sched* s = t_sched;
    s->enter(s->cur->tid);
    // returning ends the fiber: uc_link resumes the scheduler
}

// Launches from several host threads are serialised (shared memory is static).
inline void launch(dim3 grid, dim3 block, size_t smem, const std::function<void()>& body) {
    std::lock_guard<std::mutex> guard(launch_mutex());
    static std::vector<char*> stacks;  // reused across launches
    const unsigned nthreads = block.x;
    auto& buf = dyn_buf();
    if (buf.size() < smem + 64) buf.assign(smem + 64, 0);
    while (stacks.size() < nthreads) stacks.push_back(static_cast<char*>(std::malloc(FIBER_STACK)));
    std::vector<Fiber> fib(nthreads);
    Sched sched;
    Sched* prev = t_sched;
    t_sched = &sched;
    for (unsigned b = 0; b < grid.x; b++) {
        Block blk;
        blk.bar = std::make_unique<Barrier>(nthreads);
        for (unsigned w = 0; w < (nthreads + 31) / 32; w++) blk.warps.push_back(std::make_unique<Warp>());
        sched.enter = [&, b](unsigned t) {
            t_block = &blk;
            t_warp = blk.warps[t / 32].get();
            t_tid = dim3(t);
            t_bid = dim3(b);
            t_bdim = block;
            t_gdim = grid;
            body();
        };
        for (unsigned t = 0; t < nthreads; t++) {
            Fiber& f = fib[t];
            f.tid = t;
            f.parked = false;
            f.stack = stacks[t];
            getcontext(&f.ctx);
            f.ctx.uc_stack.ss_sp = f.stack;
            f.ctx.uc_stack.ss_size = FIBER_STACK;
            f.ctx.uc_link = &sched.main;
            makecontext(&f.ctx, fiber_main, 0);
            sched.ready.push_back(&f);
        }
        unsigned finished = 0;
        while (!sched.ready.empty()) {
            Fiber* f = sched.ready.front();
            sched.ready.pop_front();
            sched.cur = f;
            // the identity of the fiber being resumed (thread-locals are per OS thread)
            t_block = &blk;
            t_warp = blk.warps[f->tid / 32].get();
            t_tid = dim3(f->tid);
            t_bid = dim3(b);
            t_bdim = block;
            t_gdim = grid;
            swapcontext(&sched.main, &f->ctx);
            // back here when the fiber parked at a barrier or finished
            if (!f->parked) finished++;
        }
        if (finished != nthreads) {
            std::fprintf(stderr, "cuda_emu: a barrier was never completed (%u of %u threads finished)\n", finished,
                         nthreads);
            std::abort();
        }
    }
    t_sched = prev;
}

}  // namespace emu

#define threadIdx (emu::t_tid)
#define blockIdx (emu::t_bid)
#define blockDim (emu::t_bdim)
#define gridDim (emu::t_gdim)

inline void __syncthreads() { emu::t_block->bar->arrive_and_wait(); }
inline void __syncwarp(unsigned = 0xffffffffu) { emu::t_warp->bar.arrive_and_wait(); }

template <class T>
inline T emu_exchange(T v, int src) {
    static_assert(sizeof(T) <= 8, "shuffle width");
    emu::Warp* w = emu::t_warp;
    int lane = emu::t_tid.x & 31;
    uint64_t raw = 0;
    std::memcpy(&raw, &v, sizeof(T));
    w->slot[lane] = raw;
    w->bar.arrive_and_wait();
    uint64_t got = w->slot[src & 31];
    w->bar.arrive_and_wait();
    T r;
    std::memcpy(&r, &got, sizeof(T));
    return r;
}
template <class T>
inline T __shfl_sync(unsigned, T v, int src) {
    return emu_exchange(v, src);
}
template <class T>
inline T __shfl_xor_sync(unsigned, T v, int m) {
    return emu_exchange(v, (int)(emu::t_tid.x & 31) ^ m);
}
template <class T>
inline T __shfl_up_sync(unsigned, T v, unsigned d) {
    int lane = emu::t_tid.x & 31;
    int src = lane - (int)d >= 0 ? lane - (int)d : lane;
    return emu_exchange(v, src);
}
template <class T>
inline T __shfl_down_sync(unsigned, T v, unsigned d) {
    int lane = emu::t_tid.x & 31;
    int src = lane + (int)d < 32 ? lane + (int)d : lane;
    return emu_exchange(v, src);
}
inline unsigned __ballot_sync(unsigned, int pred) {
    emu::Warp* w = emu::t_warp;
    int lane = emu::t_tid.x & 31;
    w->slot[lane] = pred ? 1 : 0;
    w->bar.arrive_and_wait();
    unsigned m = 0;
    for (int i = 0; i < 32; i++)
        if (w->slot[i]) m |= 1u << i;
    w->bar.arrive_and_wait();
    return m;
}
inline unsigned __match_any_sync(unsigned, unsigned v) {
    emu::Warp* w = emu::t_warp;
    int lane = emu::t_tid.x & 31;
    w->slot[lane] = v;
    w->bar.arrive_and_wait();
    unsigned m = 0;
    for (int i = 0; i < 32; i++)
        if (w->slot[i] == v) m |= 1u << i;
    w->bar.arrive_and_wait();
    return m;
}
inline unsigned __reduce_or_sync(unsigned, unsigned v) {
    emu::Warp* w = emu::t_warp;
    int lane = emu::t_tid.x & 31;
    w->slot[lane] = v;
    w->bar.arrive_and_wait();
    unsigned m = 0;
    for (int i = 0; i < 32; i++) m |= (unsigned)w->slot[i];
    w->bar.arrive_and_wait();
    return m;
}
inline int __any_sync(unsigned m, int pred) { return __ballot_sync(m, pred) != 0; }
inline unsigned __reduce_min_sync(unsigned, unsigned v) {
    emu::Warp* w = emu::t_warp;
    int lane = emu::t_tid.x & 31;
    w->slot[lane] = v;
    w->bar.arrive_and_wait();
    unsigned m = 0xffffffffu;
    for (int i = 0; i < 32; i++) m = (unsigned)w->slot[i] < m ? (unsigned)w->slot[i] : m;
    w->bar.arrive_and_wait();
    return m;
}
inline int __popc(unsigned v) { return __builtin_popcount(v); }
inline unsigned __byte_perm(unsigned x, unsigned y, unsigned s) {  // PTX prmt, default mode
    const uint64_t v = ((uint64_t)y << 32) | x;
    unsigned r = 0;
    for (int i = 0; i < 4; i++) r |= (unsigned)((v >> (8 * ((s >> (4 * i)) & 7))) & 0xff) << (8 * i);
    return r;
}
inline int __ffs(int v) { return __builtin_ffs(v); }
inline unsigned __funnelshift_r(unsigned lo, unsigned hi, unsigned sh) {
    sh &= 31;
    return sh ? (lo >> sh) | (hi << (32 - sh)) : lo;
}
inline unsigned __funnelshift_lc(unsigned lo, unsigned hi, unsigned sh) {
    if (sh > 32) sh = 32;
    const unsigned long long v = ((unsigned long long)hi << 32) | lo;
    return (unsigned)((v << sh) >> 32);
}
inline unsigned __brev(unsigned v) {
    unsigned r = 0;
    for (int i = 0; i < 32; i++) r |= ((v >> i) & 1u) << (31 - i);
    return r;
}
template <class T>
inline T __ldg(const T* p) {
    return *p;
}
template <typename T>
inline T __ldcg(const T* p) {
    return *p;
}
inline unsigned atomicAdd(unsigned* p, unsigned v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
    return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
inline unsigned atomicOr(unsigned* p, unsigned v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicMin(unsigned* p, unsigned v) {
    unsigned cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return cur;
}
inline unsigned long long atomicMin(unsigned long long* p, unsigned long long v) {
    unsigned long long cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return cur;
}
inline unsigned atomicCAS(unsigned* p, unsigned cmp, unsigned v) {
    __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}

// ---- runtime API (device memory is host memory)
inline cudaError_t cudaMalloc(void** p, size_t n) {
#ifdef RRG_STRICT_ALLOC
    *p = std::malloc(n ? n : 1);  // exact size (16-byte aligned): an address checker sees overruns
#else
    *p = std::aligned_alloc(256, (n + 255) & ~(size_t)255);
#endif
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
inline cudaError_t cudaMallocHost(void** p, size_t n) { return cudaMalloc(p, n); }
inline cudaError_t cudaMemGetInfo(size_t* free_b, size_t* total_b) {  // a nominal 8 GiB device
    *free_b = 8ull << 30;
    *total_b = 8ull << 30;
    return cudaSuccess;
}
inline cudaError_t cudaFreeHost(void* p) { return cudaFree(p); }
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
    if (n) std::memmove(d, s, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind k, cudaStream_t = nullptr) {
    return cudaMemcpy(d, s, n, k);
}
inline cudaError_t cudaMemset(void* d, int v, size_t n) {
    std::memset(d, v, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemsetAsync(void* d, int v, size_t n, cudaStream_t = nullptr) { return cudaMemset(d, v, n); }
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T& sym, const void* src, size_t n, size_t off = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
    std::memcpy((char*)&sym + off, src, n);
    return cudaSuccess;
}
template <class T>
inline cudaError_t cudaGetSymbolAddress(void** p, T& sym) {
    *p = (void*)&sym;
    return cudaSuccess;
}
inline cudaError_t cudaStreamCreateWithFlags(cudaStream_t* s, unsigned) {
    *s = (void*)0x1;
    return cudaSuccess;
}
inline cudaError_t cudaStreamCreateWithPriority(cudaStream_t* s, unsigned, int) {
    *s = (void*)0x1;
    return cudaSuccess;
}
inline cudaError_t cudaDeviceGetStreamPriorityRange(int* least, int* greatest) {
    *least = 0;
    *greatest = -1;
    return cudaSuccess;
}
inline cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
struct emu_event {
    int x;
};
inline cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned) {
    *e = new emu_event{0};
    return cudaSuccess;
}
inline cudaError_t cudaEventCreate(cudaEvent_t* e) {
    *e = new emu_event{0};
    return cudaSuccess;
}
inline cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t = nullptr) { return cudaSuccess; }
enum { cudaEventRecordDefault = 0, cudaEventRecordExternal = 1 };
enum cudaStreamCaptureStatus { cudaStreamCaptureStatusNone = 0, cudaStreamCaptureStatusActive = 1 };
inline cudaError_t cudaStreamIsCapturing(cudaStream_t, cudaStreamCaptureStatus* st) {
    *st = cudaStreamCaptureStatusNone;
    return cudaSuccess;
}
inline cudaError_t cudaEventRecordWithFlags(cudaEvent_t, cudaStream_t = nullptr, unsigned = 0) { return cudaSuccess; }
inline cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned = 0) { return cudaSuccess; }
inline cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) {
    *ms = 0.f;
    return cudaSuccess;
}
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaEventDestroy(cudaEvent_t e) {
    delete e;
    return cudaSuccess;
}
inline cudaError_t cudaGetDevice(int* d) {
    *d = 0;
    return cudaSuccess;
}
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr a, int) {
    // RRG_EMU_SMS: the SM count to report (default 2), so the CPU build can
    // lay out work as a full-size device would
    static const int sms = getenv("RRG_EMU_SMS") ? atoi(getenv("RRG_EMU_SMS")) : 2;
    *v = a == cudaDevAttrMultiProcessorCount ? sms : 232448;
    return cudaSuccess;
}
template <class F>
inline cudaError_t cudaFuncSetAttribute(F, cudaFuncAttribute, int) {
    return cudaSuccess;
}
template <class F>
inline cudaError_t cudaOccupancyMaxActiveBlocksPerMultiprocessor(int* n, F, int, size_t) {
    *n = 1;
    return cudaSuccess;
}
inline const char* cudaGetErrorString(cudaError_t e) { return e ? "emulated error" : "no error"; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }

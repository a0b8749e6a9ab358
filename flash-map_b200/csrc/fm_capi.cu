// fm_capi.cu -- the extern "C" boundary of libflashmap_b200.so: table
// lifetime, host<->device transfers, the round loop of the mutating
// operations, error mapping and len bookkeeping.  Replaces the reference's
// src/gpu.rs (bajpainaman/flash-map 0.5.0); see include/flashmap_b200.h.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/flashmap_b200.h"
#include "fm_internal.h"

using fm::Ctl;
using fm::OpScratch;

namespace {

thread_local std::string tl_err;

int fail(int code, const std::string& msg) {
    tl_err = msg;
    return code;
}

int cuda_fail(int code, const char* what, cudaError_t e) {
    return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Host-side failure injection (fm_inject_fault): one armed site and the
// number of passes through it still to let by.  The failing CUDA call is not
// made; the site returns the error that call would have returned.
std::atomic<uint32_t> g_fault_site{FM_FAULT_NONE};
std::atomic<int64_t> g_fault_after{-1};

bool fault_at(uint32_t site) {
    if (g_fault_site.load(std::memory_order_relaxed) != site) return false;
    if (g_fault_after.fetch_sub(1) != 0) return false;
    g_fault_site.store(FM_FAULT_NONE);
    return true;
}

// cudaMalloc behind the allocation fault site.
cudaError_t dev_alloc(void** p, size_t bytes) {
    if (fault_at(FM_FAULT_ALLOC)) return cudaErrorMemoryAllocation;
    return cudaMalloc(p, bytes);
}

// cudaMemcpyAsync behind the transfer fault site.
cudaError_t copy_async(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
    if (fault_at(FM_FAULT_TRANSFER)) return cudaErrorInvalidValue;
    return cudaMemcpyAsync(dst, src, bytes, kind, s);
}

// Device chunk of one mutating call: op indices are u32 and 0xFFFFFFFF marks
// an idle segment slot, so a call is split into sequential chunks (which is
// exactly the sequential semantics) of at most this many operations.
constexpr uint64_t OP_CHUNK = 1ull << 30;
#ifndef FM_DIRECT_LOAD
#define FM_DIRECT_LOAD 0.97  // load from which an insert call skips the rounds
#endif
// Queue mode: an insert of at least FM_QUEUE_INS_OPS keys, or one that can
// take its table to FM_QUEUE_INS_LOAD, runs between persistent launches on the
// direct passes (launch overhead is small beside it, and its components can
// outgrow a warp); from FM_DIRECT_LOAD on it runs on the component path.
#ifndef FM_QUEUE_INS_OPS
#define FM_QUEUE_INS_OPS (1u << 18)
#endif
#ifndef FM_QUEUE_INS_LOAD
#define FM_QUEUE_INS_LOAD 0.9
#endif
// Queue mode: a remove of at least FM_QUEUE_REM_OPS keys runs between
// persistent launches too (the direct passes, then FM_QUEUE_REM_ROUNDS grid
// rounds and the tail for what they leave).
#ifndef FM_QUEUE_REM_OPS
#define FM_QUEUE_REM_OPS (1u << 18)
#endif
// ... and a lookup of at least FM_QUEUE_GET_OPS keys runs as the plain lookup
// kernel between persistent launches (its occupancy there is the tuned one).
#ifndef FM_QUEUE_GET_OPS
#define FM_QUEUE_GET_OPS (1u << 16)
#endif
#ifndef FM_QUEUE_REM_ROUNDS
#define FM_QUEUE_REM_ROUNDS 4u
#endif
#ifndef FM_HANDOFF_LOAD
#define FM_HANDOFF_LOAD 0.9  // load from which the insert tail hands stalled rounds back
#endif

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Host-API pipelining: a host call is split into pieces whose host->device
// copy, kernels and device->host copy overlap with the neighbouring pieces'
// (two streams alternate for get; a copy stream prefetches the next piece of
// a mutating call while the current one runs).  Splitting a mutating batch
// into consecutive pieces keeps the sequential semantics.
constexpr uint64_t HOST_GET_PIECE = 1ull << 19;  // queries per get piece
constexpr uint64_t HOST_MUT_PIECE = 1ull << 16;  // ops per insert/remove piece

struct GetCtx {
    cudaStream_t s[2] = {nullptr, nullptr};
    uint8_t* d_buf[2] = {nullptr, nullptr};
    size_t cap[2] = {0, 0};
};

template <class T>
cudaError_t grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = need + need / 4;
    cudaError_t e = dev_alloc((void**)&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
}

bool aligned(const void* p, uintptr_t a) { return ((uintptr_t)p % a) == 0; }

// Per-table kernel timing: event pairs recorded around each launch while on,
// read back and summed per kernel class by fm_kernel_times.
struct KTimer {
    std::mutex mu;
    bool on = false;
    struct Rec {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> spare;
    double ms[fm::KC_N] = {};
    uint64_t launches[fm::KC_N] = {};

    cudaEvent_t take() {
        if (!spare.empty()) {
            cudaEvent_t e = spare.back();
            spare.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        return cudaEventCreate(&e) == cudaSuccess ? e : nullptr;
    }
    cudaError_t collect() {
        cudaError_t err = cudaSuccess;
        for (const Rec& r : recs) {
            float x = 0.f;
            cudaError_t e = cudaEventSynchronize(r.b);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&x, r.a, r.b);
            if (e == cudaSuccess) {
                ms[r.cls] += x;
                launches[r.cls] += 1;
            } else if (err == cudaSuccess) {
                err = e;
            }
            spare.push_back(r.a);
            spare.push_back(r.b);
        }
        recs.clear();
        return err;
    }
    ~KTimer() {
        for (const Rec& r : recs) cudaEventDestroy(r.a), cudaEventDestroy(r.b);
        for (cudaEvent_t e : spare) cudaEventDestroy(e);
    }
};

thread_local KTimer* tl_timer = nullptr;
thread_local cudaEvent_t tl_open[fm::KC_N] = {};

}  // namespace

bool fm::kt_active() { return tl_timer != nullptr; }

void fm::kt_mark(int cls, bool begin, cudaStream_t s) {
    KTimer* k = tl_timer;
    if (!k || cls < 0 || cls >= KC_N) return;
    std::lock_guard<std::mutex> g(k->mu);
    if (begin) {
        cudaEvent_t e = k->take();
        if (e && cudaEventRecord(e, s) == cudaSuccess) tl_open[cls] = e;
        else if (e) k->spare.push_back(e);
        return;
    }
    cudaEvent_t a = tl_open[cls];
    tl_open[cls] = nullptr;
    if (!a) return;
    cudaEvent_t b = k->take();
    if (b && cudaEventRecord(b, s) == cudaSuccess) {
        k->recs.push_back({cls, a, b});
    } else {
        k->spare.push_back(a);
        if (b) k->spare.push_back(b);
    }
}

struct fm_table {
    int device = 0;
    uint64_t cap = 0, mask = 0;
    uint32_t ksz = 0, vsz = 0, mode = 0;
    fm::Shape shape = fm::SHAPE_GENERIC;
    uint32_t* d_flags = nullptr;
    uint8_t* d_keys = nullptr;
    uint8_t* d_vals = nullptr;
    uint32_t* d_seg_min = nullptr;
    uint32_t* d_seg_cnt = nullptr;
    Ctl* d_ctl = nullptr;
    Ctl* h_ctl = nullptr;    // pinned mirror for readbacks
    uint32_t last_rounds = 0;  // rounds of the last mutating call (statistics)
    std::atomic<uint64_t> len{0};
    cudaStream_t stream = nullptr;  // mutating calls
    std::mutex mu;                  // serialises mutating calls and their scratch
    OpScratch sc{};
    size_t sc_bytes = 0;
    uint8_t* sc_base = nullptr;
    uint8_t* d_in = nullptr;  // host-API staging for mutating calls (two pieces)
    size_t d_in_cap = 0;
    cudaStream_t copy_stream = nullptr;  // prefetch of the next piece
    cudaEvent_t piece_ready[2] = {nullptr, nullptr};
    std::mutex pool_mu;
    std::vector<GetCtx*> pool;
    KTimer timer;

    fm::TableView view() const {
        fm::TableView v;
        v.flags = d_flags;
        v.keys = d_keys;
        v.vals = d_vals;
        v.seg_min = d_seg_min;
        v.seg_cnt = d_seg_cnt;
        v.mask = mask;
        v.ksz = ksz;
        v.vsz = vsz;
        v.hash_mode = mode;
        return v;
    }

    // Shape for a call whose caller-provided buffers are `ptrs`: the
    // vectorised instantiations need 16-byte aligned record arrays.
    fm::Shape shape_for(std::initializer_list<const void*> ptrs) const {
        if (shape == fm::SHAPE_GENERIC) return shape;
        for (const void* p : ptrs)
            if (p && !aligned(p, 16)) return fm::SHAPE_GENERIC;
        return shape;
    }
};

namespace {

// Makes the table's timer current on this thread for one API call.
struct TimerScope {
    KTimer* prev;
    explicit TimerScope(fm_table* t) : prev(tl_timer) { tl_timer = (t && t->timer.on) ? &t->timer : nullptr; }
    ~TimerScope() { tl_timer = prev; }
};

int ensure_scratch(fm_table* t, uint64_t n) {
    if (t->sc.cap_ops >= n) return FM_OK;
    // pend[0], pend[1] (u32) | op_slot (u64) | op_word (u32) | op_flag (u8) | op_pt (PT_MAX u32) |
    // long_list (u32) per op, then the component buffer and the remove chunk summaries (per table)
    const uint64_t per_op = 4 + 4 + 8 + 4 + 1 + 4 * fm::PT_MAX + 4;
    const uint64_t want = n + n / 4 + 1024;
    const size_t bytes = (size_t)(want * per_op + 9 * 256 + fm::cmp_bytes(t->mask) + 4 * fm::rsum_words(t->mask));
    if (t->sc_base) cudaFree(t->sc_base);
    t->sc_base = nullptr;
    t->sc = OpScratch{};
    cudaError_t e = dev_alloc((void**)&t->sc_base, bytes);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_GPU_ALLOC, "scratch allocation", e);
    uint8_t* p = t->sc_base;
    auto carve = [&](size_t b) {
        uint8_t* r = p;
        p += (b + 255) & ~(size_t)255;
        return r;
    };
    t->sc.op_slot = (uint64_t*)carve(want * 8);
    t->sc.pend[0] = (uint32_t*)carve(want * 4);
    t->sc.pend[1] = (uint32_t*)carve(want * 4);
    t->sc.op_word = (uint32_t*)carve(want * 4);
    t->sc.op_pt = (uint32_t*)carve(want * 4 * fm::PT_MAX);
    t->sc.op_flag = carve(want);
    t->sc.long_list = (uint32_t*)carve(want * 4);
    t->sc.comp = carve(fm::cmp_bytes(t->mask));
    t->sc.rsum = (uint32_t*)carve(4 * fm::rsum_words(t->mask));
    t->sc.cap_ops = want;
    t->sc_bytes = bytes;
    // op_word doubles as the insert inflow bound: idle value 0xFFFFFFFF.
    e = cudaMemsetAsync(t->sc.op_word, 0xFF, want * 4, t->stream);
    // the remove chunk marks: IDLE between calls
    if (e == cudaSuccess) e = cudaMemsetAsync(t->sc.rsum, 0xFF, 4 * fm::rsum_words(t->mask), t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_GPU_ALLOC, "scratch init", e);
    return FM_OK;
}

// The least op index marking each 32-slot chunk (the second half of the
// remove summaries) back to idle: a remove that fails part way can leave
// marks set, and a stale mark below an op's index would block that op in
// every later remove.
cudaError_t reset_rsum_marks(fm_table* t, cudaStream_t s) {
    if (!t->sc.rsum) return cudaSuccess;
    const uint64_t nch = fm::rsum_chunks(t->mask);
    return cudaMemsetAsync(t->sc.rsum + nch, 0xFF, nch * 4, s);
}

// After a failed call the segment registrations and the per-op scratch may be
// left set; put every one of them back to idle.
void recover(fm_table* t, cudaStream_t s) {
    cudaMemsetAsync(t->d_seg_min, 0xFF, t->cap * 4, s);
    cudaMemsetAsync(t->d_seg_cnt, 0, t->cap * 4, s);
    if (t->sc.op_word) cudaMemsetAsync(t->sc.op_word, 0xFF, t->sc.cap_ops * 4, s);
    reset_rsum_marks(t, s);
    cudaStreamSynchronize(s);
}

// The round driver shared by insert and remove.  Each pass launches two
// grid-wide rounds and the single-block tail back to back, then reads the
// control block once: a zero pending count for the next round means done.
// Counts, lists and per-round flags stay in device memory between rounds.
int run_rounds_inner(fm_table* t, bool insert, const uint8_t* d_k, const uint8_t* d_v, uint64_t n,
                     cudaStream_t s, uint64_t* out_count, uint32_t* err_bits) {
    uint64_t total = 0;
    *err_bits = 0;
    const fm::Shape sh = t->shape_for({d_k, d_v});
    int rc = ensure_scratch(t, n < OP_CHUNK ? n : OP_CHUNK);
    if (rc) return rc;
    fm::TableView v = t->view();
    for (uint64_t base = 0; base < n; base += OP_CHUNK) {
        const uint32_t m = (uint32_t)((n - base) < OP_CHUNK ? (n - base) : OP_CHUNK);
        const uint8_t* kk = d_k + base * t->ksz;
        const uint8_t* vv = d_v ? d_v + base * t->vsz : nullptr;
        cudaError_t e = cudaMemsetAsync(t->d_ctl, 0, fm::CTL_CALL_BYTES, s);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "round setup", e);
        uint32_t r = 0;
        uint32_t left = m;
        if (!insert) {
            // no rounds: ops grouped by the first EMPTY slot after their home
            // (lone ops at once, each group in index order); ops the kernels
            // leave (no EMPTY slot anywhere, groups too large) run in rounds
            e = fm::launch_rem_direct(v, sh, kk, m, t->sc, t->d_ctl, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && fault_at(FM_FAULT_ROUND)) e = cudaErrorLaunchFailure;
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "remove", e);
            if (t->h_ctl->err & fm::ERR_SCRATCH) return fail(FM_ERR_KERNEL_LAUNCH, "stale segment registration");
            r = t->h_ctl->serial[0] ? 0u : 1u;
            left = t->h_ctl->serial[0] ? m : t->h_ctl->npend[1];
            if (left == 0) {
                total += t->h_ctl->total_count();
                *err_bits |= t->h_ctl->err;
                t->last_rounds = 0;
                continue;
            }
            e = fm::launch_rem_summary(v, t->sc, t->d_ctl, s);
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "round setup", e);
        }
        // a chunk that can take the table to FM_DIRECT_LOAD or beyond runs as
        // components from the start: rounds stall there, and their tiles'
        // short chain buffers walk chains of thousands of entries again and
        // again
        const double reach = (double)(t->len.load() + total + m) / (double)t->cap;
        const bool direct = insert && reach >= FM_DIRECT_LOAD;
        // below FM_HANDOFF_LOAD the tail's own one-at-a-time order is cheaper
        // than a hand-back (a readback and a scan of the table)
        const bool handoff = reach >= FM_HANDOFF_LOAD;
        if (insert && !direct && sh != fm::SHAPE_GENERIC && t->sc.comp) {
            // no rounds: lone ops run at once, ops sharing free slots run in
            // index order per component; what the kernels leave (a table with
            // no free slot for some op, components too large for a warp) runs
            // on the component path
            e = fm::launch_ins_direct(v, sh, kk, vv, m, t->sc, t->d_ctl, reach, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && fault_at(FM_FAULT_ROUND)) e = cudaErrorLaunchFailure;
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "insert", e);
            if (t->h_ctl->err & fm::ERR_SCRATCH) return fail(FM_ERR_KERNEL_LAUNCH, "stale segment registration");
            const uint32_t rest_r = t->h_ctl->serial[0] ? 0u : 1u;
            const uint32_t rest_n = t->h_ctl->serial[0] ? m : t->h_ctl->npend[1];
            if (rest_n) {
                e = fm::launch_ins_comp(v, sh, kk, vv, m, rest_r, rest_n, t->sc, t->d_ctl, s);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "component insert", e);
            }
            total += t->h_ctl->total_count();
            *err_bits |= t->h_ctl->err;
            t->last_rounds = t->h_ctl->rounds;
            continue;
        }
        for (;;) {
            if (direct) {
                e = fm::launch_ins_comp(v, sh, kk, vv, m, 0, m, t->sc, t->d_ctl, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "component insert", e);
                break;
            }
            e = insert ? fm::launch_ins_rounds(v, sh, kk, vv, m, r, 2, left, t->sc, t->d_ctl, s)
                       : fm::launch_rem_rounds(v, sh, kk, m, r, 2, left, t->sc, t->d_ctl, s);
            r += 2;
            if (e == cudaSuccess)
                e = insert ? fm::launch_ins_tail(v, sh, kk, vv, m, r, t->sc, t->d_ctl, s, handoff)
                           : fm::launch_rem_tail(v, sh, kk, m, r, t->sc, t->d_ctl, s);
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, insert ? "insert rounds" : "remove rounds", e);
            e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && fault_at(FM_FAULT_ROUND)) e = cudaErrorLaunchFailure;
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "round readback", e);
            if (t->h_ctl->err & fm::ERR_SCRATCH) return fail(FM_ERR_KERNEL_LAUNCH, "stale segment registration");
            if (t->h_ctl->err & fm::ERR_NO_PROGRESS) return fail(FM_ERR_PROBE_LIMIT, "round made no progress");
            if (insert && t->h_ctl->tail_handoff) {
                // the tail stopped progressing: its round's ops run as components
                const uint32_t rh = t->h_ctl->tail_handoff - 1;
                e = fm::launch_ins_comp(v, sh, kk, vv, m, rh, t->h_ctl->npend[rh & 1], t->sc, t->d_ctl, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "component insert", e);
                break;
            }
            uint32_t now = t->h_ctl->npend[r & 1];
            if (insert && now > 0 && t->h_ctl->serial[(r - 1) & 1]) {
                // the table is full: the remaining ops run one at a time in index order
                e = fm::launch_ins_comp(v, sh, kk, vv, m, r, now, t->sc, t->d_ctl, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "serial insert", e);
                now = t->h_ctl->npend[r & 1];
            }
            if (now == 0) break;
            if (now >= left)  // every round runs at least the lowest pending op
                return fail(FM_ERR_PROBE_LIMIT, "round made no progress");
            if (insert && (uint64_t)now * 8 > (uint64_t)left * 7) {
                // under 1/8 of the ops per pass (ops crowded onto few free
                // slots, a near-full table): the rest one at a time in index
                // order within each component, which a round boundary allows
                e = fm::launch_ins_comp(v, sh, kk, vv, m, r, now, t->sc, t->d_ctl, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "serial insert", e);
                break;
            }
            left = now;
        }
        total += t->h_ctl->total_count();
        *err_bits |= t->h_ctl->err;
        t->last_rounds = t->h_ctl->rounds;
    }
    *out_count = total;
    return FM_OK;
}

// Runs a mutating call.  On FM_OK with *limit set, every op ran but at least
// one insert walk stopped at the full-table step limit (reported to the
// caller as FM_ERR_PROBE_LIMIT after len is updated).
int run_rounds(fm_table* t, bool insert, const uint8_t* d_k, const uint8_t* d_v, uint64_t n, cudaStream_t s,
               uint64_t* out_count, bool* limit) {
    uint32_t bits = 0;
    int rc = run_rounds_inner(t, insert, d_k, d_v, n, s, out_count, &bits);
    if (rc) {
        std::string msg = tl_err;
        recover(t, s);
        tl_err = msg;
        return rc;
    }
    *limit = (bits & fm::ERR_WALK_LIMIT) != 0;
    return FM_OK;
}

int limit_error() {
    return fail(FM_ERR_PROBE_LIMIT,
                "insert walk passed 2*capacity+2 slots without a free slot (table full; the reference's "
                "insert loop would not terminate here)");
}

GetCtx* acquire_ctx(fm_table* t) {
    {
        std::lock_guard<std::mutex> g(t->pool_mu);
        if (!t->pool.empty()) {
            GetCtx* c = t->pool.back();
            t->pool.pop_back();
            return c;
        }
    }
    GetCtx* c = new GetCtx();
    for (int i = 0; i < 2; i++) {
        if (cudaStreamCreateWithFlags(&c->s[i], cudaStreamNonBlocking) != cudaSuccess) {
            if (i) cudaStreamDestroy(c->s[0]);
            delete c;
            return nullptr;
        }
    }
    return c;
}

void release_ctx(fm_table* t, GetCtx* c) {
    std::lock_guard<std::mutex> g(t->pool_mu);
    t->pool.push_back(c);
}

uint32_t max_dist_of(const uint32_t* flags, uint64_t cap) {
    uint32_t m = 0;
    for (uint64_t i = 0; i < cap; i++)
        if ((flags[i] & 0xFu) == fm::ST_OCC && (flags[i] >> 4) > m) m = flags[i] >> 4;
    return m;
}

}  // namespace

extern "C" {

const char* fm_last_error(void) { return tl_err.c_str(); }

uint64_t fm_launch_count(void) { return fm::launch_count(); }

int fm_inject_fault(uint32_t site, uint32_t after) {
    if (site > FM_FAULT_ROUND) return fail(FM_ERR_INVALID_ARG, "unknown fault site");
    g_fault_site.store(FM_FAULT_NONE);
    g_fault_after.store((int64_t)after);
    g_fault_site.store(site);
    return FM_OK;
}

int fm_create(uint64_t capacity, uint32_t key_size, uint32_t value_size, uint32_t hash_mode, int device_id,
              fm_table** out) {
    if (!out) return fail(FM_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (capacity == 0) return fail(FM_ERR_ZERO_CAPACITY, "capacity must be positive");  // gpu.rs:50-52
    if (capacity > (1ull << 32)) return fail(FM_ERR_INVALID_ARG, "capacity above 2^32 slots is not supported");
    if (hash_mode > 1) return fail(FM_ERR_INVALID_ARG, "unknown hash mode");
    uint64_t cap = 1;
    while (cap < capacity) cap <<= 1;  // next_power_of_two (gpu.rs:54)
    const fm::Shape sh = fm::pick_shape(key_size, value_size);
    if (sh == fm::SHAPE_GENERIC && (key_size > fm::GENERIC_MAX_KV || value_size > fm::GENERIC_MAX_KV))
        return fail(FM_ERR_INVALID_ARG, "key or value larger than 256 bytes (FM_MAX_KV_SIZE, kernels.cu:32)");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_CUDA_INIT, "cudaGetDeviceCount", e);
    if (device_id < 0 || device_id >= ndev) return fail(FM_ERR_CUDA_INIT, "no such CUDA device");
    DeviceGuard dg(device_id);
    if (!dg.ok) return fail(FM_ERR_CUDA_INIT, "cudaSetDevice failed");
    fm_table* t = new fm_table();
    t->device = device_id;
    t->cap = cap;
    t->mask = cap - 1;
    t->ksz = key_size;
    t->vsz = value_size;
    t->mode = hash_mode;
    t->shape = sh;
    auto bail = [&](int code, const char* what, cudaError_t err) {
        int rc = cuda_fail(code, what, err);
        fm_destroy(t);
        return rc;
    };
    if ((e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(FM_ERR_CUDA_INIT, "stream", e);
    if ((e = cudaStreamCreateWithFlags(&t->copy_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(FM_ERR_CUDA_INIT, "stream", e);
    for (int i = 0; i < 2; i++)
        if ((e = cudaEventCreateWithFlags(&t->piece_ready[i], cudaEventDisableTiming)) != cudaSuccess)
            return bail(FM_ERR_CUDA_INIT, "event", e);
    const size_t kb = (size_t)cap * (key_size ? key_size : 1);
    const size_t vb = (size_t)cap * (value_size ? value_size : 1);
    if ((e = dev_alloc((void**)&t->d_flags, cap * 4)) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "flags", e);
    if ((e = dev_alloc((void**)&t->d_keys, kb)) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "keys", e);
    if ((e = dev_alloc((void**)&t->d_vals, vb)) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "values", e);
    if ((e = dev_alloc((void**)&t->d_seg_min, cap * 4)) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "seg_min", e);
    if ((e = dev_alloc((void**)&t->d_seg_cnt, cap * 4)) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "seg_cnt", e);
    if ((e = dev_alloc((void**)&t->d_ctl, sizeof(Ctl))) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "ctl", e);
    if ((e = cudaMallocHost((void**)&t->h_ctl, sizeof(Ctl))) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "ctl", e);
    memset(t->h_ctl, 0, sizeof(Ctl));
    // Zeroed SoA table: all flags EMPTY (gpu.rs:81-92).
    cudaMemsetAsync(t->d_flags, 0, cap * 4, t->stream);
    cudaMemsetAsync(t->d_keys, 0, kb, t->stream);
    cudaMemsetAsync(t->d_vals, 0, vb, t->stream);
    cudaMemsetAsync(t->d_seg_min, 0xFF, cap * 4, t->stream);
    cudaMemsetAsync(t->d_seg_cnt, 0, cap * 4, t->stream);
    cudaMemsetAsync(t->d_ctl, 0, sizeof(Ctl), t->stream);
    if ((e = cudaStreamSynchronize(t->stream)) != cudaSuccess) return bail(FM_ERR_GPU_ALLOC, "table init", e);
    *out = t;
    return FM_OK;
}

void fm_destroy(fm_table* t) {
    if (!t) return;
    DeviceGuard dg(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    for (GetCtx* c : t->pool) {
        for (int i = 0; i < 2; i++) {
            cudaStreamSynchronize(c->s[i]);
            cudaStreamDestroy(c->s[i]);
            if (c->d_buf[i]) cudaFree(c->d_buf[i]);
        }
        delete c;
    }
    if (t->copy_stream) {
        cudaStreamSynchronize(t->copy_stream);
        cudaStreamDestroy(t->copy_stream);
    }
    for (int i = 0; i < 2; i++)
        if (t->piece_ready[i]) cudaEventDestroy(t->piece_ready[i]);
    cudaFree(t->d_flags);
    cudaFree(t->d_keys);
    cudaFree(t->d_vals);
    cudaFree(t->d_seg_min);
    cudaFree(t->d_seg_cnt);
    cudaFree(t->d_ctl);
    if (t->h_ctl) cudaFreeHost(t->h_ctl);
    if (t->sc_base) cudaFree(t->sc_base);
    if (t->d_in) cudaFree(t->d_in);
    if (t->stream) cudaStreamDestroy(t->stream);
    delete t;
}

uint64_t fm_len(const fm_table* t) { return t ? t->len.load() : 0; }
uint64_t fm_capacity(const fm_table* t) { return t ? t->cap : 0; }
double fm_load_factor(const fm_table* t) { return t ? (double)t->len.load() / (double)t->cap : 0.0; }
int fm_device(const fm_table* t) { return t ? t->device : -1; }

int fm_bulk_get(fm_table* t, const void* keys, uint64_t n, void* out_values, uint8_t* out_found) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    if (n == 0) return FM_OK;
    if (!keys || (!out_values && t->vsz) || !out_found) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    GetCtx* c = acquire_ctx(t);
    if (!c) return fail(FM_ERR_CUDA_INIT, "stream creation failed");
    // pieces alternate between two streams and staging buffers: piece i+1's
    // keys upload while piece i's lookups and downloads run
    const uint64_t piece = n < HOST_GET_PIECE ? n : HOST_GET_PIECE;
    const size_t kb = (size_t)piece * t->ksz, vb = (size_t)piece * t->vsz;
    const size_t off_v = (kb + 255) & ~(size_t)255;
    const size_t off_f = off_v + ((vb + 255) & ~(size_t)255);
    int rc = FM_OK;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && !rc; i++)
        if ((e = grow(c->d_buf[i], c->cap[i], off_f + piece)) != cudaSuccess) rc = cuda_fail(FM_ERR_GPU_ALLOC, "get buffers", e);
    const uint8_t* hk = (const uint8_t*)keys;
    uint8_t* hv = (uint8_t*)out_values;
    for (uint64_t base = 0, i = 0; base < n && !rc; base += piece, ++i) {
        const uint64_t m = (n - base) < piece ? (n - base) : piece;
        const int sl = (int)(i & 1);
        cudaStream_t st = c->s[sl];
        uint8_t* dq = c->d_buf[sl];
        uint8_t* dv = c->d_buf[sl] + off_v;
        uint8_t* df = c->d_buf[sl] + off_f;
        if ((e = copy_async(dq, hk + base * t->ksz, m * t->ksz, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            rc = cuda_fail(FM_ERR_TRANSFER, "htod keys", e);
        if (!rc && (e = fm::launch_get_cfg(t->view(), t->shape, dq, m, dv, df,
                                           fm::tuned_get_cfg(t->shape, fm_load_factor(t)), st)) != cudaSuccess)
            rc = cuda_fail(FM_ERR_KERNEL_LAUNCH, "bulk_get", e);
        if (!rc && t->vsz &&
            (e = copy_async(hv + base * t->vsz, dv, m * t->vsz, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            rc = cuda_fail(FM_ERR_TRANSFER, "dtoh values", e);
        if (!rc && (e = copy_async(out_found + base, df, m, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            rc = cuda_fail(FM_ERR_TRANSFER, "dtoh found", e);
    }
    for (int i = 0; i < 2; i++)
        if ((e = cudaStreamSynchronize(c->s[i])) != cudaSuccess && !rc) rc = cuda_fail(FM_ERR_TRANSFER, "bulk_get sync", e);
    release_ctx(t, c);
    return rc;
}

static int precheck(fm_table* t, uint64_t n) {
    // len + n > capacity * MAX_LOAD_FACTOR (1.0) -> TableFull (gpu.rs:198-206)
    const uint64_t len = t->len.load();
    if (len + n > t->cap) {
        char buf[160];
        snprintf(buf, sizeof buf, "table full: %llu occupied of %llu capacity (load factor %.1f%%)",
                 (unsigned long long)len, (unsigned long long)t->cap, (double)len / (double)t->cap * 100.0);
        return fail(FM_ERR_TABLE_FULL, buf);
    }
    return FM_OK;
}

namespace {

// A host-buffer insert (values != nullptr or vsz == 0) or remove, in pieces:
// the copy stream uploads piece i+1 into the other staging half while the
// rounds of piece i run on the table's stream.  *out is the count of the
// pieces that completed, also when a later piece fails (those pieces are in
// the table; the failing piece may be in part).
int host_pieces(fm_table* t, bool insert, const void* keys, const void* values, uint64_t n, uint64_t* out,
                bool* limit) {
    *out = 0;
    *limit = false;
    const uint64_t piece = n < HOST_MUT_PIECE ? n : HOST_MUT_PIECE;
    const size_t kb = (size_t)piece * t->ksz, vb = insert ? (size_t)piece * t->vsz : 0;
    const size_t off_v = (kb + 255) & ~(size_t)255;
    const size_t half = (off_v + vb + 256) & ~(size_t)255;
    cudaError_t e = grow(t->d_in, t->d_in_cap, 2 * half);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_GPU_ALLOC, insert ? "insert buffers" : "remove buffers", e);
    const uint8_t* hk = (const uint8_t*)keys;
    const uint8_t* hv = (const uint8_t*)values;
    auto upload = [&](uint64_t base, int sl) -> cudaError_t {
        const uint64_t m = (n - base) < piece ? (n - base) : piece;
        uint8_t* d = t->d_in + sl * half;
        cudaError_t err = copy_async(d, hk + base * t->ksz, m * t->ksz, cudaMemcpyHostToDevice, t->copy_stream);
        if (err == cudaSuccess && vb)
            err = copy_async(d + off_v, hv + base * t->vsz, m * t->vsz, cudaMemcpyHostToDevice, t->copy_stream);
        if (err == cudaSuccess) err = cudaEventRecord(t->piece_ready[sl], t->copy_stream);
        return err;
    };
    // the staging halves may still be read by the previous call's kernels
    if ((e = cudaStreamSynchronize(t->stream)) != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "sync", e);
    if ((e = upload(0, 0)) != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "htod", e);
    uint64_t total = 0;
    bool lim = false;
    for (uint64_t base = 0, i = 0; base < n; base += piece, ++i) {
        const int sl = (int)(i & 1);
        const uint64_t m = (n - base) < piece ? (n - base) : piece;
        int rc = FM_OK;
        if ((e = cudaStreamWaitEvent(t->stream, t->piece_ready[sl], 0)) != cudaSuccess)
            rc = cuda_fail(FM_ERR_TRANSFER, "piece wait", e);
        // the other half was last read by piece i-1, whose rounds have returned
        if (!rc && base + piece < n && (e = upload(base + piece, sl ^ 1)) != cudaSuccess)
            rc = cuda_fail(FM_ERR_TRANSFER, "htod", e);
        uint8_t* d = t->d_in + sl * half;
        uint64_t c = 0;
        bool l = false;
        if (!rc)
            rc = run_rounds(t, insert, d, insert && t->vsz ? d + off_v : (insert ? d : nullptr), m, t->stream, &c,
                            &l);
        if (rc) {
            const std::string msg = tl_err;
            cudaStreamSynchronize(t->copy_stream);
            cudaStreamSynchronize(t->stream);
            *out = total;
            tl_err = msg;
            return rc;
        }
        total += c;
        lim = lim || l;
        *out = total;
    }
    *out = total;
    *limit = lim;
    return FM_OK;
}

}  // namespace

int fm_bulk_insert(fm_table* t, const void* keys, const void* values, uint64_t n, uint64_t* num_new) {
    if (!t || !num_new) return fail(FM_ERR_INVALID_ARG, "NULL argument");
    *num_new = 0;
    if (n == 0) return FM_OK;  // gpu.rs:194-196
    if (!keys || (!values && t->vsz)) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    std::lock_guard<std::mutex> g(t->mu);
    int rc = precheck(t, n);  // whole batch, before any piece runs
    if (rc) return rc;
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    uint64_t added = 0;
    bool limit = false;
    rc = host_pieces(t, true, keys, values, n, &added, &limit);
    t->len += added;  // on failure: the pieces that completed
    if (rc) return rc;
    *num_new = added;
    return limit ? limit_error() : FM_OK;
}

int fm_bulk_remove(fm_table* t, const void* keys, uint64_t n, uint64_t* num_removed) {
    if (!t || !num_removed) return fail(FM_ERR_INVALID_ARG, "NULL argument");
    *num_removed = 0;
    if (n == 0) return FM_OK;
    if (!keys) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    std::lock_guard<std::mutex> g(t->mu);
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    uint64_t removed = 0;
    bool limit = false;
    int rc = host_pieces(t, false, keys, nullptr, n, &removed, &limit);
    t->len -= removed;  // on failure: the pieces that completed
    if (rc) return rc;
    *num_removed = removed;
    return FM_OK;
}

int fm_clear(fm_table* t) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    std::lock_guard<std::mutex> g(t->mu);
    DeviceGuard dg(t->device);
    cudaError_t e = cudaMemsetAsync(t->d_flags, 0, t->cap * 4, t->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(&t->d_ctl->dmax, 0, 8, t->stream);  // dmax, tomb_claimed
    if (e == cudaSuccess) e = reset_rsum_marks(t, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "clear", e);
    t->len.store(0);
    return FM_OK;
}

int fm_bulk_get_device(fm_table* t, const void* d_keys, uint64_t n, void* d_out_values, uint8_t* d_out_found,
                       void* stream) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    if (n == 0) return FM_OK;
    if (!d_keys || (!d_out_values && t->vsz)) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    const fm::Shape sh = t->shape_for({d_keys, d_out_values});
    cudaError_t e = fm::launch_get_cfg(t->view(), sh, (const uint8_t*)d_keys, n, (uint8_t*)d_out_values, d_out_found,
                                       fm::tuned_get_cfg(sh, fm_load_factor(t)), (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "bulk_get_device", e);
    return FM_OK;
}

int fm_bulk_get_values_device(fm_table* t, const void* d_keys, uint64_t n, void* d_out_values, void* stream) {
    return fm_bulk_get_device(t, d_keys, n, d_out_values, nullptr, stream);
}

static int insert_device(fm_table* t, const void* d_keys, const void* d_values, uint64_t n, uint64_t* num_new,
                         void* stream, bool counted) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    if (num_new) *num_new = 0;
    if (n == 0) return FM_OK;
    if (!d_keys || (!d_values && t->vsz)) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    std::lock_guard<std::mutex> g(t->mu);
    if (counted) {
        int rc = precheck(t, n);
        if (rc) return rc;
    }
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    uint64_t added = 0;
    bool limit = false;
    int rc = run_rounds(t, true, (const uint8_t*)d_keys, (const uint8_t*)d_values, n, (cudaStream_t)stream, &added,
                        &limit);
    if (rc) return rc;
    if (counted) {
        t->len += added;
        if (num_new) *num_new = added;
    } else {
        t->len += n;  // gpu.rs:670
    }
    return limit ? limit_error() : FM_OK;
}

int fm_bulk_insert_device(fm_table* t, const void* d_keys, const void* d_values, uint64_t n, uint64_t* num_new,
                          void* stream) {
    if (!num_new) return fail(FM_ERR_INVALID_ARG, "num_new is NULL");
    return insert_device(t, d_keys, d_values, n, num_new, stream, true);
}

int fm_bulk_insert_device_uncounted(fm_table* t, const void* d_keys, const void* d_values, uint64_t n,
                                    void* stream) {
    return insert_device(t, d_keys, d_values, n, nullptr, stream, false);
}

int fm_bulk_remove_device(fm_table* t, const void* d_keys, uint64_t n, uint64_t* num_removed, void* stream) {
    if (!t || !num_removed) return fail(FM_ERR_INVALID_ARG, "NULL argument");
    *num_removed = 0;
    if (n == 0) return FM_OK;
    if (!d_keys) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    std::lock_guard<std::mutex> g(t->mu);
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    uint64_t removed = 0;
    bool limit = false;
    int rc = run_rounds(t, false, (const uint8_t*)d_keys, nullptr, n, (cudaStream_t)stream, &removed, &limit);
    if (rc) return rc;
    t->len -= removed;
    *num_removed = removed;
    return FM_OK;
}

int fm_recount(fm_table* t, uint64_t* out) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    std::lock_guard<std::mutex> g(t->mu);
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    cudaError_t e = cudaMemsetAsync(&t->d_ctl->occupied, 0, 8, t->stream);
    if (e == cudaSuccess) e = fm::launch_count(t->view(), t->d_ctl, t->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, t->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "recount", e);
    const uint64_t c = t->h_ctl->occupied;
    t->len.store(c);
    if (out) *out = c;
    return FM_OK;
}

int fm_snapshot(fm_table* t, uint32_t* flags, void* keys, void* values) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    std::lock_guard<std::mutex> g(t->mu);
    DeviceGuard dg(t->device);
    cudaError_t e = cudaSuccess;
    if (flags) e = cudaMemcpyAsync(flags, t->d_flags, t->cap * 4, cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess && keys && t->ksz)
        e = cudaMemcpyAsync(keys, t->d_keys, t->cap * t->ksz, cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess && values && t->vsz)
        e = cudaMemcpyAsync(values, t->d_vals, t->cap * t->vsz, cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "snapshot", e);
    return FM_OK;
}

int fm_load(fm_table* t, const uint32_t* flags, const void* keys, const void* values, uint64_t len) {
    if (!t || !flags) return fail(FM_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> g(t->mu);
    DeviceGuard dg(t->device);
    cudaError_t e = cudaMemcpyAsync(t->d_flags, flags, t->cap * 4, cudaMemcpyHostToDevice, t->stream);
    if (e == cudaSuccess && keys && t->ksz)
        e = cudaMemcpyAsync(t->d_keys, keys, t->cap * t->ksz, cudaMemcpyHostToDevice, t->stream);
    if (e == cudaSuccess && values && t->vsz)
        e = cudaMemcpyAsync(t->d_vals, values, t->cap * t->vsz, cudaMemcpyHostToDevice, t->stream);
    // dmax bounds every stored distance; the history of a loaded table is
    // unknown, so tombstone reuse is assumed.
    uint32_t persist[2] = {max_dist_of(flags, t->cap), 1u};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&t->d_ctl->dmax, persist, 8, cudaMemcpyHostToDevice, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "load", e);
    t->len.store(len);
    return FM_OK;
}

int fm_copy(fm_table* dst, const fm_table* src, void* stream) {
    if (!dst || !src) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    if (dst == src) return FM_OK;
    if (dst->cap != src->cap || dst->ksz != src->ksz || dst->vsz != src->vsz || dst->device != src->device)
        return fail(FM_ERR_INVALID_ARG, "tables differ in capacity, record sizes or device");
    std::lock_guard<std::mutex> g(dst->mu);
    DeviceGuard dg(dst->device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(dst->d_flags, src->d_flags, src->cap * 4, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && src->ksz)
        e = cudaMemcpyAsync(dst->d_keys, src->d_keys, src->cap * src->ksz, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && src->vsz)
        e = cudaMemcpyAsync(dst->d_vals, src->d_vals, src->cap * src->vsz, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)  // dmax, tomb_claimed
        e = cudaMemcpyAsync(&dst->d_ctl->dmax, &src->d_ctl->dmax, 8, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "copy", e);
    dst->len.store(src->len.load());
    return FM_OK;
}

int fm_kernel_timing(fm_table* t, int on) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    std::lock_guard<std::mutex> g(t->timer.mu);
    t->timer.on = on != 0;
    return FM_OK;
}

static_assert(FM_KERNEL_CLASSES == (unsigned)fm::KC_N, "kernel classes of the header and the library");

int fm_kernel_times(fm_table* t, double* total_ms, uint64_t* launches, uint32_t n) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    DeviceGuard dg(t->device);
    std::lock_guard<std::mutex> g(t->timer.mu);
    cudaError_t e = t->timer.collect();
    for (uint32_t i = 0; i < n && i < (uint32_t)fm::KC_N; i++) {
        if (total_ms) total_ms[i] = t->timer.ms[i];
        if (launches) launches[i] = t->timer.launches[i];
    }
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "kernel timing", e);
    return FM_OK;
}

int fm_kernel_times_reset(fm_table* t) {
    if (!t) return fail(FM_ERR_INVALID_ARG, "table is NULL");
    DeviceGuard dg(t->device);
    std::lock_guard<std::mutex> g(t->timer.mu);
    cudaError_t e = t->timer.collect();
    for (int i = 0; i < fm::KC_N; i++) t->timer.ms[i] = 0.0, t->timer.launches[i] = 0;
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "kernel timing", e);
    return FM_OK;
}

const char* fm_kernel_class_name(uint32_t cls) {
    // insert classes: the direct kernels (k_dx_*) or the round kernels (k_ins_p1..p4)
    static const char* names[fm::KC_N] = {"k_get",      "ins_find",   "ins_flow",     "ins_exec",
                                          "ins_warp",   "k_ins_tail", "k_ins_serial", "k_rem_p1",
                                          "k_rem_p2",   "k_rem_p3",   "k_rem_tail",   "k_count",
                                          "rem_group"};
    return cls < (uint32_t)fm::KC_N ? names[cls] : nullptr;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free insert (no counterpart in the reference).
//
// Some callers must not allocate device memory once they are running: a
// serving process that reserves all its device memory up front under a fixed
// budget, or one whose caching allocator (PyTorch's, say) holds the free
// memory, where a cudaMalloc made here at insert time could fail and a
// cudaFree would synchronize the whole device and stall the caller's other
// streams.  For them, fm_bulk_insert_device_noalloc runs the round-based
// insert kernels with every per-call buffer (round control block, pending
// lists, per-op words) taken from the file-scope device array below, sized for
// FM_NOALLOC_MAX_OPS operations (about 2.5 MB, held by every GPU that loads
// the library until the process exits).  It never calls cudaMalloc, cudaFree
// or another allocating routine.
//
// It is called from an ordinary host thread: like fm_bulk_insert_device it
// launches kernels, copies control words back and waits on the caller's
// stream, so it cannot run inside a CUDA host function.  The first call on a
// device sets the array up (looks up its device address with that device
// current, marks the per-op words idle) and synchronizes the device; make that
// first call before any stream capture on the device.  All calls share the
// one array: calls whose GPU work overlaps -- on any table of the same device
// -- race on it, so serialize them (one stream, or an event between calls).
// Near a full table, where rounds stop making progress, the remaining ops run
// one at a time on one block (the tail or k_ins_serial): the component path of
// the allocating insert needs a per-table buffer this array does not hold.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr uint64_t NA_OPS = FM_NOALLOC_MAX_OPS;
constexpr size_t NA_CTL = 0;
constexpr size_t NA_PEND0 = na_align(sizeof(Ctl));
constexpr size_t NA_PEND1 = NA_PEND0 + na_align(NA_OPS * 4);
constexpr size_t NA_SLOT = NA_PEND1 + na_align(NA_OPS * 4);
constexpr size_t NA_WORD = NA_SLOT + na_align(NA_OPS * 8);
constexpr size_t NA_PT = NA_WORD + na_align(NA_OPS * 4);
constexpr size_t NA_FLAG = NA_PT + na_align(NA_OPS * 4 * fm::PT_MAX);
constexpr size_t NA_LONG = NA_FLAG + na_align(NA_OPS);
constexpr size_t NA_BYTES = NA_LONG + na_align(NA_OPS * 4);

}  // namespace

// The scratch of fm_bulk_insert_device_noalloc.  In host code this name is
// not a device address; na_setup() looks the address up per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

namespace {

constexpr int NA_MAX_DEVICES = 64;
std::mutex na_mu;
uint8_t* na_base[NA_MAX_DEVICES] = {};

// Once per device, with that device current: the array's device address, and
// the per-op words set idle (the insert kernels leave them idle after use).
int na_setup(int dev, uint8_t** out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) return fail(FM_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> g(na_mu);
    if (!na_base[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_CUDA_INIT, "cudaGetSymbolAddress(noalloc scratch)", e);
        e = cudaMemset((uint8_t*)p + NA_WORD, 0xFF, NA_OPS * 4);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return cuda_fail(FM_ERR_CUDA_INIT, "noalloc scratch init", e);
        na_base[dev] = (uint8_t*)p;
    }
    *out = na_base[dev];
    return FM_OK;
}

int noalloc_rounds(fm_table* t, const uint8_t* d_k, const uint8_t* d_v, uint32_t m, cudaStream_t s, uint8_t* base,
                   uint64_t* out_count, bool* limit) {
    Ctl* ctl = (Ctl*)(base + NA_CTL);
    OpScratch sc{};
    sc.pend[0] = (uint32_t*)(base + NA_PEND0);
    sc.pend[1] = (uint32_t*)(base + NA_PEND1);
    sc.op_slot = (uint64_t*)(base + NA_SLOT);
    sc.op_word = (uint32_t*)(base + NA_WORD);
    sc.op_pt = (uint32_t*)(base + NA_PT);
    sc.op_flag = base + NA_FLAG;
    sc.long_list = (uint32_t*)(base + NA_LONG);
    sc.cap_ops = NA_OPS;
    const fm::Shape sh = t->shape_for({d_k, d_v});
    const fm::TableView v = t->view();
    // per-call fields start at zero; the table's persistent facts (largest
    // stored distance, tombstone reuse) travel in and back out
    cudaError_t e = cudaMemsetAsync(ctl, 0, fm::CTL_CALL_BYTES, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ctl->dmax, &t->d_ctl->dmax, 8, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "noalloc setup", e);
    uint32_t r = 0, left = m;
    for (;;) {
        e = fm::launch_ins_rounds(v, sh, d_k, d_v, m, r, 2, left, sc, ctl, s);
        r += 2;
        if (e == cudaSuccess) e = fm::launch_ins_tail(v, sh, d_k, d_v, m, r, sc, ctl, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "noalloc insert rounds", e);
        if (t->h_ctl->err & fm::ERR_SCRATCH) return fail(FM_ERR_KERNEL_LAUNCH, "stale segment registration");
        if (t->h_ctl->err & fm::ERR_NO_PROGRESS) return fail(FM_ERR_PROBE_LIMIT, "round made no progress");
        uint32_t now = t->h_ctl->npend[r & 1];
        if (now > 0 && t->h_ctl->serial[(r - 1) & 1]) {
            e = fm::launch_ins_serial(v, sh, d_k, d_v, m, r, sc, ctl, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(t->h_ctl, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "noalloc serial insert", e);
            now = t->h_ctl->npend[r & 1];
        }
        if (now == 0) break;
        if (now >= left) return fail(FM_ERR_PROBE_LIMIT, "round made no progress");
        left = now;
    }
    e = cudaMemcpyAsync(&t->d_ctl->dmax, &ctl->dmax, 8, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "noalloc finish", e);
    *out_count = t->h_ctl->total_count();
    *limit = (t->h_ctl->err & fm::ERR_WALK_LIMIT) != 0;
    return FM_OK;
}

}  // namespace

extern "C" int fm_bulk_insert_device_noalloc(fm_table* t, const void* d_keys, const void* d_values, uint64_t n,
                                             uint64_t* num_new, void* stream) {
    if (!t || !num_new) return fail(FM_ERR_INVALID_ARG, "NULL argument");
    *num_new = 0;
    if (n == 0) return FM_OK;
    if (n > NA_OPS) {
        char buf[160];
        snprintf(buf, sizeof buf, "fm_bulk_insert_device_noalloc: %llu ops exceed FM_NOALLOC_MAX_OPS (%llu); "
                 "split the batch or use fm_bulk_insert_device", (unsigned long long)n, (unsigned long long)NA_OPS);
        return fail(FM_ERR_INVALID_ARG, buf);
    }
    if (!d_keys || (!d_values && t->vsz)) return fail(FM_ERR_INVALID_ARG, "NULL buffer");
    std::lock_guard<std::mutex> g(t->mu);
    int rc = precheck(t, n);
    if (rc) return rc;
    DeviceGuard dg(t->device);
    TimerScope ts(t);
    uint8_t* base = nullptr;
    rc = na_setup(t->device, &base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t added = 0;
    bool limit = false;
    rc = noalloc_rounds(t, (const uint8_t*)d_keys, (const uint8_t*)d_values, (uint32_t)n, s, base, &added, &limit);
    if (rc) {
        const std::string msg = tl_err;
        cudaMemsetAsync(t->d_seg_min, 0xFF, t->cap * 4, s);
        cudaMemsetAsync(t->d_seg_cnt, 0, t->cap * 4, s);
        cudaMemsetAsync(base + NA_WORD, 0xFF, NA_OPS * 4, s);
        cudaStreamSynchronize(s);
        tl_err = msg;
        return rc;
    }
    t->len += added;
    *num_new = added;
    return limit ? limit_error() : FM_OK;
}

// ---------------------------------------------------------------------------
// Batched form (no counterpart in gpu.rs): a queue of bulk operations over
// many tables of one device, executed with the sequential result of running
// them one by one in queue order.
//
// Planning (fm_batch_create): an op goes into the wave after the previous op
// on its table, except that a get following a get on the same table joins
// that get's wave (lookups do not change the table).  So the ops of a wave
// touch distinct tables (several gets of one table aside) and are independent.
// Each wave launches one grouped lookup kernel per record shape and one
// grouped round pipeline per shape for its inserts and for its removes
// (precheck against the table's count at that point of the batch, grid
// rounds, a block-per-op tail that runs to completion, result write-back).
// An eager run drives each group's grid rounds from the host, two at a time,
// and records how many it needed; a capture launches the recorded counts with
// no host synchronisation, so the whole batch replays from one CUDA graph.
// ---------------------------------------------------------------------------

static_assert(fm::STATUS_TABLE_FULL == FM_ERR_TABLE_FULL && fm::STATUS_PROBE_LIMIT == FM_ERR_PROBE_LIMIT &&
                  fm::STATUS_KERNEL == FM_ERR_KERNEL_LAUNCH,
              "device status codes");

// Device and pinned host memory of a batch, carved from one block each and
// kept for reuse when the batch is destroyed (allocating pinned memory costs
// milliseconds and freeing device memory synchronises the device, which a
// server creating a batch per step would pay every step).
struct BatchArena {
    int device = -1;
    uint8_t* d = nullptr;
    size_t dcap = 0;
    uint8_t* h = nullptr;
    size_t hcap = 0;
};

namespace {
std::mutex g_arena_mu;
std::vector<BatchArena> g_arenas;  // free arenas
constexpr size_t ARENA_KEEP = 8;

BatchArena arena_take(int device, size_t dneed, size_t hneed, cudaError_t* err) {
    {
        std::lock_guard<std::mutex> g(g_arena_mu);
        for (size_t i = 0; i < g_arenas.size(); i++) {
            if (g_arenas[i].device == device && g_arenas[i].dcap >= dneed && g_arenas[i].hcap >= hneed) {
                BatchArena a = g_arenas[i];
                g_arenas.erase(g_arenas.begin() + i);
                *err = cudaSuccess;
                return a;
            }
        }
    }
    BatchArena a;
    a.device = device;
    a.dcap = dneed + dneed / 2;
    a.hcap = hneed + hneed / 2;
    *err = cudaMalloc((void**)&a.d, a.dcap);
    if (*err == cudaSuccess) *err = cudaMallocHost((void**)&a.h, a.hcap);
    return a;
}

void arena_give(BatchArena a) {
    if (!a.d && !a.h) return;
    {
        std::lock_guard<std::mutex> g(g_arena_mu);
        if (g_arenas.size() < ARENA_KEEP) {
            g_arenas.push_back(a);
            return;
        }
    }
    if (a.d) cudaFree(a.d);
    if (a.h) cudaFreeHost(a.h);
}
}  // namespace

struct fm_batch {
    BatchArena arena;
    int device = 0;
    std::vector<fm_op> ops;
    std::vector<fm_table*> tables;      // distinct tables, batch order
    std::vector<uint32_t> table_of;     // op -> index in tables
    struct Group {
        uint32_t wave;
        uint32_t kind;
        fm::Shape shape;
        uint32_t lane = 0;              // stream lane of its tables
        std::vector<uint32_t> members;  // op indices
        size_t desc_off = 0;            // GroupGet[] / GroupOp[] in the descriptor buffer
        size_t prefix_off = 0;          // gets: uint64 prefix[n+1]
        uint64_t total = 0;             // gets: queries; mutating: sum of sizes
        fm::GetCfg cfg;
        uint32_t rounds = 0;            // mutating: grid rounds the last eager run needed (0: none yet)
        bool serial = false;            // inserts: the eager run finished them one at a time
        std::vector<uint32_t> comp;     // ... of these, the members run as components (more than TAIL_MAX left)
    };
    std::vector<Group> groups;          // in execution order
    uint32_t waves = 0;
    // Tables are spread over up to BATCH_LANES streams forked from the
    // caller's stream (balanced by their ops' sizes): a table's ops stay in
    // order on its lane, and lanes run at the same time, so a long op on one
    // table does not hold up the waves of the others.
    static constexpr uint32_t BATCH_LANES = 8;
    uint32_t nlanes = 1;
    cudaStream_t lane_s[BATCH_LANES] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[BATCH_LANES] = {};
    size_t desc_bytes = 0;
    uint8_t* d_desc = nullptr;          // descriptors (device)
    uint8_t* h_desc = nullptr;          // descriptors (pinned host)
    unsigned long long* d_len = nullptr;   // per table
    unsigned long long* d_res = nullptr;   // per op
    int* d_status = nullptr;               // per op
    uint8_t* h_io = nullptr;               // pinned: len[tables], res[ops], status[ops]
    uint32_t* d_pend = nullptr;            // pending counts (eager runs): GROUP_MAX + 1 words
    uint32_t* h_pend = nullptr;
    // Queue mode (every op of a compile-time record shape): every op as
    // device-driven kernels on stream lanes (qlanes), or the ops as chains of
    // phases drained by one persistent launch per record shape and segment,
    // the large ops as device-driven steps between the launches.
    bool qmode = false;
    bool qlanes = false;  // queue mode: every op a device-driven step on a stream lane
    std::vector<cudaEvent_t> step_ev;  // qlanes: recorded after each step another lane waits for
    struct QStep {
        uint32_t lane = 0;      // qlanes: its stream lane
        std::vector<uint32_t> wait;  // qlanes: earlier steps on other lanes it waits for
        bool signal = false;    // qlanes: a later step on another lane waits for it
        bool external = false;  // an insert or remove run between persistent launches
        bool remove = false;    // external: a remove
        bool get = false;       // external: a lookup
        bool direct = false;    // external insert: the direct passes (else the component path)
        double load = 0.0;      // external: the load it can reach (tuned tile width)
        uint32_t op = 0;        // external: the op
        fm::Shape shape = fm::SHAPE_GENERIC;
        uint32_t ph0 = 0, nph = 0;  // persistent launch: its phases (and done counters)
        uint64_t units = 0;
        uint32_t ext = 0;       // external: index of its GroupOp descriptor
        uint32_t rounds = FM_QUEUE_REM_ROUNDS;  // external remove: grid rounds (eager runs record theirs)
    };
    std::vector<QStep> qsteps;
    std::vector<fm::QPhase> qphases;
    std::vector<uint32_t> qext_ops;  // op index of each external descriptor
    size_t q_ops_off = 0, q_ph_off = 0, q_ext_off = 0;  // in the descriptor buffer
    uint32_t* d_done = nullptr;      // one counter per phase
    fm::QState* d_qstate = nullptr;  // one per step
    fm::QState* h_qstate = nullptr;
    fm::QProf* d_prof = nullptr;     // per-phase timing (fm_batch_profile), one per phase
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches_per_run = 0;
    cudaStream_t last_stream = nullptr;
    bool pending = false;

    unsigned long long* h_len() { return reinterpret_cast<unsigned long long*>(h_io); }
    unsigned long long* h_res() { return h_len() + tables.size(); }
    int* h_status() { return reinterpret_cast<int*>(h_res() + ops.size()); }
    size_t io_bytes() const { return (tables.size() + ops.size()) * 8 + ops.size() * 4; }
};

namespace {

bool batch_aligned(const fm_op& o) {
    for (const void* p : {(const void*)o.d_keys, (const void*)o.d_values, (const void*)o.d_out_values})
        if (p && !aligned(p, 16)) return false;
    return true;
}

// Fills the descriptor buffer from the current table state (scratch pointers
// can move when a table's scratch grows between runs).
int batch_fill(fm_batch* b) {
    for (size_t i = 0; i < b->tables.size(); i++) b->h_len()[i] = b->tables[i]->len.load();
    // Scratch first, sized for each table's largest mutating op: growing it
    // reallocates, so no descriptor may be filled before the last growth.
    std::vector<uint64_t> need(b->tables.size(), 0);
    for (size_t i = 0; i < b->ops.size(); i++)
        if (b->ops[i].kind != FM_OP_GET) need[b->table_of[i]] = std::max(need[b->table_of[i]], b->ops[i].n);
    for (size_t i = 0; i < b->tables.size(); i++) {
        if (!need[i]) continue;
        int rc = ensure_scratch(b->tables[i], need[i]);
        if (rc) return rc;
    }
    for (auto& g : b->groups) {
        if (g.kind == FM_OP_GET) {
            auto* d = reinterpret_cast<fm::GroupGet*>(b->h_desc + g.desc_off);
            auto* pre = reinterpret_cast<uint64_t*>(b->h_desc + g.prefix_off);
            uint64_t acc = 0;
            double load = 0.0;
            for (size_t k = 0; k < g.members.size(); k++) {
                const fm_op& o = b->ops[g.members[k]];
                fm_table* t = o.table;
                d[k].t = t->view();
                d[k].keys = (const uint8_t*)o.d_keys;
                d[k].out_vals = (uint8_t*)o.d_out_values;
                d[k].out_found = o.d_out_found;
                pre[k] = acc;
                acc += o.n;
                load = std::max(load, (double)t->len.load() / (double)t->cap);
            }
            pre[g.members.size()] = acc;
            g.total = acc;
            g.cfg = fm::tuned_get_cfg(g.shape, load);
            // one thread per query needs 8-slot windows
            for (uint32_t m : g.members)
                if (b->ops[m].table->mask < 7 && g.cfg.lanes == 1) g.cfg.lanes = 8;
        } else {
            auto* d = reinterpret_cast<fm::GroupOp*>(b->h_desc + g.desc_off);
            uint64_t sum = 0;
            for (size_t k = 0; k < g.members.size(); k++) {
                const uint32_t oi = g.members[k];
                const fm_op& o = b->ops[oi];
                fm_table* t = o.table;
                d[k].t = t->view();
                d[k].keys = (const uint8_t*)o.d_keys;
                d[k].vals = (const uint8_t*)o.d_values;
                d[k].sc = t->sc;
                d[k].ctl = t->d_ctl;
                d[k].len = b->d_len + b->table_of[oi];
                d[k].result = b->d_res + oi;
                d[k].status = b->d_status + oi;
                d[k].n = (uint32_t)o.n;
                d[k].counted = 1;
                sum += o.n;
            }
            g.total = sum;
        }
    }
    return FM_OK;
}

// Queue mode: the op descriptors from the current table state (scratch sized
// for each table's largest mutating op first: growing it reallocates).
int queue_fill(fm_batch* b) {
    for (size_t i = 0; i < b->tables.size(); i++) b->h_len()[i] = b->tables[i]->len.load();
    std::vector<uint64_t> need(b->tables.size(), 0);
    for (size_t i = 0; i < b->ops.size(); i++)
        if (b->ops[i].kind != FM_OP_GET) need[b->table_of[i]] = std::max(need[b->table_of[i]], b->ops[i].n);
    for (size_t i = 0; i < b->tables.size(); i++) {
        if (!need[i]) continue;
        int rc = ensure_scratch(b->tables[i], need[i]);
        if (rc) return rc;
    }
    auto* q = reinterpret_cast<fm::QOp*>(b->h_desc + b->q_ops_off);
    for (size_t i = 0; i < b->ops.size(); i++) {
        const fm_op& o = b->ops[i];
        fm_table* t = o.table;
        fm::QOp& d = q[i];
        d.t = t->view();
        d.keys = (const uint8_t*)o.d_keys;
        d.vals = (const uint8_t*)o.d_values;
        d.out_vals = (uint8_t*)o.d_out_values;
        d.out_found = o.d_out_found;
        d.sc = t->sc;
        d.ctl = t->d_ctl;
        d.len = b->d_len + b->table_of[i];
        d.result = b->d_res + i;
        d.status = b->d_status + i;
        d.n = (uint32_t)o.n;
        d.kind = o.kind;
        d.counted = 1;
    }
    auto* g = reinterpret_cast<fm::GroupOp*>(b->h_desc + b->q_ext_off);
    for (size_t k = 0; k < b->qext_ops.size(); k++) {
        const uint32_t i = b->qext_ops[k];
        const fm::QOp& d = q[i];
        g[k].t = d.t;
        g[k].keys = d.keys;
        g[k].vals = d.vals;
        g[k].sc = d.sc;
        g[k].ctl = d.ctl;
        g[k].len = d.len;
        g[k].result = d.result;
        g[k].status = d.status;
        g[k].n = d.n;
        g[k].counted = 1;
    }
    memcpy(b->h_desc + b->q_ph_off, b->qphases.data(), b->qphases.size() * sizeof(fm::QPhase));
    return FM_OK;
}

// Queue mode: uploads, the steps in order on stream s, downloads.  adaptive
// (eager runs): an external remove runs grid rounds two at a time until at
// most TAIL_MAX ops are pending (a readback per pair) and records how many it
// needed; otherwise (capture) the recorded count is used.
int queue_enqueue(fm_batch* b, cudaStream_t s, bool adaptive) {
    cudaError_t e = cudaMemcpyAsync(b->d_desc, b->h_desc, b->desc_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_len, b->h_len(), b->tables.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_res, 0, b->ops.size() * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status, 0, b->ops.size() * 4, s);
    if (e == cudaSuccess && !b->qphases.empty()) e = cudaMemsetAsync(b->d_done, 0, b->qphases.size() * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_qstate, 0, b->qsteps.size() * sizeof(fm::QState), s);
    if (e == cudaSuccess && b->d_prof) {
        const size_t np = b->qphases.size();
        e = cudaMemsetAsync(b->d_prof, 0, np * sizeof(fm::QProf), s);
        if (e == cudaSuccess)  // first-start times to the largest value (atomicMin)
            e = cudaMemset2DAsync(&b->d_prof[0].t0, sizeof(fm::QProf), 0xFF, sizeof(unsigned long long), np, s);
    }
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "batch upload", e);
    const auto* dq = reinterpret_cast<const fm::QOp*>(b->d_desc + b->q_ops_off);
    const auto* dph = reinterpret_cast<const fm::QPhase*>(b->d_desc + b->q_ph_off);
    const auto* dg = reinterpret_cast<const fm::GroupOp*>(b->d_desc + b->q_ext_off);
    const auto* hg = reinterpret_cast<const fm::GroupOp*>(b->h_desc + b->q_ext_off);
    const cudaStream_t s0 = s;
    const bool fork = b->qlanes && b->nlanes > 1;
    if (fork) {  // the lanes start after the uploads on the caller's stream
        e = cudaEventRecord(b->ev_fork, s0);
        for (uint32_t l = 0; e == cudaSuccess && l < b->nlanes; l++) e = cudaStreamWaitEvent(b->lane_s[l], b->ev_fork, 0);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch lanes", e);
    }
    // a step that a later step on another lane waits for records its event
    // on its lane right after its work (before the next step is enqueued)
    auto signal = [&](size_t k) -> cudaError_t {
        if (!fork || !b->qsteps[k].signal) return cudaSuccess;
        return cudaEventRecord(b->step_ev[k], b->lane_s[b->qsteps[k].lane]);
    };
    for (size_t si = 0; si < b->qsteps.size(); si++) {
        if (si > 0 && (e = signal(si - 1)) != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch lanes", e);
        fm_batch::QStep& st = b->qsteps[si];
        s = fork ? b->lane_s[st.lane] : s0;
        if (fork)
            for (uint32_t d : st.wait)
                if ((e = cudaStreamWaitEvent(s, b->step_ev[d], 0)) != cudaSuccess)
                    return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch lanes", e);
        if (!st.external) {
            fm::QProf* pr = b->d_prof ? b->d_prof + st.ph0 : nullptr;
            e = fm::launch_queue(st.shape, dph + st.ph0, st.nph, st.units, dq, b->d_done + st.ph0, b->d_qstate + si,
                                 pr, s);
        } else {
            // precheck; the direct passes with the component path over what
            // they leave (pend[1]), or the component path over every op; then
            // the write-back (its rounds see no op left)
            if (st.get) {
                const fm::QOp& q = reinterpret_cast<const fm::QOp*>(b->h_desc + b->q_ops_off)[st.op];
                e = fm::launch_get_cfg(q.t, st.shape, q.keys, q.n, q.out_vals, q.out_found,
                                       fm::tuned_get_cfg(st.shape, st.load), s);
                fm::count_launches(1);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch queue", e);
                continue;
            }
            const fm::GroupOp& h = hg[st.ext];
            if (st.remove) {
                // the direct remove, the rounds over what it leaves (pend[1]),
                // the tail, the write-back
                e = fm::launch_grp_rem(st.shape, dg + st.ext, 1, h.n, fm::GRP_BEGIN, 0, 0, s);
                if (e == cudaSuccess) e = fm::launch_rem_direct_ctl(h.t, st.shape, h.keys, h.n, h.sc, h.ctl, s);
                uint32_t r = 1;  // round r reads Ctl::npend[r & 1]
                if (adaptive) {
                    fm_table* tb = b->ops[st.op].table;
                    while (e == cudaSuccess) {
                        e = cudaMemcpyAsync(tb->h_ctl, h.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
                        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                        if (e != cudaSuccess || tb->h_ctl->npend[r & 1] <= fm::TAIL_MAX) break;
                        e = fm::launch_grp_rem(st.shape, dg + st.ext, 1, h.n, fm::GRP_ROUNDS, r, 2, s);
                        r += 2;
                    }
                    st.rounds = r - 1;
                } else if (st.rounds) {
                    e = fm::launch_grp_rem(st.shape, dg + st.ext, 1, h.n, fm::GRP_ROUNDS, 1, st.rounds, s);
                    r += st.rounds;
                }
                if (e == cudaSuccess) e = fm::launch_grp_rem(st.shape, dg + st.ext, 1, h.n, fm::GRP_END, r, 0, s);
                if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch queue", e);
                continue;
            }
            e = fm::launch_grp_ins(st.shape, dg + st.ext, 1, h.n, fm::GRP_BEGIN, 0, 0, s);
            if (e == cudaSuccess && st.direct) {
                e = fm::launch_ins_direct_ctl(h.t, st.shape, h.keys, h.vals, h.n, h.sc, h.ctl, st.load, s);
                if (e == cudaSuccess)
                    e = fm::launch_ins_comp(h.t, st.shape, h.keys, h.vals, fm::CMP_N0_CTL, 1, h.n, h.sc, h.ctl, s);
            } else if (e == cudaSuccess) {
                e = fm::launch_ins_comp(h.t, st.shape, h.keys, h.vals, fm::CMP_N0_CTL, 0, h.n, h.sc, h.ctl, s);
            }
            if (e == cudaSuccess) e = cudaMemsetAsync(&h.ctl->n0, 0, sizeof(uint32_t), s);
            if (e == cudaSuccess) e = fm::launch_grp_ins(st.shape, dg + st.ext, 1, h.n, fm::GRP_END, 0, 0, s);
        }
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch queue", e);
    }
    if (!b->qsteps.empty() && (e = signal(b->qsteps.size() - 1)) != cudaSuccess)
        return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch lanes", e);
    s = s0;
    if (fork) {  // join the lanes back before the downloads
        for (uint32_t l = 0; e == cudaSuccess && l < b->nlanes; l++) {
            e = cudaEventRecord(b->ev_join[l], b->lane_s[l]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->ev_join[l], 0);
        }
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch lanes", e);
    }
    e = cudaMemcpyAsync(b->h_len(), b->d_len, b->tables.size() * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_res(), b->d_res, b->ops.size() * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_status(), b->d_status, b->ops.size() * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_qstate, b->d_qstate, b->qsteps.size() * sizeof(fm::QState), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "batch download", e);
    return FM_OK;
}

// Queue mode runs every op as device-driven kernels on BATCH_LANES stream
// lanes forked from the caller's stream (queue_plan: a table's writes in
// order on its lane, lookups spread over the lanes between them), or, with
// FLASHMAP_BATCH_MODE=queue, drains the ops through the persistent kernel.
bool queue_lanes_wanted() {
    const char* m = getenv("FLASHMAP_BATCH_MODE");
    return !(m && !strcmp(m, "queue"));
}

// Queue mode plan: segments of ops closed by the inserts that run between
// persistent launches (large or able to fill their table); per segment
// and record shape, the phases of every table's chain of ops listed level by
// level (the first phase of every chain, then the second, ...), each waiting
// for the one before it in its chain.
void queue_plan(fm_batch* b, const std::vector<uint32_t>& lane_of) {
    const uint32_t nops = (uint32_t)b->ops.size();
    std::vector<double> est(b->tables.size());
    for (size_t i = 0; i < b->tables.size(); i++) est[i] = (double)b->tables[i]->len.load();
    if (b->qlanes) {
        // every op a device-driven step: a table's inserts and removes on its
        // lane in queue order; a lookup after the table's last write, on the
        // table's lane or, with fewer tables than lanes, on the next lane in
        // turn; a write after the table's lookups since its last write (on
        // whatever lanes they ran)
        const bool spread = b->tables.size() < b->nlanes;
        std::vector<int32_t> last_w(b->tables.size(), -1);         // step of the table's last write
        std::vector<std::vector<uint32_t>> gets(b->tables.size());  // its lookup steps since then
        uint32_t rr = 0;
        for (uint32_t i = 0; i < nops; i++) {
            const fm_op& o = b->ops[i];
            if (o.n == 0) continue;  // nothing to run; result 0, status OK
            const uint32_t ti = b->table_of[i];
            const double cap = (double)b->tables[ti]->cap;
            fm_batch::QStep st;
            st.external = true;
            // with fewer tables than lanes, lookups fill the idle lanes
            st.lane = (o.kind == FM_OP_GET && spread) ? (rr++ % b->nlanes) : lane_of[ti];
            const uint32_t me = (uint32_t)b->qsteps.size();
            auto after = [&](uint32_t d) {
                if (b->qsteps[d].lane == st.lane) return;  // stream order
                st.wait.push_back(d);
                b->qsteps[d].signal = true;
            };
            if (last_w[ti] >= 0) after((uint32_t)last_w[ti]);
            if (o.kind == FM_OP_GET) {
                gets[ti].push_back(me);
            } else {
                for (uint32_t d : gets[ti]) after(d);
                gets[ti].clear();
                last_w[ti] = (int32_t)me;
            }
            st.op = i;
            st.shape = o.table->shape;
            st.get = o.kind == FM_OP_GET;
            st.remove = o.kind == FM_OP_REMOVE;
            if (o.kind == FM_OP_INSERT) est[ti] = std::min(est[ti] + (double)o.n, cap);
            st.direct = est[ti] < FM_DIRECT_LOAD * cap;
            st.load = est[ti] / cap;
            st.ext = (uint32_t)b->qext_ops.size();
            b->qext_ops.push_back(i);
            b->qsteps.push_back(st);
        }
        return;
    }
    std::vector<uint32_t> seg;
    auto flush = [&]() {
        for (int shi = 0; shi < (int)fm::SHAPE_GENERIC; shi++) {
            const fm::Shape sh = (fm::Shape)shi;
            // per table, its chain of (op, phase kind, units)
            std::vector<std::vector<fm::QPhase>> chain(b->tables.size());
            bool any = false;
            for (uint32_t i : seg) {
                const fm_op& o = b->ops[i];
                if (o.table->shape != sh) continue;
                any = true;
                auto& c = chain[b->table_of[i]];
                const uint32_t n = (uint32_t)o.n;
                auto add = [&](uint32_t kind) {
                    fm::QPhase p{};
                    p.op = i;
                    p.kind = kind;
                    p.units = fm::queue_units(kind, n);
                    p.per = fm::queue_per(kind, n);
                    c.push_back(p);
                };
                if (o.kind == FM_OP_GET) {
                    add(fm::QP_GET);
                } else if (o.kind == FM_OP_INSERT) {
                    for (uint32_t k : {fm::QP_BEGIN, fm::QP_IFIND, fm::QP_IFLOW, fm::QP_IEXEC, fm::QP_IWARP,
                                       fm::QP_IBIG, fm::QP_END})
                        add(k);
                } else {
                    for (uint32_t k : {fm::QP_BEGIN, fm::QP_RFIND, fm::QP_REXEC, fm::QP_END}) add(k);
                }
            }
            if (!any) continue;
            fm_batch::QStep st;
            st.shape = sh;
            st.ph0 = (uint32_t)b->qphases.size();
            std::vector<int32_t> last(b->tables.size(), -1);  // index (within the step) of the chain's last phase
            size_t maxlen = 0;
            for (auto& c : chain) maxlen = std::max(maxlen, c.size());
            uint64_t base = 0;
            for (size_t lvl = 0; lvl < maxlen; lvl++) {
                for (size_t ti = 0; ti < chain.size(); ti++) {
                    if (lvl >= chain[ti].size()) continue;
                    fm::QPhase p = chain[ti][lvl];
                    p.dep = last[ti];
                    p.base = base;
                    base += p.units;
                    last[ti] = (int32_t)(b->qphases.size() - st.ph0);
                    b->qphases.push_back(p);
                }
            }
            st.nph = (uint32_t)(b->qphases.size() - st.ph0);
            st.units = base;
            b->qsteps.push_back(st);
        }
        seg.clear();
    };
    for (uint32_t i = 0; i < nops; i++) {
        const fm_op& o = b->ops[i];
        if (o.n == 0) continue;  // nothing to run; result 0, status OK
        const uint32_t ti = b->table_of[i];
        if (o.kind == FM_OP_INSERT) {
            const double cap = (double)b->tables[ti]->cap;
            est[ti] += (double)o.n;
            if (est[ti] >= FM_QUEUE_INS_LOAD * cap || o.n >= FM_QUEUE_INS_OPS) {
                est[ti] = std::min(est[ti], cap);
                flush();
                fm_batch::QStep st;
                st.external = true;
                st.direct = est[ti] < FM_DIRECT_LOAD * cap;
                st.load = est[ti] / cap;
                st.op = i;
                st.shape = o.table->shape;
                st.ext = (uint32_t)b->qext_ops.size();
                b->qext_ops.push_back(i);
                b->qsteps.push_back(st);
                continue;
            }
        }
        if ((o.kind == FM_OP_REMOVE && o.n >= FM_QUEUE_REM_OPS) || (o.kind == FM_OP_GET && o.n >= FM_QUEUE_GET_OPS)) {
            flush();
            fm_batch::QStep st;
            st.external = true;
            st.remove = o.kind == FM_OP_REMOVE;
            st.get = o.kind == FM_OP_GET;
            st.load = std::min(est[ti], (double)b->tables[ti]->cap) / (double)b->tables[ti]->cap;
            st.op = i;
            st.shape = o.table->shape;
            st.ext = (uint32_t)b->qext_ops.size();
            b->qext_ops.push_back(i);
            b->qsteps.push_back(st);
            continue;
        }
        seg.push_back(i);
    }
    flush();
}

// Enqueues the batch on stream s: descriptor and count upload, the waves,
// result download.  adaptive (eager runs): each insert/remove group runs grid
// rounds two at a time until at most TAIL_MAX ops are pending (a 4-byte
// readback per pair) and records how many it needed; otherwise (capture) the
// recorded count is used (3 when there is none), so the stream carries no
// host synchronisation.  Either way the block-per-op tail completes every op.
int batch_enqueue(fm_batch* b, cudaStream_t s, bool adaptive) {
    cudaError_t e = cudaMemcpyAsync(b->d_desc, b->h_desc, b->desc_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_len, b->h_len(), b->tables.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_res, 0, b->ops.size() * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status, 0, b->ops.size() * 4, s);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "batch upload", e);
    const cudaStream_t s0 = s;
    // an upper bound of each table's count as the waves go (inserts add
    // their size): inserts that can take a table to FM_DIRECT_LOAD run as
    // components from the start, as plain calls do
    std::vector<double> est(b->tables.size());
    for (size_t i = 0; i < b->tables.size(); i++) est[i] = (double)b->h_len()[i];
    if (b->nlanes > 1) {  // fork the lanes off the caller's stream
        e = cudaEventRecord(b->ev_fork, s0);
        for (uint32_t l = 0; e == cudaSuccess && l < b->nlanes; l++) e = cudaStreamWaitEvent(b->lane_s[l], b->ev_fork, 0);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch fork", e);
    }
    for (auto& g : b->groups) {
        const uint32_t n = (uint32_t)g.members.size();
        s = b->nlanes > 1 ? b->lane_s[g.lane] : s0;
        if (g.kind == FM_OP_GET) {
            e = fm::launch_grp_get(g.shape, reinterpret_cast<const fm::GroupGet*>(b->d_desc + g.desc_off),
                                   reinterpret_cast<const uint64_t*>(b->d_desc + g.prefix_off), n, g.total, g.cfg, s);
            if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch wave", e);
            continue;
        }
        const auto* d = reinterpret_cast<const fm::GroupOp*>(b->d_desc + g.desc_off);
        auto* L = g.kind == FM_OP_INSERT ? &fm::launch_grp_ins : &fm::launch_grp_rem;
        e = L(g.shape, d, n, g.total, fm::GRP_BEGIN, 0, 0, s);
        if (g.kind == FM_OP_INSERT) {
            const auto* hd = reinterpret_cast<const fm::GroupOp*>(b->h_desc + g.desc_off);
            for (uint32_t k = 0; e == cudaSuccess && k < n; k++) {
                const uint32_t ti = b->table_of[g.members[k]];
                const double cap = (double)b->tables[ti]->cap;
                est[ti] += (double)hd[k].n;
                if (est[ti] < FM_DIRECT_LOAD * cap) continue;
                est[ti] = std::min(est[ti], cap);
                // the member's ops as components, then a zero op count so the
                // group's rounds pass it by (its counts stay for the finish)
                e = fm::launch_ins_comp(hd[k].t, g.shape, hd[k].keys, hd[k].vals, fm::CMP_N0_CTL, 0, hd[k].n, hd[k].sc,
                                        hd[k].ctl, s);
                if (e == cudaSuccess) e = cudaMemsetAsync(&hd[k].ctl->n0, 0, sizeof(uint32_t), s);
            }
        } else {
            // removes: each member's chunk summaries (built when its windows are long)
            const auto* hd = reinterpret_cast<const fm::GroupOp*>(b->h_desc + g.desc_off);
            for (uint32_t k = 0; e == cudaSuccess && k < n; k++) e = fm::launch_rem_summary(hd[k].t, hd[k].sc, hd[k].ctl, s);
        }
        uint32_t r = 0;
        if (adaptive) {
            // every round runs the lowest pending op of each group: bounded
            const uint64_t bound = 2 * g.total + 4;
            uint64_t prev = g.total;
            while (e == cudaSuccess) {
                e = L(g.shape, d, n, g.total, fm::GRP_ROUNDS, r, 2, s);
                r += 2;
                if (e == cudaSuccess) e = fm::launch_grp_pending(d, n, r, b->d_pend, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_pend, b->d_pend, 4, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                // done, few enough for the tail, or under 1/8 progress (the
                // tail then finishes the rest one at a time)
                if (e != cudaSuccess || *b->h_pend <= fm::TAIL_MAX || r >= bound) break;
                if (g.kind == FM_OP_INSERT && (uint64_t)*b->h_pend * 8 > (uint64_t)prev * 7) {
                    // under 1/8 of the ops per pass (ops crowded onto few free
                    // slots): the rest one at a time in index order
                    g.serial = true;
                    break;
                }
                prev = *b->h_pend;
            }
            g.rounds = r;
            g.comp.clear();
            if (e == cudaSuccess && g.serial) {
                // members with many ops left run as components (the rest in
                // the block-per-op serial launch)
                e = fm::launch_grp_pending_each(d, n, r, b->d_pend, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_pend, b->d_pend, n * 4, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                for (uint32_t k = 0; e == cudaSuccess && k < n; k++)
                    if (b->h_pend[k] > fm::TAIL_MAX) g.comp.push_back(k);
            }
        } else {
            const uint32_t nr = g.rounds ? g.rounds : 3u;
            e = L(g.shape, d, n, g.total, fm::GRP_ROUNDS, 0, nr, s);
            r = nr;
        }
        if (e == cudaSuccess && g.serial) {
            const auto* hd = reinterpret_cast<const fm::GroupOp*>(b->h_desc + g.desc_off);
            for (uint32_t k : g.comp) {
                if (e != cudaSuccess) break;
                const fm::GroupOp& o = hd[k];
                e = fm::launch_ins_comp(o.t, g.shape, o.keys, o.vals, fm::CMP_N0_CTL, r, o.n, o.sc, o.ctl, s);
            }
            if (e == cudaSuccess) e = L(g.shape, d, n, g.total, fm::GRP_SERIAL, r, 0, s);
        }
        if (e == cudaSuccess) e = L(g.shape, d, n, g.total, fm::GRP_END, r, 0, s);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch wave", e);
    }
    s = s0;
    if (b->nlanes > 1) {  // join them back
        for (uint32_t l = 0; e == cudaSuccess && l < b->nlanes; l++) {
            e = cudaEventRecord(b->ev_join[l], b->lane_s[l]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->ev_join[l], 0);
        }
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch join", e);
    }
    e = cudaMemcpyAsync(b->h_len(), b->d_len, b->tables.size() * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_res(), b->d_res, b->ops.size() * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_status(), b->d_status, b->ops.size() * 4, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "batch download", e);
    return FM_OK;
}

}  // namespace

extern "C" {

int fm_batch_create(const fm_op* ops, uint32_t nops, fm_batch** out) {
    if (!out) return fail(FM_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!ops || nops == 0) return fail(FM_ERR_INVALID_ARG, "empty batch");
    fm_batch* b = new fm_batch();
    b->ops.assign(ops, ops + nops);
    b->device = ops[0].table ? ops[0].table->device : 0;
    std::vector<int> last_wave;
    std::vector<uint32_t> last_kind;
    std::vector<uint32_t> op_wave;
    for (uint32_t i = 0; i < nops; i++) {
        const fm_op& o = ops[i];
        auto bad = [&](const char* why) {
            delete b;
            return fail(FM_ERR_INVALID_ARG, std::string("batch op ") + std::to_string(i) + ": " + why);
        };
        if (!o.table) return bad("table is NULL");
        if (o.table->device != b->device) return bad("tables on different devices");
        if (o.kind > FM_OP_REMOVE) return bad("unknown kind");
        if (o.n > 0xFFFFFFFFull - 1) return bad("more than 2^32-2 keys in one op");
        if (o.n && !o.d_keys) return bad("NULL keys");
        if (o.n && o.kind == FM_OP_INSERT && o.table->vsz && !o.d_values) return bad("NULL values");
        uint32_t ti = 0;
        while (ti < b->tables.size() && b->tables[ti] != o.table) ti++;
        if (ti == b->tables.size()) {
            b->tables.push_back(o.table);
            last_wave.push_back(-1);
            last_kind.push_back(0xFFu);
        }
        b->table_of.push_back(ti);
        int w;
        if (last_wave[ti] < 0) w = 0;
        else if (o.kind == FM_OP_GET && last_kind[ti] == FM_OP_GET) w = last_wave[ti];
        else w = last_wave[ti] + 1;
        last_wave[ti] = w;
        last_kind[ti] = o.kind;
        if ((uint32_t)w + 1 > b->waves) b->waves = (uint32_t)w + 1;
        op_wave.push_back((uint32_t)w);
    }
    // queue mode: every op with keys of a compile-time record shape, 16-byte
    // aligned buffers and fewer than 2^31 keys
    b->qmode = true;
    for (uint32_t i = 0; i < nops && b->qmode; i++) {
        const fm_op& o = ops[i];
        if (o.n == 0) continue;
        if (o.table->shape == fm::SHAPE_GENERIC || !batch_aligned(o) || o.n >= (1ull << 31)) b->qmode = false;
    }
    if (b->qmode) {
        // lanes: tables by decreasing work (sum of op sizes, mutations
        // weighted up), each to the lane with the least work so far
        const uint32_t ntab = (uint32_t)b->tables.size();
        std::vector<uint32_t> lane_of(ntab, 0);
        b->qlanes = queue_lanes_wanted();
        b->nlanes = b->qlanes ? fm_batch::BATCH_LANES : 1;
        {
            std::vector<double> work(ntab, 0.0);
            for (uint32_t i = 0; i < nops; i++)
                work[b->table_of[i]] += (double)ops[i].n * (ops[i].kind == FM_OP_GET ? 1.0 : 4.0);
            std::vector<uint32_t> order(ntab);
            for (uint32_t i = 0; i < ntab; i++) order[i] = i;
            std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return work[x] > work[y]; });
            std::vector<double> lane_work(b->nlanes, 0.0);
            for (uint32_t ti : order) {
                uint32_t best = 0;
                for (uint32_t l = 1; l < b->nlanes; l++)
                    if (lane_work[l] < lane_work[best]) best = l;
                lane_of[ti] = best;
                lane_work[best] += work[ti];
            }
        }
        queue_plan(b, lane_of);
        size_t off = 0;
        auto take = [&](size_t bytes) {
            const size_t o = off;
            off = (off + bytes + 255) & ~(size_t)255;
            return o;
        };
        b->q_ops_off = take(nops * sizeof(fm::QOp));
        b->q_ph_off = take(std::max<size_t>(1, b->qphases.size()) * sizeof(fm::QPhase));
        b->q_ext_off = take(std::max<size_t>(1, b->qext_ops.size()) * sizeof(fm::GroupOp));
        b->desc_bytes = off;
        DeviceGuard dg(b->device);
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        const size_t nst = std::max<size_t>(1, b->qsteps.size());
        const size_t o_len = al(b->desc_bytes), o_res = o_len + al(b->tables.size() * 8),
                     o_st = o_res + al(nops * 8), o_done = o_st + al(nops * 4),
                     o_qs = o_done + al(std::max<size_t>(1, b->qphases.size()) * 4),
                     dneed = o_qs + al(nst * sizeof(fm::QState));
        const size_t h_io = al(b->desc_bytes), h_qs = h_io + al(b->io_bytes()), hneed = h_qs + al(nst * sizeof(fm::QState));
        cudaError_t e = cudaSuccess;
        b->arena = arena_take(b->device, dneed, hneed, &e);
        if (e != cudaSuccess) {
            fm_batch_destroy(b);
            return cuda_fail(FM_ERR_GPU_ALLOC, "batch buffers", e);
        }
        b->d_desc = b->arena.d;
        b->d_len = reinterpret_cast<unsigned long long*>(b->arena.d + o_len);
        b->d_res = reinterpret_cast<unsigned long long*>(b->arena.d + o_res);
        b->d_status = reinterpret_cast<int*>(b->arena.d + o_st);
        b->d_done = reinterpret_cast<uint32_t*>(b->arena.d + o_done);
        b->d_qstate = reinterpret_cast<fm::QState*>(b->arena.d + o_qs);
        b->h_desc = b->arena.h;
        b->h_io = b->arena.h + h_io;
        b->h_qstate = reinterpret_cast<fm::QState*>(b->arena.h + h_qs);
        memset(b->h_desc, 0, b->desc_bytes);
        memset(b->h_io, 0, b->io_bytes());
        if (b->nlanes > 1) {
            e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
            for (uint32_t l = 0; e == cudaSuccess && l < b->nlanes; l++) {
                e = cudaStreamCreateWithFlags(&b->lane_s[l], cudaStreamNonBlocking);
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[l], cudaEventDisableTiming);
            }
            b->step_ev.assign(b->qsteps.size(), nullptr);
            for (size_t k = 0; e == cudaSuccess && k < b->qsteps.size(); k++)
                if (b->qsteps[k].signal) e = cudaEventCreateWithFlags(&b->step_ev[k], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                fm_batch_destroy(b);
                return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch streams", e);
            }
        }
        *out = b;
        return FM_OK;
    }
    // lanes: tables by decreasing work (sum of op sizes, mutations weighted
    // up), each to the lane with the least work so far
    const uint32_t ntab = (uint32_t)b->tables.size();
    b->nlanes = ntab < fm_batch::BATCH_LANES ? ntab : fm_batch::BATCH_LANES;
    std::vector<double> work(ntab, 0.0);
    for (uint32_t i = 0; i < nops; i++)
        work[b->table_of[i]] += (double)ops[i].n * (ops[i].kind == FM_OP_GET ? 1.0 : 4.0);
    std::vector<uint32_t> order(ntab), lane_of(ntab, 0);
    for (uint32_t i = 0; i < ntab; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return work[x] > work[y]; });
    std::vector<double> lane_work(b->nlanes, 0.0);
    for (uint32_t ti : order) {
        uint32_t best = 0;
        for (uint32_t l = 1; l < b->nlanes; l++)
            if (lane_work[l] < lane_work[best]) best = l;
        lane_of[ti] = best;
        lane_work[best] += work[ti];
    }
    for (uint32_t i = 0; i < nops; i++) {
        const fm_op& o = ops[i];
        if (o.n == 0) continue;  // nothing to launch; result 0, status OK
        const uint32_t w = op_wave[i], lane = lane_of[b->table_of[i]];
        const fm::Shape sh = batch_aligned(o) ? o.table->shape : fm::SHAPE_GENERIC;
        // the group of (lane, wave, kind, shape), split at GROUP_MAX members
        fm_batch::Group* g = nullptr;
        for (auto it = b->groups.rbegin(); it != b->groups.rend(); ++it) {
            if (it->wave == w && it->lane == lane && it->kind == o.kind && it->shape == sh &&
                it->members.size() < fm::GROUP_MAX) {
                g = &*it;
                break;
            }
        }
        if (!g) {
            b->groups.push_back(fm_batch::Group{w, o.kind, sh, lane, {}});
            g = &b->groups.back();
        }
        g->members.push_back(i);
    }
    // execution order: by wave (groups of one wave are independent)
    std::stable_sort(b->groups.begin(), b->groups.end(),
                     [](const fm_batch::Group& x, const fm_batch::Group& y) { return x.wave < y.wave; });
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (off + bytes + 255) & ~(size_t)255;
        return o;
    };
    for (auto& g : b->groups) {
        if (g.kind == FM_OP_GET) {
            g.desc_off = take(g.members.size() * sizeof(fm::GroupGet));
            g.prefix_off = take((g.members.size() + 1) * 8);
        } else {
            g.desc_off = take(g.members.size() * sizeof(fm::GroupOp));
        }
    }
    b->desc_bytes = off ? off : 256;
    DeviceGuard dg(b->device);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_len = al(b->desc_bytes), o_res = o_len + al(b->tables.size() * 8), o_st = o_res + al(nops * 8),
                 o_pend = o_st + al(nops * 4), dneed = o_pend + al(4 * (fm::GROUP_MAX + 1));
    const size_t h_io = al(b->desc_bytes), h_pend = h_io + al(b->io_bytes()),
                 hneed = h_pend + al(4 * (fm::GROUP_MAX + 1));
    cudaError_t e = cudaSuccess;
    b->arena = arena_take(b->device, dneed, hneed, &e);
    if (e != cudaSuccess) {
        fm_batch_destroy(b);
        return cuda_fail(FM_ERR_GPU_ALLOC, "batch buffers", e);
    }
    b->d_desc = b->arena.d;
    b->d_len = reinterpret_cast<unsigned long long*>(b->arena.d + o_len);
    b->d_res = reinterpret_cast<unsigned long long*>(b->arena.d + o_res);
    b->d_status = reinterpret_cast<int*>(b->arena.d + o_st);
    b->d_pend = reinterpret_cast<uint32_t*>(b->arena.d + o_pend);
    b->h_desc = b->arena.h;
    b->h_io = b->arena.h + h_io;
    b->h_pend = reinterpret_cast<uint32_t*>(b->arena.h + h_pend);
    memset(b->h_desc, 0, b->desc_bytes);
    memset(b->h_io, 0, b->io_bytes());
    if (b->nlanes > 1) {
        e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
        for (uint32_t l = 0; e == cudaSuccess && l < b->nlanes; l++) {
            e = cudaStreamCreateWithFlags(&b->lane_s[l], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[l], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {
            fm_batch_destroy(b);
            return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch streams", e);
        }
    }
    *out = b;
    return FM_OK;
}

uint32_t fm_batch_waves(const fm_batch* b) { return b ? b->waves : 0; }

int fm_batch_capture(fm_batch* b, void* stream) {
    if (!b) return fail(FM_ERR_INVALID_ARG, "batch is NULL");
    if (b->pending) return fail(FM_ERR_INVALID_ARG, "batch still running: call fm_batch_wait first");
    DeviceGuard dg(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = b->qmode ? queue_fill(b) : batch_fill(b);  // allocations (scratch growth) happen here, outside the capture
    if (rc) return rc;
    if (b->exec) cudaGraphExecDestroy(b->exec), b->exec = nullptr;
    if (b->graph) cudaGraphDestroy(b->graph), b->graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "begin capture", e);
    const unsigned long long l0 = fm::launch_count();
    rc = b->qmode ? queue_enqueue(b, s, false) : batch_enqueue(b, s, false);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "end capture", e);
    b->launches_per_run = fm::launch_count() - l0;
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "graph instantiate", e);
    return FM_OK;
}

int fm_batch_run(fm_batch* b, void* stream) {
    if (!b) return fail(FM_ERR_INVALID_ARG, "batch is NULL");
    if (b->pending) return fail(FM_ERR_INVALID_ARG, "batch still running: call fm_batch_wait first");
    DeviceGuard dg(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    // tables must not have host-side work in flight on their own streams
    for (fm_table* t : b->tables) cudaStreamSynchronize(t->stream);
    int rc;
    if (b->exec) {
        rc = b->qmode ? queue_fill(b) : batch_fill(b);
        if (rc) return rc;
        cudaError_t e = cudaGraphLaunch(b->exec, s);
        if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "graph launch", e);
        fm::count_launches((unsigned)b->launches_per_run);
    } else {
        TimerScope ts(b->tables.size() == 1 ? b->tables[0] : nullptr);
        if (b->qmode) {
            rc = queue_fill(b);
            if (!rc) rc = queue_enqueue(b, s, true);
        } else {
            rc = batch_fill(b);
            if (!rc) rc = batch_enqueue(b, s, true);
        }
        if (rc) return rc;
    }
    b->last_stream = s;
    b->pending = true;
    return FM_OK;
}

int fm_batch_wait(fm_batch* b, fm_op* ops) {
    if (!b) return fail(FM_ERR_INVALID_ARG, "batch is NULL");
    if (!b->pending) return fail(FM_ERR_INVALID_ARG, "batch was not run");
    DeviceGuard dg(b->device);
    cudaError_t e = cudaStreamSynchronize(b->last_stream);
    b->pending = false;
    if (e != cudaSuccess) return cuda_fail(FM_ERR_KERNEL_LAUNCH, "batch", e);
    int rc = FM_OK;
    for (size_t i = 0; i < b->tables.size(); i++) b->tables[i]->len.store(b->h_len()[i]);
    if (b->qmode)
        for (size_t si = 0; si < b->qsteps.size(); si++)
            if (b->h_qstate[si].err) rc = fail(FM_ERR_DEVICE_TIMEOUT, "batch queue: a dependency wait ran out");
    for (size_t i = 0; i < b->ops.size(); i++) {
        const int st = b->h_status()[i];
        if (ops) {
            ops[i].result = b->h_res()[i];
            ops[i].status = st;
        }
        if (st == FM_ERR_KERNEL_LAUNCH) {
            recover(b->ops[i].table, b->ops[i].table->stream);
            rc = fail(FM_ERR_KERNEL_LAUNCH, "batch op " + std::to_string(i) + ": round scheduling error");
        }
    }
    return rc;
}

void fm_batch_destroy(fm_batch* b) {
    if (!b) return;
    DeviceGuard dg(b->device);
    if (b->pending && b->last_stream) cudaStreamSynchronize(b->last_stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (uint32_t l = 0; l < fm_batch::BATCH_LANES; l++) {
        if (b->lane_s[l]) cudaStreamDestroy(b->lane_s[l]);
        if (b->ev_join[l]) cudaEventDestroy(b->ev_join[l]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    for (cudaEvent_t ev : b->step_ev)
        if (ev) cudaEventDestroy(ev);
    if (b->d_prof) cudaFree(b->d_prof);
    arena_give(b->arena);
    delete b;
}

int fm_batch_profile(fm_batch* b, int on) {
    if (!b) return fail(FM_ERR_INVALID_ARG, "batch is NULL");
    if (!b->qmode) return fail(FM_ERR_INVALID_ARG, "batch profile: the batch runs as waves, not as a queue");
    if (b->pending) return fail(FM_ERR_INVALID_ARG, "batch still running: call fm_batch_wait first");
    if (b->exec) return fail(FM_ERR_INVALID_ARG, "batch profile: set it before fm_batch_capture");
    DeviceGuard dg(b->device);
    if (!on) {
        if (b->d_prof) cudaFree(b->d_prof);
        b->d_prof = nullptr;
        return FM_OK;
    }
    if (b->d_prof || b->qphases.empty()) return FM_OK;
    const cudaError_t e = cudaMalloc((void**)&b->d_prof, b->qphases.size() * sizeof(fm::QProf));
    if (e != cudaSuccess) {
        b->d_prof = nullptr;
        return cuda_fail(FM_ERR_GPU_ALLOC, "batch profile buffer", e);
    }
    return FM_OK;
}

int fm_batch_phase_times(fm_batch* b, uint64_t* rows, uint32_t max_rows, uint32_t* nrows) {
    if (!b || !nrows) return fail(FM_ERR_INVALID_ARG, "batch or nrows is NULL");
    if (b->pending) return fail(FM_ERR_INVALID_ARG, "batch still running: call fm_batch_wait first");
    *nrows = 0;
    if (!b->d_prof) return FM_OK;
    DeviceGuard dg(b->device);
    std::vector<fm::QProf> h(b->qphases.size());
    const cudaError_t e = cudaMemcpy(h.data(), b->d_prof, h.size() * sizeof(fm::QProf), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(FM_ERR_TRANSFER, "batch profile read", e);
    uint32_t r = 0;
    for (size_t si = 0; si < b->qsteps.size(); si++) {
        const fm_batch::QStep& st = b->qsteps[si];
        if (st.external) continue;
        for (uint32_t k = 0; k < st.nph && r < max_rows; k++, r++) {
            const fm::QPhase& p = b->qphases[st.ph0 + k];
            const fm::QProf& q = h[st.ph0 + k];
            uint64_t* w = rows + (size_t)r * 8;
            w[0] = si;
            w[1] = p.kind;
            w[2] = p.op;
            w[3] = p.units;
            w[4] = q.t0;
            w[5] = q.t1;
            w[6] = q.wait;
            w[7] = q.busy;
        }
    }
    *nrows = r;
    return FM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner for the lookup kernels (no counterpart in the reference).  For
// each compile-time record shape and load bucket it fills a sample table of
// 2^20 slots to the bucket's load with seeded keys, times every candidate --
// lanes per query in {1, 4, 8, 16, 32} x resident blocks per SM in
// {8, 16, 32, 64} -- on 2^20 queries (half present) with CUDA events, keeps
// the fastest, and uses it for every later lookup (plain and batched) on a
// table of that shape whose load falls in the bucket.  Results can be saved
// to and loaded from a text file (one "shape bucket lanes blocks_per_sm"
// line each).
// ---------------------------------------------------------------------------
namespace {

struct ShapeKV {
    fm::Shape sh;
    uint32_t k, v;
};
const ShapeKV kTuneShapes[] = {{fm::SHAPE_8_8, 8, 8},
                               {fm::SHAPE_32_128, 32, 128},
                               {fm::SHAPE_32_64, 32, 64},
                               {fm::SHAPE_32_32, 32, 32},
                               {fm::SHAPE_8_32, 8, 32}};
const double kBucketLoad[fm::LOAD_BUCKETS] = {0.5, 0.7, 0.88};

int tune_load(const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return 0;
    // one line per shape and load bucket: shape bucket lanes blocks_per_sm
    // [queries per thread, 1 when absent]
    // ("ins shape bucket tile": the insert warp pass's tile width)
    int n = 0;
    char line[128];
    while (fgets(line, sizeof line, f)) {
        int sh, b, lanes, bps, qpt = 1;
        if (sscanf(line, "ins %d %d %d", &sh, &b, &lanes) == 3) {
            if (sh < 0 || sh >= fm::SHAPE_GENERIC || b < 0 || b >= fm::LOAD_BUCKETS) continue;
            fm::InsCfg c;
            c.tile = lanes;
            fm::set_tuned_ins_cfg((fm::Shape)sh, b, c);
            ++n;
            continue;
        }
        if (sscanf(line, "%d %d %d %d %d", &sh, &b, &lanes, &bps, &qpt) < 4) continue;
        if (sh < 0 || sh > fm::SHAPE_GENERIC || b < 0 || b >= fm::LOAD_BUCKETS) continue;
        fm::GetCfg c;
        c.lanes = lanes;
        c.blocks_per_sm = bps;
        c.qpt = qpt;
        fm::set_tuned_get_cfg((fm::Shape)sh, b, c);
        ++n;
    }
    fclose(f);
    return n;
}

}  // namespace

extern "C" {

int fm_autotune(int device, const char* cache_path) {
    if (cache_path && tune_load(cache_path) > 0) return FM_OK;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device < 0 || device >= ndev) return fail(FM_ERR_CUDA_INIT, "no such CUDA device");
    DeviceGuard dg(device);
    const uint64_t cap = 1ull << 20, nq = 1ull << 20;
    // candidates: lanes per query (with one lane, 1, 2 or 4 queries per
    // thread in lockstep) x resident blocks per SM
    const int lanes[] = {1, 1, 1, 4, 8, 16, 32};
    const int qpts[] = {1, 2, 4, 1, 1, 1, 1};
    const int bpss[] = {8, 16, 32, 64};
    std::string out;
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    uint8_t *dk = nullptr, *dv = nullptr, *dq = nullptr, *dout = nullptr, *dfound = nullptr;
    int rc = FM_OK;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&a)) != cudaSuccess || (e = cudaEventCreate(&b)) != cudaSuccess)
        return cuda_fail(FM_ERR_CUDA_INIT, "autotune", e);
    for (const ShapeKV& sk : kTuneShapes) {
        const uint64_t nfill = (uint64_t)(cap * kBucketLoad[fm::LOAD_BUCKETS - 1]) + 8;
        if ((e = cudaMalloc(&dk, nfill * sk.k)) != cudaSuccess || (e = cudaMalloc(&dv, nfill * sk.v)) != cudaSuccess ||
            (e = cudaMalloc(&dq, nq * sk.k)) != cudaSuccess || (e = cudaMalloc(&dout, nq * sk.v)) != cudaSuccess ||
            (e = cudaMalloc(&dfound, nq)) != cudaSuccess) {
            rc = cuda_fail(FM_ERR_GPU_ALLOC, "autotune buffers", e);
            break;
        }
        fm::launch_fill_random(dk, nfill * sk.k, 11, s);
        fm::launch_fill_random(dv, nfill * sk.v, 12, s);
        fm_table* t = nullptr;
        if ((rc = fm_create(cap, sk.k, sk.v, FM_HASH_IDENTITY, device, &t)) != FM_OK) break;
        uint64_t filled = 0;
        for (int bk = 0; bk < fm::LOAD_BUCKETS && rc == FM_OK; bk++) {
            const uint64_t target = (uint64_t)(cap * kBucketLoad[bk]);
            uint64_t added = 0;
            rc = fm_bulk_insert_device(t, dk + filled * sk.k, dv + filled * sk.v, target - filled, &added, s);
            if (rc) break;
            filled = target;
            // queries: half present (inserted keys, strided), half fresh
            fm::launch_fill_random(dq, nq * sk.k, 13 + bk, s);
            const uint64_t half = nq / 2 < filled ? nq / 2 : filled;
            cudaMemcpy2DAsync(dq, 2 * sk.k, dk, sk.k * (filled / half), sk.k, half, cudaMemcpyDeviceToDevice, s);
            float best = 1e30f;
            fm::GetCfg bestc;
            for (int li = 0; li < (int)(sizeof(lanes) / sizeof(lanes[0])); li++) {
                for (int bps : bpss) {
                    fm::GetCfg c;
                    c.lanes = lanes[li];
                    c.qpt = qpts[li];
                    c.blocks_per_sm = bps;
                    float ms = 1e30f;
                    for (int rep = 0; rep < 3; rep++) {
                        cudaEventRecord(a, s);
                        fm::launch_get_cfg(t->view(), t->shape, dq, nq, dout, dfound, c, s);
                        cudaEventRecord(b, s);
                        if ((e = cudaEventSynchronize(b)) != cudaSuccess) break;
                        float x = 0.f;
                        cudaEventElapsedTime(&x, a, b);
                        if (rep > 0 && x < ms) ms = x;  // the first run warms up
                    }
                    if (e != cudaSuccess) break;
                    if (ms < best) best = ms, bestc = c;
                }
            }
            if (e != cudaSuccess) {
                rc = cuda_fail(FM_ERR_KERNEL_LAUNCH, "autotune", e);
                break;
            }
            fm::set_tuned_get_cfg(sk.sh, bk, bestc);
            out += std::to_string((int)sk.sh) + " " + std::to_string(bk) + " " + std::to_string(bestc.lanes) + " " +
                   std::to_string(bestc.blocks_per_sm) + " " + std::to_string(bestc.qpt) + "\n";
            // the insert warp pass's tile width: a call of nins fresh keys
            // (the queries' second half) from this state, restored from a
            // device copy before every candidate
            {
                const uint64_t nins = nq / 2 < cap / 50 ? nq / 2 : cap / 50;
                const uint8_t* ik = dq + (nq / 2) * sk.k;
                fm_table* bk_t = nullptr;
                if ((rc = fm_create(cap, sk.k, sk.v, FM_HASH_IDENTITY, device, &bk_t)) != FM_OK) break;
                rc = fm_copy(bk_t, t, s);
                const int tiles[] = {8, 16, 32};
                float best_i = 1e30f;
                int best_t = 32;
                for (int tw : tiles) {
                    fm::InsCfg ic;
                    ic.tile = tw;
                    fm::set_tuned_ins_cfg(sk.sh, bk, ic);
                    float ms_i = 1e30f;
                    for (int rep = 0; rep < 3 && rc == FM_OK; rep++) {
                        if ((rc = fm_copy(t, bk_t, s)) != FM_OK) break;
                        uint64_t added = 0;
                        cudaEventRecord(a, s);
                        rc = fm_bulk_insert_device(t, ik, dv, nins, &added, s);
                        cudaEventRecord(b, s);
                        if (rc != FM_OK || (e = cudaEventSynchronize(b)) != cudaSuccess) break;
                        float x = 0.f;
                        cudaEventElapsedTime(&x, a, b);
                        if (rep > 0 && x < ms_i) ms_i = x;  // the first run warms up
                    }
                    if (rc != FM_OK || e != cudaSuccess) break;
                    if (ms_i < best_i) best_i = ms_i, best_t = tw;
                }
                if (rc == FM_OK) rc = fm_copy(t, bk_t, s);  // the filled state for the next bucket
                fm_destroy(bk_t);
                if (rc != FM_OK) break;
                if (e != cudaSuccess) {
                    rc = cuda_fail(FM_ERR_KERNEL_LAUNCH, "autotune", e);
                    break;
                }
                fm::InsCfg ic;
                ic.tile = best_t;
                fm::set_tuned_ins_cfg(sk.sh, bk, ic);
                out += "ins " + std::to_string((int)sk.sh) + " " + std::to_string(bk) + " " + std::to_string(best_t) +
                       "\n";
            }
        }
        fm_destroy(t);
        cudaFree(dk), cudaFree(dv), cudaFree(dq), cudaFree(dout), cudaFree(dfound);
        dk = dv = dq = dout = dfound = nullptr;
        if (rc) break;
    }
    cudaFree(dk), cudaFree(dv), cudaFree(dq), cudaFree(dout), cudaFree(dfound);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamDestroy(s);
    if (rc) return rc;
    if (cache_path) {
        FILE* f = fopen(cache_path, "w");
        if (f) {
            fputs(out.c_str(), f);
            fclose(f);
        }
    }
    return FM_OK;
}

int fm_tuned_get_config(uint32_t key_size, uint32_t value_size, double load, int* lanes, int* blocks_per_sm) {
    const fm::GetCfg c = fm::tuned_get_cfg(fm::pick_shape(key_size, value_size), load);
    if (lanes) *lanes = c.lanes;
    if (blocks_per_sm) *blocks_per_sm = c.blocks_per_sm;
    return FM_OK;
}

}  // extern "C"

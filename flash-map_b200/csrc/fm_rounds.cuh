// fm_rounds.cuh -- plumbing shared by the round-based mutating kernels
// (fm_insert.cu, fm_remove.cu): which ops a round sees, list appends, and the
// per-round fields of the control block.
#pragma once
#include "fm_internal.h"

namespace fm {

constexpr int RBLOCK = 256;

// Warp-aggregated append of `j` to `list`: one atomic per warp.  Works in
// divergent code (the ballot covers the lanes that reach it together).
__device__ __forceinline__ void append(uint32_t* list, uint32_t* counter, uint32_t j, bool take) {
    const uint32_t active = __activemask();
    const uint32_t m = __ballot_sync(active, take);
    if (!take) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    list[base + __popc(m & ((1u << lane) - 1u))] = j;
}

// A tile of T consecutive lanes of a warp working on one operation.
template <int T>
struct Tile {
    static_assert(T == 4 || T == 8 || T == 16 || T == 32, "tile width");
    static constexpr uint32_t TM = (T == 32) ? 0xFFFFFFFFu : ((1u << T) - 1u);
    static constexpr int W = T;  // lanes
    uint32_t lane;   // 0..T-1
    uint32_t base;   // first lane of the tile in its warp
    uint32_t wmask;  // the tile's lanes as a warp mask
    __device__ __forceinline__ Tile() {
        lane = threadIdx.x & (T - 1);
        base = (threadIdx.x & 31u) & ~(uint32_t)(T - 1);
        wmask = TM << base;
    }
    __device__ __forceinline__ uint32_t ballot(bool p) const { return (__ballot_sync(wmask, p) >> base) & TM; }
    template <class X>
    __device__ __forceinline__ X shfl(X v, uint32_t src) const {
        return __shfl_sync(wmask, v, base + src);
    }
    __device__ __forceinline__ void sync() const { __syncwarp(wmask); }
};

// The whole block as one crew of W threads (tile_moves over a block).
template <int W_>
struct BlockCrew {
    static constexpr int W = W_;
    uint32_t lane;
    __device__ __forceinline__ BlockCrew() : lane(threadIdx.x) {}
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Pending list of round r (a select, so the scratch struct stays in registers).
__device__ __forceinline__ uint32_t* pend_of(const OpScratch& sc, uint32_t r) {
    return (r & 1u) ? sc.pend[1] : sc.pend[0];
}

// The ops of round r: round 0 is the identity over the call's n0 ops.
struct RoundOps {
    const uint32_t* list;  // nullptr: identity
    uint32_t n;
    __device__ __forceinline__ uint32_t op(uint32_t i) const { return list ? list[i] : i; }
};

__device__ __forceinline__ RoundOps round_ops(const OpScratch& sc, const Ctl* ctl, uint32_t r, uint32_t n0) {
    RoundOps o;
    if (r == 0) {
        o.list = nullptr;
        o.n = n0;
    } else {
        o.list = pend_of(sc, r);
        o.n = *(volatile const uint32_t*)&ctl->npend[r & 1];
    }
    return o;
}

// Clear the next round's fields (called by one thread of the first phase of
// round r; nothing reads them until the last phase of round r appends).
__device__ __forceinline__ void reset_next_round(Ctl* ctl, uint32_t r) {
    const uint32_t nx = (r + 1) & 1;
    ctl->npend[nx] = 0;
    ctl->serial[nx] = 0;
    ctl->nlong[nx] = 0;
}

// Block-aggregated append: one global atomic per block per call.  Every
// thread of the block calls it (block-uniform control flow); each thread
// appends at most one entry.
struct AppendSmem {
    uint32_t n[2];     // per-call counters, alternating (the idle one is reset in passing)
    uint32_t base[2];
    uint32_t buf[2][RBLOCK];
    uint32_t phase;
};

__device__ __forceinline__ void append_init(AppendSmem& s) {
    if (threadIdx.x == 0) {
        s.n[0] = s.n[1] = 0;
        s.phase = 0;
    }
    __syncthreads();
}

// Two block barriers per call: entries go to a shared buffer, thread 0 takes
// the block's range with one global atomic, then the buffer is copied out
// while the other buffer's counter is cleared for the next call.
__device__ __forceinline__ void block_append(uint32_t* list, uint32_t* counter, uint32_t j, bool take, AppendSmem& s) {
    const uint32_t ph = s.phase;
    if (take) s.buf[ph][atomicAdd(&s.n[ph], 1u)] = j;
    __syncthreads();
    const uint32_t n = s.n[ph];
    if (threadIdx.x == 0) {
        if (n) s.base[ph] = atomicAdd(counter, n);
        s.n[ph ^ 1] = 0;
        s.phase = ph ^ 1;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) list[s.base[ph] + k] = s.buf[ph][k];
}

// Block sum of v added to one of the spread counters.  Block-uniform call.
__device__ __forceinline__ void block_add_count(Ctl* ctl, uint32_t v, uint32_t* s_tmp /* >= blockDim/32 */) {
    v = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31u) == 0) s_tmp[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; w++) s += s_tmp[w];
        if (s) atomicAdd(&ctl->count_part[blockIdx.x % COUNT_PARTS][0], (unsigned long long)s);
    }
}

// Order-preserving block compaction: writes the j of every thread with
// `take` to out[] in thread order and returns the count.  Block-uniform call;
// s_woff holds 33 words (32 warp offsets and the total).
__device__ __forceinline__ uint32_t block_compact(uint32_t j, bool take, uint32_t* out, uint32_t* s_woff) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, take);
    if (lane == 0) s_woff[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; w++) {
            const uint32_t c = s_woff[w];
            s_woff[w] = acc;
            acc += c;
        }
        s_woff[32] = acc;
    }
    __syncthreads();
    const uint32_t total = s_woff[32];
    if (take) out[s_woff[warp] + __popc(m & ((1u << lane) - 1u))] = j;
    __syncthreads();
    return total;
}

// ---- grouped launches ------------------------------------------------------

// Exclusive prefix of the ops' item counts into s_pre[0..nops] (block-wide;
// every thread calls it; count(o) is read once per op).  Returns the total.
template <class Count>
__device__ __forceinline__ uint32_t group_prefix(uint32_t nops, Count count, uint32_t* s_pre) {
    if (threadIdx.x < 32) {
        uint32_t carry = 0;
        for (uint32_t b = 0; b < nops; b += 32) {
            const uint32_t o = b + threadIdx.x;
            uint32_t v = o < nops ? count(o) : 0u;
            uint32_t incl = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if ((int)threadIdx.x >= d) incl += x;
            }
            if (o < nops) s_pre[o] = carry + incl - v;
            carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
        if (threadIdx.x == 0) s_pre[nops] = carry;
    }
    __syncthreads();
    return s_pre[nops];
}

// The op holding flat item `flat` (largest o with s_pre[o] <= flat).
__device__ __forceinline__ uint32_t group_find(const uint32_t* s_pre, uint32_t nops, uint32_t flat) {
    uint32_t lo = 0, hi = nops;  // s_pre[lo] <= flat < s_pre[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_pre[mid] <= flat) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Append of `j` to op o's list, aggregated over the lanes of a warp working
// on the same op (one atomic per op per warp).
__device__ __forceinline__ void append_peer(uint32_t* list, uint32_t* counter, uint32_t j, bool take, uint32_t o) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, o);
    const uint32_t m = __ballot_sync(peers, take);
    if (!take) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    list[base + __popc(m & ((1u << lane) - 1u))] = j;
}

// Adds v to op o's spread counter, aggregated over the warp's lanes on o.
__device__ __forceinline__ void add_peer(Ctl* ctl, uint32_t v, uint32_t o) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, o);
    const uint32_t sum = __reduce_add_sync(peers, v);
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1) && sum)
        atomicAdd(&ctl->count_part[blockIdx.x % COUNT_PARTS][0], (unsigned long long)sum);
}

namespace {

// Per op: reset the call's control fields, then the precheck of
// gpu.rs:198-206 against the table's count at this point of the batch.
__global__ void k_grp_setup(const GroupOp* __restrict__ ops, int is_insert) {
    const GroupOp& g = ops[blockIdx.x];
    uint32_t* w = reinterpret_cast<uint32_t*>(g.ctl);
    for (uint32_t i = threadIdx.x; i < CTL_CALL_BYTES / 4; i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t n0 = g.n;
        int st = STATUS_OK;
        if (is_insert && g.counted && *g.len + g.n > g.t.mask + 1) {
            n0 = 0;
            st = STATUS_TABLE_FULL;
        }
        g.ctl->n0 = n0;
        *g.status = st;
        *g.result = 0;
    }
}

// Per op: the result, the table's count and the status.
__global__ void k_grp_finish(const GroupOp* __restrict__ ops, uint32_t nops, int is_insert) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nops) return;
    const GroupOp& g = ops[o];
    if (*g.status != STATUS_OK) return;  // rejected by the precheck
    const unsigned long long c = g.ctl->total_count();
    *g.result = c;
    if (is_insert) *g.len += g.counted ? c : (unsigned long long)g.n;
    else *g.len -= c;
    const uint32_t err = g.ctl->err;
    if (err & (ERR_SCRATCH | ERR_NO_PROGRESS)) *g.status = STATUS_KERNEL;
    else if (err & ERR_WALK_LIMIT) *g.status = STATUS_PROBE_LIMIT;
}

}  // namespace

// Iteration count of a uniform grid-stride loop (every thread of a warp runs
// the same number of iterations, so warp collectives stay legal).
__device__ __forceinline__ uint32_t grid_iters(uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    return (n + stride - 1) / stride;
}

}  // namespace fm

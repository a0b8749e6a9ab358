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

// Iteration count of a uniform grid-stride loop (every thread of a warp runs
// the same number of iterations, so warp collectives stay legal).
__device__ __forceinline__ uint32_t grid_iters(uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    return (n + stride - 1) / stride;
}

}  // namespace fm

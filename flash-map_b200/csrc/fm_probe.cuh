// fm_probe.cuh -- single-thread probes shared by the plain kernels and the
// persistent batch kernel: the lookup of one query and the remove of one key,
// each on one thread with aligned 8-slot metadata windows.
#pragma once
#include "fm_internal.h"

namespace fm {

template <int KB>
__device__ __forceinline__ uint64_t home_of(const TableView& t, const uint8_t* keys, uint32_t j, RegKey<KB>& key) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    key.load(keys + (uint64_t)j * ksz, ksz);
    return key.hash(ksz, t.hash_mode) & t.mask;
}

#ifndef FM_GET_WCOPY
#define FM_GET_WCOPY 1  // k_get_thread moves values a warp at a time
#endif

// The probe of one lookup on one thread: the slot holding the key, or NONE64.
template <int KB>
__device__ __forceinline__ uint64_t get_probe_thread(const TableView& t, const uint8_t* __restrict__ qk);

// bulk_get with one thread per query (compile-time shapes, capacity >= 8).
// Each step reads the 8-slot metadata window that holds the probe position as
// two 16-byte loads (one 32-byte sector, aligned), walks it in registers, and
// compares keys only where the stored distance equals the probe depth.  With
// one query per thread about eight times as many queries are in flight per SM
// as with one query per 8-lane tile, which is what a chain of dependent
// random reads (key -> metadata -> key -> value) needs.
template <int KB, int VB>
__device__ __forceinline__ void get_query_thread(const TableView& t, const uint8_t* __restrict__ qk,
                                                 uint8_t* __restrict__ ov, uint8_t* __restrict__ of) {
    const uint64_t hit = get_probe_thread<KB>(t, qk);
    if (ov) {
        RegVal<VB> v;
        if (hit != NONE64) v.load_ro(t.vals + hit * VB);
        else v.zero();
        v.store(ov, VB);
    }
    if (of) *of = hit != NONE64 ? 1 : 0;
}

template <int KB>
__device__ __forceinline__ uint64_t get_probe_thread(const TableView& t, const uint8_t* __restrict__ qk) {
    const uint64_t mask = t.mask;
    RegKey<KB> key;
    key.load(qk, KB);
    const uint64_t h = key.hash(KB, t.hash_mode) & mask;
    uint64_t wb = h & ~7ull;
    uint64_t hit = NONE64;
    bool done = false;
    while (!done) {
        const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
        const uint4 a = __ldg(fp), b = __ldg(fp + 1);
        const uint32_t f8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        // the window in registers: candidates (stored distance == depth)
        // before the first terminator -- probe past the capacity, EMPTY, or
        // OCCUPIED with depth > dist (rayon_cpu.rs:91-111); tombstones are
        // skipped
        uint32_t cand = 0;
#pragma unroll
        for (int l = 0; l < 8; l++) {
            const uint64_t pos = wb + l;
            if (done || pos < h) continue;
            const uint64_t p = pos - h;
            const uint32_t f = f8[l];
            const uint32_t s = st_of(f);
            if (p > mask || s == ST_EMPTY || (s == ST_OCC && p > dist_of(f))) done = true;
            else if (s == ST_OCC && dist_matches(f, p)) cand |= 1u << l;
        }
        // the candidates in walk order
        while (cand) {
            const int l = __ffs(cand) - 1;
            cand &= cand - 1;
            const uint64_t slot = (wb + l) & mask;
            if (key.eq(t.keys + slot * KB, KB)) {
                hit = slot;
                done = true;
                break;
            }
        }
        wb += 8;
    }
    return hit;
}

// Q lookups per thread probed in lockstep (compile-time shapes, capacity >=
// 8): queries q0, q0 + stride, ... below q1.  Each step loads the 8-slot
// metadata window of every query still probing (Q independent loads in
// flight), then compares candidate keys one candidate per query per pass, so
// a thread keeps Q chains of dependent reads going where get_query_thread
// keeps one: what a kernel with few resident threads per SM needs.  Table
// loads are plain (coherent) loads -- the persistent batch kernel runs
// lookups after writes made by other blocks of the same launch; the query
// keys are read through the read-only path.  Semantics as get_query_thread.
template <int KB, int VB, int Q>
__device__ __forceinline__ void get_queries_lockstep(const TableView& t, const uint8_t* __restrict__ keys,
                                                     uint64_t q0, uint64_t stride, uint64_t q1,
                                                     uint8_t* __restrict__ ov, uint8_t* __restrict__ of) {
    const uint64_t mask = t.mask;
    RegKey<KB> key[Q];
    uint64_t h[Q], wb[Q], hit[Q];
    uint32_t act = 0;
#pragma unroll
    for (int i = 0; i < Q; i++) {
        const uint64_t q = q0 + (uint64_t)i * stride;
        h[i] = 0;
        hit[i] = NONE64;
        if (q < q1) {
            key[i].load(keys + q * KB, KB);
            h[i] = key[i].hash(KB, t.hash_mode) & mask;
            act |= 1u << i;
        }
        wb[i] = h[i] & ~7ull;
    }
    while (act) {
        uint4 wa[Q], wz[Q];
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (act >> i & 1u) {
                const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb[i] & mask));
                wa[i] = fp[0];
                wz[i] = fp[1];
            }
        }
        uint32_t cand[Q];
        uint32_t stop = 0;
#pragma unroll
        for (int i = 0; i < Q; i++) {
            cand[i] = 0;
            if (!(act >> i & 1u)) continue;
            const uint32_t f8[8] = {wa[i].x, wa[i].y, wa[i].z, wa[i].w, wz[i].x, wz[i].y, wz[i].z, wz[i].w};
            bool done = false;
#pragma unroll
            for (int l = 0; l < 8; l++) {
                const uint64_t pos = wb[i] + l;
                if (done || pos < h[i]) continue;
                const uint64_t p = pos - h[i];
                const uint32_t f = f8[l];
                const uint32_t s = st_of(f);
                if (p > mask || s == ST_EMPTY || (s == ST_OCC && p > dist_of(f))) done = true;
                else if (s == ST_OCC && dist_matches(f, p)) cand[i] |= 1u << l;
            }
            if (done) stop |= 1u << i;
        }
        // candidates in walk order, one per query per pass
        for (;;) {
            uint32_t more = 0;
#pragma unroll
            for (int i = 0; i < Q; i++) {
                if (!cand[i]) continue;
                const uint64_t slot = (wb[i] + (uint64_t)(__ffs(cand[i]) - 1)) & mask;
                if (key[i].eq(t.keys + slot * KB, KB)) {
                    hit[i] = slot;
                    cand[i] = 0;
                    stop |= 1u << i;
                } else {
                    cand[i] &= cand[i] - 1;
                }
                more |= cand[i];
            }
            if (!more) break;
        }
        act &= ~stop;
#pragma unroll
        for (int i = 0; i < Q; i++) wb[i] += 8;
    }
    // values: a few hits' loads in flight before their stores
    constexpr int VG = VB >= 64 ? 1 : Q;
#pragma unroll
    for (int g = 0; g < Q; g += VG) {
        RegVal<VB> v[VG];
#pragma unroll
        for (int i = 0; i < VG; i++) {
            if (g + i >= Q) break;
            if (ov && hit[g + i] != NONE64) v[i].load(t.vals + hit[g + i] * VB, VB);
            else v[i].zero();
        }
#pragma unroll
        for (int i = 0; i < VG; i++) {
            if (g + i >= Q) break;
            const uint64_t q = q0 + (uint64_t)(g + i) * stride;
            if (q >= q1) continue;
            if (ov) v[i].store(ov + q * VB, VB);
            if (of) of[q] = hit[g + i] != NONE64 ? 1 : 0;
        }
    }
}

// Sorts a[0..n) ascending in shared memory (a holds the next power of two
// >= n words): bitonic network over that power of two, padded with
// 0xFFFFFFFF.  Block-uniform call.
static __device__ __noinline__ void block_sort_u32(uint32_t* a, uint32_t n) {
    uint32_t P = 1;
    while (P < n) P <<= 1;
    for (uint32_t i = n + threadIdx.x; i < P; i += blockDim.x) a[i] = 0xFFFFFFFFu;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t d = k >> 1; d > 0; d >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                const uint32_t m = i ^ d;
                if (m > i) {
                    const uint32_t x = a[i], y = a[m];
                    if ((x > y) == ((i & k) == 0)) {
                        a[i] = y;
                        a[m] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// First EMPTY slot at or after home h, NONE64 when the table has none (two
// aligned 8-slot windows per round trip with capacity >= 8).
__device__ __forceinline__ uint64_t rx_first_empty(const TableView& t, uint64_t h) {
    const uint64_t mask = t.mask;
    if (mask >= 7) {
        uint64_t wb = h & ~7ull;
        for (uint64_t w = 0; w <= (mask >> 4) + 1; ++w, wb += 16) {
            const uint4* p0 = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
            const uint4* p1 = reinterpret_cast<const uint4*>(t.flags + ((wb + 8) & mask));
            const uint4 a = p0[0], b = p0[1], c = p1[0], d = p1[1];
            const uint32_t f16[16] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w};
#pragma unroll
            for (int l = 0; l < 16; l++) {
                const uint64_t pos = wb + l;
                if (pos < h) continue;
                if (pos - h > mask) return NONE64;
                if (st_of(f16[l]) == ST_EMPTY) return pos & mask;
            }
        }
        return NONE64;
    }
    for (uint64_t p = 0; p <= mask; ++p)
        if (st_of(t.flags[(h + p) & mask]) == ST_EMPTY) return (h + p) & mask;
    return NONE64;
}

// The probe of one remove (rayon_cpu.rs:273-328): skip TOMBSTONEs, stop at
// EMPTY or at the Robin Hood exit (OCCUPIED with depth > stored distance) or
// at the first OCCUPIED slot holding the key (its stored distance equal to the
// depth).  Returns that slot (NONE64: a miss) and, in *stop, the slot where
// the probe stopped (the match, the terminator, or NONE64 when it went round
// the whole table).  With `commit` the match becomes the whole word TOMBSTONE.
template <int KB>
__device__ __forceinline__ uint64_t rx_look(const TableView& t, const RegKey<KB>& key, uint64_t h, bool commit,
                                            uint64_t* stop) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint64_t mask = t.mask;
    if (mask >= 7) {
        for (uint64_t wb = h & ~7ull;; wb += 8) {
            const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
            const uint4 a = fp[0], b = fp[1];
            const uint32_t f8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int l = 0; l < 8; l++) {
                const uint64_t pos = wb + l;
                if (pos < h) continue;
                const uint64_t p = pos - h;
                if (p > mask) {
                    *stop = NONE64;
                    return NONE64;
                }
                const uint32_t f = f8[l];
                const uint32_t st = st_of(f);
                const uint64_t slot = pos & mask;
                if (st == ST_EMPTY || (st == ST_OCC && p > dist_of(f))) {
                    *stop = slot;
                    return NONE64;
                }
                if (st == ST_OCC && dist_matches(f, p) && key.eq(t.keys + slot * ksz, ksz)) {
                    if (commit) t.flags[slot] = ST_TOMB;
                    *stop = slot;
                    return slot;
                }
            }
        }
    }
    for (uint64_t p = 0; p <= mask; ++p) {
        const uint64_t slot = (h + p) & mask;
        const uint32_t f = t.flags[slot];
        const uint32_t st = st_of(f);
        if (st == ST_EMPTY || (st == ST_OCC && p > dist_of(f))) {
            *stop = slot;
            return NONE64;
        }
        if (st == ST_OCC && dist_matches(f, p) && key.eq(t.keys + slot * ksz, ksz)) {
            if (commit) t.flags[slot] = ST_TOMB;
            *stop = slot;
            return slot;
        }
    }
    *stop = NONE64;
    return NONE64;
}

// The sequential remove of one key: 1 when it tombstoned a slot.
template <int KB>
__device__ __forceinline__ uint32_t rx_probe(const TableView& t, const RegKey<KB>& key, uint64_t h) {
    uint64_t stop;
    return rx_look<KB>(t, key, h, true, &stop) != NONE64 ? 1u : 0u;
}

// Up to 32 removes (the indices in ops[0..cnt), in index order) on one warp
// with the sequential result: every lane probes its op on the table as it is
// (no writes), then the warp commits the ops in index order.  An op whose
// probe range [home, stop] (measured from its home, the whole table when its
// probe went round it) holds a slot an earlier op of these tombstoned probes
// again on the current table; any other op's probe is unchanged by them
// (removes change nothing but those slots).  Returns the count removed (on
// every lane).  Warp-uniform call; the table may have no EMPTY slot.
template <int KB>
__device__ __forceinline__ uint32_t rx_chunk32(const TableView& t, const uint8_t* keys, const uint32_t* ops,
                                               uint32_t cnt) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t mask = t.mask;
    RegKey<KB> key;
    uint64_t h = 0, stop = NONE64, tgt = NONE64;
    if (lane < cnt) {
        h = home_of<KB>(t, keys, ops[lane], key);
        tgt = rx_look<KB>(t, key, h, false, &stop);
    }
    const uint64_t span = stop == NONE64 ? mask : ((stop - h) & mask);  // probe range, from home
    bool done_t = false;  // this lane's op tombstoned tgt
    uint32_t removed = 0;
    for (uint32_t i = 0; i < cnt; i++) {
        const uint64_t hi = __shfl_sync(0xFFFFFFFFu, h, i);
        const uint64_t si = __shfl_sync(0xFFFFFFFFu, span, i);
        const bool hit_range = done_t && ((tgt - hi) & mask) <= si;
        const bool conflict = __ballot_sync(0xFFFFFFFFu, lane < i && hit_range) != 0;
        if (lane == i) {
            if (conflict) {
                uint64_t st2;
                tgt = rx_look<KB>(t, key, h, true, &st2);
            } else if (tgt != NONE64) {
                t.flags[tgt] = ST_TOMB;
            }
            if (tgt != NONE64) {
                done_t = true;
                ++removed;
            }
        }
        __syncwarp();
    }
    return __reduce_add_sync(0xFFFFFFFFu, removed);
}

// Ops of a group of removes (equal first EMPTY slot) a warp runs itself; up
// to RX_THREAD of them one thread runs.
constexpr uint32_t RX_GMAX = 256;
#ifndef FM_RX_THREAD
#define FM_RX_THREAD 16
#endif
constexpr uint32_t RX_THREAD = FM_RX_THREAD;
constexpr uint32_t RX_BMAX = 8192;  // ops of a group one block sorts in shared memory

template <int KB>
__device__ __noinline__ uint32_t rx_group_run(const TableView& t, const uint8_t* keys, uint64_t E, uint32_t g,
                                              uint32_t* s_grp);

// The removes of the group at EMPTY slot E (c ops listed from seg_min[E]
// through the per-op words) on one warp: lane 0 gathers the list into
// s_grp (registrations set idle), the warp sorts it by index, then, 32 at a
// time, every lane probes its op on the table as it is (no writes) and the
// warp commits the ops in index order: an op whose probe range [home, stop]
// holds a slot that an earlier op of its chunk tombstoned probes again on the
// current table; any other op's probe is unchanged by them (removes change
// nothing but those slots), so its result stands.  Returns the ops removed
// (the group's total, on every lane);
// a group of more than RX_GMAX ops goes to pend[1] instead (0 returned).
// Warp-uniform call.
template <int KB>
__device__ __noinline__ uint32_t rx_group(const TableView& t, const uint8_t* keys, uint32_t n0, const OpScratch& sc,
                                          Ctl* ctl, uint64_t E, uint32_t c, uint32_t* s_grp) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t g = 0;
    if (lane == 0) {
        uint32_t x = t.seg_min[E];
        for (uint32_t q = 0; q < c && x != IDLE; q++) {
            if (x >= n0) {
                atomicOr(&ctl->err, ERR_SCRATCH);
                break;
            }
            const uint32_t nx = sc.op_word[x];
            sc.op_word[x] = IDLE;
            if (c <= RX_GMAX) s_grp[g++] = x;
            else sc.pend[1][atomicAdd(&ctl->npend[1], 1u)] = x;
            x = nx;
        }
        t.seg_min[E] = IDLE;
        t.seg_cnt[E] = 0;
    }
    g = __shfl_sync(0xFFFFFFFFu, g, 0);
    __syncwarp();
    return rx_group_run<KB>(t, keys, E, g, s_grp);
}

// The g ops of a group (indices in s_grp[0..g), any order, g <= RX_GMAX) at
// EMPTY slot E, sorted into index order by the warp and run in chunks of 32
// as rx_group describes.  Returns the count removed (on every lane).
template <int KB>
__device__ __noinline__ uint32_t rx_group_run(const TableView& t, const uint8_t* keys, uint64_t E, uint32_t g,
                                              uint32_t* s_grp) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t mask = t.mask;
    if (g == 0) return 0;
    // index order: the rank of each entry among the group
    uint32_t v[RX_GMAX / 32], r[RX_GMAX / 32];
#pragma unroll
    for (int u = 0; u < (int)(RX_GMAX / 32); u++) {
        const uint32_t q = lane + 32 * u;
        v[u] = q < g ? s_grp[q] : 0u;
        r[u] = 0;
    }
    for (uint32_t q = 0; q < g; q++) {
        const uint32_t y = s_grp[q];
#pragma unroll
        for (int u = 0; u < (int)(RX_GMAX / 32); u++) r[u] += y < v[u] ? 1u : 0u;
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < (int)(RX_GMAX / 32); u++)
        if (lane + 32 * u < g) s_grp[r[u]] = v[u];
    __syncwarp();
    uint32_t removed = 0;
    for (uint32_t c0 = 0; c0 < g; c0 += 32) {
        const uint32_t cnt = min(32u, g - c0);
        const bool mine = lane < cnt;
        RegKey<KB> key;
        uint64_t h = 0, stop = 0, tgt = NONE64;
        if (mine) {
            h = home_of<KB>(t, keys, s_grp[c0 + lane], key);
            tgt = rx_look<KB>(t, key, h, false, &stop);
        }
        // distances before E: a slot s lies in [h, stop] when d(h) >= d(s) >= d(stop)
        const uint64_t dh = (E - h) & mask;
        const uint64_t ds = stop == NONE64 ? 0 : ((E - stop) & mask);
        uint64_t dt = tgt == NONE64 ? NONE64 : ((E - tgt) & mask);
        bool done_t = false;  // this lane's op has tombstoned its target (in this chunk)
        for (uint32_t i = 0; i < cnt; i++) {
            const uint64_t hi = __shfl_sync(0xFFFFFFFFu, dh, i);
            const uint64_t si = __shfl_sync(0xFFFFFFFFu, ds, i);
            const bool hit_range = done_t && dt != NONE64 && dt <= hi && dt >= si;
            const bool conflict = __ballot_sync(0xFFFFFFFFu, (int)lane < (int)i && hit_range) != 0;
            if (lane == i) {
                if (conflict) {  // an earlier op changed a slot of this probe: probe again
                    uint64_t st2;
                    tgt = rx_look<KB>(t, key, h, true, &st2);
                    dt = tgt == NONE64 ? NONE64 : ((E - tgt) & mask);
                } else if (tgt != NONE64) {
                    t.flags[tgt] = ST_TOMB;
                }
                if (tgt != NONE64) {
                    done_t = true;
                    ++removed;
                }
            }
            __syncwarp();
        }
    }
    return __reduce_add_sync(0xFFFFFFFFu, removed);  // each lane counted the ops it committed
}

}  // namespace fm

// fm_kernels.cu -- sm_100a kernels of the FlashMap B200 backend.
//
// Semantics: every kernel reproduces the reference's sequential results
// (bajpainaman/flash-map 0.5.0, src/rayon_cpu.rs:82-328 applied one operation
// at a time in batch index order) bit for bit, including in-batch duplicate
// keys (later position wins), tombstone reuse and the Robin Hood early exit.
//
//  * get     (k_get): read-only, one tile of T lanes per query.  The tile reads
//            T consecutive metadata words per step (one 32-byte sector for
//            T = 8), finds the first terminating slot with a ballot, compares
//            keys only in slots whose stored distance equals the probe depth,
//            and copies the value with 16-byte vector moves spread over the
//            tile's lanes.  Mirrors kernels.cu:365-556 / rayon_cpu.rs:82-126.
//  * insert  (k_ins_probe / k_ins_walk / k_ins_exec, in rounds): an insert
//            only reads and writes slots in [home, F] where F is the first
//            EMPTY-or-TOMBSTONE slot at or after home, so operations whose
//            segments end at different free slots commute.  Each round runs
//            the lowest-index op of every segment unless an earlier op could
//            still flow into that segment once free slots before it are
//            consumed (bounded by a forward walk from every segment holding
//            two or more pending ops).  rayon_cpu.rs:133-270.
//  * remove  (k_rem_scan / k_rem_check / k_rem_reset, in rounds): an op runs
//            unless an earlier pending op has a possible target inside its
//            dependency window.  rayon_cpu.rs:273-328.
#include <atomic>

#include "fm_internal.h"

namespace fm {

namespace {

constexpr int BLOCK = 256;
int g_num_sms = 0;
std::atomic<unsigned long long> g_launches{0};

__device__ __forceinline__ uint32_t warp_min_u32(uint32_t v) { return __reduce_min_sync(0xFFFFFFFFu, v); }

// Warp-aggregated append of `j` to a list: one atomic per warp.
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

// ---------------------------------------------------------------------------
// Tile-cooperative value moves.
// ---------------------------------------------------------------------------
template <int VB, int T>
__device__ __forceinline__ void tile_copy(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, uint32_t vsz,
                                          uint32_t lane) {
    if constexpr (VB == 0) {
        for (uint32_t i = lane; i < vsz; i += T) dst[i] = src[i];
    } else if constexpr (VB % 16 == 0) {
#pragma unroll
        for (uint32_t i = lane; i < VB / 16; i += T)
            reinterpret_cast<uint4*>(dst)[i] = __ldg(reinterpret_cast<const uint4*>(src) + i);
    } else if constexpr (VB % 8 == 0) {
#pragma unroll
        for (uint32_t i = lane; i < VB / 8; i += T)
            reinterpret_cast<uint2*>(dst)[i] = __ldg(reinterpret_cast<const uint2*>(src) + i);
    } else {
#pragma unroll
        for (uint32_t i = lane; i < VB / 4; i += T)
            reinterpret_cast<uint32_t*>(dst)[i] = __ldg(reinterpret_cast<const uint32_t*>(src) + i);
    }
}

template <int VB, int T>
__device__ __forceinline__ void tile_zero(uint8_t* __restrict__ dst, uint32_t vsz, uint32_t lane) {
    if constexpr (VB == 0) {
        for (uint32_t i = lane; i < vsz; i += T) dst[i] = 0;
    } else if constexpr (VB % 16 == 0) {
#pragma unroll
        for (uint32_t i = lane; i < VB / 16; i += T) reinterpret_cast<uint4*>(dst)[i] = make_uint4(0, 0, 0, 0);
    } else if constexpr (VB % 8 == 0) {
#pragma unroll
        for (uint32_t i = lane; i < VB / 8; i += T) reinterpret_cast<uint2*>(dst)[i] = make_uint2(0, 0);
    } else {
#pragma unroll
        for (uint32_t i = lane; i < VB / 4; i += T) reinterpret_cast<uint32_t*>(dst)[i] = 0u;
    }
}

// ---------------------------------------------------------------------------
// bulk_get: one T-lane tile per query.
// ---------------------------------------------------------------------------
template <int KB, int VB, int T>
__global__ void __launch_bounds__(BLOCK) k_get(TableView t, const uint8_t* __restrict__ qkeys, uint64_t n,
                                               uint8_t* __restrict__ out_vals, uint8_t* __restrict__ out_found) {
    static_assert(T == 4 || T == 8 || T == 16 || T == 32, "tile width");
    constexpr uint32_t TM = (T == 32) ? 0xFFFFFFFFu : ((1u << T) - 1u);
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint32_t vsz = VB ? (uint32_t)VB : t.vsz;
    const uint32_t lane = threadIdx.x & (T - 1);
    const uint32_t tbase = (threadIdx.x & 31u) & ~(uint32_t)(T - 1);
    const uint32_t tmask = TM << tbase;
    const uint64_t mask = t.mask;
    const uint64_t ntiles = ((uint64_t)gridDim.x * blockDim.x) / T;
    for (uint64_t q = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / T; q < n; q += ntiles) {
        RegKey<KB> key;
        key.load(qkeys + q * ksz, ksz);
        const uint64_t h = key.hash(ksz, t.hash_mode) & mask;
        uint64_t wbase = h & ~(uint64_t)(T - 1);  // sector-aligned window start
        uint64_t hit = NONE64;
        for (;;) {
            const uint64_t pos = wbase + lane;
            const bool before = pos < h;
            const uint64_t p = pos - h;
            const uint64_t slot = pos & mask;
            const uint32_t f = __ldg(t.flags + slot);
            const uint32_t s = st_of(f);
            const bool past = !before && p > mask;
            // Terminators: EMPTY, or OCCUPIED with p > dist (rayon_cpu.rs:97-111);
            // the probe also ends once p passes the capacity (rayon_cpu.rs:91).
            const bool term = !before && (past || s == ST_EMPTY || (s == ST_OCC && p > dist_of(f)));
            const bool cand = !before && !past && s == ST_OCC && dist_matches(f, p);
            const uint32_t tm = (__ballot_sync(tmask, term) >> tbase) & TM;
            const uint32_t lim = tm ? (uint32_t)(__ffs(tm) - 1) : (uint32_t)T;
            const bool m = cand && lane < lim && key.eq(t.keys + slot * ksz, ksz);
            const uint32_t mm = (__ballot_sync(tmask, m) >> tbase) & TM;
            if (mm) {
                hit = __shfl_sync(tmask, slot, tbase + __ffs(mm) - 1);
                break;
            }
            if (tm) break;
            wbase += T;
        }
        if (out_vals) {
            uint8_t* dst = out_vals + q * vsz;
            if (hit != NONE64) tile_copy<VB, T>(dst, t.vals + hit * vsz, vsz, lane);
            else tile_zero<VB, T>(dst, vsz, lane);
        }
        if (out_found && lane == 0) out_found[q] = hit != NONE64 ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Insert, round phase 1: find each pending op's terminating free slot F and
// register the op there (lowest index and count per segment).
// ---------------------------------------------------------------------------
template <int KB>
__global__ void __launch_bounds__(BLOCK) k_ins_probe(TableView t, const uint8_t* __restrict__ keys,
                                                     const uint32_t* __restrict__ pend, uint32_t npend,
                                                     uint64_t* __restrict__ op_slot, Ctl* ctl) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint64_t mask = t.mask;
    uint32_t my_min = IDLE;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t iters = (npend + stride - 1) / stride;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t i = i0 + it * stride;
        if (i < npend) {
            const uint32_t j = pend[i];
            RegKey<KB> key;
            key.load(keys + (uint64_t)j * ksz, ksz);
            const uint64_t h = key.hash(ksz, t.hash_mode) & mask;
            uint64_t F = NONE64;
            for (uint64_t p = 0; p <= mask; ++p) {
                const uint64_t s = (h + p) & mask;
                if (is_free(t.flags[s])) {
                    F = s;
                    break;
                }
            }
            op_slot[j] = F;
            if (F == NONE64) {
                atomicExch(&ctl->serial, 1u);  // no free slot anywhere: run one op per round
            } else {
                atomicMin(&t.seg_min[F], j);
                atomicAdd(&t.seg_cnt[F], 1u);
            }
            my_min = min(my_min, j);
        }
    }
    my_min = warp_min_u32(my_min);
    if ((threadIdx.x & 31u) == 0 && my_min != IDLE) atomicMin(&ctl->gmin, my_min);
}

// ---------------------------------------------------------------------------
// Insert, round phase 2: leaders; forward flow walks from crowded segments.
// A segment holding c >= 2 pending ops can push up to c-1 of them past its
// free slot; a walker carries that flow forward over the following segments
// (each absorbs one op at its free slot, adds its own pending ops) and marks
// every segment it reaches with a lower bound on the indices that could
// arrive.  That segment's leader waits while an earlier op could arrive.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(BLOCK) k_ins_walk(TableView t, const uint32_t* __restrict__ pend, uint32_t npend,
                                                    uint32_t nops, const uint64_t* __restrict__ op_slot,
                                                    uint32_t* op_block, uint8_t* __restrict__ op_leader, Ctl* ctl) {
    const uint64_t mask = t.mask;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npend; i += gridDim.x * blockDim.x) {
        const uint32_t j = pend[i];
        const uint64_t F = op_slot[j];
        const bool leader = F != NONE64 && t.seg_min[F] == j;
        op_leader[j] = leader ? 1 : 0;
        if (!leader) continue;
        const uint32_t c = t.seg_cnt[F];
        if (c < 2) continue;
        uint64_t flow = c - 1;
        uint32_t L = j;
        uint64_t pos = F + 1;
        uint64_t walked = 0;
        for (;;) {
            // Scan at most the capacity-1 slots after F; coming back to F means
            // the flow wraps the whole table.
            uint64_t F2 = NONE64;
            while (walked < mask) {
                const uint64_t s = pos & mask;
                ++pos;
                ++walked;
                if (is_free(t.flags[s])) {
                    F2 = s;
                    break;
                }
            }
            if (F2 == NONE64) {  // the flow wraps the whole table: fall back to one op per round
                atomicExch(&ctl->serial, 1u);
                break;
            }
            const uint32_t c2 = t.seg_cnt[F2];
            if (c2) {
                const uint32_t l2 = t.seg_min[F2];
                if (l2 >= nops) {  // registrations come only from this call's ops
                    atomicOr(&ctl->err, ERR_SCRATCH);
                    break;
                }
                atomicMin(&op_block[l2], L);
                L = min(L, l2);
            }
            flow = flow + c2 - 1;
            if (flow == 0) break;
        }
    }
}

// The sequential insert of one key (rayon_cpu.rs:157-264), run by one thread
// on the segment it owns this round.  Returns 1 when a free slot was claimed.
template <int KB, int VB>
__device__ __forceinline__ int exec_insert(const TableView& t, const uint8_t* kin, const uint8_t* vin,
                                           uint32_t& maxd, bool& tomb, bool& limit_hit) {
    const uint64_t mask = t.mask;
    RegKey<KB> ck;
    ck.load(kin, KB);
    RegVal<VB> cv;
    cv.load(vin, VB);
    uint64_t h = ck.hash(KB, t.hash_mode) & mask;
    uint64_t p = 0;
    const uint64_t step_limit = 2 * (mask + 1) + 2;
    for (uint64_t step = 0;; ++step) {
        if (p > mask) return 0;  // drop (rayon_cpu.rs:167-169)
        if (step > step_limit) {  // full table: the reference's loop may never end
            limit_hit = true;
            return 0;
        }
        const uint64_t idx = (h + p) & mask;
        const uint32_t f = t.flags[idx];
        const uint32_t s = st_of(f);
        if (s == ST_OCC) {
            if (dist_matches(f, p) && ck.eq(t.keys + idx * KB, KB)) {
                cv.store(t.vals + idx * VB, VB);  // update in place
                return 0;
            }
            const uint64_t d = dist_of(f);
            if (p > d) {  // Robin Hood eviction
                RegKey<KB> tk;
                tk.load_table(t.keys + idx * KB, KB);
                RegVal<VB> tv;
                tv.load(t.vals + idx * VB, VB);
                ck.store(t.keys + idx * KB, KB);
                cv.store(t.vals + idx * VB, VB);
                t.flags[idx] = mk_flag(ST_OCC, p);
                maxd = max(maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
                ck = tk;
                cv = tv;
                h = ck.hash(KB, t.hash_mode) & mask;
                p = d + 1;
                continue;
            }
            ++p;
            continue;
        }
        if (s == ST_EMPTY || s == ST_TOMB) {
            ck.store(t.keys + idx * KB, KB);
            cv.store(t.vals + idx * VB, VB);
            t.flags[idx] = mk_flag(ST_OCC, p);
            maxd = max(maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
            tomb = tomb || s == ST_TOMB;
            return 1;
        }
        ++p;
    }
}

// Run-time sizes (up to GENERIC_MAX_KV bytes each): the carried entry lives in
// a local buffer and is swapped with the slot byte by byte.
__device__ __forceinline__ int exec_insert_generic(const TableView& t, const uint8_t* kin, const uint8_t* vin,
                                                   uint32_t& maxd, bool& tomb, bool& limit_hit) {
    const uint64_t mask = t.mask;
    const uint32_t ksz = t.ksz, vsz = t.vsz;
    uint8_t ck[GENERIC_MAX_KV];
    uint8_t cv[GENERIC_MAX_KV];
    copy_bytes(ck, kin, ksz);
    copy_bytes(cv, vin, vsz);
    uint64_t h = hash_bytes(ck, ksz, t.hash_mode) & mask;
    uint64_t p = 0;
    const uint64_t step_limit = 2 * (mask + 1) + 2;
    for (uint64_t step = 0;; ++step) {
        if (p > mask) return 0;
        if (step > step_limit) {
            limit_hit = true;
            return 0;
        }
        const uint64_t idx = (h + p) & mask;
        const uint32_t f = t.flags[idx];
        const uint32_t s = st_of(f);
        uint8_t* sk = t.keys + idx * ksz;
        uint8_t* sv = t.vals + idx * vsz;
        if (s == ST_OCC) {
            bool eq = dist_matches(f, p);
            for (uint32_t i = 0; eq && i < ksz; i++) eq = sk[i] == ck[i];
            if (eq) {
                copy_bytes(sv, cv, vsz);
                return 0;
            }
            const uint64_t d = dist_of(f);
            if (p > d) {
                for (uint32_t i = 0; i < ksz; i++) {
                    uint8_t x = sk[i];
                    sk[i] = ck[i];
                    ck[i] = x;
                }
                for (uint32_t i = 0; i < vsz; i++) {
                    uint8_t x = sv[i];
                    sv[i] = cv[i];
                    cv[i] = x;
                }
                t.flags[idx] = mk_flag(ST_OCC, p);
                maxd = max(maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
                h = hash_bytes(ck, ksz, t.hash_mode) & mask;
                p = d + 1;
                continue;
            }
            ++p;
            continue;
        }
        if (s == ST_EMPTY || s == ST_TOMB) {
            copy_bytes(sk, ck, ksz);
            copy_bytes(sv, cv, vsz);
            t.flags[idx] = mk_flag(ST_OCC, p);
            maxd = max(maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
            tomb = tomb || s == ST_TOMB;
            return 1;
        }
        ++p;
    }
}

// ---------------------------------------------------------------------------
// Insert, round phase 3: unblocked leaders run; everyone clears its segment
// registration; ops that did not run go to the next round's list.
// ---------------------------------------------------------------------------
template <int KB, int VB>
__global__ void __launch_bounds__(BLOCK) k_ins_exec(TableView t, const uint8_t* __restrict__ keys,
                                                    const uint8_t* __restrict__ vals,
                                                    const uint32_t* __restrict__ pend, uint32_t npend,
                                                    uint32_t* __restrict__ pend_next,
                                                    const uint64_t* __restrict__ op_slot, uint32_t* op_block,
                                                    const uint8_t* __restrict__ op_leader, Ctl* ctl) {
    const bool serial = *(volatile uint32_t*)&ctl->serial != 0;
    const uint32_t gmin = *(volatile uint32_t*)&ctl->gmin;
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint32_t vsz = VB ? (uint32_t)VB : t.vsz;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t iters = (npend + stride - 1) / stride;
    uint32_t maxd = 0, claimed = 0;
    bool tomb = false, limit_hit = false;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t i = i0 + it * stride;
        const bool valid = i < npend;
        uint32_t j = 0;
        bool run = false;
        if (valid) {
            j = pend[i];
            run = serial ? (j == gmin) : (op_leader[j] != 0 && op_block[j] > j);
            if (run) {
                if constexpr (KB == 0 || VB == 0)
                    claimed += exec_insert_generic(t, keys + (uint64_t)j * ksz, vals + (uint64_t)j * vsz, maxd, tomb,
                                                   limit_hit);
                else
                    claimed += exec_insert<KB, VB>(t, keys + (uint64_t)j * ksz, vals + (uint64_t)j * vsz, maxd, tomb,
                                                   limit_hit);
            }
            const uint64_t F = op_slot[j];
            if (F != NONE64) {
                t.seg_min[F] = IDLE;
                t.seg_cnt[F] = 0;
            }
            op_block[j] = IDLE;
        }
        append(pend_next, &ctl->npend_next, j, valid && !run);
    }
    const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, claimed);
    const uint32_t md = __reduce_max_sync(0xFFFFFFFFu, maxd);
    const bool tb = __any_sync(0xFFFFFFFFu, tomb);
    const bool lh = __any_sync(0xFFFFFFFFu, limit_hit);
    if ((threadIdx.x & 31u) == 0) {
        if (lh) atomicOr(&ctl->err, ERR_WALK_LIMIT);
        if (c) atomicAdd(&ctl->count, (unsigned long long)c);
        if (md > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, md);
        if (tb) ctl->tomb_claimed = 1u;
    }
}

// ---------------------------------------------------------------------------
// Remove, round phase 1: probe, then mark every possible target of the op
// (slots holding its key within [home, min(first EMPTY - 1, X + dmax)], X the
// current target or home) with the op's index.
// ---------------------------------------------------------------------------
template <int KB>
__global__ void __launch_bounds__(BLOCK) k_rem_scan(TableView t, const uint8_t* __restrict__ keys,
                                                    const uint32_t* __restrict__ pend, uint32_t npend,
                                                    OpScratch sc, const Ctl* __restrict__ ctl) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint64_t mask = t.mask;
    const uint64_t dmax = ctl->dmax;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npend; i += gridDim.x * blockDim.x) {
        const uint32_t j = pend[i];
        RegKey<KB> key;
        key.load(keys + (uint64_t)j * ksz, ksz);
        const uint64_t h = key.hash(ksz, t.hash_mode) & mask;
        uint64_t tp = NONE64;  // probe depth of the current target
        uint64_t p = 0;
        bool empty_hit = false;
        for (; p <= mask; ++p) {
            const uint64_t s = (h + p) & mask;
            const uint32_t f = t.flags[s];
            const uint32_t st = st_of(f);
            if (st == ST_EMPTY) {
                empty_hit = true;
                break;
            }
            if (st == ST_OCC) {
                if (p > dist_of(f)) break;
                if (dist_matches(f, p) && key.eq(t.keys + s * ksz, ksz)) {
                    tp = p;
                    break;
                }
            }
        }
        uint64_t lim = (tp != NONE64 ? tp : 0) + dmax;
        if (lim > mask) lim = mask;
        uint32_t npt = 0;
        uint64_t wend;
        auto mark = [&](uint64_t q) {
            const uint64_t s = (h + q) & mask;
            atomicMin(&t.seg_min[s], j);
            if (npt < PT_MAX) sc.op_pt[(uint64_t)j * PT_MAX + npt] = (uint32_t)q;
            ++npt;
        };
        if (empty_hit) {
            wend = p == 0 ? 0 : min(p - 1, lim);
            if (p == 0) wend = NONE64;  // home slot EMPTY: nothing to watch
        } else {
            if (tp != NONE64) mark(tp);
            uint64_t q = (tp != NONE64 ? tp : p) + 1;
            wend = min(p, lim);
            for (; q <= lim; ++q) {
                const uint64_t s = (h + q) & mask;
                const uint32_t f = t.flags[s];
                const uint32_t st = st_of(f);
                if (st == ST_EMPTY) break;
                wend = q;
                if (st == ST_OCC && dist_matches(f, q) && key.eq(t.keys + s * ksz, ksz)) mark(q);
            }
        }
        sc.op_slot[j] = tp != NONE64 ? ((h + tp) & mask) : NONE64;
        sc.op_word[j] = wend == NONE64 ? IDLE : (uint32_t)wend;
        sc.op_flag[j] = (uint8_t)min(npt, 255u);
    }
}

// Remove, round phase 2: an op runs unless an earlier pending op marked a slot
// inside its window; a running op with a target writes the tombstone word.
template <int KB>
__global__ void __launch_bounds__(BLOCK) k_rem_check(TableView t, const uint8_t* __restrict__ keys,
                                                     const uint32_t* __restrict__ pend, uint32_t npend,
                                                     uint32_t* __restrict__ pend_next, OpScratch sc, Ctl* ctl) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint64_t mask = t.mask;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t iters = (npend + stride - 1) / stride;
    uint32_t removed = 0;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t i = i0 + it * stride;
        const bool valid = i < npend;
        uint32_t j = 0;
        bool run = false;
        if (valid) {
            j = pend[i];
            RegKey<KB> key;
            key.load(keys + (uint64_t)j * ksz, ksz);
            const uint64_t h = key.hash(ksz, t.hash_mode) & mask;
            const uint32_t wend = sc.op_word[j];
            run = true;
            if (wend != IDLE) {
                for (uint64_t q = 0; q <= wend; ++q) {
                    if (t.seg_min[(h + q) & mask] < j) {
                        run = false;
                        break;
                    }
                }
            }
            if (run) {
                const uint64_t ts = sc.op_slot[j];
                if (ts != NONE64) {
                    t.flags[ts] = ST_TOMB;  // whole word 2: TOMBSTONE, dist 0 (rayon_cpu.rs:306-313)
                    ++removed;
                }
            }
        }
        append(pend_next, &ctl->npend_next, j, valid && !run);
    }
    const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, removed);
    if ((threadIdx.x & 31u) == 0 && c) atomicAdd(&ctl->count, (unsigned long long)c);
}

// Remove, round phase 3: clear this round's marks.
template <int KB>
__global__ void __launch_bounds__(BLOCK) k_rem_reset(TableView t, const uint8_t* __restrict__ keys,
                                                     const uint32_t* __restrict__ pend, uint32_t npend,
                                                     OpScratch sc) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint64_t mask = t.mask;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npend; i += gridDim.x * blockDim.x) {
        const uint32_t j = pend[i];
        const uint32_t npt = sc.op_flag[j];
        const uint32_t wend = sc.op_word[j];
        sc.op_word[j] = IDLE;  // the word is the insert's inflow bound between calls
        if (npt == 0) continue;
        RegKey<KB> key;
        key.load(keys + (uint64_t)j * ksz, ksz);
        const uint64_t h = key.hash(ksz, t.hash_mode) & mask;
        if (npt <= PT_MAX) {
            for (uint32_t k = 0; k < npt; k++) t.seg_min[(h + sc.op_pt[(uint64_t)j * PT_MAX + k]) & mask] = IDLE;
        } else {
            for (uint64_t q = 0; q <= wend; ++q) {
                const uint64_t s = (h + q) & mask;
                if (t.seg_min[s] != IDLE) t.seg_min[s] = IDLE;
            }
        }
    }
}

__global__ void k_iota(uint32_t* p, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

// Count OCCUPIED slots (kernels.cu:328-337), reduced per block.
__global__ void __launch_bounds__(BLOCK) k_count(const uint32_t* __restrict__ flags, uint64_t cap, Ctl* ctl) {
    uint32_t c = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x)
        c += st_of(__ldg(flags + i)) == ST_OCC;
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    __shared__ uint32_t part[BLOCK / 32];
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < BLOCK / 32; w++) s += part[w];
        if (s) atomicAdd(&ctl->occupied, (unsigned long long)s);
    }
}

unsigned grid_for(uint64_t threads, unsigned per_sm) {
    const uint64_t want = (threads + BLOCK - 1) / BLOCK;
    const uint64_t cap = (uint64_t)num_sms() * per_sm;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

template <int KB, int VB>
cudaError_t get_shape(const TableView& t, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of, cudaStream_t s) {
    constexpr int T = 8;
    k_get<KB, VB, T><<<grid_for(n * T, 16), BLOCK, 0, s>>>(t, q, n, ov, of);
    g_launches += 1;
    return cudaGetLastError();
}

template <int KB, int VB>
cudaError_t ins_round_shape(const TableView& t, const uint8_t* keys, const uint8_t* vals, const uint32_t* pend,
                            uint32_t npend, uint32_t nops, uint32_t* pend_next, const OpScratch& sc, Ctl* ctl,
                            cudaStream_t s) {
    const unsigned g = grid_for(npend, 8);
    k_ins_probe<KB><<<g, BLOCK, 0, s>>>(t, keys, pend, npend, sc.op_slot, ctl);
    k_ins_walk<<<g, BLOCK, 0, s>>>(t, pend, npend, nops, sc.op_slot, sc.op_word, sc.op_flag, ctl);
    k_ins_exec<KB, VB><<<g, BLOCK, 0, s>>>(t, keys, vals, pend, npend, pend_next, sc.op_slot, sc.op_word,
                                           sc.op_flag, ctl);
    g_launches += 3;
    return cudaGetLastError();
}

template <int KB>
cudaError_t rem_round_shape(const TableView& t, const uint8_t* keys, const uint32_t* pend, uint32_t npend,
                            uint32_t* pend_next, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    const unsigned g = grid_for(npend, 8);
    k_rem_scan<KB><<<g, BLOCK, 0, s>>>(t, keys, pend, npend, sc, ctl);
    k_rem_check<KB><<<g, BLOCK, 0, s>>>(t, keys, pend, npend, pend_next, sc, ctl);
    k_rem_reset<KB><<<g, BLOCK, 0, s>>>(t, keys, pend, npend, sc);
    g_launches += 3;
    return cudaGetLastError();
}

}  // namespace

unsigned long long launch_count() { return g_launches.load(); }

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        g_num_sms = v > 0 ? v : 148;
    }
    return g_num_sms;
}

Shape pick_shape(uint32_t k, uint32_t v) {
    if (k == 8 && v == 8) return SHAPE_8_8;
    if (k == 32 && v == 128) return SHAPE_32_128;
    if (k == 32 && v == 64) return SHAPE_32_64;
    if (k == 32 && v == 32) return SHAPE_32_32;
    if (k == 8 && v == 32) return SHAPE_8_32;
    return SHAPE_GENERIC;
}

cudaError_t launch_get(const TableView& t, Shape sh, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of,
                       cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    switch (sh) {
        case SHAPE_8_8: return get_shape<8, 8>(t, q, n, ov, of, s);
        case SHAPE_32_128: return get_shape<32, 128>(t, q, n, ov, of, s);
        case SHAPE_32_64: return get_shape<32, 64>(t, q, n, ov, of, s);
        case SHAPE_32_32: return get_shape<32, 32>(t, q, n, ov, of, s);
        case SHAPE_8_32: return get_shape<8, 32>(t, q, n, ov, of, s);
        default: return get_shape<0, 0>(t, q, n, ov, of, s);
    }
}

cudaError_t launch_iota(uint32_t* p, uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_iota<<<grid_for(n, 8), BLOCK, 0, s>>>(p, n);
    g_launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_ins_round(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals,
                             const uint32_t* pend, uint32_t npend, uint32_t nops, uint32_t* pend_next,
                             const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    switch (sh) {
        case SHAPE_8_8: return ins_round_shape<8, 8>(t, keys, vals, pend, npend, nops, pend_next, sc, ctl, s);
        case SHAPE_32_128: return ins_round_shape<32, 128>(t, keys, vals, pend, npend, nops, pend_next, sc, ctl, s);
        case SHAPE_32_64: return ins_round_shape<32, 64>(t, keys, vals, pend, npend, nops, pend_next, sc, ctl, s);
        case SHAPE_32_32: return ins_round_shape<32, 32>(t, keys, vals, pend, npend, nops, pend_next, sc, ctl, s);
        case SHAPE_8_32: return ins_round_shape<8, 32>(t, keys, vals, pend, npend, nops, pend_next, sc, ctl, s);
        default: return ins_round_shape<0, 0>(t, keys, vals, pend, npend, nops, pend_next, sc, ctl, s);
    }
}

cudaError_t launch_rem_round(const TableView& t, Shape sh, const uint8_t* keys, const uint32_t* pend,
                             uint32_t npend, uint32_t* pend_next, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    switch (sh) {
        case SHAPE_8_8:
        case SHAPE_8_32: return rem_round_shape<8>(t, keys, pend, npend, pend_next, sc, ctl, s);
        case SHAPE_32_128:
        case SHAPE_32_64:
        case SHAPE_32_32: return rem_round_shape<32>(t, keys, pend, npend, pend_next, sc, ctl, s);
        default: return rem_round_shape<0>(t, keys, pend, npend, pend_next, sc, ctl, s);
    }
}

cudaError_t launch_count(const TableView& t, Ctl* ctl, cudaStream_t s) {
    k_count<<<grid_for(t.mask + 1, 4), BLOCK, 0, s>>>(t.flags, t.mask + 1, ctl);
    g_launches += 1;
    return cudaGetLastError();
}

}  // namespace fm

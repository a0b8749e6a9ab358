// fm_insert.cu -- deterministic bulk insert for sm_100a.
//
// Semantics: the reference's sequential insert (src/rayon_cpu.rs:153-264; the
// same walk as src/kernels.cu:224-313 run one key at a time) applied to the
// batch in index order: Robin Hood eviction, update of an equal key in place,
// claim of the first EMPTY or TOMBSTONE slot, drop past the capacity, and
// in-batch duplicate keys resolved to the later position.
//
// Why rounds: an insert only reads and writes slots in [home, F], where F is
// the first free (EMPTY or TOMBSTONE) slot at or after its home, so ops whose
// segments end at different free slots touch disjoint slots and commute.  A
// round runs the lowest-index pending op of every segment ("leader") unless an
// earlier op could still reach that segment: a segment holding c >= 2 pending
// ops can push up to c-1 of them past its free slot once it is consumed, so a
// forward walk from every such segment carries that flow over the following
// segments (each absorbs one op at its free slot and adds its own) and marks
// the leaders it reaches with a lower bound on the op indices that could
// arrive.  The lowest pending op is never blocked, so every round makes
// progress.  When a round finds an op with no free slot anywhere (only an
// uncounted insert can overfill a table) or a flow that wraps the whole
// table, it runs nothing and the remaining ops are applied one at a time in
// index order by a single thread (serial_process).
//
// Control: two grid-wide rounds are launched back to back (counts and lists
// live in device memory, double-buffered by round parity), then one block
// runs every remaining round with block barriers between phases when at most
// TAIL_MAX ops are left.  The host reads the control block once per pass.
// Grid kernels aggregate list appends and counts per block so no address
// takes more than one atomic per block.
#include <climits>
#include <limits>
#include <cstdlib>
#include <type_traits>
#include <utility>

#include "fm_rounds.cuh"
#include "fm_probe.cuh"

namespace fm {
namespace {

// First free (EMPTY or TOMBSTONE) slot at or after home, NONE64 if the table
// has none.  With capacity >= 8 the metadata is read in aligned 8-slot
// windows (one 32-byte sector as two 16-byte loads) and scanned in registers.
template <int KB>
__device__ __forceinline__ uint64_t find_free(const TableView& t, const uint8_t* keys, uint32_t j) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    RegKey<KB> key;
    key.load(keys + (uint64_t)j * ksz, ksz);
    const uint64_t h = key.hash(ksz, t.hash_mode) & t.mask;
    if (t.mask >= 7) {
        // two windows per round trip
        uint64_t wb = h & ~7ull;
        for (uint64_t w = 0; w <= (t.mask >> 4) + 1; ++w, wb += 16) {
            const uint4* p0 = reinterpret_cast<const uint4*>(t.flags + (wb & t.mask));
            const uint4* p1 = reinterpret_cast<const uint4*>(t.flags + ((wb + 8) & t.mask));
            const uint4 a = p0[0], b = p0[1], c = p1[0], d = p1[1];
            const uint32_t f16[16] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w};
#pragma unroll
            for (int l = 0; l < 16; l++) {
                const uint64_t pos = wb + l;
                if (pos < h) continue;
                if (pos - h > t.mask) return NONE64;
                if (is_free(f16[l])) return pos & t.mask;
            }
        }
        return NONE64;
    }
    for (uint64_t p = 0; p <= t.mask; ++p) {
        const uint64_t s = (h + p) & t.mask;
        if (is_free(t.flags[s])) return s;
    }
    return NONE64;
}

// The same from a known home h.  With capacity >= 64: two aligned 8-slot
// windows in the first round trip (most walks end there), then four per
// round trip, so a long walk takes fewer trips; smaller tables two windows
// per trip, or slot by slot below 8 slots.
__device__ __forceinline__ uint64_t find_free_from(const TableView& t, uint64_t h) {
    const uint64_t mask = t.mask;
    if (mask >= 63) {
        uint64_t wb = h & ~7ull;
        {
            const uint4* p0 = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
            const uint4* p1 = reinterpret_cast<const uint4*>(t.flags + ((wb + 8) & mask));
            const uint4 a = p0[0], b = p0[1], c = p1[0], d = p1[1];
            const uint32_t f16[16] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w};
#pragma unroll
            for (int l = 0; l < 16; l++)
                if (wb + l >= h && is_free(f16[l])) return (wb + l) & mask;
        }
        for (wb += 16; wb - h <= mask; wb += 32) {
            uint4 x[8];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint4* pq = reinterpret_cast<const uint4*>(t.flags + ((wb + 8 * q) & mask));
                x[2 * q] = pq[0];
                x[2 * q + 1] = pq[1];
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const uint32_t f4[4] = {x[q].x, x[q].y, x[q].z, x[q].w};
#pragma unroll
                for (int l = 0; l < 4; l++) {
                    const uint64_t pos = wb + 4 * q + l;
                    if (pos - h > mask) return NONE64;
                    if (is_free(f4[l])) return pos & mask;
                }
            }
        }
        return NONE64;
    }
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
                if (is_free(f16[l])) return pos & mask;
            }
        }
        return NONE64;
    }
    for (uint64_t p = 0; p <= mask; ++p) {
        const uint64_t s = (h + p) & mask;
        if (is_free(t.flags[s])) return s;
    }
    return NONE64;
}

__device__ __forceinline__ void register_op(const TableView& t, uint32_t j, uint64_t F, uint64_t* op_slot) {
    op_slot[j] = F;
    if (F != NONE64) {
        atomicMin(&t.seg_min[F], j);
        atomicAdd(&t.seg_cnt[F], 1u);
    }
}

// Phase 2 for op j: records whether j leads its segment and, for a crowded
// segment, walks the flow forward.  Returns bit 0 when the flow wraps the
// whole table (serial round), bit 1 on a registration from another call.
__device__ __forceinline__ uint32_t walk_op(const TableView& t, uint32_t j, uint32_t nops, const uint64_t* op_slot,
                                            uint32_t* op_block, uint8_t* op_leader) {
    const uint64_t mask = t.mask;
    const uint64_t F = op_slot[j];
    const bool leader = F != NONE64 && t.seg_min[F] == j;
    op_leader[j] = leader ? 1 : 0;
    if (!leader) return 0;
    const uint32_t c = t.seg_cnt[F];
    if (c < 2) return 0;
    uint64_t flow = c - 1;
    uint32_t L = j;
    uint64_t pos = F + 1;
    uint64_t walked = 0;
    for (;;) {
        // At most the capacity-1 slots after F; coming back to F means the
        // flow wraps the whole table.
        uint64_t F2 = NONE64;
        if (mask >= 7) {  // aligned 8-slot windows, one 32-byte sector each
            for (uint64_t wb = pos & ~7ull; F2 == NONE64 && walked < mask; wb += 8) {
                const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
                const uint4 a = fp[0], b = fp[1];
                const uint32_t f8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    if (F2 != NONE64 || wb + l < pos || walked >= mask) continue;
                    ++walked;
                    if (is_free(f8[l])) F2 = wb + l;
                }
            }
            if (F2 != NONE64) {
                pos = F2 + 1;
                F2 &= mask;
            }
        } else {
            while (walked < mask) {
                const uint64_t s = pos & mask;
                ++pos;
                ++walked;
                if (is_free(t.flags[s])) {
                    F2 = s;
                    break;
                }
            }
        }
        if (F2 == NONE64) return 1u;
        const uint32_t c2 = t.seg_cnt[F2];
        if (c2) {
            const uint32_t l2 = t.seg_min[F2];
            if (l2 >= nops) return 2u;  // registrations come only from this call's ops
            atomicMin(&op_block[l2], L);
            L = min(L, l2);
        }
        flow = flow + c2 - 1;
        if (flow == 0) return 0;
    }
}

struct ExecAcc {
    uint32_t claimed = 0;
    uint32_t maxd = 0;
    bool tomb = false;
    bool limit = false;
};

template <int VB>
__device__ __forceinline__ void swap_value(uint8_t* p, RegVal<VB>& cv);

// The sequential insert of one key, run by one thread on the segment it owns
// this round.  Returns 1 when a free slot was claimed.
template <int KB, int VB>
__device__ __noinline__ int exec_insert_key(const TableView& t, RegKey<KB> ck, const uint8_t* vin, ExecAcc& a) {
    const uint64_t mask = t.mask;
    RegVal<VB> cv;
    cv.load(vin, VB);
    uint64_t h = ck.hash(KB, t.hash_mode) & mask;
    uint64_t p = 0;
    const uint64_t step_limit = 2 * (mask + 1) + 2;
    for (uint64_t step = 0;; ++step) {
        if (p > mask) return 0;  // drop (rayon_cpu.rs:167-169)
        if (step > step_limit) {  // no free slot: the reference's loop may never end
            a.limit = true;
            return 0;
        }
        const uint64_t idx = (h + p) & mask;
        const uint32_t f = t.flags[idx];
        const uint32_t s = st_of(f);
        if (s == ST_OCC) {
            if (dist_matches(f, p) && ck.eq(t.keys + idx * KB, KB)) {
                cv.store(t.vals + idx * VB, VB);  // update in place (rayon_cpu.rs:178-182)
                return 0;
            }
            const uint64_t d = dist_of(f);
            if (p > d) {  // Robin Hood eviction (rayon_cpu.rs:184-217)
                RegKey<KB> tk;
                tk.load_table(t.keys + idx * KB, KB);
                ck.store(t.keys + idx * KB, KB);
                swap_value<VB>(t.vals + idx * VB, cv);
                t.flags[idx] = mk_flag(ST_OCC, p);
                a.maxd = max(a.maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
                ck = tk;
                h = ck.hash(KB, t.hash_mode) & mask;
                p = d + 1;
                continue;
            }
            ++p;
            continue;
        }
        if (s == ST_EMPTY || s == ST_TOMB) {  // claim (rayon_cpu.rs:228-251)
            ck.store(t.keys + idx * KB, KB);
            cv.store(t.vals + idx * VB, VB);
            t.flags[idx] = mk_flag(ST_OCC, p);
            a.maxd = max(a.maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
            a.tomb = a.tomb || s == ST_TOMB;
            return 1;
        }
        ++p;
    }
}

template <int KB, int VB>
__device__ __forceinline__ int exec_insert(const TableView& t, const uint8_t* kin, const uint8_t* vin, ExecAcc& a) {
    RegKey<KB> ck;
    ck.load(kin, KB);
    return exec_insert_key<KB, VB>(t, ck, vin, a);
}

// Swap a value held in registers with the value at p (in halves of at most
// 64 bytes, so the temporary stays small).
template <int VB>
__device__ __forceinline__ void swap_value(uint8_t* p, RegVal<VB>& cv) {
    constexpr int CW = (VB % 16 == 0) ? 4 : ((VB % 8 == 0) ? 2 : 1);  // words per chunk
    constexpr int NCH = VB / (4 * CW);
    constexpr int HALF = NCH > 4 ? 4 : NCH;
#pragma unroll
    for (int c0 = 0; c0 < NCH; c0 += HALF) {
        uint32_t tmp[HALF * CW];
#pragma unroll
        for (int c = 0; c < HALF && c0 + c < NCH; c++) {
            if constexpr (CW == 4) {
                const uint4 v = reinterpret_cast<const uint4*>(p)[c0 + c];
                tmp[4 * c] = v.x; tmp[4 * c + 1] = v.y; tmp[4 * c + 2] = v.z; tmp[4 * c + 3] = v.w;
            } else if constexpr (CW == 2) {
                const uint2 v = reinterpret_cast<const uint2*>(p)[c0 + c];
                tmp[2 * c] = v.x; tmp[2 * c + 1] = v.y;
            } else {
                tmp[c] = reinterpret_cast<const uint32_t*>(p)[c0 + c];
            }
        }
#pragma unroll
        for (int c = 0; c < HALF && c0 + c < NCH; c++) {
            const int w = (c0 + c) * CW;
            if constexpr (CW == 4)
                reinterpret_cast<uint4*>(p)[c0 + c] = make_uint4(cv.w[w], cv.w[w + 1], cv.w[w + 2], cv.w[w + 3]);
            else if constexpr (CW == 2)
                reinterpret_cast<uint2*>(p)[c0 + c] = make_uint2(cv.w[w], cv.w[w + 1]);
            else
                reinterpret_cast<uint32_t*>(p)[c0 + c] = cv.w[w];
#pragma unroll
            for (int i = 0; i < CW; i++) cv.w[w + i] = tmp[c * CW + i];
        }
    }
}

// One move of a whole entry (or just its value) from a source to a slot, in
// groups of at most 64 bytes so the temporary stays small.  Every thread of a
// warp runs the same loop, so their loads issue together.
template <int KB, int VB>
__device__ __forceinline__ void move_entry(const TableView& t, const uint8_t* ksrc, const uint8_t* vsrc, uint64_t dst,
                                           bool value_only, bool src_ro) {
    constexpr int CW = (KB % 16 == 0 && VB % 16 == 0) ? 16 : ((KB % 8 == 0 && VB % 8 == 0) ? 8 : 4);
    using Ch = typename std::conditional<CW == 16, uint4, typename std::conditional<CW == 8, uint2, uint32_t>::type>::type;
    constexpr int NK = KB / CW, NV = VB / CW;
    if (!value_only) {
        Ch k[NK];
#pragma unroll
        for (int c = 0; c < NK; c++)
            k[c] = src_ro ? __ldg(reinterpret_cast<const Ch*>(ksrc) + c) : reinterpret_cast<const Ch*>(ksrc)[c];
#pragma unroll
        for (int c = 0; c < NK; c++) reinterpret_cast<Ch*>(t.keys + dst * KB)[c] = k[c];
    }
    constexpr int G = (64 / CW) > 0 ? (64 / CW) : 1;
#pragma unroll
    for (int c0 = 0; c0 < NV; c0 += G) {
        Ch v[G];
#pragma unroll
        for (int c = 0; c < G; c++)
            if (c0 + c < NV)
                v[c] = src_ro ? __ldg(reinterpret_cast<const Ch*>(vsrc) + c0 + c)
                              : reinterpret_cast<const Ch*>(vsrc)[c0 + c];
#pragma unroll
        for (int c = 0; c < G; c++)
            if (c0 + c < NV) reinterpret_cast<Ch*>(t.vals + dst * VB)[c0 + c] = v[c];
    }
}

#ifndef FM_TH_MAXK
#define FM_TH_MAXK 3
#endif
#ifndef FM_TH_MAXC
#define FM_TH_MAXC 2
#endif
constexpr int TH_MAXK = FM_TH_MAXK;  // evictions per op on the thread path
constexpr int TH_MAXC = FM_TH_MAXC;  // possible updates per op on the thread path

// The sequential insert of one key by one thread, for the common short walk
// (capacity >= 8, rounds that are not serial, so the walk ends at or before
// the op's free slot and visits each slot once).  Dependent memory round
// trips: the two aligned 8-slot metadata windows from home (one trip), the
// key compares at the slots where the stored distance equals the probe depth
// (one trip), then one per entry move.
//   1. walk the 16 metadata words in registers, recording the eviction slots
//      (slot P_i takes the entry carried there; the evicted resident continues
//      at the next slot with depth dist+1) and the possible updates;
//   2. compare the carried key at those slots, the first match in walk order
//      ending the walk as an in-place update;
//   3. move entries, highest first: the end slot gets the entry evicted at
//      P_(k-1), P_i the one evicted at P_(i-1), P_0 the new entry; then the
//      metadata words.
// A walk that leaves the two windows, needs more than TH_MAXK evictions or
// more than TH_MAXC compares returns -1 having written nothing.  The small
// arrays are written through unrolled selects so they stay in registers.
template <int KB, int VB>
__device__ __noinline__ int exec_insert_thread(const TableView& t, const RegKey<KB>& key, const uint8_t* kin,
                                               const uint8_t* vin, ExecAcc& a) {
    const uint64_t mask = t.mask;
    uint64_t ev_pos[TH_MAXK];
    uint32_t ev_p[TH_MAXK];
    uint64_t cd_pos[TH_MAXC];
    uint32_t cd_stage[TH_MAXC];
#pragma unroll
    for (int i = 0; i < TH_MAXK; i++) ev_pos[i] = 0, ev_p[i] = 0;
#pragma unroll
    for (int i = 0; i < TH_MAXC; i++) cd_pos[i] = 0, cd_stage[i] = 0;
    uint32_t k = 0, nc = 0;
    int kind = 0;  // 1 claim, 2 update, 3 drop, 4 too long for this path
    uint64_t end_pos = 0, end_p = 0;
    bool end_tomb = false;
    const uint64_t h = key.hash(KB, t.hash_mode) & mask;
    const uint64_t wb = h & ~7ull;
    const uint4* w0 = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
    const uint4* w1 = reinterpret_cast<const uint4*>(t.flags + ((wb + 8) & mask));
    const uint4 fa = w0[0], fb = w0[1], fc = w1[0], fd = w1[1];
    const uint32_t f16[16] = {fa.x, fa.y, fa.z, fa.w, fb.x, fb.y, fb.z, fb.w,
                              fc.x, fc.y, fc.z, fc.w, fd.x, fd.y, fd.z, fd.w};
    uint64_t p = 0;
#pragma unroll
    for (int l = 0; l < 16; l++) {
        const uint64_t pos = wb + l;
        if (kind != 0 || pos < h) continue;
        const uint32_t f = f16[l];
        const uint32_t s = st_of(f);
        if (p > mask) {
            kind = 3;  // drop (rayon_cpu.rs:167-169)
        } else if (s == ST_EMPTY || s == ST_TOMB) {
            kind = 1;
            end_pos = pos;
            end_p = p;
            end_tomb = s == ST_TOMB;
        } else if (s == ST_OCC) {
            if (dist_matches(f, p)) {
                if (nc < TH_MAXC) {
#pragma unroll
                    for (int i = 0; i < TH_MAXC; i++)
                        if (i == (int)nc) cd_pos[i] = pos, cd_stage[i] = k;
                    ++nc;
                } else {
                    kind = 4;
                }
                ++p;
            } else if (p > dist_of(f)) {
                if (k < TH_MAXK) {
#pragma unroll
                    for (int i = 0; i < TH_MAXK; i++)
                        if (i == (int)k) ev_pos[i] = pos, ev_p[i] = (uint32_t)p;
                    ++k;
                    p = dist_of(f) + 1;
                } else {
                    kind = 4;
                }
            } else {
                ++p;
            }
        } else {
            ++p;
        }
    }
    if (kind == 0 || kind == 4) return -1;  // nothing written; the warp-per-op pass runs it
    // 2. possible updates: every compare's loads in one round trip, then the
    // first match in walk order (slots at or past a claimed end are not reached)
    {
        RegKey<KB> sk[TH_MAXC], ck[TH_MAXC];
#pragma unroll
        for (int c = 0; c < TH_MAXC; c++) {
            if (c < (int)nc) {
                sk[c].load_table(t.keys + (cd_pos[c] & mask) * KB, KB);
                uint32_t st = cd_stage[c];
                uint64_t src = 0;
#pragma unroll
                for (int i = 0; i < TH_MAXK; i++)
                    if (i + 1 == (int)st) src = ev_pos[i];
                // the entry carried at that point, still at its old slot
                if (st) ck[c].load_table(t.keys + (src & mask) * KB, KB);
                else ck[c] = key;
            }
        }
        bool found = false;
#pragma unroll
        for (int c = 0; c < TH_MAXC; c++) {
            if (found || c >= (int)nc) continue;
            if (kind == 1 && cd_pos[c] >= end_pos) continue;
            if (ck[c].same(sk[c])) {
                found = true;
                kind = 2;
                end_pos = cd_pos[c];
                k = cd_stage[c];
            }
        }
    }
    // 3. moves, highest first (kind 3: the last carried entry is dropped)
    const int M = (kind == 3) ? (int)k : (int)k + 1;
#pragma unroll
    for (int m = TH_MAXK; m >= 0; m--) {
        if (m >= M) continue;
        uint64_t dst = end_pos, src = 0;
#pragma unroll
        for (int i = 0; i < TH_MAXK; i++) {
            if (i == m && m < (int)k) dst = ev_pos[i];
            if (i + 1 == m) src = ev_pos[i];
        }
        dst &= mask;
        const bool value_only = (m == (int)k) && kind == 2;
        if (m == 0) {
            move_entry<KB, VB>(t, kin, vin, dst, value_only, true);
        } else {
            src &= mask;
            move_entry<KB, VB>(t, t.keys + src * KB, t.vals + src * VB, dst, value_only, false);
        }
    }
    uint32_t md = 0;
#pragma unroll
    for (int m = 0; m < TH_MAXK; m++) {
        if (m < (int)k) {
            t.flags[ev_pos[m] & mask] = mk_flag(ST_OCC, ev_p[m]);
            md = max(md, min(ev_p[m], DIST_MASK));
        }
    }
    if (kind == 1) {
        t.flags[end_pos & mask] = mk_flag(ST_OCC, end_p);
        md = max(md, (uint32_t)min(end_p, (uint64_t)DIST_MASK));
        a.tomb = a.tomb || end_tomb;
    }
    a.maxd = max(a.maxd, md);
    return kind == 1 ? 1 : 0;
}

// Run-time sizes (up to GENERIC_MAX_KV bytes each): the carried entry lives in
// a local buffer and is swapped with the slot byte by byte.
__device__ __forceinline__ int exec_insert_generic(const TableView& t, const uint8_t* kin, const uint8_t* vin,
                                                   ExecAcc& a) {
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
            a.limit = true;
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
                    const uint8_t x = sk[i];
                    sk[i] = ck[i];
                    ck[i] = x;
                }
                for (uint32_t i = 0; i < vsz; i++) {
                    const uint8_t x = sv[i];
                    sv[i] = cv[i];
                    cv[i] = x;
                }
                t.flags[idx] = mk_flag(ST_OCC, p);
                a.maxd = max(a.maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
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
            a.maxd = max(a.maxd, (uint32_t)min(p, (uint64_t)DIST_MASK));
            a.tomb = a.tomb || s == ST_TOMB;
            return 1;
        }
        ++p;
    }
}

// Phase 3 for op j (one thread per op): run it if it leads an unblocked
// segment of a non-serial round, then clear its registration.  Returns 0 when
// it did not run, 1 when it ran and 2 when its walk is too long for the
// thread path and `defer` allows handing it to the tile pass (it then counts
// as run: its segment is disjoint from every other segment of the round, so
// running it after them gives the same result); without `defer` such a walk
// takes the scalar path.
template <int KB, int VB>
__device__ __forceinline__ int finish_op(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t j,
                                         bool serial, const OpScratch& sc, ExecAcc& a, bool defer) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint32_t vsz = VB ? (uint32_t)VB : t.vsz;
    if constexpr (KB == 0 || VB == 0) {
        const bool run = !serial && sc.op_flag[j] != 0 && sc.op_word[j] > j;
        if (run) a.claimed += exec_insert_generic(t, keys + (uint64_t)j * ksz, vals + (uint64_t)j * vsz, a);
        const uint64_t F = sc.op_slot[j];
        if (F != NONE64) {
            t.seg_min[F] = IDLE;
            t.seg_cnt[F] = 0;
        }
        sc.op_word[j] = IDLE;
        return run ? 1 : 0;
    } else {
        // independent loads issued together: decision words, registration, key
        const uint8_t lead = sc.op_flag[j];
        const uint32_t blk = sc.op_word[j];
        const uint64_t F = sc.op_slot[j];
        RegKey<KB> key;
        key.load(keys + (uint64_t)j * ksz, ksz);
        const bool run = !serial && lead != 0 && blk > j;
        int code = run ? 1 : 0;
        if (run) {
            // windows need capacity >= 8; consecutive walk positions need
            // probe depths below 2^28 (the stored distance width)
            int c = -1;
            if (t.mask >= 7 && t.mask < (uint64_t)DIST_MASK)
                c = exec_insert_thread<KB, VB>(t, key, keys + (uint64_t)j * ksz, vals + (uint64_t)j * vsz, a);
            if (c < 0 && defer) code = 2;
            else if (c < 0) c = exec_insert_key<KB, VB>(t, key, vals + (uint64_t)j * vsz, a);
            if (c > 0) a.claimed += c;
        }
        if (F != NONE64) {
            t.seg_min[F] = IDLE;
            t.seg_cnt[F] = 0;
        }
        sc.op_word[j] = IDLE;
        return code;
    }
}

// Rare facts, once per warp: the largest stored distance, tombstone reuse and
// the full-table walk limit.
__device__ __forceinline__ void publish_rare(Ctl* ctl, uint32_t maxd, bool tomb, bool limit) {
    maxd = __reduce_max_sync(0xFFFFFFFFu, maxd);
    tomb = __any_sync(0xFFFFFFFFu, tomb);
    limit = __any_sync(0xFFFFFFFFu, limit);
    if ((threadIdx.x & 31u) == 0) {
        if (maxd > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, maxd);
        if (tomb && !*(volatile uint32_t*)&ctl->tomb_claimed) ctl->tomb_claimed = 1u;
        if (limit) atomicOr(&ctl->err, ERR_WALK_LIMIT);
    }
}

// ---- tile-cooperative execute (compile-time shapes) -----------------------
//
// A tile of T lanes runs one insert whose walk is too long for one thread.
//
// The walk in closed form.  Write the carried entry's state as its home
// H = position - depth.  At an OCCUPIED slot holding a resident with home
// h = position - dist: dist == depth is h == H (a possible update), and
// depth > dist is h > H (an eviction, after which the carried entry is that
// resident, so H becomes h); otherwise the walk moves on with H unchanged.
// So H is the running maximum of the residents' homes from the op's own home
// on, the evictions are the slots whose home exceeds the running maximum
// before them, the possible updates those whose home equals it, and the walk
// ends at the first EMPTY/TOMBSTONE slot or where position - H passes the
// capacity (drop).  A tile reads 4T slots per round trip (one 16-byte load
// per lane) and classifies them with one max-scan, one count-scan and
// ballots, whatever the number of evictions.
//
// Then: the possible updates of each window are compared before the next
// window is read (the first equal key, in walk order, ends the walk as an
// in-place update), and the records move highest first in batches of round
// trips -- the end slot gets the entry evicted at P_(k-1), P_i the one
// evicted at P_(i-1), P_0 the new entry -- sources read before their slots
// are written.  The tile keeps up to TMAXCH eviction slots; a longer chain's
// last chunk is moved first, then each earlier piece of the chain is found
// again by a walk from home (slots before a piece's end are untouched by the
// later moves) and moved, last to first.

constexpr int TMAXCH = 256;  // eviction slots held per tile
constexpr int TMAXC = 128;   // possible updates of one window (>= 4T)
constexpr uint32_t NOSRC = 0xFFFFFFFFu;

template <int MAXCH_, int MAXC_ = TMAXC>
struct ChainBuf {
    static constexpr int MAXCH = MAXCH_;
    static constexpr int MAXC = MAXC_;
    uint32_t pos[MAXCH];    // eviction slots of the current chunk
    uint32_t p[MAXCH];      // depth stored at each of them
    uint32_t cpos[MAXC];    // possible updates of the current window: slot,
    uint32_t cstage[MAXC];  //   evictions before it,
    uint32_t csrc[MAXC];    //   slot holding the carried key (NOSRC: the new key)
    uint32_t src_base;      // slot evicted just before the chunk's first stage
};
using TileChain = ChainBuf<TMAXCH>;
// The one-op-at-a-time path's buffer (dynamic shared memory, 67 KB): chains
// of up to SMAXCH - 128 evictions need no second walk.
constexpr int SMAXCH = 8192;
using SerialChain = ChainBuf<SMAXCH>;

template <int T>
__device__ __forceinline__ uint64_t find_free_tile(const TableView& t, uint64_t h, const Tile<T>& tl) {
    const uint64_t mask = t.mask;
    uint64_t wb = h & ~(uint64_t)(T - 1);
    for (;;) {
        const uint64_t pos = wb + tl.lane;
        const bool before = pos < h;
        const uint64_t p = pos - h;
        const uint32_t f = t.flags[pos & mask];
        const bool past = !before && p > mask;
        const uint32_t fm = tl.ballot(!before && !past && is_free(f));
        if (fm) return (wb + __ffs(fm) - 1) & mask;
        if (tl.ballot(past)) return NONE64;
        wb += T;
    }
}

// Chunk type for moving KB/VB-byte records.
template <int KB, int VB>
struct ChunkOf {
    static constexpr int CK = (KB % 16 == 0 && VB % 16 == 0) ? 16 : ((KB % 8 == 0 && VB % 8 == 0) ? 8 : 4);
    using type = typename std::conditional<CK == 16, uint4, typename std::conditional<CK == 8, uint2, uint32_t>::type>::type;
    static constexpr int NK = KB / CK;
    static constexpr int NV = VB / CK;
    static constexpr int NC = NK + NV;
};

// Chunk c (CK bytes) of a key held in registers.
template <int KB, class Ch, int CK>
__device__ __forceinline__ Ch key_chunk(const RegKey<KB>& key, int c) {
    Ch x;
    uint32_t* w = reinterpret_cast<uint32_t*>(&x);
#pragma unroll
    for (int i = 0; i < CK / 4; i++) w[i] = key.w[c * (CK / 4) + i];
    return x;
}

// Inclusive scans over the T lanes of a tile.
template <int T>
__device__ __forceinline__ uint32_t tile_sum(uint32_t v, const Tile<T>& tl) {
#pragma unroll
    for (int d = 1; d < T; d <<= 1) {
        const uint32_t o = __shfl_up_sync(tl.wmask, v, d, T);
        if ((int)tl.lane >= d) v += o;
    }
    return v;
}
template <int T, class P>
__device__ __forceinline__ P tile_max(P v, const Tile<T>& tl) {
#pragma unroll
    for (int d = 1; d < T; d <<= 1) {
        const P o = __shfl_up_sync(tl.wmask, v, d, T);
        if ((int)tl.lane >= d) v = max(v, o);
    }
    return v;
}

// Record moves m = hi down to lo (absolute stage numbers, lo >= chunk_base)
// of a chain whose stages from chunk_base sit in s.pos: move m writes
// dest(m) = P_m (m < k) or the end slot (m == k) from source(m) = P_(m-1), the
// slot `src_base` for m == chunk_base > 0, or the new entry for m == 0.  MB
// moves per round trip, every lane holding up to CPL chunks.
template <int KB, int VB, int CPL, class Crew, class C>
__device__ __forceinline__ void tile_moves(const TableView& t, const RegKey<KB>& key, const uint8_t* vin,
                                           const C& s, uint32_t chunk_base, int hi, int lo, uint32_t k,
                                           int kind, uint64_t end_slot, uint32_t src_base, const Crew& tl) {
    constexpr int T = Crew::W;
    using CO = ChunkOf<KB, VB>;
    using Ch = typename CO::type;
    constexpr int CK = CO::CK, NK = CO::NK, NC = CO::NC;
    constexpr int MB = (CPL * T) / NC > 0 ? (CPL * T) / NC : 1;
    constexpr int CL = (MB * NC + T - 1) / T;
    const uint32_t lane = tl.lane;
    for (int top = hi; top >= lo; top -= MB) {
        const int bot = top - MB + 1 > lo ? top - MB + 1 : lo;
        const int nchunks = (top - bot + 1) * NC;
        Ch buf[CL];
#pragma unroll
        for (int u = 0; u < CL; u++) {
            const int g = (int)lane + u * T;
            if (g < nchunks) {
                const int m = bot + g / NC, c = g % NC;
                const bool value_only = (m == (int)k) && kind == 2;
                if (value_only && c < NK) continue;
                if (m == 0 && c < NK) {
                    buf[u] = key_chunk<KB, Ch, CK>(key, c);
                    continue;
                }
                const uint8_t* src;
                if (m == 0) {
                    src = vin + (c - NK) * CK;
                } else {
                    const uint64_t ss = (m == (int)chunk_base) ? src_base : s.pos[m - 1 - chunk_base];
                    src = c < NK ? t.keys + ss * KB + c * CK : t.vals + ss * VB + (c - NK) * CK;
                }
                buf[u] = *reinterpret_cast<const Ch*>(src);
            }
        }
        tl.sync();
#pragma unroll
        for (int u = 0; u < CL; u++) {
            const int g = (int)lane + u * T;
            if (g < nchunks) {
                const int m = bot + g / NC, c = g % NC;
                const bool value_only = (m == (int)k) && kind == 2;
                if (value_only && c < NK) continue;
                const uint64_t ds = (m < (int)k) ? s.pos[m - chunk_base] : end_slot;
                uint8_t* dst = c < NK ? t.keys + ds * KB + c * CK : t.vals + ds * VB + (c - NK) * CK;
                *reinterpret_cast<Ch*>(dst) = buf[u];
            }
        }
        tl.sync();
    }
}

// Walks an insert chain from home with a tile, window by window.
//   find: to the end of the walk, comparing each window's possible updates
//         before reading the next; keeps the eviction slots of the last chunk
//         (stages from chunk_base) in s.pos; returns 1 claim, 2 update,
//         3 drop, 5 (never in a non-serial round) walk past the bound.
//   otherwise: records the eviction slots of stages [lo, hi) and stops.
// Positions are kept relative to the first window's base in the signed type
// P: int (32-bit scans) for tables below 2^30 slots, 64-bit above.
template <int KB, int T, class C, class P>
__device__ int tile_walk_p(const TableView& t, const RegKey<KB>& key, C& s, const Tile<T>& tl, bool find,
                           uint32_t lo, uint32_t hi, uint32_t& k, uint32_t& chunk_base, uint32_t& src_base,
                           uint64_t& end_slot, uint64_t& end_p, bool& end_tomb) {
    constexpr int MAXCH = C::MAXCH;
    static_assert(C::MAXC >= 4 * T && MAXCH >= 8 * T, "a window's updates and evictions must fit the buffers");
    const uint64_t mask = t.mask;
    constexpr P PMIN = std::numeric_limits<P>::min();
    const uint64_t h = key.hash(KB, t.hash_mode) & mask;
    const uint64_t wb0 = h & ~(uint64_t)(4 * T - 1);  // origin of the relative positions
    const P hr = (P)(h - wb0);
    P M = hr;  // the carried entry's home
    uint32_t g = 0;              // evictions so far
    uint32_t last_ev = NOSRC;    // slot of the last eviction
    int kind = 0;
    chunk_base = find ? 0 : lo;
    src_base = NOSRC;
    if (!find && tl.lane == 0) s.src_base = NOSRC;
    uint64_t wb = h & ~(uint64_t)(4 * T - 1);
    // a walk of a non-serial round ends within one pass over the table; the
    // bound only guards against a broken invariant (reported, nothing written)
    const uint64_t wb_end = wb + 2 * (mask + 1) + 4 * T;
    while (kind == 0) {
        if (wb > wb_end) {
            kind = 5;
            break;
        }
        if (find && g - chunk_base > (uint32_t)(MAXCH - 4 * T)) {  // room for this window's evictions
            src_base = last_ev;
            chunk_base = g;
        }
        const uint64_t base = wb + 4 * tl.lane;
        const uint4 fw = *reinterpret_cast<const uint4*>(t.flags + (base & mask));
        const uint32_t f[4] = {fw.x, fw.y, fw.z, fw.w};
        // homes of the occupied slots on the walk, and the running maximum
        const P br = (P)(base - wb0);
        P hh[4];
        P lm = PMIN;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            hh[i] = (br + i >= hr && st_of(f[i]) == ST_OCC) ? br + i - (P)dist_of(f[i]) : PMIN;
            lm = max(lm, hh[i]);
        }
        const P incl = tile_max<T, P>(lm, tl);
        P mx = __shfl_up_sync(tl.wmask, incl, 1, T);
        mx = tl.lane == 0 ? M : max(M, mx);
        // classify: end (free or drop), eviction, possible update
        uint32_t endb = 0, evb = 0, cdb = 0, pend[4];
        P mi[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            mi[i] = mx;
            const uint64_t depth = (uint64_t)(br + i - mx);
            pend[i] = (uint32_t)depth;
            if (br + i >= hr) {
                const uint32_t st = st_of(f[i]);
                if (depth > mask || st == ST_EMPTY || st == ST_TOMB) endb |= 1u << i;
                else if (hh[i] > mx) evb |= 1u << i;
                else if (hh[i] == mx) cdb |= 1u << i;
            }
            mx = max(mx, hh[i]);
        }
        const uint32_t em = tl.ballot(endb != 0);
        const uint32_t elane = em ? (uint32_t)(__ffs(em) - 1) : (uint32_t)T;
        const uint32_t myi = endb ? (uint32_t)(__ffs(endb) - 1) : 4u;
        // only the slots before the end
        if (tl.lane > elane) evb = cdb = 0;
        else if (tl.lane == elane) evb &= (1u << myi) - 1u, cdb &= (1u << myi) - 1u;
        // evictions in walk order: global stage numbers and the eviction slots
        const uint32_t ne = __popc(evb);
        const uint32_t einc = tile_sum<T>(ne, tl);
        const uint32_t etot = tl.shfl(einc, T - 1);
        uint32_t gi = g + einc - ne;
        // the last eviction before each slot (for the possible updates' carried key)
        P lastpos = evb ? br + (P)(31 - __clz(evb)) : (P)-1;
        const P linc = tile_max<T, P>(lastpos, tl);
        P lprev = __shfl_up_sync(tl.wmask, linc, 1, T);
        if (tl.lane == 0) lprev = -1;
        uint32_t co = 0;
        uint32_t nc_tot = 0;
        if (find) {
            const uint32_t ncd = __popc(cdb);
            const uint32_t cinc = tile_sum<T>(ncd, tl);
            nc_tot = tl.shfl(cinc, T - 1);
            co = cinc - ncd;
        }
        uint32_t stg = gi;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint64_t pos = base + i;
            if ((evb >> i) & 1u) {
                if (stg >= chunk_base && stg < (find ? chunk_base + MAXCH : hi)) {
                    s.pos[stg - chunk_base] = (uint32_t)(pos & mask);
                    s.p[stg - chunk_base] = pend[i];
                }
                if (!find && stg + 1 == lo) s.src_base = (uint32_t)(pos & mask);
                lprev = br + i;
                ++stg;
            } else if (find && ((cdb >> i) & 1u)) {
                s.cpos[co] = (uint32_t)(pos & mask);
                s.cstage[co] = stg;
                s.csrc[co] = lprev >= 0 ? (uint32_t)((wb0 + (uint64_t)lprev) & mask)
                                        : (last_ev == NOSRC ? NOSRC : last_ev);
                ++co;
            }
        }
        tl.sync();
        // compare this window's possible updates, T per round trip
        if (find && nc_tot) {
            int found = -1;
            for (uint32_t b0 = 0; b0 < nc_tot && found < 0; b0 += T) {
                const uint32_t c = b0 + tl.lane;
                bool eq = false;
                if (c < nc_tot) {
                    const uint8_t* sk = t.keys + (uint64_t)s.cpos[c] * KB;
                    const uint32_t src = s.csrc[c];
                    if (src == NOSRC) {
                        eq = key.eq(sk, KB);
                    } else {
                        RegKey<KB> ck;  // the carried entry's key, still at its old slot
                        ck.load_table(t.keys + (uint64_t)src * KB, KB);
                        eq = ck.eq(sk, KB);
                    }
                }
                const uint32_t mm = tl.ballot(eq);
                if (mm) found = (int)(b0 + __ffs(mm) - 1);
            }
            if (found >= 0) {
                kind = 2;
                end_slot = s.cpos[found];
                k = s.cstage[found];
                tl.sync();
                break;
            }
        }
        // advance: evictions, last eviction slot, carried home
        if (etot) {
            const P lw = tl.shfl(linc, T - 1);
            last_ev = (uint32_t)((wb0 + (uint64_t)lw) & mask);
        }
        g += etot;
        const P mall = tl.shfl(incl, T - 1);
        if (em) {
            // the end slot: its depth is position - running max before it
            const uint32_t dsel = myi == 0 ? pend[0] : (myi == 1 ? pend[1] : (myi == 2 ? pend[2] : pend[3]));
            const uint32_t fsel = myi == 0 ? f[0] : (myi == 1 ? f[1] : (myi == 2 ? f[2] : f[3]));
            const uint32_t ef = tl.shfl(fsel, elane);
            const uint64_t epos = wb + 4 * elane + tl.shfl(myi, elane);
            // depth as a full 64-bit value (pend holds its low 32 bits)
            const P mend = tl.shfl(myi == 0 ? mi[0] : (myi == 1 ? mi[1] : (myi == 2 ? mi[2] : mi[3])), elane);
            const uint64_t edepth = (uint64_t)((P)(epos - wb0) - mend);
            (void)dsel;
            kind = (edepth > mask) ? 3 : 1;
            end_slot = epos & mask;
            end_p = edepth;
            end_tomb = st_of(ef) == ST_TOMB;
            k = g;
            if (!find) kind = 4;
            break;
        }
        M = max(M, mall);
        if (!find && g >= hi) {
            kind = 4;
            break;
        }
        wb += 4 * T;
    }
    if (!find) src_base = s.src_base;
    tl.sync();
    return kind;
}

template <int KB, int T, class C>
__device__ __forceinline__ int tile_walk(const TableView& t, const RegKey<KB>& key, C& s, const Tile<T>& tl,
                                         bool find, uint32_t lo, uint32_t hi, uint32_t& k, uint32_t& chunk_base,
                                         uint32_t& src_base, uint64_t& end_slot, uint64_t& end_p, bool& end_tomb) {
    if (t.mask < (1ull << 30))
        return tile_walk_p<KB, T, C, int>(t, key, s, tl, find, lo, hi, k, chunk_base, src_base, end_slot, end_p,
                                          end_tomb);
    return tile_walk_p<KB, T, C, long long>(t, key, s, tl, find, lo, hi, k, chunk_base, src_base, end_slot, end_p,
                                            end_tomb);
}

// One insert by a tile (capacity >= 4T, rounds that are not serial).
template <int KB, int VB, int T, class C = TileChain>
__device__ __forceinline__ int exec_tile(const TableView& t, const RegKey<KB>& key,
                                         const uint8_t* __restrict__ vals_in, uint32_t j, const Tile<T>& tl,
                                         C& s, ExecAcc& a) {
    constexpr int CPL = 4;
    constexpr int MAXCH = C::MAXCH;
    const uint8_t* vin = vals_in + (uint64_t)j * VB;
    uint32_t k = 0, chunk_base = 0, src_base = NOSRC;
    uint64_t end_slot = 0, end_p = 0;
    bool end_tomb = false;
    const int kind =
        tile_walk<KB, T, C>(t, key, s, tl, true, 0, 0, k, chunk_base, src_base, end_slot, end_p, end_tomb);
    if (kind == 5) return 5;  // no free slot within a pass: nothing written
    uint32_t md = 0;
    // last chunk: moves from the end (or the last eviction) down to chunk_base
    {
        const int hi = (kind == 3) ? (int)k - 1 : (int)k;
        tile_moves<KB, VB, CPL>(t, key, vin, s, chunk_base, hi, (int)chunk_base, k, kind, end_slot, src_base, tl);
        for (uint32_t m = chunk_base + tl.lane; m < k; m += T) {
            t.flags[s.pos[m - chunk_base]] = mk_flag(ST_OCC, s.p[m - chunk_base]);
            md = max(md, min(s.p[m - chunk_base], DIST_MASK));
        }
        tl.sync();
    }
    // earlier stages, MAXCH at a time from the top, each found again by a
    // walk from home
    for (uint32_t top = chunk_base; top > 0;) {
        const uint32_t lo = top > (uint32_t)MAXCH ? top - MAXCH : 0u;
        uint32_t k2, cb2, sb2;
        uint64_t es2, ep2;
        bool et2;
        tile_walk<KB, T, C>(t, key, s, tl, false, lo, top, k2, cb2, sb2, es2, ep2, et2);
        tile_moves<KB, VB, CPL>(t, key, vin, s, lo, (int)top - 1, (int)lo, k, kind, end_slot, sb2, tl);
        for (uint32_t m = tl.lane; m < top - lo; m += T) {
            t.flags[s.pos[m]] = mk_flag(ST_OCC, s.p[m]);
            md = max(md, min(s.p[m], DIST_MASK));
        }
        tl.sync();
        top = lo;
    }
    if (tl.lane == 0 && kind == 1) {
        t.flags[end_slot] = mk_flag(ST_OCC, end_p);
        md = max(md, (uint32_t)min(end_p, (uint64_t)DIST_MASK));
        a.claimed += 1;
        a.tomb = a.tomb || end_tomb;
    }
    a.maxd = max(a.maxd, md);
    return kind;
}

// The walk's outcome, broadcast from warp 0 to the block.
struct SerialOut {
    int kind;
    uint32_t k, chunk_base, src_base;
    uint64_t end_slot, end_p;
    int tomb;
};

constexpr int SERIAL_THREADS = 512;

// One insert by a whole block of W threads (compile-time sizes,
// capacity >= 128): warp 0 walks the chain into the large buffer, then every
// thread moves records (204 account-shape records per round trip with 512
// threads) and writes flags.  A chain longer than the buffer moves its last
// chunk first and each earlier chunk after warp 0 finds it again; a walk
// that finds no free slot within a pass (overfull table) takes the scalar
// walk.
// Block-uniform call.
template <int KB, int VB, int W = SERIAL_THREADS>
__device__ void exec_serial_block(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t j,
                                  SerialChain& s, SerialOut& so, ExecAcc& a) {
    RegKey<KB> key;
    key.load(keys + (uint64_t)j * KB, KB);
    const uint8_t* vin = vals + (uint64_t)j * VB;
    if (threadIdx.x < 32) {
        const Tile<32> tl;
        uint32_t k = 0, cb = 0, sb = NOSRC;
        uint64_t es = 0, ep = 0;
        bool et = false;
        const int kind = tile_walk<KB, 32, SerialChain>(t, key, s, tl, true, 0, 0, k, cb, sb, es, ep, et);
        if (tl.lane == 0) {
            so.kind = kind;
            so.k = k;
            so.chunk_base = cb;
            so.src_base = sb;
            so.end_slot = es;
            so.end_p = ep;
            so.tomb = et ? 1 : 0;
        }
    }
    __syncthreads();
    const int kind = so.kind;
    if (kind == 5) {
        if (threadIdx.x == 0) a.claimed += exec_insert_key<KB, VB>(t, key, vin, a);
        __syncthreads();
        return;
    }
    const uint32_t k = so.k, cb = so.chunk_base;
    const int hi = kind == 3 ? (int)k - 1 : (int)k;
    const BlockCrew<W> crew;
    // the last chunk of the chain (stages from cb) first
    tile_moves<KB, VB, 4>(t, key, vin, s, cb, hi, (int)cb, k, kind, so.end_slot, so.src_base, crew);
    uint32_t md = 0;
    for (uint32_t m = cb + threadIdx.x; m < k; m += blockDim.x) {
        t.flags[s.pos[m - cb]] = mk_flag(ST_OCC, s.p[m - cb]);
        md = max(md, min(s.p[m - cb], DIST_MASK));
    }
    __syncthreads();
    // a chain longer than the buffer: earlier chunks from the top, each found
    // again by warp 0 walking from home (slots before a chunk's end are
    // untouched by the later chunks' moves), moved by the whole block
    for (uint32_t top = cb; top > 0;) {
        const uint32_t lo = top > (uint32_t)SMAXCH ? top - SMAXCH : 0u;
        if (threadIdx.x < 32) {
            const Tile<32> tl;
            uint32_t k2, cb2, sb2;
            uint64_t es2, ep2;
            bool et2;
            tile_walk<KB, 32, SerialChain>(t, key, s, tl, false, lo, top, k2, cb2, sb2, es2, ep2, et2);
            if (tl.lane == 0) so.src_base = sb2;
        }
        __syncthreads();
        tile_moves<KB, VB, 4>(t, key, vin, s, lo, (int)top - 1, (int)lo, k, kind, so.end_slot, so.src_base, crew);
        for (uint32_t m = threadIdx.x; m < top - lo; m += blockDim.x) {
            t.flags[s.pos[m]] = mk_flag(ST_OCC, s.p[m]);
            md = max(md, min(s.p[m], DIST_MASK));
        }
        __syncthreads();
        top = lo;
    }
    if (threadIdx.x == 0 && kind == 1) {
        t.flags[so.end_slot] = mk_flag(ST_OCC, so.end_p);
        md = max(md, (uint32_t)min(so.end_p, (uint64_t)DIST_MASK));
        a.claimed += 1;
        a.tomb = a.tomb || so.tomb != 0;
    }
    a.maxd = max(a.maxd, md);
    __syncthreads();  // the next op reads these writes
}

// Applies the c ops of s_list in that order on this block, each as
// serial_process (below) describes.  Block-uniform call; W = blockDim.x
// when s_big is given.
template <int KB, int VB, int W>
__device__ void serial_apply(const TableView& t, const uint8_t* keys, const uint8_t* vals, const uint32_t* s_list,
                             uint32_t c, const OpScratch& sc, ExecAcc& a, TileChain* s_chain, SerialChain* s_big,
                             SerialOut* s_out) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint32_t vsz = VB ? (uint32_t)VB : t.vsz;
    if constexpr (KB == 0 || VB == 0) {
        if (threadIdx.x == 0) {
            for (uint32_t k = 0; k < c; k++) {
                const uint32_t jj = s_list[k];
                sc.op_flag[jj] = 0;
                a.claimed += exec_insert_generic(t, keys + (uint64_t)jj * ksz, vals + (uint64_t)jj * vsz, a);
            }
        }
    } else if (s_big && t.mask >= 4 * 32 - 1) {
        for (uint32_t k = 0; k < c; k++) {
            const uint32_t jj = s_list[k];
            if (threadIdx.x == 0) sc.op_flag[jj] = 0;
            exec_serial_block<KB, VB, W>(t, keys, vals, jj, *s_big, *s_out, a);
        }
    } else {
        if (threadIdx.x < 32) {
            const Tile<32> tl;
            for (uint32_t k = 0; k < c; k++) {
                const uint32_t jj = s_list[k];
                if (tl.lane == 0) sc.op_flag[jj] = 0;
                RegKey<KB> key;
                key.load(keys + (uint64_t)jj * KB, KB);
                int kind = 5;
                if (s_chain && t.mask >= 4 * 32 - 1) kind = exec_tile<KB, VB, 32>(t, key, vals, jj, tl, *s_chain, a);
                if (kind == 5 && tl.lane == 0) a.claimed += exec_insert_key<KB, VB>(t, key, vals + (uint64_t)jj * VB, a);
                tl.sync();  // the next op reads this one's writes
            }
        }
    }
}

// Applies the ops of `list` (n ops; nullptr = the identity over n ops) one at
// a time in index order -- the sequential semantics, for rounds that found an
// op with no free slot or a flow wrapping the table.  With compile-time
// record sizes each op runs on warp 0 as a tile walk (128 slots per round
// trip); an op whose walk finds no free slot within a pass over the table
// (a table overfilled by uncounted inserts) writes nothing there and reruns
// as the scalar walk, which applies the step limit.  Run-time sizes use the
// scalar walk on thread 0.  Registrations must already be clear.
// Block-uniform call; s_buf holds blockDim.x words, s_woff 33, s_chain one
// tile chain buffer (compile-time sizes; may be null for the scalar walk).
// With s_big (a block of SERIAL_THREADS threads) each op runs on the whole
// block instead (exec_serial_block).
template <int KB, int VB>
__device__ void serial_process(const TableView& t, const uint8_t* keys, const uint8_t* vals, const uint32_t* list,
                               uint32_t n, uint32_t n0, const OpScratch& sc, ExecAcc& a, uint32_t* s_buf,
                               uint32_t* s_woff, TileChain* s_chain, SerialChain* s_big = nullptr,
                               SerialOut* s_out = nullptr) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sc.op_flag[list ? list[i] : i] = 3;
    __syncthreads();
    for (uint32_t base = 0; base < n0; base += blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        const bool take = j < n0 && sc.op_flag[j] == 3;
        const uint32_t c = block_compact(j, take, s_buf, s_woff);
        serial_apply<KB, VB, SERIAL_THREADS>(t, keys, vals, s_buf, c, sc, a, s_chain, s_big, s_out);
        __syncthreads();
    }
}


// ---- grid-wide round phases ---------------------------------------------

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_ins_p1(TableView t, const uint8_t* __restrict__ keys, uint32_t n0,
                                                   uint32_t r, OpScratch sc, Ctl* ctl) {
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    if (blockIdx.x == 0 && threadIdx.x == 0) reset_next_round(ctl, r);
    bool no_free = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops.n; i += gridDim.x * blockDim.x) {
        const uint32_t j = ops.op(i);
        const uint64_t F = find_free<KB>(t, keys, j);
        register_op(t, j, F, sc.op_slot);
        no_free = no_free || F == NONE64;
    }
    if (no_free) ctl->serial[r & 1] = 1u;
}

__global__ void __launch_bounds__(RBLOCK) k_ins_p2(TableView t, uint32_t n0, uint32_t r, uint32_t nops,
                                                   OpScratch sc, Ctl* ctl) {
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops.n; i += gridDim.x * blockDim.x) {
        const uint32_t bits = walk_op(t, ops.op(i), nops, sc.op_slot, sc.op_word, sc.op_flag);
        if (bits & 1u) ctl->serial[r & 1] = 1u;
        if (bits & 2u) atomicOr(&ctl->err, ERR_SCRATCH);
    }
}

#ifndef FM_P3_MIN_BLOCKS
#define FM_P3_MIN_BLOCKS 3  // resident blocks per SM the thread-per-op pass is compiled for
#endif
template <int KB, int VB>
__global__ void __launch_bounds__(RBLOCK, FM_P3_MIN_BLOCKS) k_ins_p3(TableView t, const uint8_t* __restrict__ keys,
                                                   const uint8_t* __restrict__ vals, uint32_t n0, uint32_t r,
                                                   OpScratch sc, Ctl* ctl) {
    __shared__ AppendSmem s_app;
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    append_init(s_app);
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    const bool serial = *(volatile uint32_t*)&ctl->serial[r & 1] != 0;
    uint32_t* out = pend_of(sc, r + 1);
    uint32_t* out_n = &ctl->npend[(r + 1) & 1];
    uint32_t* long_n = &ctl->nlong[r & 1];
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t iters = grid_iters(ops.n);
    ExecAcc a;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t i = i0 + it * stride;
        const bool valid = i < ops.n;
        uint32_t j = 0;
        bool ran = false;
        if (valid) {
            j = ops.op(i);
            const int code = finish_op<KB, VB>(t, keys, vals, j, serial, sc, a, true);
            if constexpr (KB != 0 && VB != 0) append(sc.long_list, long_n, j, code == 2);
            ran = code != 0;
        }
        block_append(out, out_n, j, valid && !ran, s_app);
    }
    block_add_count(ctl, a.claimed, s_tmp);
    publish_rare(ctl, a.maxd, a.tomb, a.limit);
    if (blockIdx.x == 0 && threadIdx.x == 0 && ops.n) atomicAdd(&ctl->rounds, 1u);
}

// ---- tile-cooperative phases (compile-time shapes) -----------------------

// Phase 3 for op j on a tile (the single-block tail): run the tile walk if j
// leads an unblocked segment; clear the registration.  Returns whether it ran.
template <int KB, int VB, int T>
__device__ __forceinline__ bool finish_tile(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t j,
                                            bool serial, const OpScratch& sc, const Tile<T>& tl, TileChain& s,
                                            ExecAcc& a) {
    // independent loads issued together: decision words, registration, key
    const uint8_t lead = sc.op_flag[j];
    const uint32_t blk = sc.op_word[j];
    const uint64_t F = sc.op_slot[j];
    RegKey<KB> key;
    key.load(keys + (uint64_t)j * KB, KB);
    const bool run = !serial && lead != 0 && blk > j;
    if (run) {
        if (t.mask >= 4 * T - 1) {
            if (exec_tile<KB, VB, T>(t, key, vals, j, tl, s, a) == 5) a.limit = true;
        } else {
            if (tl.lane == 0) a.claimed += exec_insert_key<KB, VB>(t, key, vals + (uint64_t)j * VB, a);
        }
    }
    tl.sync();
    if (tl.lane == 0) {
        if (F != NONE64) {
            t.seg_min[F] = IDLE;
            t.seg_cnt[F] = 0;
        }
        sc.op_word[j] = IDLE;
    }
    return run;
}

// Phase 4: the inserts of round r whose walks were too long for one thread,
// one T-lane tile each (T = 8 or 16 share every warp instruction between 4
// or 2 inserts; the closed-form walk keeps their control flow together).
// Their segments are disjoint from each other and from every op run in
// phase 3.
template <int T>
using P4Chain = ChainBuf<(8 * T > 64 ? 8 * T : 64), 4 * T>;

#ifndef FM_P4_MIN_BLOCKS
#define FM_P4_MIN_BLOCKS 2  // resident blocks per SM the long-walk pass is compiled for (no spills at 2)
#endif
template <int KB, int VB, int T>
__global__ void __launch_bounds__(RBLOCK, FM_P4_MIN_BLOCKS) k_ins_p4(TableView t, const uint8_t* __restrict__ keys,
                                                      const uint8_t* __restrict__ vals, uint32_t r, OpScratch sc,
                                                      Ctl* ctl) {
    constexpr int NT = RBLOCK / T;
    __shared__ P4Chain<T> s_chain[NT];
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    const uint32_t n = *(volatile const uint32_t*)&ctl->nlong[r & 1];
    if (n == 0) return;  // block-uniform
    const Tile<T> tl;
    const uint32_t ti = threadIdx.x / T;
    const uint32_t ntiles = gridDim.x * NT;
    ExecAcc a;
    // uniform trip count per warp (all tiles of a warp loop together)
    const uint32_t iters = (n + ntiles - 1) / ntiles;
    const uint32_t first = blockIdx.x * NT + ti;
    // two-deep prefetch: the next op's key and the op after's list entry
    // load while this op walks (their round trips overlap the walk)
    uint32_t jn = first < n ? sc.long_list[first] : 0u;
    RegKey<KB> kn;
    if (first < n) kn.load(keys + (uint64_t)jn * KB, KB);
    uint32_t jnn = first + ntiles < n ? sc.long_list[first + ntiles] : 0u;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t i = first + it * ntiles;
        const uint32_t j = jn;
        const RegKey<KB> key = kn;
        if (i + ntiles < n) {
            jn = jnn;
            kn.load(keys + (uint64_t)jn * KB, KB);
            if (i + 2 * ntiles < n) jnn = sc.long_list[i + 2 * ntiles];
        }
        if (i < n) {
            if (t.mask >= 4 * T - 1) {
                if (exec_tile<KB, VB, T, P4Chain<T>>(t, key, vals, j, tl, s_chain[ti], a) == 5) a.limit = true;
            } else {
                if (tl.lane == 0) a.claimed += exec_insert_key<KB, VB>(t, key, vals + (uint64_t)j * VB, a);
            }
        }
        tl.sync();
    }
    block_add_count(ctl, a.claimed, s_tmp);
    publish_rare(ctl, a.maxd, a.tomb, a.limit);
}

// Lanes per insert of the long-walk pass: 32, 16 or 8 (compile-time setting
// FM_P4_LANES; default 32, the fastest measured on B200 at load 0.8: 8 and 16
// lanes share warp instructions between inserts but walk more windows and
// move fewer records per round trip).
#ifndef FM_P4_LANES
#define FM_P4_LANES 32
#endif
static_assert(FM_P4_LANES == 8 || FM_P4_LANES == 16 || FM_P4_LANES == 32, "FM_P4_LANES: 8, 16 or 32");
constexpr int p4_lanes() { return FM_P4_LANES; }

// ---- single-block tails ----------------------------------------------------
//
// One block runs every remaining round of the call (phases separated by block
// barriers) when at most TAIL_MAX ops are pending, or returns at once.  A
// serial round hands its ops to serial_process.  On completion both pending
// counts are zero (the host's done marker).  With `handoff`, rounds that stop
// progressing are handed back instead of run one at a time here: the tail
// stops at a round boundary with that round's ops pending and records the
// round in Ctl::tail_handoff (the host then runs them as components).

template <int KB, int VB, int T>
__device__ __forceinline__ void ins_tail_body(const TableView& t, const uint8_t* __restrict__ keys,
                                              const uint8_t* __restrict__ vals, uint32_t n0, uint32_t r0,
                                              uint32_t nops, const OpScratch& sc, Ctl* ctl, uint32_t limit,
                                              bool handoff) {
    // tiles holding a chain buffer (T > 1): as many as the static shared
    // memory allows; the block's other warps idle in the tile phases
    constexpr int NT = T > 1 ? (TAIL_THREADS / T < 12 ? TAIL_THREADS / T : 12) : 1;
    __shared__ uint32_t s_n, s_next, s_serial, s_err;
    __shared__ TileChain s_chain[T > 1 ? NT : 1];
    __shared__ uint32_t s_buf[TAIL_THREADS];
    __shared__ uint32_t s_woff[33];
    if (threadIdx.x == 0) {
        s_n = (r0 == 0) ? n0 : *(volatile uint32_t*)&ctl->npend[r0 & 1];
        s_err = 0;
    }
    __syncthreads();
    uint32_t n = s_n;
    if (n == 0 || n > limit) return;
    ExecAcc a;
    uint32_t r = r0;
    uint32_t rounds = 0;
    uint32_t handed = 0;  // ops handed back at round r (handoff)
    // tiles (T > 1) or single threads (T == 1) as the unit of work
    const uint32_t unit = T > 1 ? threadIdx.x / T : threadIdx.x;
    const uint32_t nunits = T > 1 ? (uint32_t)NT : blockDim.x;
    const bool leader_lane = T > 1 ? (threadIdx.x & (T - 1)) == 0 : true;
    for (;;) {
        const uint32_t* in = (r == 0) ? nullptr : pend_of(sc, r);
        uint32_t* out = pend_of(sc, r + 1);
        if (threadIdx.x == 0) {
            s_next = 0;
            s_serial = 0;
        }
        __syncthreads();
        for (uint32_t i = unit; unit < nunits && i < n; i += nunits) {
            const uint32_t j = in ? in[i] : i;
            uint64_t F;
            if constexpr (T > 1) {
                const Tile<(T > 1 ? T : 8)> tl;
                RegKey<KB> key;
                key.load(keys + (uint64_t)j * KB, KB);
                F = find_free_tile<(T > 1 ? T : 8)>(t, key.hash(KB, t.hash_mode) & t.mask, tl);
            } else {
                F = find_free<KB>(t, keys, j);
            }
            if (leader_lane) {
                register_op(t, j, F, sc.op_slot);
                if (F == NONE64) s_serial = 1u;
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t bits = walk_op(t, in ? in[i] : i, nops, sc.op_slot, sc.op_word, sc.op_flag);
            if (bits & 1u) s_serial = 1u;
            if (bits & 2u) atomicOr(&s_err, ERR_SCRATCH);
        }
        __syncthreads();
        const bool serial = s_serial != 0;
        if (s_err) break;
        if (serial) {
            // clear the round's registrations, then apply its ops in index order
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint32_t j = in ? in[i] : i;
                const uint64_t F = sc.op_slot[j];
                if (F != NONE64) {
                    t.seg_min[F] = IDLE;
                    t.seg_cnt[F] = 0;
                }
                sc.op_word[j] = IDLE;
            }
            __syncthreads();
            if (handoff && in) {
                handed = n;
                break;
            }
            serial_process<KB, VB>(t, keys, vals, in, n, n0, sc, a, s_buf, s_woff, T > 1 ? &s_chain[0] : nullptr);
            ++rounds;
            break;
        }
        for (uint32_t i = unit; unit < nunits && i < n; i += nunits) {
            const uint32_t j = in ? in[i] : i;
            bool ran;
            if constexpr (T > 1) {
                const Tile<(T > 1 ? T : 8)> tl;
                ran = finish_tile<KB, VB, (T > 1 ? T : 8)>(t, keys, vals, j, false, sc, tl, s_chain[unit], a);
            } else {
                ran = finish_op<KB, VB>(t, keys, vals, j, false, sc, a, false) != 0;
            }
            if (!ran && leader_lane) out[atomicAdd(&s_next, 1u)] = j;
        }
        __syncthreads();
        const uint32_t nn = s_next;
        ++r;
        ++rounds;
        if (nn == 0) break;
        if (nn >= n) {  // every non-serial round runs its smallest op
            if (threadIdx.x == 0) atomicOr(&s_err, ERR_NO_PROGRESS);
            break;
        }
        if (rounds >= 4 && (uint64_t)nn * 8 > (uint64_t)n * 7) {
            // under 1/8 of the ops per round (ops crowded onto few free slots,
            // a near-full table): the rest in index order, one at a time
            __syncthreads();
            if (handoff) {
                handed = nn;
                break;
            }
            serial_process<KB, VB>(t, keys, vals, pend_of(sc, r), nn, n0, sc, a, s_buf, s_woff,
                                   T > 1 ? &s_chain[0] : nullptr);
            ++rounds;
            break;
        }
        n = nn;
        __syncthreads();  // everyone has read s_next before it is reset
    }
    __syncthreads();
    if (a.claimed) atomicAdd(&ctl->count, (unsigned long long)a.claimed);
    if (a.maxd > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, a.maxd);
    if (a.tomb) ctl->tomb_claimed = 1u;
    if (a.limit) atomicOr(&ctl->err, ERR_WALK_LIMIT);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_err) {
            atomicOr(&ctl->err, s_err);
        } else {
            ctl->npend[r0 & 1] = 0;  // done marker read by the host
            ctl->npend[(r0 + 1) & 1] = 0;
            if (handed) {
                ctl->npend[r & 1] = handed;
                ctl->tail_handoff = r + 1;
            }
        }
        atomicAdd(&ctl->rounds, rounds);
    }
}

template <int KB, int VB, int T>
__global__ void __launch_bounds__(TAIL_THREADS) k_ins_tail(TableView t, const uint8_t* __restrict__ keys,
                                                           const uint8_t* __restrict__ vals, uint32_t n0,
                                                           uint32_t r0, uint32_t nops, OpScratch sc, Ctl* ctl,
                                                           bool handoff) {
    ins_tail_body<KB, VB, T>(t, keys, vals, n0, r0, nops, sc, ctl, TAIL_MAX, handoff);
}

// Host-launched fallback for a serial round whose pending count is above
// TAIL_MAX: applies round r's ops in index order.
template <int KB, int VB>
__global__ void __launch_bounds__(SERIAL_THREADS) k_ins_serial(TableView t, const uint8_t* __restrict__ keys,
                                                               const uint8_t* __restrict__ vals, uint32_t n0,
                                                               uint32_t r, OpScratch sc, Ctl* ctl) {
    __shared__ uint32_t s_buf[SERIAL_THREADS];
    __shared__ uint32_t s_woff[33];
    __shared__ TileChain s_chain;
    __shared__ SerialOut s_out;
    extern __shared__ __align__(16) unsigned char s_dyn[];  // SerialChain (compile-time sizes)
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    ExecAcc a;
    serial_process<KB, VB>(t, keys, vals, ops.list, ops.n, n0, sc, a, s_buf, s_woff, &s_chain,
                           (KB && VB) ? reinterpret_cast<SerialChain*>(s_dyn) : nullptr, &s_out);
    __syncthreads();
    if (a.claimed) atomicAdd(&ctl->count, (unsigned long long)a.claimed);
    if (a.maxd > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, a.maxd);
    if (a.tomb) ctl->tomb_claimed = 1u;
    if (a.limit) atomicOr(&ctl->err, ERR_WALK_LIMIT);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->npend[r & 1] = 0;
        ctl->npend[(r + 1) & 1] = 0;
        atomicAdd(&ctl->rounds, 1u);
    }
}

// Dynamic shared memory of a serial kernel (its attribute is set before each
// launch: a host-side call).
template <class K>
size_t serial_smem(K kernel, bool big) {
    if (!big) return 0;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SerialChain));
    return sizeof(SerialChain);
}

// ---- components: the one-at-a-time order spread over the GPU ---------------
//
// When rounds stall (ops crowded onto few free slots of a near-full table),
// the remaining ops must run in index order -- but only ops that can reach
// the same slots need that order.  An insert reads and writes only [home, F']
// with F' the first free slot at or after its home when it runs, and fills
// F' when its key is new.  With d(s) the pending ops whose first free slot is
// s now, a carry walk over the table in slot order bounds the free slots they
// fill: a free slot passes on c' = max(0, c + d(s) - 1) of the c ops that
// arrive at it, an occupied slot passes c on.  A free slot with d(s) > 0 and
// no arriving carry starts a component, which ends at the first free slot
// that passes on 0.  A component's ops fill free slots within it only and read
// nothing below their homes, so components touch disjoint slots and may run
// at the same time.  Counting updates as demand only raises carries (merging
// components), which keeps this true.  Each component's ops run in index
// order on one block; components go to the resident blocks by a hash of
// their start.
//
// The walk is a scan of the functions c -> max(a, c + b), which compose
// associatively: per chunk of CMP_CHUNK slots (32 per thread), then one block
// over the chunks.  The carry into slot 0 comes round the ring: with the
// ring's composition (A, B) and B < 0 (fewer demanding ops than free slots)
// it is A.  Otherwise (B >= 0, or an op with no free slot at all) every op
// goes to block 0, which is the plain one-at-a-time order.
constexpr int CMP_THREADS = 256;
constexpr uint32_t CMP_PER_T = (uint32_t)CMP_CHUNK / CMP_THREADS;  // slots per thread
constexpr long long CMP_NEG = -(1ll << 60);
constexpr uint32_t CMP_UNK = 0xFFFFFFFEu;  // demand slot whose component starts in an earlier chunk
constexpr uint32_t CMP_OPS_PER_T = 16;
constexpr uint32_t CMP_OPS_PER_BLOCK = CMP_THREADS * CMP_OPS_PER_T;  // op indices per compaction block
constexpr int CMP_EXEC_THREADS = 256;
static_assert(CMP_PER_T == 32, "cmp_load reads 32 slots per thread");

struct CFn {  // c -> max(a, c + b)
    long long a, b;
};
__device__ __forceinline__ CFn cfn_id() { return CFn{CMP_NEG, 0}; }
// f, then g
__device__ __forceinline__ CFn cfn_then(const CFn& f, const CFn& g) {
    return CFn{max(g.a, f.a + g.b), f.b + g.b};
}
__device__ __forceinline__ long long cfn_apply(const CFn& f, long long c) { return max(f.a, c + f.b); }

struct CmpHdr {
    uint32_t fallback;  // 1: every op to block 0
    uint32_t np;        // ops in the ordered list
};

// The call's op count: the argument, or the grouped call's count in its
// control block (CMP_N0_CTL).
__device__ __forceinline__ uint32_t cmp_n0(uint32_t n0, const Ctl* ctl) {
    return n0 != CMP_N0_CTL ? n0 : *(volatile const uint32_t*)&ctl->n0;
}

// The component buffer: header, then per chunk its function, the carry into
// it, its last component start + 1 and the last start before it + 1 (0: none).
struct CmpView {
    CmpHdr* hdr;
    CFn* fn;
    long long* carry;
    uint32_t* last;
    uint32_t* prev;
    uint32_t nch;
    __device__ __forceinline__ CmpView(uint8_t* base, uint64_t mask) {
        nch = (uint32_t)cmp_chunks(mask);
        hdr = reinterpret_cast<CmpHdr*>(base);
        fn = reinterpret_cast<CFn*>(base + 256);
        carry = reinterpret_cast<long long*>(fn + nch);
        last = reinterpret_cast<uint32_t*>(carry + nch);
        prev = last + nch;
    }
};

// Metadata and demand of the 32 slots from s0 (a multiple of 32); slots past
// the table read as occupied.
__device__ __forceinline__ void cmp_load(const TableView& t, uint64_t s0, uint32_t (&fl)[CMP_PER_T],
                                         uint32_t (&dm)[CMP_PER_T]) {
    if (s0 + CMP_PER_T - 1 <= t.mask) {
        const uint4* pf = reinterpret_cast<const uint4*>(t.flags + s0);
        const uint4* pc = reinterpret_cast<const uint4*>(t.seg_cnt + s0);
#pragma unroll
        for (int q = 0; q < (int)CMP_PER_T / 4; q++) {
            const uint4 f = pf[q], c = pc[q];
            fl[4 * q] = f.x, fl[4 * q + 1] = f.y, fl[4 * q + 2] = f.z, fl[4 * q + 3] = f.w;
            dm[4 * q] = c.x, dm[4 * q + 1] = c.y, dm[4 * q + 2] = c.z, dm[4 * q + 3] = c.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < (int)CMP_PER_T; i++) {
            const uint64_t s = s0 + i;
            fl[i] = s <= t.mask ? t.flags[s] : ST_OCC;
            dm[i] = s <= t.mask ? t.seg_cnt[s] : 0u;
        }
    }
}

__device__ __forceinline__ CFn cmp_thread_fn(const uint32_t (&fl)[CMP_PER_T], const uint32_t (&dm)[CMP_PER_T]) {
    CFn f = cfn_id();
#pragma unroll
    for (int i = 0; i < (int)CMP_PER_T; i++)
        if (is_free(fl[i])) f = cfn_then(f, CFn{0, (long long)dm[i] - 1});
    return f;
}

// Exclusive in-order scan of one function per thread over the block; `total`
// gets the block's composition.  s_w: 32 entries.
__device__ CFn cmp_block_scan(CFn f, CFn* s_w, CFn& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    CFn inc = f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        CFn g;
        g.a = __shfl_up_sync(0xFFFFFFFFu, inc.a, off);
        g.b = __shfl_up_sync(0xFFFFFFFFu, inc.b, off);
        if ((int)lane >= off) inc = cfn_then(g, inc);
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        CFn v = lane < nw ? s_w[lane] : cfn_id();
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            CFn g;
            g.a = __shfl_up_sync(0xFFFFFFFFu, v.a, off);
            g.b = __shfl_up_sync(0xFFFFFFFFu, v.b, off);
            if ((int)lane >= off) v = cfn_then(g, v);
        }
        s_w[lane] = v;  // inclusive over the warps
    }
    __syncthreads();
    CFn ex;
    ex.a = __shfl_up_sync(0xFFFFFFFFu, inc.a, 1);
    ex.b = __shfl_up_sync(0xFFFFFFFFu, inc.b, 1);
    if (lane == 0) ex = cfn_id();
    if (warp > 0) ex = cfn_then(s_w[warp - 1], ex);
    total = s_w[nw - 1];
    __syncthreads();
    return ex;
}

// Exclusive max-scan (ex: the largest value of the threads before) and the
// block's largest value.  s_m: 32 entries.
__device__ uint32_t cmp_block_max(uint32_t v, uint32_t* s_m, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t g = __shfl_up_sync(0xFFFFFFFFu, inc, off);
        if ((int)lane >= off) inc = max(inc, g);
    }
    if (lane == 31) s_m[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? s_m[lane] : 0u;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t g = __shfl_up_sync(0xFFFFFFFFu, w, off);
            if ((int)lane >= off) w = max(w, g);
        }
        s_m[lane] = w;
    }
    __syncthreads();
    uint32_t ex = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
    if (lane == 0) ex = 0u;
    if (warp > 0) ex = max(ex, s_m[warp - 1]);
    total = s_m[nw - 1];
    __syncthreads();
    return ex;
}

// Exclusive sum-scan and the block's sum.  s_m: 32 entries.
__device__ uint32_t cmp_block_sum(uint32_t v, uint32_t* s_m, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t g = __shfl_up_sync(0xFFFFFFFFu, inc, off);
        if ((int)lane >= off) inc += g;
    }
    if (lane == 31) s_m[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? s_m[lane] : 0u;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t g = __shfl_up_sync(0xFFFFFFFFu, w, off);
            if ((int)lane >= off) w += g;
        }
        s_m[lane] = w;
    }
    __syncthreads();
    uint32_t ex = inc - v;
    if (warp > 0) ex += s_m[warp - 1];
    total = s_m[nw - 1];
    __syncthreads();
    return ex;
}

// 1. Each pending op of round r: its first free slot (op_slot), its mark
// (op_flag 3) and its demand on that slot (seg_cnt).
template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_cmp_find(TableView t, const uint8_t* __restrict__ keys, uint32_t n0,
                                                     uint32_t r, OpScratch sc, Ctl* ctl, uint32_t force) {
    const RoundOps ops = round_ops(sc, ctl, r, cmp_n0(n0, ctl));
    bool fb = force != 0u && blockIdx.x == 0 && threadIdx.x == 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops.n; i += gridDim.x * blockDim.x) {
        const uint32_t j = ops.op(i);
        const uint64_t F = find_free<KB>(t, keys, j);
        sc.op_slot[j] = F;
        sc.op_flag[j] = 3;
        if (F == NONE64) fb = true;
        else atomicAdd(&t.seg_cnt[F], 1u);
    }
    if (fb) reinterpret_cast<CmpHdr*>(sc.comp)->fallback = 1u;
}

// 2. Each chunk's composition.
__global__ void __launch_bounds__(CMP_THREADS) k_cmp_fn(TableView t, uint8_t* comp) {
    __shared__ CFn s_w[32];
    CmpView cv(comp, t.mask);
    const uint64_t s0 = (uint64_t)blockIdx.x * CMP_CHUNK + (uint64_t)threadIdx.x * CMP_PER_T;
    uint32_t fl[CMP_PER_T], dm[CMP_PER_T];
    cmp_load(t, s0, fl, dm);
    CFn total;
    cmp_block_scan(cmp_thread_fn(fl, dm), s_w, total);
    if (threadIdx.x == 0) cv.fn[blockIdx.x] = total;
}

// 3. One block: the carry into every chunk, from the carry round the ring.
__global__ void __launch_bounds__(1024) k_cmp_carry(uint8_t* comp, uint64_t mask) {
    __shared__ CFn s_w[32];
    CmpView cv(comp, mask);
    const uint32_t per = (cv.nch + blockDim.x - 1) / blockDim.x;
    const uint32_t c0 = min(threadIdx.x * per, cv.nch), c1 = min(c0 + per, cv.nch);
    CFn f = cfn_id();
    for (uint32_t c = c0; c < c1; c++) f = cfn_then(f, cv.fn[c]);
    CFn total;
    const CFn ex = cmp_block_scan(f, s_w, total);
    if (total.b >= 0 || total.a < 0) {  // block-uniform
        if (threadIdx.x == 0) cv.hdr->fallback = 1u;
        return;
    }
    long long carry = cfn_apply(ex, total.a);
    for (uint32_t c = c0; c < c1; c++) {
        cv.carry[c] = carry;
        carry = cfn_apply(cv.fn[c], carry);
    }
}

// 4. Component starts: every demand slot gets its component's start in
// seg_min (CMP_UNK when it lies in an earlier chunk); each chunk its last start.
__global__ void __launch_bounds__(CMP_THREADS) k_cmp_starts(TableView t, uint8_t* comp) {
    __shared__ CFn s_w[32];
    __shared__ uint32_t s_m[32];
    CmpView cv(comp, t.mask);
    if (*(volatile uint32_t*)&cv.hdr->fallback) return;  // block-uniform
    const uint64_t s0 = (uint64_t)blockIdx.x * CMP_CHUNK + (uint64_t)threadIdx.x * CMP_PER_T;
    uint32_t fl[CMP_PER_T], dm[CMP_PER_T];
    cmp_load(t, s0, fl, dm);
    CFn total;
    const CFn ex = cmp_block_scan(cmp_thread_fn(fl, dm), s_w, total);
    const long long cin = cfn_apply(ex, cv.carry[blockIdx.x]);
    long long c = cin;
    uint32_t last = 0;
#pragma unroll
    for (int i = 0; i < (int)CMP_PER_T; i++) {
        if (is_free(fl[i])) {
            if (dm[i] && c == 0) last = (uint32_t)(s0 + i) + 1u;
            c = max(0ll, c + (long long)dm[i] - 1);
        }
    }
    uint32_t tot;
    uint32_t cur = cmp_block_max(last, s_m, tot);
    c = cin;
#pragma unroll
    for (int i = 0; i < (int)CMP_PER_T; i++) {
        if (is_free(fl[i])) {
            if (dm[i]) {
                if (c == 0) cur = (uint32_t)(s0 + i) + 1u;
                t.seg_min[s0 + i] = cur ? cur - 1u : CMP_UNK;
            }
            c = max(0ll, c + (long long)dm[i] - 1);
        }
    }
    if (threadIdx.x == 0) cv.last[blockIdx.x] = tot;
}

// 5. One block: the last start before every chunk, round the ring.
__global__ void __launch_bounds__(1024) k_cmp_prev(uint8_t* comp, uint64_t mask) {
    __shared__ uint32_t s_m[32];
    CmpView cv(comp, mask);
    if (*(volatile uint32_t*)&cv.hdr->fallback) return;
    const uint32_t per = (cv.nch + blockDim.x - 1) / blockDim.x;
    const uint32_t c0 = min(threadIdx.x * per, cv.nch), c1 = min(c0 + per, cv.nch);
    uint32_t m = 0;
    for (uint32_t c = c0; c < c1; c++) m = max(m, cv.last[c]);
    uint32_t tot;
    uint32_t ex = cmp_block_max(m, s_m, tot);
    for (uint32_t c = c0; c < c1; c++) {
        cv.prev[c] = ex ? ex : tot;
        ex = max(ex, cv.last[c]);
    }
}

// 6. Each pending op's block: a hash of its component's start (0 for all on
// the fallback).
__global__ void __launch_bounds__(RBLOCK) k_cmp_own(TableView t, uint32_t n0, uint32_t r, OpScratch sc, Ctl* ctl,
                                                    uint32_t nblk) {
    const RoundOps ops = round_ops(sc, ctl, r, cmp_n0(n0, ctl));
    CmpView cv(sc.comp, t.mask);
    const bool fb = *(volatile uint32_t*)&cv.hdr->fallback != 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops.n; i += gridDim.x * blockDim.x) {
        const uint32_t j = ops.op(i);
        uint32_t o = 0;
        if (!fb) {
            const uint64_t F = sc.op_slot[j];
            uint32_t v = t.seg_min[F];
            if (v == CMP_UNK) v = cv.prev[F / CMP_CHUNK] - 1u;
            o = (uint32_t)(((uint64_t)(v * 2654435761u) * nblk) >> 32);
        }
        sc.op_word[j] = o;
    }
}

// 7. The marked ops in index order (long_list): counts per block of op
// indices (kept in op_pt), one block's scan of them, then the writes.
__device__ __forceinline__ uint32_t cmp_marks(const OpScratch& sc, uint32_t n0, uint32_t j0) {
    uint32_t m = 0;
    if (j0 + CMP_OPS_PER_T <= n0) {
        const uint4 w = *reinterpret_cast<const uint4*>(sc.op_flag + j0);
        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int q = 0; q < 16; q++)
            if (((ws[q >> 2] >> (8 * (q & 3))) & 0xFFu) == 3u) m |= 1u << q;
    } else {
        for (uint32_t q = 0; q < CMP_OPS_PER_T && j0 + q < n0; q++)
            if (sc.op_flag[j0 + q] == 3) m |= 1u << q;
    }
    return m;
}

__global__ void __launch_bounds__(CMP_THREADS) k_cmp_count(OpScratch sc, uint32_t n0, const Ctl* ctl) {
    __shared__ uint32_t s_m[32];
    n0 = cmp_n0(n0, ctl);
    const uint32_t j0 = blockIdx.x * CMP_OPS_PER_BLOCK + threadIdx.x * CMP_OPS_PER_T;
    uint32_t tot;
    cmp_block_sum(__popc(cmp_marks(sc, n0, j0)), s_m, tot);
    if (threadIdx.x == 0) sc.op_pt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_cmp_offsets(OpScratch sc, uint32_t nb) {
    __shared__ uint32_t s_m[32];
    const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
    const uint32_t b0 = min(threadIdx.x * per, nb), b1 = min(b0 + per, nb);
    uint32_t v = 0;
    for (uint32_t b = b0; b < b1; b++) v += sc.op_pt[b];
    uint32_t tot;
    uint32_t ex = cmp_block_sum(v, s_m, tot);
    for (uint32_t b = b0; b < b1; b++) {
        const uint32_t c = sc.op_pt[b];
        sc.op_pt[b] = ex;
        ex += c;
    }
    if (threadIdx.x == 0) reinterpret_cast<CmpHdr*>(sc.comp)->np = tot;
}

__global__ void __launch_bounds__(CMP_THREADS) k_cmp_list(OpScratch sc, uint32_t n0, const Ctl* ctl) {
    __shared__ uint32_t s_m[32];
    n0 = cmp_n0(n0, ctl);
    const uint32_t j0 = blockIdx.x * CMP_OPS_PER_BLOCK + threadIdx.x * CMP_OPS_PER_T;
    uint32_t m = cmp_marks(sc, n0, j0);
    uint32_t tot;
    uint32_t at = sc.op_pt[blockIdx.x] + cmp_block_sum(__popc(m), s_m, tot);
    while (m) {
        const int q = __ffs(m) - 1;
        m &= m - 1u;
        sc.long_list[at++] = j0 + (uint32_t)q;
    }
}

// 8. Every block runs the ops it owns in index order.
template <int KB, int VB>
__global__ void __launch_bounds__(CMP_EXEC_THREADS, 2) k_ins_comp(TableView t, const uint8_t* __restrict__ keys,
                                                                  const uint8_t* __restrict__ vals, uint32_t r,
                                                                  OpScratch sc, Ctl* ctl) {
    __shared__ uint32_t s_buf[CMP_EXEC_THREADS];
    __shared__ uint32_t s_woff[33];
    __shared__ TileChain s_chain;
    __shared__ SerialOut s_out;
    extern __shared__ __align__(16) unsigned char s_dyn[];  // SerialChain (compile-time sizes)
    const CmpHdr* hdr = reinterpret_cast<const CmpHdr*>(sc.comp);
    const uint32_t np = *(volatile const uint32_t*)&hdr->np;
    const bool fb = *(volatile const uint32_t*)&hdr->fallback != 0u;
    ExecAcc a;
    if (!fb || blockIdx.x == 0) {  // block-uniform
        for (uint32_t base = 0; base < np; base += blockDim.x) {
            const uint32_t i = base + threadIdx.x;
            const uint32_t j = i < np ? sc.long_list[i] : 0u;
            const bool take = i < np && sc.op_word[j] == blockIdx.x;
            const uint32_t c = block_compact(j, take, s_buf, s_woff);
            serial_apply<KB, VB, CMP_EXEC_THREADS>(t, keys, vals, s_buf, c, sc, a, &s_chain,
                                                   (KB && VB) ? reinterpret_cast<SerialChain*>(s_dyn) : nullptr,
                                                   &s_out);
            __syncthreads();
        }
    }
    if (a.claimed) atomicAdd(&ctl->count, (unsigned long long)a.claimed);
    if (a.maxd > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, a.maxd);
    if (a.tomb) ctl->tomb_claimed = 1u;
    if (a.limit) atomicOr(&ctl->err, ERR_WALK_LIMIT);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->npend[r & 1] = 0;
        ctl->npend[(r + 1) & 1] = 0;
        atomicAdd(&ctl->rounds, 1u);
    }
}

// 9. Registrations and inflow words back to idle.
__global__ void __launch_bounds__(RBLOCK) k_cmp_clean(TableView t, OpScratch sc) {
    const uint32_t np = *(volatile const uint32_t*)&reinterpret_cast<const CmpHdr*>(sc.comp)->np;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const uint32_t j = sc.long_list[i];
        const uint64_t F = sc.op_slot[j];
        if (F != NONE64) {
            t.seg_min[F] = IDLE;
            t.seg_cnt[F] = 0;
        }
        sc.op_word[j] = IDLE;
    }
}

// ---- direct insert: components found from each op's free slot -------------
//
// The plain insert call below the component load, without rounds.  An insert
// reads and writes only [home, F'] (F' its first free slot when it runs) and
// fills F' when its key is new (the argument of the component path above).
// With F each op's first free slot before the call, the ops that can touch
// common slots are those joined by a chain of free slots over which their
// demand carries; here the chains are found from the ops' own free slots
// instead of by a scan of the table:
//   find  (a thread per op)  F, then the op joins F's list: seg_cnt[F] counts
//         the ops at F, seg_min[F] heads a list linked through op_word, and
//         the first op to arrive leads F (op_flag 1).
//   flow  (a thread per leader of an F holding c >= 2 ops)  walks the free
//         slots after F carrying c - 1 ops, each slot taking one and adding
//         its own ops, and marks every later F it reaches (DX_ABS in seg_cnt)
//         as part of this component, until the carry is 0.
//   exec  (a thread per op)  an op alone at an unmarked F runs at once: its
//         walk [home, F] from the metadata, the possible updates compared,
//         the records moved two per round trip; a walk too long for one
//         thread, and the leader of an unmarked F with c >= 2, go to the warp
//         pass's list; the other ops wait for their component.
//   warp  (a warp per list entry)  a long lone op runs as a tile walk; a
//         component gathers its ops from the lists of its free slots (the
//         flow walk again), sorts them by index and runs them one after
//         another as tile walks.
// Components touch disjoint slots, so all of this runs at once.  A call that
// finds an op with no free slot or a flow round the whole table leaves every
// op to the component path (Ctl::serial[0]); a component with more ops than a
// warp gathers leaves its ops to it (pend[1], Ctl::npend[1]).  Every
// registration and list word is idle again when the four kernels end.
constexpr uint32_t DX_ABS = 0x80000000u;   // seg_cnt: the free slot is in an earlier slot's component
constexpr uint32_t DX_CNT = 0x7FFFFFFFu;
constexpr uint32_t DX_ROOT = 0x80000000u;  // warp-pass list entry: a component's leader
#ifndef FM_DX_LCH
#define FM_DX_LCH 4
#endif
#ifndef FM_DX_LTRIPS
#define FM_DX_LTRIPS 4
#endif
constexpr int DX_LCH = FM_DX_LCH;          // evictions of a walk on the thread path
constexpr int DX_LCMP = 6;                 // possible updates of a walk on the thread path
constexpr int DX_LTRIPS = FM_DX_LTRIPS;    // 16-slot metadata reads of a walk on the thread path
constexpr int DX_GATHER = 64;              // ops of a component the warp pass runs itself
constexpr int DX_THREADS = 256;            // threads of an exec block

// Programmatic dependent launch between the direct kernels (compile-time
// setting FM_DX_PDL, default on): each kernel lets the next one launch as
// soon as all its blocks have started, and the next one waits for it to
// finish (and its writes to be visible) before reading anything it wrote, so
// launch latency overlaps execution instead of adding to it.
#ifndef FM_DX_PDL
#define FM_DX_PDL 1
#endif
__device__ __forceinline__ void dx_wait_prev() {
#if FM_DX_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
__device__ __forceinline__ void dx_let_next() {
#if FM_DX_PDL
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// First free slot at or after unwrapped position a, looking at no more than
// `budget` slots (less the slots looked at); NONE64 when none lies within it.
__device__ __forceinline__ uint64_t dx_next_free(const TableView& t, uint64_t a, uint64_t& budget) {
    const uint64_t mask = t.mask;
    if (mask >= 7) {
        for (uint64_t wb = a & ~7ull; budget > 0; wb += 8) {
            const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
            const uint4 x = fp[0], y = fp[1];
            const uint32_t f8[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
            uint64_t hit = NONE64;
#pragma unroll
            for (int l = 0; l < 8; l++) {
                if (hit != NONE64 || wb + l < a || budget == 0) continue;
                --budget;
                if (is_free(f8[l])) hit = wb + l;
            }
            if (hit != NONE64) return hit;
        }
        return NONE64;
    }
    for (; budget > 0; ++a) {
        --budget;
        if (is_free(t.flags[a & mask])) return a;
    }
    return NONE64;
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_dx_find(TableView t, const uint8_t* __restrict__ keys, uint32_t n0_arg,
                                                    OpScratch sc, Ctl* ctl) {
    dx_let_next();
    const uint32_t n0 = cmp_n0(n0_arg, ctl);
    bool no_free = false;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n0; j += gridDim.x * blockDim.x) {
        RegKey<KB> key;
        key.load(keys + (uint64_t)j * KB, KB);
        const uint64_t h = key.hash(KB, t.hash_mode) & t.mask;
        const uint64_t F = find_free_from(t, h);
        sc.op_slot[j] = F;
        sc.op_pt[(uint64_t)j * PT_MAX] = (uint32_t)h;  // the exec pass starts from it
        uint8_t lead = 0;
        uint32_t next = IDLE;
        if (F == NONE64) {
            no_free = true;
        } else {
            lead = atomicAdd(&t.seg_cnt[F], 1u) == 0u ? 1 : 0;
            next = atomicExch(&t.seg_min[F], j);
        }
        sc.op_word[j] = next;
        sc.op_flag[j] = lead;
    }
    if (no_free) ctl->serial[0] = 1u;
}

__global__ void __launch_bounds__(RBLOCK) k_dx_flow(TableView t, uint32_t n0_arg, OpScratch sc, Ctl* ctl) {
    dx_wait_prev();
    dx_let_next();
    if (*(volatile uint32_t*)&ctl->serial[0]) return;  // every op goes to the component path
    const uint32_t n0 = cmp_n0(n0_arg, ctl);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n0; j += gridDim.x * blockDim.x) {
        if (!sc.op_flag[j]) continue;
        const uint64_t F = sc.op_slot[j];
        const uint32_t c = t.seg_cnt[F] & DX_CNT;
        if (c < 2) continue;
        uint64_t flow = c - 1, a = F + 1, budget = t.mask;  // back at F: the flow wraps the table
        for (;;) {
            const uint64_t at = dx_next_free(t, a, budget);
            if (at == NONE64) {
                ctl->serial[0] = 1u;
                break;
            }
            const uint64_t F2 = at & t.mask;
            const uint32_t w2 = t.seg_cnt[F2];
            const uint32_t c2 = w2 & DX_CNT;
            if (c2) {
                if (t.seg_min[F2] >= n0) {  // registrations come only from this call's ops
                    atomicOr(&ctl->err, ERR_SCRATCH);
                    break;
                }
                if (!(w2 & DX_ABS)) atomicOr(&t.seg_cnt[F2], DX_ABS);
            }
            flow = flow + c2 - 1;
            if (flow == 0) break;
            a = at + 1;
        }
    }
}

// The thread path's per-thread lists (shared memory, one column per thread):
// eviction slots and depths, possible-update slots and the evictions before
// each.
struct DxLaneSmem {
    uint32_t pos[DX_LCH][DX_THREADS];
    uint32_t dep[DX_LCH][DX_THREADS];
    uint32_t cpos[DX_LCMP][DX_THREADS];
    uint32_t cst[DX_LCMP][DX_THREADS];
};

// A record (key and value) held in registers for a move.
template <int KB, int VB>
struct DxRec {
    RegKey<KB> k;
    RegVal<VB> v;
    __device__ __forceinline__ void load_in(const uint8_t* kp, const uint8_t* vp) {
        k.load(kp, KB);
        v.load_ro(vp);
    }
    __device__ __forceinline__ void load_slot(const TableView& t, uint64_t s, bool value_only) {
        if (!value_only) k.load_table(t.keys + s * KB, KB);
        v.load(t.vals + s * VB, VB);
    }
    __device__ __forceinline__ void store_slot(const TableView& t, uint64_t s, bool value_only) const {
        if (!value_only) k.store(t.keys + s * KB, KB);
        v.store(t.vals + s * VB, VB);
    }
};

// One op alone at its free slot F (nothing of another op lies in [home, F]),
// on one thread.  Every slot in [home, F) is occupied (F is the first free
// slot at or after home), so the walk is in closed form: with H the home of
// the carried entry (the op's home first), a resident whose home r exceeds H
// is evicted (the carried entry takes its slot at depth position - H, and the
// resident is carried on: H = r), one with r == H is a possible update, and F
// takes the last carried entry.  The possible updates are compared first on
// the keys' first 8 bytes, all in one round trip, and in full only where
// those agree (the first equal key in walk order ends the walk in place);
// then the records move highest first, DX_MB per round trip: move m writes
// P_m (the m-th eviction slot; the end slot for the last) from P_(m-1) (the
// new entry for m = 0), and a batch loads all its sources before it stores,
// which keeps each slot's read before its write.  Returns 1 (claimed F), 0
// (updated in place) or -1 with nothing written when the walk needs more than
// DX_LTRIPS metadata reads, DX_LCH evictions or DX_LCMP possible updates, or
// when the metadata does not show F as the first free slot.  Needs capacity
// >= 8 and below 2^28 slots.
// The first metadata window of a walk from home h (two aligned 8-slot
// windows), loaded while the caller's other loads are in flight.
struct DxWin {
    uint4 a, b, c, d;
    __device__ __forceinline__ void load(const TableView& t, uint64_t w) {
        const uint4* p0 = reinterpret_cast<const uint4*>(t.flags + (w & t.mask));
        const uint4* p1 = reinterpret_cast<const uint4*>(t.flags + ((w + 8) & t.mask));
        a = p0[0], b = p0[1], c = p1[0], d = p1[1];
    }
};

template <int KB, int VB>
__device__ __noinline__ int dx_lane(const TableView& t, const RegKey<KB>& key, uint64_t h, uint64_t F,
                                    const DxWin& w0, const uint8_t* kin, const uint8_t* vin, DxLaneSmem& sl,
                                    ExecAcc& acc) {
    constexpr int MB = (KB + VB) <= 16 ? 8 : ((KB + VB) <= 64 ? 4 : 2);  // moves per round trip
    const uint64_t mask = t.mask;
    const uint32_t me = threadIdx.x;
    const uint64_t e = h + ((F - h) & mask);  // F, unwrapped
    const uint64_t wb = h & ~7ull;
    if (e - wb >= 16ull * DX_LTRIPS) return -1;
    uint32_t k = 0, nc = 0;
    long long H = (long long)h;
    bool end_tomb = false;
    for (uint64_t w = wb; w <= e; w += 16) {
        DxWin win = w0;
        if (w != wb) win.load(t, w);
        const uint4 fa = win.a, fb = win.b, fc = win.c, fd = win.d;
        const uint32_t f16[16] = {fa.x, fa.y, fa.z, fa.w, fb.x, fb.y, fb.z, fb.w,
                                  fc.x, fc.y, fc.z, fc.w, fd.x, fd.y, fd.z, fd.w};
#pragma unroll
        for (int l = 0; l < 16; l++) {
            const uint64_t pos = w + l;
            if (pos < h || pos > e) continue;
            if (pos == e) {
                if (!is_free(f16[l])) return -1;  // not the free slot the find pass saw
                end_tomb = st_of(f16[l]) == ST_TOMB;
                continue;
            }
            if (st_of(f16[l]) != ST_OCC) return -1;  // a free slot before F: likewise
            const long long r = (long long)pos - (long long)dist_of(f16[l]);
            if (r > H) {
                if (k == (uint32_t)DX_LCH) return -1;
                sl.pos[k][me] = (uint32_t)(pos & mask);
                sl.dep[k][me] = (uint32_t)((long long)pos - H);
                ++k;
                H = r;
            } else if (r == H) {
                if (nc == (uint32_t)DX_LCMP) return -1;
                sl.cpos[nc][me] = (uint32_t)(pos & mask);
                sl.cst[nc][me] = k;
                ++nc;
            }
        }
    }
    // possible updates: 8-byte prefixes of the resident and the carried keys
    // in one round trip, full keys only where the prefixes agree
    int kind = 1;
    uint64_t end_slot = e & mask;
    uint32_t kk = k;
    if (nc) {
        uint2 rp[DX_LCMP], cp[DX_LCMP];
        const uint2 kp = make_uint2(key.w[0], KB >= 8 ? key.w[1] : 0u);
#pragma unroll
        for (int c = 0; c < DX_LCMP; c++) {
            if (c < (int)nc) {
                rp[c] = *reinterpret_cast<const uint2*>(t.keys + (uint64_t)sl.cpos[c][me] * KB);
                const uint32_t st = sl.cst[c][me];
                cp[c] = st ? *reinterpret_cast<const uint2*>(t.keys + (uint64_t)sl.pos[st - 1][me] * KB) : kp;
            }
        }
        for (int c = 0; c < (int)nc; c++) {
            bool agree = false;
#pragma unroll
            for (int q = 0; q < DX_LCMP; q++)
                if (q == c) agree = rp[q].x == cp[q].x && rp[q].y == cp[q].y;
            if (!agree) continue;
            const uint32_t st = sl.cst[c][me];
            const uint64_t cs = sl.cpos[c][me];
            RegKey<KB> ck;
            if (st) ck.load_table(t.keys + (uint64_t)sl.pos[st - 1][me] * KB, KB);
            else ck = key;
            if (ck.eq(t.keys + cs * KB, KB)) {
                kind = 2, end_slot = cs, kk = st;
                break;
            }
        }
    }
    // moves, highest first, MB per round trip
    for (int top = (int)kk; top >= 0; top -= MB) {
        DxRec<KB, VB> rec[MB];
#pragma unroll
        for (int b = 0; b < MB; b++) {
            const int m = top - b;
            if (m < 0) continue;
            const bool vo = kind == 2 && m == (int)kk;  // the update writes the value only
            if (m == 0) rec[b].load_in(kin, vin);
            else rec[b].load_slot(t, sl.pos[m - 1][me], vo);
        }
#pragma unroll
        for (int b = 0; b < MB; b++) {
            const int m = top - b;
            if (m < 0) continue;
            const bool vo = kind == 2 && m == (int)kk;
            const uint64_t d = m < (int)kk ? (uint64_t)sl.pos[m][me] : end_slot;
            rec[b].store_slot(t, d, vo);
        }
    }
    uint32_t md = 0;
    for (uint32_t i = 0; i < kk; i++) {
        const uint32_t d = sl.dep[i][me];
        t.flags[sl.pos[i][me]] = mk_flag(ST_OCC, d);
        md = max(md, d);
    }
    if (kind == 1) {
        const uint64_t d = (uint64_t)((long long)e - H);
        t.flags[end_slot] = mk_flag(ST_OCC, d);
        md = max(md, (uint32_t)d);
        acc.tomb = acc.tomb || end_tomb;
    }
    acc.maxd = max(acc.maxd, md);
    return kind == 1 ? 1 : 0;
}

// The exec pass: one thread per op (uniform trip count per warp, for the
// warp-aggregated appends).
template <int KB, int VB>
__global__ void __launch_bounds__(DX_THREADS, 2) k_dx_exec(TableView t, const uint8_t* __restrict__ keys,
                                                           const uint8_t* __restrict__ vals, uint32_t n0_arg,
                                                           OpScratch sc, Ctl* ctl) {
    __shared__ DxLaneSmem s_lane;
    __shared__ uint32_t s_tmp[DX_THREADS / 32];
    dx_wait_prev();
    dx_let_next();
    const uint32_t n0 = cmp_n0(n0_arg, ctl);
    // with the count in the control block (a device-driven call) the ops of a
    // call that found no free slot go to pend[1] for the component path
    // launched after this pass; otherwise the host reruns every op
    const bool to_pend = n0_arg == CMP_N0_CTL;
    const bool serial = *(volatile uint32_t*)&ctl->serial[0] != 0;
    const bool lanes_ok = t.mask >= 7 && t.mask < (uint64_t)DIST_MASK;
    ExecAcc a;
    // ops taken 32 at a time per warp from a counter (Ctl::exec_next, zero at
    // the start of the call): the grid is the resident blocks, and a warp that
    // drew long walks does not hold up a static share of the ops
    for (;;) {
        uint32_t j0 = 0;
        if ((threadIdx.x & 31u) == 0) j0 = atomicAdd(&ctl->exec_next, 32u);
        j0 = __shfl_sync(0xFFFFFFFFu, j0, 0);
        if (j0 >= n0) break;
        const uint32_t j = j0 + (threadIdx.x & 31u);
        uint32_t item = 0;
        bool defer = false;
        if (j < n0 && serial && to_pend) sc.pend[1][atomicAdd(&ctl->npend[1], 1u)] = j;
        if (j < n0) {
            // independent loads together: free slot, home, key; then the
            // registration count with the first metadata window
            const uint64_t F = sc.op_slot[j];
            const uint64_t h = sc.op_pt[(uint64_t)j * PT_MAX];
            RegKey<KB> key;
            key.load(keys + (uint64_t)j * KB, KB);
            if (F != NONE64) {
                DxWin w0;
                if (lanes_ok && !serial) w0.load(t, h & ~7ull);
                const uint32_t w = t.seg_cnt[F];
                if (serial) {  // registrations back to idle; the component path runs every op
                    t.seg_min[F] = IDLE;
                    t.seg_cnt[F] = 0;
                    sc.op_word[j] = IDLE;
                } else if (w == 1u) {  // alone at F, and F in no other op's component
                    int c = -1;
                    if (lanes_ok)
                        c = dx_lane<KB, VB>(t, key, h, F, w0, keys + (uint64_t)j * KB, vals + (uint64_t)j * VB,
                                            s_lane, a);
                    if (c < 0) defer = true, item = j;
                    else a.claimed += (uint32_t)c;
                    t.seg_min[F] = IDLE;
                    t.seg_cnt[F] = 0;
                    sc.op_word[j] = IDLE;
                } else if (sc.op_flag[j] && !(w & DX_ABS)) {
                    defer = true, item = j | DX_ROOT;
                }
            }
        }
        append(sc.long_list, &ctl->nlong[0], item, defer);
    }
    block_add_count(ctl, a.claimed, s_tmp);
    publish_rare(ctl, a.maxd, a.tomb, a.limit);
}

// One op on a warp: the tile walk (the scalar walk on small tables).
template <int KB, int VB, int T = 32>
__device__ __forceinline__ void dx_run_tile(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t j,
                                            const Tile<T>& tl, P4Chain<T>& s, ExecAcc& a) {
    RegKey<KB> key;
    key.load(keys + (uint64_t)j * KB, KB);
    if (t.mask >= 4 * T - 1) {
        if (exec_tile<KB, VB, T, P4Chain<T>>(t, key, vals, j, tl, s, a) == 5) a.limit = true;
    } else if (tl.lane == 0) {
        a.claimed += exec_insert_key<KB, VB>(t, key, vals + (uint64_t)j * VB, a);
    }
    tl.sync();  // the next op on this warp reads these writes
}

// The ops of the component led by op j, gathered by lane 0 from the lists of
// j's free slot F and of every free slot the flow from F reaches (the flow
// pass's walk again: nothing in the component has run), their registrations
// and list words set idle on the way; then sorted into index order by the
// warp.  Returns their count, or 0 when there are more than DX_GATHER (their
// ops then go to pend[1] for the component path).
template <int T = 32>
__device__ __noinline__ uint32_t dx_gather(const TableView& t, uint32_t j, uint32_t n0, const OpScratch& sc,
                                           Ctl* ctl, uint32_t* s_ops, const Tile<T>& tl) {
    uint32_t g = 0;
    if (tl.lane == 0) {
        const uint64_t mask = t.mask;
        uint64_t F = sc.op_slot[j];
        uint64_t a = F, budget = mask;
        uint64_t flow = 0;
        for (;;) {
            const uint32_t c = t.seg_cnt[F] & DX_CNT;
            uint32_t x = t.seg_min[F];
            if (c) {
                t.seg_min[F] = IDLE;
                t.seg_cnt[F] = 0;
            }
            for (uint32_t q = 0; q < c && x != IDLE; q++) {
                if (x >= n0) {
                    atomicOr(&ctl->err, ERR_SCRATCH);
                    break;
                }
                const uint32_t nx = sc.op_word[x];
                sc.op_word[x] = IDLE;
                if (g == (uint32_t)DX_GATHER) {  // too many for this warp: all of them to the component path
                    const uint32_t at = atomicAdd(&ctl->npend[1], (uint32_t)DX_GATHER);
                    for (int i = 0; i < DX_GATHER; i++) sc.pend[1][at + i] = s_ops[i];
                }
                if (g < (uint32_t)DX_GATHER) s_ops[g] = x;
                else sc.pend[1][atomicAdd(&ctl->npend[1], 1u)] = x;
                ++g;
                x = nx;
            }
            flow = flow + c - 1;
            if (flow == 0) break;
            const uint64_t at = dx_next_free(t, a + 1, budget);
            if (at == NONE64) break;  // the flow pass found no wrap: not reached
            a = at;
            F = at & mask;
        }
    }
    g = tl.shfl(g, 0);
    tl.sync();
    if (g > (uint32_t)DX_GATHER) return 0;
    // index order: each lane ranks DX_GATHER / T entries
    constexpr int PER = DX_GATHER / T;
    const uint32_t lane = tl.lane;
    uint32_t v[PER], r[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) {
        v[u] = lane + T * u < g ? s_ops[lane + T * u] : 0u;
        r[u] = 0;
    }
    for (uint32_t q = 0; q < g; q++) {
        const uint32_t x = s_ops[q];
#pragma unroll
        for (int u = 0; u < PER; u++) r[u] += x < v[u] ? 1u : 0u;
    }
    tl.sync();
#pragma unroll
    for (int u = 0; u < PER; u++)
        if (lane + T * u < g) s_ops[r[u]] = v[u];
    tl.sync();
    return g;
}

// Ops registered at the free slots the flow from unwrapped position a still
// reaches, carrying `flow` ops past it (the flow pass's walk, reads only).
__device__ __forceinline__ uint32_t dx_flow_rest(const TableView& t, uint64_t a, uint64_t budget, uint64_t flow) {
    uint32_t rest = 0;
    while (flow > 0) {
        const uint64_t at = dx_next_free(t, a + 1, budget);
        if (at == NONE64) break;
        const uint32_t c = t.seg_cnt[at & t.mask] & DX_CNT;
        rest += c;
        flow = flow + c - 1;
        a = at;
    }
    return rest;
}

// dx_gather for the persistent batch: a component of more than DX_GATHER ops
// is gathered into a range of pend[1] reserved for it (Ctl::big_ops) and
// listed in pend[0] (offset, count; Ctl::nbig) for the block pass (QP_IBIG)
// instead of leaving its ops to a single block at the op's end.  Returns the
// count gathered into s_ops in index order, or 0 for a listed component.
__device__ __noinline__ uint32_t dx_gather_q(const TableView& t, uint32_t j, uint32_t n0, const OpScratch& sc,
                                             Ctl* ctl, uint32_t* s_ops, const Tile<32>& tl) {
    uint32_t g = 0;
    if (tl.lane == 0) {
        const uint64_t mask = t.mask;
        uint64_t F = sc.op_slot[j];
        uint64_t a = F, budget = mask;
        uint64_t flow = 0;
        uint32_t* big = nullptr;  // the reserved range, once the component outgrows s_ops
        uint32_t room = 0;
        for (;;) {
            const uint32_t c = t.seg_cnt[F] & DX_CNT;
            uint32_t x = t.seg_min[F];
            for (uint32_t q = 0; q < c && x != IDLE; q++) {
                if (x >= n0) {
                    atomicOr(&ctl->err, ERR_SCRATCH);
                    break;
                }
                if (g == (uint32_t)DX_GATHER && !big) {
                    // the rest of this slot's list and of the slots the flow
                    // reaches (registrations still in place)
                    room = g + (c - q) + dx_flow_rest(t, a, budget, flow + c - 1);
                    big = sc.pend[1] + atomicAdd(&ctl->big_ops, room);
                    for (uint32_t i = 0; i < g; i++) big[i] = s_ops[i];
                }
                const uint32_t nx = sc.op_word[x];
                sc.op_word[x] = IDLE;
                if (!big) s_ops[g] = x;
                else if (g < room) big[g] = x;
                else atomicOr(&ctl->err, ERR_SCRATCH);  // more ops than registered: never expected
                ++g;
                x = nx;
            }
            if (c) {
                t.seg_min[F] = IDLE;
                t.seg_cnt[F] = 0;
            }
            flow = flow + c - 1;
            if (flow == 0) break;
            const uint64_t at = dx_next_free(t, a + 1, budget);
            if (at == NONE64) break;  // the flow pass found no wrap: not reached
            a = at;
            F = at & mask;
        }
        if (big) {
            const uint32_t k = atomicAdd(&ctl->nbig, 1u);
            sc.pend[0][2 * k] = (uint32_t)(big - sc.pend[1]);
            sc.pend[0][2 * k + 1] = min(g, room);
            g = 0;
        }
    }
    g = tl.shfl(g, 0);
    tl.sync();
    if (g == 0) return 0;
    constexpr int PER = DX_GATHER / 32;
    const uint32_t lane = tl.lane;
    uint32_t v[PER], r[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) {
        v[u] = lane + 32 * u < g ? s_ops[lane + 32 * u] : 0u;
        r[u] = 0;
    }
    for (uint32_t q = 0; q < g; q++) {
        const uint32_t x = s_ops[q];
#pragma unroll
        for (int u = 0; u < PER; u++) r[u] += x < v[u] ? 1u : 0u;
    }
    tl.sync();
#pragma unroll
    for (int u = 0; u < PER; u++)
        if (lane + 32 * u < g) s_ops[r[u]] = v[u];
    tl.sync();
    return g;
}

// The warp pass: a tile of T lanes per entry of the list the exec pass built
// (T: 32, 16 or 8, chosen per record shape and load by the autotuner; a
// narrower tile reads fewer slots per round trip but runs more entries at
// once).
template <int KB, int VB, int T>
__global__ void __launch_bounds__(RBLOCK, FM_P4_MIN_BLOCKS) k_dx_warp(TableView t, const uint8_t* __restrict__ keys,
                                                                      const uint8_t* __restrict__ vals, uint32_t n0_arg,
                                                                      OpScratch sc, Ctl* ctl) {
    constexpr int NT = RBLOCK / T;
    __shared__ P4Chain<T> s_chain[NT];
    __shared__ uint32_t s_ops[NT][DX_GATHER];
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    dx_wait_prev();
    const uint32_t n = *(volatile const uint32_t*)&ctl->nlong[0];
    if (n == 0) return;  // block-uniform
    const uint32_t n0 = cmp_n0(n0_arg, ctl);
    const Tile<T> tl;
    const uint32_t ti = threadIdx.x / T;
    ExecAcc a;
    // entries taken a warp's worth at a time from a counter (Ctl::nlong[1],
    // zero at the start of the call): long entries do not hold up a static
    // share of the list; all tiles of a warp loop together
    constexpr uint32_t TPW = 32 / T;
    for (;;) {
        uint32_t i0 = 0;
        if ((threadIdx.x & 31u) == 0) i0 = atomicAdd(&ctl->nlong[1], TPW);
        i0 = __shfl_sync(0xFFFFFFFFu, i0, 0);
        if (i0 >= n) break;
        const uint32_t i = i0 + (threadIdx.x & 31u) / T;
        uint32_t g = 0;  // a lone op, or a component's ops in index order
        if (i < n) {
            const uint32_t item = sc.long_list[i];
            if (item & DX_ROOT) {
                g = dx_gather<T>(t, item & ~DX_ROOT, n0, sc, ctl, s_ops[ti], tl);
            } else {
                if (tl.lane == 0) s_ops[ti][0] = item;
                g = 1;
            }
        }
        tl.sync();
        for (uint32_t q = 0; q < g; q++) dx_run_tile<KB, VB, T>(t, keys, vals, s_ops[ti][q], tl, s_chain[ti], a);
        __syncwarp();
    }
    block_add_count(ctl, a.claimed, s_tmp);
    publish_rare(ctl, a.maxd, a.tomb, a.limit);
}

// ---- persistent batch: one launch drains a queue of bulk ops ---------------
//
// The host plans every op of a batch into a chain of phases (QPhase, in
// fm_internal.h), each of some number of work units, and lists the phases of
// all ops in an order where every phase follows the phase it waits for: the
// previous phase of its op, or the last phase of the previous op on its
// table.  k_queue's blocks take units from one counter in that order; a block
// that takes a unit waits (bounded) until the phase it depends on has
// finished all its units, runs the unit and counts it finished.  A unit is
// taken only by a running block and waits only for units handed out before
// it, so the waits end whether or not all blocks are resident at once.
//
// Units (all block-wide, QTHREADS threads):
//   QP_GET    up to QG_UNIT queries, QG_Q per thread probed in lockstep;
//   QP_BEGIN  the op's control block reset and, for a counted insert, the
//             TableFull precheck against the table's count at this point;
//   QP_IFIND / QP_IFLOW / QP_IEXEC  up to QI_UNIT ops of the direct insert's find,
//             flow and exec passes;
//   QP_IWARP  8 warps over the exec pass's list, strided over the phase's
//             units (lone long walks and components as tile walks);
//   QP_RFIND / QP_REXEC  up to QI_UNIT ops of the direct remove;
//   QP_END    what the direct passes left (every op when some op found no
//             free slot / EMPTY slot, or the ops of oversized groups) in index
//             order on this block, then the op's result, status and the
//             table's count.
constexpr int QTHREADS = 256;
constexpr uint32_t QG_UNIT = 2048;  // largest lookup unit (queries)
constexpr uint32_t QSPREAD = 296;   // units a phase is cut into where it can be (two blocks per SM)
template <int KB>
constexpr int QG_Q = 4;  // lookups per thread in lockstep
constexpr uint32_t QI_UNIT = 512;   // largest find / flow / exec unit (ops)
constexpr uint64_t QWAIT_NS = 20000000000ull;  // bound of one dependency wait (20 s)
constexpr uint32_t QBIG_MAX = 8192;           // largest component the block pass sorts in shared memory

__device__ __forceinline__ uint64_t q_now() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct QSmem {
    union {
        DxLaneSmem exec;
        struct {
            P4Chain<32> chain[QTHREADS / 32];
            uint32_t ops[QTHREADS / 32][DX_GATHER];
        } warp;
        struct {
            uint32_t buf[QTHREADS];
            uint32_t woff[33];
            TileChain chain;
        } serial;
        uint32_t rgrp[QTHREADS / 32][RX_GMAX];
        struct {
            uint32_t list[QBIG_MAX];
            P4Chain<32> chain;
        } big;
    };
    uint32_t tmp[QTHREADS / 32];
    uint32_t word;
};
static_assert(DX_THREADS == QTHREADS, "exec pass buffers");

// A lookup on a table of fewer than 8 slots, slot by slot.
template <int KB, int VB>
__device__ __noinline__ void q_get_small(const TableView& t, const uint8_t* qk, uint8_t* ov, uint8_t* of) {
    RegKey<KB> key;
    key.load(qk, KB);
    const uint64_t h = key.hash(KB, t.hash_mode) & t.mask;
    uint64_t hit = NONE64;
    for (uint64_t p = 0; p <= t.mask; ++p) {
        const uint64_t s = (h + p) & t.mask;
        const uint32_t f = t.flags[s];
        if (st_of(f) == ST_EMPTY || (st_of(f) == ST_OCC && p > dist_of(f))) break;
        if (st_of(f) == ST_OCC && dist_matches(f, p) && key.eq(t.keys + s * KB, KB)) {
            hit = s;
            break;
        }
    }
    if (ov) {
        RegVal<VB> v;
        if (hit != NONE64) v.load(t.vals + hit * VB, VB);
        else v.zero();
        v.store(ov, VB);
    }
    if (of) *of = hit != NONE64 ? 1 : 0;
}

template <int KB, int VB>
__device__ __noinline__ void q_get(const QOp& o, uint32_t c, uint32_t per) {
    const TableView& t = o.t;
    const uint64_t q0 = (uint64_t)c * per;
    const uint64_t q1 = min((uint64_t)o.n, q0 + per);
    if (t.mask >= 7) {
        // QG_Q queries per thread in lockstep: two resident blocks of
        // QTHREADS per SM keep QG_Q times as many probes in flight
#pragma unroll 1
        for (uint64_t q = q0 + threadIdx.x; q < q1; q += (uint64_t)QTHREADS * QG_Q<KB>)
            get_queries_lockstep<KB, VB, QG_Q<KB>>(t, o.keys, q, QTHREADS, q1, o.out_vals, o.out_found);
        return;
    }
#pragma unroll 1
    for (uint64_t q = q0 + threadIdx.x; q < q1; q += QTHREADS) {
        uint8_t* ov = o.out_vals ? o.out_vals + q * VB : nullptr;
        uint8_t* of = o.out_found ? o.out_found + q : nullptr;
        q_get_small<KB, VB>(t, o.keys + q * KB, ov, of);
    }
}

__device__ __noinline__ void q_begin(const QOp& o) {
    uint32_t* w = reinterpret_cast<uint32_t*>(o.ctl);
    for (uint32_t i = threadIdx.x; i < CTL_CALL_BYTES / 4; i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t n0 = o.n;
        int st = STATUS_OK;
        if (o.kind == 1 && o.counted && *o.len + o.n > o.t.mask + 1) {  // gpu.rs:198-206
            n0 = 0;
            st = STATUS_TABLE_FULL;
        }
        o.ctl->n0 = n0;
        *o.status = st;
        *o.result = 0;
    }
}

__device__ __forceinline__ uint32_t q_n0(const QOp& o) { return *(volatile const uint32_t*)&o.ctl->n0; }

template <int KB>
__device__ __noinline__ void q_ifind(const QOp& o, uint32_t c, uint32_t per) {
    const uint32_t n0 = q_n0(o);
    const uint32_t j = c * per + threadIdx.x;
    bool no_free = false;
    for (uint32_t k = 0; k < per / QTHREADS; k++) {
        const uint32_t jj = j + k * QTHREADS;
        if (jj >= n0) break;
        RegKey<KB> key;
        key.load(o.keys + (uint64_t)jj * KB, KB);
        const uint64_t h = key.hash(KB, o.t.hash_mode) & o.t.mask;
        const uint64_t F = find_free_from(o.t, h);
        o.sc.op_slot[jj] = F;
        o.sc.op_pt[(uint64_t)jj * PT_MAX] = (uint32_t)h;
        uint8_t lead = 0;
        uint32_t next = IDLE;
        if (F == NONE64) {
            no_free = true;
        } else {
            lead = atomicAdd(&o.t.seg_cnt[F], 1u) == 0u ? 1 : 0;
            next = atomicExch(&o.t.seg_min[F], jj);
        }
        o.sc.op_word[jj] = next;
        o.sc.op_flag[jj] = lead;
    }
    if (no_free) o.ctl->serial[0] = 1u;
}

__device__ __noinline__ void q_iflow(const QOp& o, uint32_t c, uint32_t per) {
    const uint32_t n0 = q_n0(o);
    if (*(volatile uint32_t*)&o.ctl->serial[0]) return;
    const TableView& t = o.t;
    for (uint32_t k = 0; k < per / QTHREADS; k++) {
        const uint32_t j = c * per + threadIdx.x + k * QTHREADS;
        if (j >= n0) break;
        if (!o.sc.op_flag[j]) continue;
        const uint64_t F = o.sc.op_slot[j];
        const uint32_t cnt = t.seg_cnt[F] & DX_CNT;
        if (cnt < 2) continue;
        uint64_t flow = cnt - 1, a = F + 1, budget = t.mask;
        for (;;) {
            const uint64_t at = dx_next_free(t, a, budget);
            if (at == NONE64) {
                o.ctl->serial[0] = 1u;
                break;
            }
            const uint64_t F2 = at & t.mask;
            const uint32_t w2 = t.seg_cnt[F2];
            const uint32_t c2 = w2 & DX_CNT;
            if (c2) {
                if (t.seg_min[F2] >= n0) {
                    atomicOr(&o.ctl->err, ERR_SCRATCH);
                    break;
                }
                if (!(w2 & DX_ABS)) atomicOr(&t.seg_cnt[F2], DX_ABS);
            }
            flow = flow + c2 - 1;
            if (flow == 0) break;
            a = at + 1;
        }
    }
}

template <int KB, int VB>
__device__ __noinline__ void q_iexec(const QOp& o, uint32_t c, uint32_t per, QSmem& sm) {
    const uint32_t n0 = q_n0(o);
    const TableView& t = o.t;
    const bool serial = *(volatile uint32_t*)&o.ctl->serial[0] != 0;
    const bool lanes_ok = t.mask >= 7 && t.mask < (uint64_t)DIST_MASK;
    ExecAcc a;
    for (uint32_t k = 0; k < per / QTHREADS; k++) {  // block-uniform trip count
        const uint32_t j = c * per + threadIdx.x + k * QTHREADS;
        uint32_t item = 0;
        bool defer = false;
        if (j < n0) {
            const uint64_t F = o.sc.op_slot[j];
            const uint64_t h = o.sc.op_pt[(uint64_t)j * PT_MAX];
            RegKey<KB> key;
            key.load(o.keys + (uint64_t)j * KB, KB);
            if (F != NONE64) {
                DxWin w0;
                if (lanes_ok && !serial) w0.load(t, h & ~7ull);
                const uint32_t w = t.seg_cnt[F];
                if (serial) {
                    t.seg_min[F] = IDLE;
                    t.seg_cnt[F] = 0;
                    o.sc.op_word[j] = IDLE;
                } else if (w == 1u) {
                    int r = -1;
                    if (lanes_ok)
                        r = dx_lane<KB, VB>(t, key, h, F, w0, o.keys + (uint64_t)j * KB, o.vals + (uint64_t)j * VB,
                                            sm.exec, a);
                    if (r < 0) defer = true, item = j;
                    else a.claimed += (uint32_t)r;
                    t.seg_min[F] = IDLE;
                    t.seg_cnt[F] = 0;
                    o.sc.op_word[j] = IDLE;
                } else if (o.sc.op_flag[j] && !(w & DX_ABS)) {
                    defer = true, item = j | DX_ROOT;
                }
            }
        }
        append(o.sc.long_list, &o.ctl->nlong[0], item, defer);
    }
    block_add_count(o.ctl, a.claimed, sm.tmp);
    publish_rare(o.ctl, a.maxd, a.tomb, a.limit);
}

template <int KB, int VB>
__device__ __noinline__ void q_iwarp(const QOp& o, uint32_t c, uint32_t units, QSmem& sm) {
    const uint32_t n = *(volatile const uint32_t*)&o.ctl->nlong[0];
    const uint32_t n0 = q_n0(o);
    const Tile<32> tl;
    const uint32_t wi = threadIdx.x >> 5;
    ExecAcc a;
    for (uint32_t i = c * (QTHREADS / 32) + wi; i < n; i += units * (QTHREADS / 32)) {
        const uint32_t item = o.sc.long_list[i];
        uint32_t g = 1;
        if (item & DX_ROOT) {
            g = dx_gather_q(o.t, item & ~DX_ROOT, n0, o.sc, o.ctl, sm.warp.ops[wi], tl);
        } else {
            if (tl.lane == 0) sm.warp.ops[wi][0] = item;
            tl.sync();
        }
        for (uint32_t q = 0; q < g; q++)
            dx_run_tile<KB, VB>(o.t, o.keys, o.vals, sm.warp.ops[wi][q], tl, sm.warp.chain[wi], a);
    }
    block_add_count(o.ctl, a.claimed, sm.tmp);
    publish_rare(o.ctl, a.maxd, a.tomb, a.limit);
}

// The block pass: the components the warp pass listed (dx_gather_q), taken
// one at a time; each is sorted into index order in shared memory and run by
// warp 0 op after op.  A component of more than QBIG_MAX ops is marked for the
// op's end unit instead (op_flag 3, Ctl::serial[1]).
template <int KB, int VB>
__device__ __noinline__ void q_ibig(const QOp& o, QSmem& sm) {
    const TableView& t = o.t;
    ExecAcc a;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t k = atomicAdd(&o.ctl->big_next, 1u);
            sm.word = k < *(volatile uint32_t*)&o.ctl->nbig ? k : 0xFFFFFFFFu;
        }
        __syncthreads();
        const uint32_t k = sm.word;
        if (k == 0xFFFFFFFFu) break;
        const uint32_t* src = o.sc.pend[1] + o.sc.pend[0][2 * k];
        const uint32_t g = o.sc.pend[0][2 * k + 1];
        if (g > QBIG_MAX) {
            for (uint32_t i = threadIdx.x; i < g; i += blockDim.x) o.sc.op_flag[src[i]] = 3;
            if (threadIdx.x == 0) o.ctl->serial[1] = 1u;
            __syncthreads();
            continue;
        }
        for (uint32_t i = threadIdx.x; i < g; i += blockDim.x) sm.big.list[i] = src[i];
        __syncthreads();
        block_sort_u32(sm.big.list, g);
        if (threadIdx.x < 32) {
            const Tile<32> tl;
            for (uint32_t q = 0; q < g; q++) dx_run_tile<KB, VB>(t, o.keys, o.vals, sm.big.list[q], tl, sm.big.chain, a);
        }
        __syncthreads();
    }
    block_add_count(o.ctl, a.claimed, sm.tmp);
    publish_rare(o.ctl, a.maxd, a.tomb, a.limit);
}

template <int KB>
__device__ __noinline__ void q_rfind(const QOp& o, uint32_t c, uint32_t per) {
    const uint32_t n0 = q_n0(o);
    bool no_empty = false;
    for (uint32_t k = 0; k < per / QTHREADS; k++) {
        const uint32_t j = c * per + threadIdx.x + k * QTHREADS;
        if (j >= n0) break;
        RegKey<KB> key;
        const uint64_t E = rx_first_empty(o.t, home_of<KB>(o.t, o.keys, j, key));
        o.sc.op_slot[j] = E;
        uint8_t lead = 0;
        uint32_t next = IDLE;
        if (E == NONE64) {
            no_empty = true;
        } else {
            lead = atomicAdd(&o.t.seg_cnt[E], 1u) == 0u ? 1 : 0;
            next = atomicExch(&o.t.seg_min[E], j);
        }
        o.sc.op_word[j] = next;
        o.sc.op_flag[j] = lead;
    }
    if (no_empty) o.ctl->serial[0] = 1u;
}

template <int KB>
__device__ __noinline__ void q_rexec(const QOp& o, uint32_t c, uint32_t per, QSmem& sm) {
    const uint32_t n0 = q_n0(o);
    const TableView& t = o.t;
    const bool serial = *(volatile uint32_t*)&o.ctl->serial[0] != 0;
    uint32_t removed = 0;
    for (uint32_t k = 0; k < per / QTHREADS; k++) {  // block-uniform trip count
        const uint32_t j = c * per + threadIdx.x + k * QTHREADS;
        uint64_t E = NONE64;
        uint32_t cnt = 0;
        bool lead = false;
        if (j < n0) {
            E = o.sc.op_slot[j];
            if (E != NONE64) {
                if (serial) {
                    t.seg_min[E] = IDLE;
                    t.seg_cnt[E] = 0;
                    o.sc.op_word[j] = IDLE;
                } else if (o.sc.op_flag[j]) {
                    cnt = t.seg_cnt[E];
                    if (cnt == 1) {
                        RegKey<KB> key;
                        removed += rx_probe<KB>(t, key, home_of<KB>(t, o.keys, j, key));
                        t.seg_min[E] = IDLE;
                        t.seg_cnt[E] = 0;
                        o.sc.op_word[j] = IDLE;
                    } else {
                        lead = true;
                    }
                }
            }
        }
        for (uint32_t lm = __ballot_sync(0xFFFFFFFFu, lead); lm; lm &= lm - 1) {
            const int L = __ffs(lm) - 1;
            const uint64_t EL = __shfl_sync(0xFFFFFFFFu, E, L);
            const uint32_t cL = __shfl_sync(0xFFFFFFFFu, cnt, L);
            const uint32_t r = rx_group<KB>(t, o.keys, n0, o.sc, o.ctl, EL, cL, sm.rgrp[threadIdx.x >> 5]);
            if ((threadIdx.x & 31u) == 0) removed += r;
        }
    }
    block_add_count(o.ctl, removed, sm.tmp);
}

// The leftovers in index order on this block, then the result write-back.
template <int KB, int VB>
__device__ __noinline__ void q_end(const QOp& o, QSmem& sm) {
    const uint32_t n0 = q_n0(o);
    const bool serial = *(volatile uint32_t*)&o.ctl->serial[0] != 0;
    const uint32_t left = serial ? n0 : *(volatile uint32_t*)&o.ctl->npend[1];
    const uint32_t* list = serial ? nullptr : o.sc.pend[1];
    // inserts: components the block pass left (already marked op_flag 3)
    const bool marked = o.kind == 1 && !serial && *(volatile uint32_t*)&o.ctl->serial[1] != 0;
    if (left || marked) {
        if (o.kind == 1) {
            ExecAcc a;
            serial_process<KB, VB>(o.t, o.keys, o.vals, list, left, n0, o.sc, a, sm.serial.buf, sm.serial.woff,
                                   &sm.serial.chain);
            __syncthreads();
            if (a.claimed) atomicAdd(&o.ctl->count, (unsigned long long)a.claimed);
            if (a.maxd > *(volatile uint32_t*)&o.ctl->dmax) atomicMax(&o.ctl->dmax, a.maxd);
            if (a.tomb) o.ctl->tomb_claimed = 1u;
            if (a.limit) atomicOr(&o.ctl->err, ERR_WALK_LIMIT);
        } else {
            // removes: mark, list in index order, then warp 0 runs them 32 at
            // a time (parallel probes, commits in index order)
            for (uint32_t i = threadIdx.x; i < left; i += blockDim.x) o.sc.op_flag[list ? list[i] : i] = 3;
            __syncthreads();
            uint32_t removed = 0;
            for (uint32_t base = 0; base < n0; base += blockDim.x) {
                const uint32_t j = base + threadIdx.x;
                const bool take = j < n0 && o.sc.op_flag[j] == 3;
                if (take) o.sc.op_flag[j] = 0;
                const uint32_t cnt = block_compact(j, take, sm.serial.buf, sm.serial.woff);
                if (threadIdx.x < 32)
                    for (uint32_t q = 0; q < cnt; q += 32)
                        removed += rx_chunk32<KB>(o.t, o.keys, sm.serial.buf + q, min(32u, cnt - q));
                __syncthreads();
            }
            if (threadIdx.x == 0 && removed) atomicAdd(&o.ctl->count, (unsigned long long)removed);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (*o.status == STATUS_OK) {
            const unsigned long long cnt = o.ctl->total_count();
            *o.result = cnt;
            if (o.kind == 1) *o.len += o.counted ? cnt : (unsigned long long)o.n;
            else *o.len -= cnt;
            const uint32_t err = o.ctl->err;
            if (err & (ERR_SCRATCH | ERR_NO_PROGRESS)) *o.status = STATUS_KERNEL;
            else if (err & ERR_WALK_LIMIT) *o.status = STATUS_PROBE_LIMIT;
        }
        o.ctl->npend[0] = o.ctl->npend[1] = 0;
    }
}

template <int KB, int VB>
__global__ void __launch_bounds__(QTHREADS, 2) k_queue(const QPhase* __restrict__ ph, uint64_t total,
                                                       const QOp* __restrict__ ops, uint32_t* done, QState* st,
                                                       QProf* prof) {
    __shared__ QSmem sm;
    __shared__ unsigned long long s_u;
    __shared__ uint32_t s_pe;
    uint32_t cursor = 0;  // the phase of the last unit taken: units come in increasing order
    unsigned long long t_run = 0;  // (thread 0, with prof) when the current unit started
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long u = atomicAdd(&st->next, 1ull);
            s_u = u;
            if (u < total) {
                while (ph[cursor].base + ph[cursor].units <= u) ++cursor;
                s_pe = cursor;
                const unsigned long long t_take = prof ? q_now() : 0ull;
                const int32_t d = ph[cursor].dep;
                // after one wait has run out the rest skip theirs, so a broken
                // plan ends at once (reported to the host)
                if (d >= 0 && !*(volatile uint32_t*)&st->err) {
                    const uint32_t need = ph[d].units;
                    const uint64_t t0 = q_now();
                    while (*(volatile uint32_t*)&done[d] < need) {
                        __nanosleep(200);
                        if (q_now() - t0 > QWAIT_NS) {  // reported to the host; the unit still runs
                            atomicOr(&st->err, 1u);
                            break;
                        }
                    }
                    __threadfence();
                }
                if (prof) {
                    t_run = q_now();
                    atomicMin(&prof[cursor].t0, t_run);
                    atomicAdd(&prof[cursor].wait, t_run - t_take);
                }
            }
        }
        __syncthreads();
        const unsigned long long u = s_u;
        if (u >= total) break;
        const QPhase p = ph[s_pe];
        const QOp& o = ops[p.op];
        const uint32_t c = (uint32_t)(u - p.base);
        switch (p.kind) {
            case QP_GET: q_get<KB, VB>(o, c, p.per); break;
            case QP_BEGIN: q_begin(o); break;
            case QP_IFIND: q_ifind<KB>(o, c, p.per); break;
            case QP_IFLOW: q_iflow(o, c, p.per); break;
            case QP_IEXEC: q_iexec<KB, VB>(o, c, p.per, sm); break;
            case QP_IWARP: q_iwarp<KB, VB>(o, c, p.units, sm); break;
            case QP_RFIND: q_rfind<KB>(o, c, p.per); break;
            case QP_REXEC: q_rexec<KB>(o, c, p.per, sm); break;
            case QP_IBIG: q_ibig<KB, VB>(o, sm); break;
            default: q_end<KB, VB>(o, sm); break;
        }
        __threadfence();  // this unit's writes before its count
        __syncthreads();
        if (threadIdx.x == 0) {
            if (prof) {
                const unsigned long long t_end = q_now();
                atomicMax(&prof[s_pe].t1, t_end);
                atomicAdd(&prof[s_pe].busy, t_end - t_run);
            }
            atomicAdd(&done[s_pe], 1u);
        }
    }
}

constexpr int INS_T = 32;  // lanes per insert in the single-block tail

// ---- grouped rounds (batch waves) ------------------------------------------
//
// The same phases over the inserts of a batch wave (distinct tables), one
// launch per phase for all of them: a flat item index is mapped to (op, item)
// through the prefix of the ops' pending counts, list appends and counts are
// aggregated over the lanes of a warp working on the same op, and the tail
// runs one block per op until every op is done.

__device__ __forceinline__ uint32_t grp_pending(const GroupOp* ops, uint32_t o, uint32_t r) {
    const Ctl* c = ops[o].ctl;
    return r == 0 ? *(volatile const uint32_t*)&c->n0 : *(volatile const uint32_t*)&c->npend[r & 1];
}

__device__ __forceinline__ void grp_rare(Ctl* ctl, const ExecAcc& a) {
    if (a.maxd > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, a.maxd);
    if (a.tomb && !*(volatile uint32_t*)&ctl->tomb_claimed) ctl->tomb_claimed = 1u;
    if (a.limit) atomicOr(&ctl->err, ERR_WALK_LIMIT);
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_grp_ins_p1(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r) {
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    const uint32_t total = group_prefix(nops, [&](uint32_t o) { return grp_pending(ops, o, r); }, s_pre);
    if (blockIdx.x == 0)
        for (uint32_t o = threadIdx.x; o < nops; o += blockDim.x) reset_next_round(ops[o].ctl, r);
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t i = f - s_pre[o];
        const uint32_t j = r == 0 ? i : pend_of(g.sc, r)[i];
        const uint64_t F = find_free<KB>(g.t, g.keys, j);
        register_op(g.t, j, F, g.sc.op_slot);
        if (F == NONE64) g.ctl->serial[r & 1] = 1u;
    }
}

__global__ void __launch_bounds__(RBLOCK) k_grp_ins_p2(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r) {
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    const uint32_t total = group_prefix(nops, [&](uint32_t o) { return grp_pending(ops, o, r); }, s_pre);
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t i = f - s_pre[o];
        const uint32_t j = r == 0 ? i : pend_of(g.sc, r)[i];
        const uint32_t bits = walk_op(g.t, j, g.n, g.sc.op_slot, g.sc.op_word, g.sc.op_flag);
        if (bits & 1u) g.ctl->serial[r & 1] = 1u;
        if (bits & 2u) atomicOr(&g.ctl->err, ERR_SCRATCH);
    }
}

template <int KB, int VB>
__global__ void __launch_bounds__(RBLOCK, 3) k_grp_ins_p3(const GroupOp* __restrict__ ops, uint32_t nops,
                                                          uint32_t r) {
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    const uint32_t total = group_prefix(nops, [&](uint32_t o) { return grp_pending(ops, o, r); }, s_pre);
    if (blockIdx.x == 0)
        for (uint32_t o = threadIdx.x; o < nops; o += blockDim.x)
            if (s_pre[o + 1] > s_pre[o]) atomicAdd(&ops[o].ctl->rounds, 1u);
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t i = f - s_pre[o];
        const uint32_t j = r == 0 ? i : pend_of(g.sc, r)[i];
        const bool serial = *(volatile uint32_t*)&g.ctl->serial[r & 1] != 0;
        ExecAcc a;
        const int code = finish_op<KB, VB>(g.t, g.keys, g.vals, j, serial, g.sc, a, KB != 0 && VB != 0);
        append_peer(pend_of(g.sc, r + 1), &g.ctl->npend[(r + 1) & 1], j, code == 0, o);
        if constexpr (KB != 0 && VB != 0) append_peer(g.sc.long_list, &g.ctl->nlong[r & 1], j, code == 2, o);
        add_peer(g.ctl, a.claimed, o);
        grp_rare(g.ctl, a);
    }
}

template <int KB, int VB>
__global__ void __launch_bounds__(RBLOCK, 3) k_grp_ins_p4(const GroupOp* __restrict__ ops, uint32_t nops,
                                                          uint32_t r) {
    constexpr int NW = RBLOCK / 32;
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    __shared__ TileChain s_chain[NW];
    const uint32_t total = group_prefix(
        nops, [&](uint32_t o) { return *(volatile const uint32_t*)&ops[o].ctl->nlong[r & 1]; }, s_pre);
    if (total == 0) return;  // block-uniform
    const Tile<32> tl;
    const uint32_t w = threadIdx.x >> 5;
    for (uint32_t f = blockIdx.x * NW + w; f < total; f += gridDim.x * NW) {  // warp-uniform
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t j = g.sc.long_list[f - s_pre[o]];
        RegKey<KB> key;
        key.load(g.keys + (uint64_t)j * KB, KB);
        ExecAcc a;
        if (g.t.mask >= 4 * 32 - 1) {
            if (exec_tile<KB, VB, 32>(g.t, key, g.vals, j, tl, s_chain[w], a) == 5) a.limit = true;
        } else {
            if (tl.lane == 0) a.claimed += exec_insert_key<KB, VB>(g.t, key, g.vals + (uint64_t)j * VB, a);
        }
        tl.sync();
        a.maxd = __reduce_max_sync(0xFFFFFFFFu, a.maxd);
        a.tomb = __any_sync(0xFFFFFFFFu, a.tomb);
        a.limit = __any_sync(0xFFFFFFFFu, a.limit);
        a.claimed = __reduce_add_sync(0xFFFFFFFFu, a.claimed);
        if (tl.lane == 0) {
            if (a.claimed) atomicAdd(&g.ctl->count_part[blockIdx.x % COUNT_PARTS][0], (unsigned long long)a.claimed);
            grp_rare(g.ctl, a);
        }
    }
}

template <int KB, int VB, int T>
__global__ void __launch_bounds__(TAIL_THREADS) k_grp_ins_tail(const GroupOp* __restrict__ ops, uint32_t r0) {
    const GroupOp& g = ops[blockIdx.x];
    const uint32_t n0 = *(volatile const uint32_t*)&g.ctl->n0;
    ins_tail_body<KB, VB, T>(g.t, g.keys, g.vals, n0, r0, g.n, g.sc, g.ctl, 0xFFFFFFFFu, false);
}

// Serial completion of a grouped call, one block per op: the op's pending
// ops of round r one at a time in index order (ops with none return).
template <int KB, int VB>
__global__ void __launch_bounds__(SERIAL_THREADS) k_grp_ins_serial(const GroupOp* __restrict__ ops, uint32_t r) {
    __shared__ uint32_t s_buf[SERIAL_THREADS];
    __shared__ uint32_t s_woff[33];
    __shared__ TileChain s_chain;
    __shared__ SerialOut s_out;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    const GroupOp& g = ops[blockIdx.x];
    const uint32_t n0 = *(volatile const uint32_t*)&g.ctl->n0;
    const uint32_t n = grp_pending(ops, blockIdx.x, r);
    if (n == 0) return;  // block-uniform
    ExecAcc a;
    serial_process<KB, VB>(g.t, g.keys, g.vals, r == 0 ? nullptr : pend_of(g.sc, r), n, n0, g.sc, a, s_buf, s_woff,
                           &s_chain, (KB && VB) ? reinterpret_cast<SerialChain*>(s_dyn) : nullptr, &s_out);
    __syncthreads();
    Ctl* ctl = g.ctl;
    if (a.claimed) atomicAdd(&ctl->count, (unsigned long long)a.claimed);
    if (a.maxd > *(volatile uint32_t*)&ctl->dmax) atomicMax(&ctl->dmax, a.maxd);
    if (a.tomb) ctl->tomb_claimed = 1u;
    if (a.limit) atomicOr(&ctl->err, ERR_WALK_LIMIT);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->npend[r & 1] = 0;
        ctl->npend[(r + 1) & 1] = 0;
    }
}

// Phases of a grouped insert call: GRP_BEGIN (control reset and precheck),
// GRP_ROUNDS grid rounds r0 .. r0+nrounds-1, GRP_END (block-per-op tail to
// completion from round r0, then the result write-back).
template <int KB, int VB>
void grp_ins_shape(const GroupOp* ops, uint32_t nops, uint64_t sum_n, int phase, uint32_t r0, uint32_t nrounds,
                   cudaStream_t s) {
    const unsigned g = grid_for(sum_n, 8);
    if (phase == GRP_BEGIN) {
        k_grp_setup<<<nops, 256, 0, s>>>(ops, 1);
        count_launches(1);
        return;
    }
    if (phase == GRP_SERIAL) {
        KtScope kt(KC_INS_SERIAL, s);
        const size_t smem = serial_smem(k_grp_ins_serial<KB, VB>, KB && VB);
        k_grp_ins_serial<KB, VB><<<nops, SERIAL_THREADS, smem, s>>>(ops, r0);
        count_launches(1);
        return;
    }
    if (phase == GRP_END) {
        {
            KtScope kt(KC_INS_TAIL, s);
            k_grp_ins_tail<KB, VB, (KB && VB) ? INS_T : 1><<<nops, TAIL_THREADS, 0, s>>>(ops, r0);
        }
        k_grp_finish<<<(nops + 255) / 256, 256, 0, s>>>(ops, nops, 1);
        count_launches(2);
        return;
    }
    for (uint32_t r = r0; r < r0 + nrounds; r++) {
        {
            KtScope kt(KC_INS_FIND, s);
            k_grp_ins_p1<KB><<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
        {
            KtScope kt(KC_INS_WALK, s);
            k_grp_ins_p2<<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
        {
            KtScope kt(KC_INS_EXEC, s);
            k_grp_ins_p3<KB, VB><<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
        if constexpr (KB != 0 && VB != 0) {
            KtScope kt(KC_INS_LONG, s);
            k_grp_ins_p4<KB, VB><<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
    }
    count_launches(nrounds * ((KB != 0 && VB != 0) ? 4 : 3));
}

// Pending count of round r of every op.
__global__ void k_grp_pending_each(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r, uint32_t* out) {
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < nops; o += gridDim.x * blockDim.x)
        out[o] = grp_pending(ops, o, r);
}

// Largest pending count of round r over the ops (one thread).
__global__ void k_grp_pending(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r, uint32_t* out) {
    uint32_t m = 0;
    for (uint32_t o = 0; o < nops; o++) m = max(m, grp_pending(ops, o, r));
    *out = m;
}

template <int KB, int VB>
void rounds_shape(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t n0, uint32_t r0,
                  uint32_t nrounds, uint32_t grid_ops, uint32_t nops, const OpScratch& sc, Ctl* ctl,
                  cudaStream_t s) {
    // one op per thread: far more ops in flight than one per tile, which is
    // what chains of dependent random reads need
    const unsigned g = grid_for(grid_ops, 8);
    // the long-walk pass: a warp per walk that a pending op may defer, up to
    // the blocks that fit on the GPU at once
    const unsigned g4 = grid_for((uint64_t)grid_ops * 32, FM_P4_MIN_BLOCKS);
    for (uint32_t r = r0; r < r0 + nrounds; r++) {
        {
            KtScope kt(KC_INS_FIND, s);
            k_ins_p1<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, r, sc, ctl);
        }
        {
            KtScope kt(KC_INS_WALK, s);
            k_ins_p2<<<g, RBLOCK, 0, s>>>(t, n0, r, nops, sc, ctl);
        }
        {
            KtScope kt(KC_INS_EXEC, s);
            k_ins_p3<KB, VB><<<g, RBLOCK, 0, s>>>(t, keys, vals, n0, r, sc, ctl);
        }
        if constexpr (KB != 0 && VB != 0) {
            KtScope kt(KC_INS_LONG, s);
            k_ins_p4<KB, VB, p4_lanes()><<<g4, RBLOCK, 0, s>>>(t, keys, vals, r, sc, ctl);
        }
    }
    count_launches((KB != 0 && VB != 0 ? 4 : 3) * nrounds);
}

template <int KB, int VB>
void tail_shape(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t n0, uint32_t r,
                uint32_t nops, const OpScratch& sc, Ctl* ctl, bool handoff, cudaStream_t s) {
    KtScope kt(KC_INS_TAIL, s);
    k_ins_tail<KB, VB, (KB && VB) ? INS_T : 1><<<1, TAIL_THREADS, 0, s>>>(t, keys, vals, n0, r, nops, sc, ctl,
                                                                          handoff);
    count_launches(1);
}

template <int KB, int VB>
void serial_shape(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t n0, uint32_t r,
                  const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    KtScope kt(KC_INS_SERIAL, s);
    const size_t smem = serial_smem(k_ins_serial<KB, VB>, KB && VB);
    k_ins_serial<KB, VB><<<1, SERIAL_THREADS, smem, s>>>(t, keys, vals, n0, r, sc, ctl);
    count_launches(1);
}

// The component path (k_cmp_* then k_ins_comp): npend bounds round r's
// pending count (sizes the per-op grids) and, with n0 = CMP_N0_CTL, the
// call's op count too.
template <int KB, int VB>
void comp_shape(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t n0, uint32_t r,
                uint32_t npend, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    KtScope kt(KC_INS_SERIAL, s);
    const size_t smem = serial_smem(k_ins_comp<KB, VB>, KB && VB);
    static int per_sm = 0;  // resident exec blocks per SM, per instantiation
    if (per_sm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_ins_comp<KB, VB>, CMP_EXEC_THREADS, smem) !=
                cudaSuccess ||
            b < 1)
            b = 1;
        per_sm = b;
    }
    const uint32_t nblk = (uint32_t)(num_sms() * per_sm);
    // start slots are kept as 32-bit words
    const bool force = t.mask >= 0xFFFFFFF0ull;
    const unsigned g = grid_for(npend, 8);
    const unsigned nch = (unsigned)cmp_chunks(t.mask);
    const uint32_t n0_max = n0 != CMP_N0_CTL ? n0 : npend;
    const unsigned nb = (unsigned)(((uint64_t)n0_max + CMP_OPS_PER_BLOCK - 1) / CMP_OPS_PER_BLOCK);
    cudaMemsetAsync(sc.comp, 0, sizeof(CmpHdr), s);
    k_cmp_find<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, r, sc, ctl, force ? 1u : 0u);
    unsigned launches = 1;
    if (!force) {
        k_cmp_fn<<<nch, CMP_THREADS, 0, s>>>(t, sc.comp);
        k_cmp_carry<<<1, 1024, 0, s>>>(sc.comp, t.mask);
        k_cmp_starts<<<nch, CMP_THREADS, 0, s>>>(t, sc.comp);
        k_cmp_prev<<<1, 1024, 0, s>>>(sc.comp, t.mask);
        launches += 4;
    }
    k_cmp_own<<<g, RBLOCK, 0, s>>>(t, n0, r, sc, ctl, nblk);
    k_cmp_count<<<nb, CMP_THREADS, 0, s>>>(sc, n0, ctl);
    k_cmp_offsets<<<1, 1024, 0, s>>>(sc, nb);
    k_cmp_list<<<nb, CMP_THREADS, 0, s>>>(sc, n0, ctl);
    k_ins_comp<KB, VB><<<nblk, CMP_EXEC_THREADS, smem, s>>>(t, keys, vals, r, sc, ctl);
    k_cmp_clean<<<g, RBLOCK, 0, s>>>(t, sc);
    count_launches(launches + 6);
}

// A launch that may start while the stream's previous kernel still runs
// (programmatic dependent launch; the kernel waits for it in dx_wait_prev),
// or a plain launch.
template <class... P, class... A>
void launch_dependent(void (*k)(P...), unsigned grid, unsigned block, cudaStream_t s, bool pdl, A&&... args) {
    if (!pdl) {
        k<<<grid, block, 0, s>>>(std::forward<A>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// The direct insert of a call (compile-time shapes): find, flow, exec, warp.
template <int KB, int VB>
constexpr Shape sh_of() {
    return (KB == 8 && VB == 8) ? SHAPE_8_8
         : (KB == 32 && VB == 128) ? SHAPE_32_128
         : (KB == 32 && VB == 64) ? SHAPE_32_64
         : (KB == 32 && VB == 32) ? SHAPE_32_32
         : (KB == 8 && VB == 32) ? SHAPE_8_32 : SHAPE_GENERIC;
}

template <int KB, int VB>
void direct_shape(const TableView& t, const uint8_t* keys, const uint8_t* vals, uint32_t n0, uint32_t nmax,
                  const OpScratch& sc, Ctl* ctl, float load, bool pdl_ok, cudaStream_t s) {
    if constexpr (KB == 0 || VB == 0) {
        return;
    } else {
        const unsigned g = grid_for(nmax, 8);
        // with per-kernel timing on, events sit between the kernels, so they
        // run as plain launches
        const bool pdl = pdl_ok && FM_DX_PDL && !kt_active();
        {
            KtScope kt(KC_INS_FIND, s);
            k_dx_find<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, sc, ctl);
        }
        {
            KtScope kt(KC_INS_WALK, s);
            launch_dependent(k_dx_flow, g, RBLOCK, s, pdl, t, n0, sc, ctl);
        }
        {
            KtScope kt(KC_INS_EXEC, s);
            const unsigned ge = grid_for(nmax, 2);  // the resident blocks at most (two per SM)
            launch_dependent(k_dx_exec<KB, VB>, ge, DX_THREADS, s, pdl, t, keys, vals, n0, sc, ctl);
        }
        {
            KtScope kt(KC_INS_LONG, s);
            const int tw = tuned_ins_cfg(sh_of<KB, VB>(), (double)load).tile;
            const unsigned gwt = grid_for((uint64_t)nmax * tw, FM_P4_MIN_BLOCKS);
            if (tw == 8) launch_dependent(k_dx_warp<KB, VB, 8>, gwt, RBLOCK, s, pdl, t, keys, vals, n0, sc, ctl);
            else if (tw == 16) launch_dependent(k_dx_warp<KB, VB, 16>, gwt, RBLOCK, s, pdl, t, keys, vals, n0, sc, ctl);
            else launch_dependent(k_dx_warp<KB, VB, 32>, gwt, RBLOCK, s, pdl, t, keys, vals, n0, sc, ctl);
        }
        count_launches(4);
    }
}

}  // namespace

#define FM_SHAPE_SWITCH(sh, CALL)                 \
    switch (sh) {                                 \
        case SHAPE_8_8: CALL(8, 8); break;        \
        case SHAPE_32_128: CALL(32, 128); break;  \
        case SHAPE_32_64: CALL(32, 64); break;    \
        case SHAPE_32_32: CALL(32, 32); break;    \
        case SHAPE_8_32: CALL(8, 32); break;      \
        default: CALL(0, 0); break;               \
    }

cudaError_t launch_ins_rounds(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                              uint32_t r0, uint32_t nrounds, uint32_t grid_ops, const OpScratch& sc, Ctl* ctl,
                              cudaStream_t s) {
#define FM_CALL(K, V) rounds_shape<K, V>(t, keys, vals, n0, r0, nrounds, grid_ops, n0, sc, ctl, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

cudaError_t launch_ins_direct(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                              const OpScratch& sc, Ctl* ctl, double load, cudaStream_t s) {
    if (sh == SHAPE_GENERIC || !sc.comp) return cudaErrorInvalidValue;
#define FM_CALL(K, V) direct_shape<K, V>(t, keys, vals, n0, n0, sc, ctl, (float)load, true, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

cudaError_t launch_ins_direct_ctl(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals,
                                  uint32_t nmax, const OpScratch& sc, Ctl* ctl, double load, cudaStream_t s) {
    if (sh == SHAPE_GENERIC || !sc.comp) return cudaErrorInvalidValue;
#define FM_CALL(K, V) direct_shape<K, V>(t, keys, vals, CMP_N0_CTL, nmax, sc, ctl, (float)load, false, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

// Tuned insert configurations, per shape and load bucket (tile 0: not measured).
InsCfg g_ins_tuned[SHAPE_GENERIC + 1][LOAD_BUCKETS];

#ifndef FM_INS_TILE
#define FM_INS_TILE 32  // the warp pass's tile width where none was tuned
#endif
InsCfg tuned_ins_cfg(Shape sh, double load) {
    InsCfg c = g_ins_tuned[sh][load_bucket(load)];
    if (c.tile != 8 && c.tile != 16 && c.tile != 32) c.tile = FM_INS_TILE;
    return c;
}

void set_tuned_ins_cfg(Shape sh, int bucket, InsCfg cfg) { g_ins_tuned[sh][bucket] = cfg; }

uint32_t queue_per(uint32_t kind, uint32_t n) {
    // about QSPREAD units per phase where the op is large enough, in whole
    // multiples of QTHREADS items, at most the kind's largest unit
    const uint32_t most = kind == QP_GET ? QG_UNIT : QI_UNIT;
    const uint32_t want = (n + QSPREAD - 1) / QSPREAD;
    const uint32_t per = (want + QTHREADS - 1) / QTHREADS * QTHREADS;
    return per < (uint32_t)QTHREADS ? QTHREADS : (per > most ? most : per);
}

uint32_t queue_units(uint32_t kind, uint32_t n) {
    switch (kind) {
        case QP_BEGIN:
        case QP_END: return 1;
        case QP_IBIG: {  // blocks that take the listed components
            const uint32_t u = n / 4096 + 1;
            return u < 64 ? u : 64;
        }
        case QP_IWARP: return (n + 63) / 64;  // 8 warps per unit: a warp per 8 ops the exec pass may list
        default: {
            const uint32_t per = queue_per(kind, n);
            return (n + per - 1) / per;
        }
    }
}

cudaError_t launch_queue(Shape sh, const QPhase* ph, uint32_t nph, uint64_t total_units, const QOp* ops,
                         uint32_t* done, QState* st, QProf* prof, cudaStream_t s) {
    if (nph == 0 || total_units == 0) return cudaSuccess;
    (void)nph;
    auto go = [&](auto kernel) {
        static int per_sm = 0;  // resident blocks per SM of this instantiation
        if (per_sm == 0) {
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, QTHREADS, 0) != cudaSuccess || b < 1) b = 1;
            per_sm = b;
        }
        const uint64_t want = (uint64_t)num_sms() * per_sm;
        const unsigned grid = (unsigned)(total_units < want ? total_units : want);
        kernel<<<grid, QTHREADS, 0, s>>>(ph, total_units, ops, done, st, prof);
    };
    switch (sh) {
        case SHAPE_8_8: go(k_queue<8, 8>); break;
        case SHAPE_32_128: go(k_queue<32, 128>); break;
        case SHAPE_32_64: go(k_queue<32, 64>); break;
        case SHAPE_32_32: go(k_queue<32, 32>); break;
        case SHAPE_8_32: go(k_queue<8, 32>); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_ins_tail(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                            uint32_t r, const OpScratch& sc, Ctl* ctl, cudaStream_t s, bool handoff) {
#define FM_CALL(K, V) tail_shape<K, V>(t, keys, vals, n0, r, n0, sc, ctl, handoff, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

cudaError_t launch_grp_ins(Shape sh, const GroupOp* ops, uint32_t nops, uint64_t sum_n, int phase, uint32_t r0,
                           uint32_t nrounds, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
#define FM_CALL(K, V) grp_ins_shape<K, V>(ops, nops, sum_n, phase, r0, nrounds, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

cudaError_t launch_grp_pending(const GroupOp* ops, uint32_t nops, uint32_t r, uint32_t* out, cudaStream_t s) {
    k_grp_pending<<<1, 1, 0, s>>>(ops, nops, r, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_grp_pending_each(const GroupOp* ops, uint32_t nops, uint32_t r, uint32_t* out, cudaStream_t s) {
    k_grp_pending_each<<<(nops + 255) / 256, 256, 0, s>>>(ops, nops, r, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_ins_serial(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                              uint32_t r, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
#define FM_CALL(K, V) serial_shape<K, V>(t, keys, vals, n0, r, sc, ctl, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

cudaError_t launch_ins_comp(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                            uint32_t r, uint32_t npend, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    if (!sc.comp) {
        if (n0 == CMP_N0_CTL) return cudaErrorInvalidValue;
        return launch_ins_serial(t, sh, keys, vals, n0, r, sc, ctl, s);
    }
#define FM_CALL(K, V) comp_shape<K, V>(t, keys, vals, n0, r, npend, sc, ctl, s)
    FM_SHAPE_SWITCH(sh, FM_CALL)
#undef FM_CALL
    return cudaGetLastError();
}

}  // namespace fm

// fm_probe.cuh -- single-thread probes shared by the plain kernels and the
// persistent batch kernel: the lookup of one query and the remove of one key,
// each on one thread with aligned 8-slot metadata windows.
#pragma once
#include "fm_internal.h"

namespace fm {

// Ops of one group (a run between EMPTY slots) the direct remove runs on one
// thread; larger groups go to the rounds (or, in a batch, to the op's last
// unit).
constexpr uint32_t RX_GATHER = 32;

template <int KB>
__device__ __forceinline__ uint64_t home_of(const TableView& t, const uint8_t* keys, uint32_t j, RegKey<KB>& key) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    key.load(keys + (uint64_t)j * ksz, ksz);
    return key.hash(ksz, t.hash_mode) & t.mask;
}

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
    if (ov) {
        RegVal<VB> v;
        if (hit != NONE64) v.load_ro(t.vals + hit * VB);
        else v.zero();
        v.store(ov, VB);
    }
    if (of) *of = hit != NONE64 ? 1 : 0;
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

// The sequential remove of one key (rayon_cpu.rs:273-328): skip TOMBSTONEs,
// stop at EMPTY or at the Robin Hood exit (OCCUPIED with depth > stored
// distance), and turn the first OCCUPIED slot holding the key (its stored
// distance equal to the depth) into the whole word TOMBSTONE.  Returns 1 when
// it did.
template <int KB>
__device__ __forceinline__ uint32_t rx_probe(const TableView& t, const RegKey<KB>& key, uint64_t h) {
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
                if (p > mask) return 0;
                const uint32_t f = f8[l];
                const uint32_t st = st_of(f);
                if (st == ST_EMPTY) return 0;
                if (st == ST_OCC) {
                    if (p > dist_of(f)) return 0;
                    const uint64_t slot = pos & mask;
                    if (dist_matches(f, p) && key.eq(t.keys + slot * ksz, ksz)) {
                        t.flags[slot] = ST_TOMB;
                        return 1;
                    }
                }
            }
        }
    }
    for (uint64_t p = 0; p <= mask; ++p) {
        const uint64_t slot = (h + p) & mask;
        const uint32_t f = t.flags[slot];
        const uint32_t st = st_of(f);
        if (st == ST_EMPTY) return 0;
        if (st == ST_OCC) {
            if (p > dist_of(f)) return 0;
            if (dist_matches(f, p) && key.eq(t.keys + slot * ksz, ksz)) {
                t.flags[slot] = ST_TOMB;
                return 1;
            }
        }
    }
    return 0;
}

}  // namespace fm

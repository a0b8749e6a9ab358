// fm_device.cuh -- device-side building blocks of the FlashMap B200 backend:
// the slot metadata word, the two key hashes, and key/value access templated
// on compile-time key/value sizes (0 = sizes known only at run time).
//
// Table layout in HBM (structure of arrays, one entry per slot, capacity a
// power of two):
//   flags[cap]      u32  (dist << 4) | state            -- probe metadata
//   keys[cap * K]   u8   key bytes, slot i at i*K
//   values[cap * V] u8   value bytes, slot i at i*V
//   seg_min[cap]    u32  insert/remove round scratch (0xFFFFFFFF when idle)
//   seg_cnt[cap]    u32  insert round scratch (0 when idle)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fm {

// Slot states and the packed metadata word.  Same encoding as the reference
// (src/kernels.cu:23-30, src/rayon_cpu.rs:23-41): the low 4 bits hold the
// state, the upper 28 bits the probe distance from the home slot.  A
// tombstone is the whole word 2 (dist 0).
constexpr uint32_t ST_EMPTY = 0u;
constexpr uint32_t ST_OCC = 1u;
constexpr uint32_t ST_TOMB = 2u;
constexpr uint32_t DIST_MASK = 0x0FFFFFFFu;
constexpr uint32_t IDLE = 0xFFFFFFFFu;
constexpr uint64_t NONE64 = ~0ull;

__device__ __forceinline__ uint32_t st_of(uint32_t f) { return f & 0xFu; }
__device__ __forceinline__ uint64_t dist_of(uint32_t f) { return (uint64_t)(f >> 4); }
// make_flag keeps the low 28 bits of the distance, as the reference's
// `(dist as u32) << 4` does.
__device__ __forceinline__ uint32_t mk_flag(uint32_t st, uint64_t dist) {
    return ((uint32_t)dist << 4) | st;
}
__device__ __forceinline__ bool is_free(uint32_t f) {
    uint32_t s = st_of(f);
    return s == ST_EMPTY || s == ST_TOMB;
}
// A stored key can equal a probing key only if its stored distance equals the
// probe depth (equal keys share a home slot); the stored distance is the depth
// modulo 2^28.
__device__ __forceinline__ bool dist_matches(uint32_t f, uint64_t p) {
    return (f >> 4) == ((uint32_t)p & DIST_MASK);
}

struct TableView {
    uint32_t* flags;
    uint8_t* keys;
    uint8_t* vals;
    uint32_t* seg_min;
    uint32_t* seg_cnt;
    uint64_t mask;
    uint32_t ksz;
    uint32_t vsz;
    uint32_t hash_mode;
};

// ---------------------------------------------------------------------------
// Hashes.  Bit-identical to src/hash.rs:30-86 (identity_hash, murmur3_hash);
// restated from the algorithm, operating on little-endian 64-bit chunks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fmix_chunk(uint64_t k) {
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

__device__ __forceinline__ uint64_t murmur_finish(uint64_t h, uint64_t rem, uint32_t ksz) {
    if (rem != 0 || (ksz & 7u) != 0) {
        rem *= 0xff51afd7ed558ccdull;
        rem ^= rem >> 33;
        h ^= rem;
    }
    h ^= (uint64_t)ksz;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h;
}

// Hash of a key given as little-endian 32-bit words (tail bytes zero).
template <int NW>
__device__ __forceinline__ uint64_t hash_words(const uint32_t (&w)[NW], uint32_t ksz, uint32_t mode) {
    if (mode == 0) {
        uint64_t lo = NW > 0 ? w[0] : 0u;
        uint64_t hi = NW > 1 ? w[1] : 0u;
        uint64_t h = lo | (hi << 32);
        if (ksz < 8) h &= (ksz == 0) ? 0ull : (~0ull >> (64 - 8 * ksz));
        return h;
    }
    uint64_t h = 0x9e3779b97f4a7c15ull;
    const uint32_t chunks = ksz / 8;
#pragma unroll
    for (int c = 0; c < NW / 2; c++) {
        if ((uint32_t)c < chunks) {
            uint64_t k = (uint64_t)w[2 * c] | ((uint64_t)w[2 * c + 1] << 32);
            h ^= fmix_chunk(k);
            h = h * 5 + 0x52dce729ull;
        }
    }
    uint64_t rem = 0;
    const uint32_t rb = ksz - chunks * 8;  // 0..7 tail bytes
    if (rb) {
        uint64_t lo = (2 * chunks < (uint32_t)NW) ? w[2 * chunks] : 0u;
        uint64_t hi = (2 * chunks + 1 < (uint32_t)NW) ? w[2 * chunks + 1] : 0u;
        rem = (lo | (hi << 32)) & (~0ull >> (64 - 8 * rb));
    }
    return murmur_finish(h, rem, ksz);
}

// Hash of a key in memory, byte by byte (any size, any alignment).
__device__ __forceinline__ uint64_t hash_bytes(const uint8_t* k, uint32_t ksz, uint32_t mode) {
    if (mode == 0) {
        uint64_t h = 0;
        uint32_t n = ksz < 8 ? ksz : 8;
        for (uint32_t i = 0; i < n; i++) h |= (uint64_t)k[i] << (8 * i);
        return h;
    }
    uint64_t h = 0x9e3779b97f4a7c15ull;
    uint32_t chunks = ksz / 8;
    for (uint32_t c = 0; c < chunks; c++) {
        uint64_t x = 0;
        for (uint32_t i = 0; i < 8; i++) x |= (uint64_t)k[c * 8 + i] << (8 * i);
        h ^= fmix_chunk(x);
        h = h * 5 + 0x52dce729ull;
    }
    uint64_t rem = 0;
    for (uint32_t i = chunks * 8; i < ksz; i++) rem |= (uint64_t)k[i] << (8 * (i - chunks * 8));
    return murmur_finish(h, rem, ksz);
}

// ---------------------------------------------------------------------------
// Keys held in registers.  KB > 0 and KB % 4 == 0: the key is NW 32-bit words
// loaded with the widest aligned vector the size allows.  KB == 0: run-time
// size, the key stays in memory and is compared byte by byte.
// ---------------------------------------------------------------------------
template <int KB>
struct RegKey {
    static constexpr int NW = KB / 4;
    uint32_t w[NW];

    // Load from a read-only input buffer (read-only data path).
    __device__ __forceinline__ void load(const uint8_t* p, uint32_t) {
        if constexpr (KB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 16; i++) {
                uint4 v = __ldg(reinterpret_cast<const uint4*>(p) + i);
                w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
            }
        } else if constexpr (KB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 8; i++) {
                uint2 v = __ldg(reinterpret_cast<const uint2*>(p) + i);
                w[2 * i] = v.x; w[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) w[i] = __ldg(reinterpret_cast<const uint32_t*>(p) + i);
        }
    }
    // Load from the table, which the same kernel may be writing.
    __device__ __forceinline__ void load_table(const uint8_t* p, uint32_t) {
        if constexpr (KB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 16; i++) {
                uint4 v = reinterpret_cast<const uint4*>(p)[i];
                w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
            }
        } else if constexpr (KB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 8; i++) {
                uint2 v = reinterpret_cast<const uint2*>(p)[i];
                w[2 * i] = v.x; w[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) w[i] = reinterpret_cast<const uint32_t*>(p)[i];
        }
    }
    // Compare with a key stored in the table (plain loads: the table may be
    // written by the same kernel).
    __device__ __forceinline__ bool eq(const uint8_t* p, uint32_t) const {
        uint32_t diff = 0;
        if constexpr (KB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 16; i++) {
                uint4 v = reinterpret_cast<const uint4*>(p)[i];
                diff |= (v.x ^ w[4 * i]) | (v.y ^ w[4 * i + 1]) | (v.z ^ w[4 * i + 2]) | (v.w ^ w[4 * i + 3]);
            }
        } else if constexpr (KB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 8; i++) {
                uint2 v = reinterpret_cast<const uint2*>(p)[i];
                diff |= (v.x ^ w[2 * i]) | (v.y ^ w[2 * i + 1]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) diff |= reinterpret_cast<const uint32_t*>(p)[i] ^ w[i];
        }
        return diff == 0;
    }
    __device__ __forceinline__ bool same(const RegKey& o) const {
        uint32_t diff = 0;
#pragma unroll
        for (int i = 0; i < NW; i++) diff |= w[i] ^ o.w[i];
        return diff == 0;
    }
    __device__ __forceinline__ void store(uint8_t* p, uint32_t) const {
        if constexpr (KB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 16; i++)
                reinterpret_cast<uint4*>(p)[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
        } else if constexpr (KB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < KB / 8; i++) reinterpret_cast<uint2*>(p)[i] = make_uint2(w[2 * i], w[2 * i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) reinterpret_cast<uint32_t*>(p)[i] = w[i];
        }
    }
    __device__ __forceinline__ uint64_t hash(uint32_t, uint32_t mode) const {
        return hash_words<NW>(w, (uint32_t)KB, mode);
    }
};

// Run-time key size: the key lives in a caller-provided byte buffer.
template <>
struct RegKey<0> {
    const uint8_t* p;
    __device__ __forceinline__ void load(const uint8_t* src, uint32_t) { p = src; }
    __device__ __forceinline__ bool eq(const uint8_t* q, uint32_t ksz) const {
        for (uint32_t i = 0; i < ksz; i++)
            if (q[i] != p[i]) return false;
        return true;
    }
    __device__ __forceinline__ void store(uint8_t* q, uint32_t ksz) const {
        for (uint32_t i = 0; i < ksz; i++) q[i] = p[i];
    }
    __device__ __forceinline__ uint64_t hash(uint32_t ksz, uint32_t mode) const {
        return hash_bytes(p, ksz, mode);
    }
};

// Byte copy helper for run-time sizes (both pointers any alignment).
__device__ __forceinline__ void copy_bytes(uint8_t* dst, const uint8_t* src, uint32_t n) {
    for (uint32_t i = 0; i < n; i++) dst[i] = src[i];
}

// A value moved through registers (KB-style sizes; VB == 0 = run-time size,
// moved through a bounded local buffer).
template <int VB>
struct RegVal {
    static constexpr int NW = VB / 4;
    uint32_t w[NW > 0 ? NW : 1];
    __device__ __forceinline__ void load(const uint8_t* p, uint32_t) {
        if constexpr (VB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < VB / 16; i++) {
                uint4 v = reinterpret_cast<const uint4*>(p)[i];
                w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
            }
        } else if constexpr (VB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < VB / 8; i++) {
                uint2 v = reinterpret_cast<const uint2*>(p)[i];
                w[2 * i] = v.x; w[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) w[i] = reinterpret_cast<const uint32_t*>(p)[i];
        }
    }
    __device__ __forceinline__ void store(uint8_t* p, uint32_t) const {
        if constexpr (VB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < VB / 16; i++)
                reinterpret_cast<uint4*>(p)[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
        } else if constexpr (VB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < VB / 8; i++) reinterpret_cast<uint2*>(p)[i] = make_uint2(w[2 * i], w[2 * i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) reinterpret_cast<uint32_t*>(p)[i] = w[i];
        }
    }
    // Load through the read-only path (the table is not written concurrently).
    __device__ __forceinline__ void load_ro(const uint8_t* p) {
        if constexpr (VB % 16 == 0) {
#pragma unroll
            for (int i = 0; i < VB / 16; i++) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(p) + i);
                w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
            }
        } else if constexpr (VB % 8 == 0) {
#pragma unroll
            for (int i = 0; i < VB / 8; i++) {
                const uint2 v = __ldg(reinterpret_cast<const uint2*>(p) + i);
                w[2 * i] = v.x; w[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < NW; i++) w[i] = __ldg(reinterpret_cast<const uint32_t*>(p) + i);
        }
    }
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < (NW > 0 ? NW : 1); i++) w[i] = 0u;
    }
};

}  // namespace fm

// fm_get.cu -- sm_100a lookup kernel of the FlashMap B200 backend, plus the
// recount kernel and launch plumbing shared by the other kernel files.
//
// bulk_get (k_get) is read-only: one tile of T lanes per query.  The tile
// reads T consecutive metadata words per step (one 32-byte sector for T = 8,
// aligned so the first step covers the sector holding the home slot), finds
// the first terminating slot with a ballot (EMPTY, or OCCUPIED with probe
// depth > stored distance: rayon_cpu.rs:97-111, kernels.cu:403-412), compares
// keys only in slots whose stored distance equals the probe depth (the only
// slots that can hold the key), and moves the value with 16-byte vector
// copies spread over the tile's lanes.  Misses write zeros.  Semantics of
// kernels.cu:365-556 / rayon_cpu.rs:82-126.
#include <atomic>

#include "fm_internal.h"

namespace fm {

namespace {

constexpr int BLOCK = 256;
int g_num_sms = 0;
std::atomic<unsigned long long> g_launches{0};

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

// bulk_get with one thread per query (compile-time shapes, capacity >= 8).
// Each step reads the 8-slot metadata window that holds the probe position as
// two 16-byte loads (one 32-byte sector, aligned), walks it in registers, and
// compares keys only where the stored distance equals the probe depth.  With
// one query per thread about eight times as many queries are in flight per SM
// as with one query per 8-lane tile, which is what a chain of dependent
// random reads (key -> metadata -> key -> value) needs.
template <int KB, int VB>
__global__ void __launch_bounds__(BLOCK) k_get_thread(TableView t, const uint8_t* __restrict__ qkeys, uint64_t n,
                                                      uint8_t* __restrict__ out_vals,
                                                      uint8_t* __restrict__ out_found) {
    const uint64_t mask = t.mask;
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (uint64_t)gridDim.x * blockDim.x) {
        RegKey<KB> key;
        key.load(qkeys + q * KB, KB);
        const uint64_t h = key.hash(KB, t.hash_mode) & mask;
        uint64_t wb = h & ~7ull;
        uint64_t hit = NONE64;
        bool done = false;
        while (!done) {
            const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
            const uint4 a = __ldg(fp), b = __ldg(fp + 1);
            const uint32_t f8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int l = 0; l < 8; l++) {
                const uint64_t pos = wb + l;
                if (done || pos < h) continue;
                const uint64_t p = pos - h;
                const uint32_t f = f8[l];
                const uint32_t s = st_of(f);
                // Terminators: probe past the capacity, EMPTY, or OCCUPIED with
                // p > dist (rayon_cpu.rs:91-111); tombstones are skipped.
                if (p > mask || s == ST_EMPTY || (s == ST_OCC && p > dist_of(f))) {
                    done = true;
                } else if (s == ST_OCC && dist_matches(f, p) && key.eq(t.keys + (pos & mask) * KB, KB)) {
                    hit = pos & mask;
                    done = true;
                }
            }
            wb += 8;
        }
        if (out_vals) {
            RegVal<VB> v;
            if (hit != NONE64) v.load_ro(t.vals + hit * VB);
            else v.zero();
            v.store(out_vals + q * VB, VB);
        }
        if (out_found) out_found[q] = hit != NONE64 ? 1 : 0;
    }
}

template <int KB, int VB>
cudaError_t get_shape(const TableView& t, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of, cudaStream_t s) {
    if constexpr (KB != 0 && VB != 0) {
        if (t.mask >= 7) {
            KtScope kt(KC_GET, s);
            k_get_thread<KB, VB><<<grid_for(n, 64), BLOCK, 0, s>>>(t, q, n, ov, of);
            g_launches += 1;
            return cudaGetLastError();
        }
    }
    constexpr int T = 8;
    KtScope kt(KC_GET, s);
    k_get<KB, VB, T><<<grid_for(n * T, 16), BLOCK, 0, s>>>(t, q, n, ov, of);
    g_launches += 1;
    return cudaGetLastError();
}

}  // namespace

unsigned long long launch_count() { return g_launches.load(); }
void count_launches(unsigned n) { g_launches += n; }

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        g_num_sms = v > 0 ? v : 148;
    }
    return g_num_sms;
}

unsigned grid_for(uint64_t threads, unsigned per_sm) {
    const uint64_t want = (threads + BLOCK - 1) / BLOCK;
    const uint64_t cap = (uint64_t)num_sms() * per_sm;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
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

cudaError_t launch_count(const TableView& t, Ctl* ctl, cudaStream_t s) {
    KtScope kt(KC_COUNT_OCC, s);
    k_count<<<grid_for(t.mask + 1, 4), BLOCK, 0, s>>>(t.flags, t.mask + 1, ctl);
    g_launches += 1;
    return cudaGetLastError();
}

}  // namespace fm

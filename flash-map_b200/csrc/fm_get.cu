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
#include "fm_probe.cuh"

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
// One query by the tile of lanes [tbase, tbase+T) of the warp; qk is the
// query key, ov / of its output value and found byte (either may be null).
template <int KB, int VB, int T>
__device__ __forceinline__ void get_query_tile(const TableView& t, const uint8_t* __restrict__ qk,
                                               uint8_t* __restrict__ ov, uint8_t* __restrict__ of) {
    static_assert(T == 4 || T == 8 || T == 16 || T == 32, "tile width");
    constexpr uint32_t TM = (T == 32) ? 0xFFFFFFFFu : ((1u << T) - 1u);
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint32_t vsz = VB ? (uint32_t)VB : t.vsz;
    const uint32_t lane = threadIdx.x & (T - 1);
    const uint32_t tbase = (threadIdx.x & 31u) & ~(uint32_t)(T - 1);
    const uint32_t tmask = TM << tbase;
    const uint64_t mask = t.mask;
    RegKey<KB> key;
    key.load(qk, ksz);
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
    if (ov) {
        if (hit != NONE64) tile_copy<VB, T>(ov, t.vals + hit * vsz, vsz, lane);
        else tile_zero<VB, T>(ov, vsz, lane);
    }
    if (of && lane == 0) *of = hit != NONE64 ? 1 : 0;
}

template <int KB, int VB, int T>
__global__ void __launch_bounds__(BLOCK) k_get(TableView t, const uint8_t* __restrict__ qkeys, uint64_t n,
                                               uint8_t* __restrict__ out_vals, uint8_t* __restrict__ out_found) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint32_t vsz = VB ? (uint32_t)VB : t.vsz;
    const uint64_t ntiles = ((uint64_t)gridDim.x * blockDim.x) / T;
    for (uint64_t q = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / T; q < n; q += ntiles)
        get_query_tile<KB, VB, T>(t, qkeys + q * ksz, out_vals ? out_vals + q * vsz : nullptr,
                                  out_found ? out_found + q : nullptr);
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

template <int KB, int VB>
__global__ void __launch_bounds__(BLOCK) k_get_thread(TableView t, const uint8_t* __restrict__ qkeys, uint64_t n,
                                                      uint8_t* __restrict__ out_vals,
                                                      uint8_t* __restrict__ out_found) {
#if FM_GET_WCOPY
    constexpr bool wcopy = VB % 16 == 0;
#else
    constexpr bool wcopy = false;
#endif
    if constexpr (wcopy) {
        // a thread probes its query; then the warp moves its 32 values
        // together, VB / 16 lanes per value, so each load and store
        // instruction covers whole 128-byte lines of several values
        constexpr uint32_t LPV = VB / 16, VPR = 32 / LPV;
        const uint32_t lane = threadIdx.x & 31u, part = lane % LPV, vsel = lane / LPV;
        const uint64_t G = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += G) {
            const uint64_t q = base + lane;
            uint64_t hit = NONE64;
            if (q < n) hit = get_probe_thread<KB>(t, qkeys + q * KB);
            if (out_found && q < n) out_found[q] = hit != NONE64 ? 1 : 0;
            if (!out_vals) continue;
#pragma unroll
            for (uint32_t r = 0; r < LPV; r++) {
                const uint32_t src = r * VPR + vsel;
                const uint64_t hs = __shfl_sync(0xFFFFFFFFu, hit, src);
                const uint64_t qs = base + src;
                if (qs < n) {
                    uint4 v = make_uint4(0u, 0u, 0u, 0u);
                    if (hs != NONE64) v = __ldg(reinterpret_cast<const uint4*>(t.vals + hs * VB) + part);
                    reinterpret_cast<uint4*>(out_vals + qs * VB)[part] = v;
                }
            }
        }
    } else {
        for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
             q += (uint64_t)gridDim.x * blockDim.x)
            get_query_thread<KB, VB>(t, qkeys + q * KB, out_vals ? out_vals + q * VB : nullptr,
                                     out_found ? out_found + q : nullptr);
    }
}

// Q queries per thread probed in lockstep (get_queries_lockstep): thread g
// takes queries g, g + G, ..., g + (Q-1)G of each span of Q*G (G threads in
// the grid), so a warp's key loads stay coalesced.
template <int KB, int VB, int Q>
__global__ void __launch_bounds__(BLOCK) k_get_lockstep(TableView t, const uint8_t* __restrict__ qkeys, uint64_t n,
                                                        uint8_t* __restrict__ out_vals,
                                                        uint8_t* __restrict__ out_found) {
    const uint64_t G = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += G * Q)
        get_queries_lockstep<KB, VB, Q>(t, qkeys, q, G, n, out_vals, out_found);
}

// Grouped lookups: the gets of a batch wave, one flat index space over their
// queries (prefix[o] = first flat index of get o), T lanes per query (T == 1:
// one thread per query).  Load-balanced over gets of any sizes.
template <int KB, int VB, int T>
__global__ void __launch_bounds__(BLOCK) k_grp_get(const GroupGet* __restrict__ ops,
                                                   const uint64_t* __restrict__ prefix, uint32_t nops,
                                                   uint64_t total) {
    const uint64_t units = ((uint64_t)gridDim.x * blockDim.x) / T;
    for (uint64_t q = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / T; q < total; q += units) {
        uint32_t lo = 0, hi = nops;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(prefix + mid) <= q) lo = mid;
            else hi = mid;
        }
        const GroupGet& g = ops[lo];
        const uint64_t i = q - __ldg(prefix + lo);
        const uint32_t ksz = KB ? (uint32_t)KB : g.t.ksz;
        const uint32_t vsz = VB ? (uint32_t)VB : g.t.vsz;
        uint8_t* ov = g.out_vals ? g.out_vals + i * vsz : nullptr;
        uint8_t* of = g.out_found ? g.out_found + i : nullptr;
        if constexpr (T == 1) get_query_thread<KB, VB>(g.t, g.keys + i * ksz, ov, of);
        else get_query_tile<KB, VB, T>(g.t, g.keys + i * ksz, ov, of);
    }
}

// Seeded pseudo-random bytes (splitmix64 of the word index), for the
// autotuner's sample tables and queries.
__global__ void k_fill_random(uint64_t* __restrict__ out, uint64_t words, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        out[i] = z ^ (z >> 31);
    }
}

// Tuned lookup configurations, per shape and load bucket (0: not measured).
GetCfg g_tuned[SHAPE_GENERIC + 1][LOAD_BUCKETS];

template <int KB, int VB, int T>
void get_launch(const TableView& t, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of, int bps,
                cudaStream_t s) {
    KtScope kt(KC_GET, s);
    if constexpr (T == 1) k_get_thread<KB, VB><<<grid_for(n, bps), BLOCK, 0, s>>>(t, q, n, ov, of);
    else k_get<KB, VB, T><<<grid_for(n * T, bps), BLOCK, 0, s>>>(t, q, n, ov, of);
    g_launches += 1;
}

template <int KB, int VB>
cudaError_t get_shape(const TableView& t, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of, GetCfg cfg,
                      cudaStream_t s) {
    int lanes = cfg.lanes;
    // one thread per query needs compile-time sizes and 8-slot windows
    if (lanes == 1 && !(KB != 0 && VB != 0 && t.mask >= 7)) lanes = 8;
    switch (lanes) {
        case 1:
            if constexpr (KB != 0 && VB != 0) {
                if (cfg.qpt == 2 || cfg.qpt == 4) {
                    KtScope kt(KC_GET, s);
                    const unsigned g = grid_for((n + cfg.qpt - 1) / cfg.qpt, cfg.blocks_per_sm);
                    if (cfg.qpt == 2) k_get_lockstep<KB, VB, 2><<<g, BLOCK, 0, s>>>(t, q, n, ov, of);
                    else k_get_lockstep<KB, VB, 4><<<g, BLOCK, 0, s>>>(t, q, n, ov, of);
                    g_launches += 1;
                } else {
                    get_launch<KB, VB, 1>(t, q, n, ov, of, cfg.blocks_per_sm, s);
                }
            }
            break;
        case 4: get_launch<KB, VB, 4>(t, q, n, ov, of, cfg.blocks_per_sm, s); break;
        case 16: get_launch<KB, VB, 16>(t, q, n, ov, of, cfg.blocks_per_sm, s); break;
        case 32: get_launch<KB, VB, 32>(t, q, n, ov, of, cfg.blocks_per_sm, s); break;
        default: get_launch<KB, VB, 8>(t, q, n, ov, of, cfg.blocks_per_sm, s); break;
    }
    return cudaGetLastError();
}

template <int KB, int VB, int T>
void grp_get_launch(const GroupGet* ops, const uint64_t* prefix, uint32_t nops, uint64_t total, int bps,
                    cudaStream_t s) {
    KtScope kt(KC_GET, s);
    k_grp_get<KB, VB, T><<<grid_for(total * T, bps), BLOCK, 0, s>>>(ops, prefix, nops, total);
    g_launches += 1;
}

template <int KB, int VB>
cudaError_t grp_get_shape(const GroupGet* ops, const uint64_t* prefix, uint32_t nops, uint64_t total, GetCfg cfg,
                          cudaStream_t s) {
    int lanes = cfg.lanes;
    if (lanes == 1 && !(KB != 0 && VB != 0)) lanes = 8;
    switch (lanes) {
        case 1:
            if constexpr (KB != 0 && VB != 0) grp_get_launch<KB, VB, 1>(ops, prefix, nops, total, cfg.blocks_per_sm, s);
            break;
        case 4: grp_get_launch<KB, VB, 4>(ops, prefix, nops, total, cfg.blocks_per_sm, s); break;
        case 16: grp_get_launch<KB, VB, 16>(ops, prefix, nops, total, cfg.blocks_per_sm, s); break;
        case 32: grp_get_launch<KB, VB, 32>(ops, prefix, nops, total, cfg.blocks_per_sm, s); break;
        default: grp_get_launch<KB, VB, 8>(ops, prefix, nops, total, cfg.blocks_per_sm, s); break;
    }
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

#define FM_GET_SWITCH(sh, CALL)                          \
    switch (sh) {                                        \
        case SHAPE_8_8: return CALL(8, 8);               \
        case SHAPE_32_128: return CALL(32, 128);         \
        case SHAPE_32_64: return CALL(32, 64);           \
        case SHAPE_32_32: return CALL(32, 32);           \
        case SHAPE_8_32: return CALL(8, 32);             \
        default: return CALL(0, 0);                      \
    }

cudaError_t launch_get_cfg(const TableView& t, Shape sh, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of,
                           GetCfg cfg, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
#define FM_CALL(K, V) get_shape<K, V>(t, q, n, ov, of, cfg, s)
    FM_GET_SWITCH(sh, FM_CALL)
#undef FM_CALL
}

GetCfg tuned_get_cfg(Shape sh, double load) {
    const GetCfg c = g_tuned[sh][load_bucket(load)];
    if (c.lanes > 0 && c.blocks_per_sm > 0) return c;
    GetCfg d;  // measured default on B200: one thread per query, 64 blocks per SM
    if (sh == SHAPE_GENERIC) d.lanes = 8, d.blocks_per_sm = 16;
    return d;
}

void set_tuned_get_cfg(Shape sh, int bucket, GetCfg cfg) {
    if (bucket >= 0 && bucket < LOAD_BUCKETS) g_tuned[sh][bucket] = cfg;
}

cudaError_t launch_get(const TableView& t, Shape sh, const uint8_t* q, uint64_t n, uint8_t* ov, uint8_t* of,
                       cudaStream_t s) {
    GetCfg cfg;
    if (sh == SHAPE_GENERIC) cfg.lanes = 8, cfg.blocks_per_sm = 16;
    return launch_get_cfg(t, sh, q, n, ov, of, cfg, s);
}

cudaError_t launch_grp_get(Shape sh, const GroupGet* ops, const uint64_t* prefix, uint32_t nops, uint64_t total,
                           GetCfg cfg, cudaStream_t s) {
    if (total == 0 || nops == 0) return cudaSuccess;
#define FM_CALL(K, V) grp_get_shape<K, V>(ops, prefix, nops, total, cfg, s)
    FM_GET_SWITCH(sh, FM_CALL)
#undef FM_CALL
}

cudaError_t launch_fill_random(void* out, uint64_t bytes, uint64_t seed, cudaStream_t s) {
    k_fill_random<<<grid_for(bytes / 8, 8), BLOCK, 0, s>>>((uint64_t*)out, bytes / 8, seed);
    return cudaGetLastError();
}

cudaError_t launch_count(const TableView& t, Ctl* ctl, cudaStream_t s) {
    KtScope kt(KC_COUNT_OCC, s);
    k_count<<<grid_for(t.mask + 1, 4), BLOCK, 0, s>>>(t.flags, t.mask + 1, ctl);
    g_launches += 1;
    return cudaGetLastError();
}

}  // namespace fm

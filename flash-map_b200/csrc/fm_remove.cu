// fm_remove.cu -- deterministic bulk remove for sm_100a.
//
// Semantics: the reference's sequential remove (src/rayon_cpu.rs:273-328;
// the probe of src/kernels.cu:565-644 run one key at a time) in batch index
// order: the first OCCUPIED slot holding the key before the first EMPTY slot
// or Robin Hood exit (p > dist) becomes the whole word TOMBSTONE (dist 0).
//
// Why rounds: removes of different keys interact only through slots one of
// them tombstones.  Every pending op marks each slot that holds its key
// within [home, min(first EMPTY - 1, X + dmax)] (X = its current target, or
// home on a miss; dmax bounds every stored distance, so no copy of a key lies
// further) with its index.  An op runs in a round unless an earlier pending
// op marked a slot of its own window (the same range), which covers both
// directions of interference: an earlier op's tombstone changing this op's
// probe, and this op's tombstone letting an earlier op's probe run on past a
// former terminator.  The lowest pending op is never blocked.
//
// Control: as fm_insert.cu (two grid rounds, then a single-block tail).
#include "fm_rounds.cuh"
#include "fm_probe.cuh"

namespace fm {
namespace {

// The call's chunk summaries, or null when the call did not build them.
__device__ __forceinline__ uint32_t* rsum_of(const OpScratch& sc, const Ctl* ctl) {
    return *(volatile const uint32_t*)&ctl->rsum_on ? sc.rsum : nullptr;
}

// Below this largest stored distance the windows are short enough that the
// summaries cost more than they save (load 0.8: about 7% on a 1.3M-key remove).
constexpr uint32_t RSUM_MIN_DMAX = 256;

// Chunk summaries of a remove call, once per call (capacity >= 32): per 32
// slots whether one is EMPTY and the largest stored distance.  Removes make
// no EMPTY slot and only lower distances, so they stay valid bounds for the
// whole call.
__global__ void __launch_bounds__(256) k_rem_sum(TableView t, OpScratch sc, Ctl* ctl) {
    if (*(volatile const uint32_t*)&ctl->dmax < RSUM_MIN_DMAX) return;  // grid-uniform
    const uint64_t nch = rsum_chunks(t.mask);
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) ctl->rsum_on = 1u;
    if (c >= nch) return;
    const uint4* p = reinterpret_cast<const uint4*>(t.flags + c * 32);
    uint32_t md = 0;
    bool empty = false;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const uint4 w = p[q];
        const uint32_t f4[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int l = 0; l < 4; l++) {
            const uint32_t st = st_of(f4[l]);
            if (st == ST_EMPTY) empty = true;
            else if (st == ST_OCC) md = max(md, (uint32_t)dist_of(f4[l]));
        }
    }
    sc.rsum[c] = (empty ? 0x80000000u : 0u) | md;
}

// Phase 1 for op j: probe, then mark every possible target.  With capacity
// >= 8 the metadata is read in aligned 8-slot windows (two 16-byte loads, one
// 32-byte sector) and scanned in registers; key compares happen only where
// the stored distance equals the probe depth.
template <int KB>
__device__ __forceinline__ void scan_op(const TableView& t, const uint8_t* keys, uint32_t j, uint64_t dmax,
                                        const OpScratch& sc, const uint32_t* rs) {
    const uint32_t ksz = KB ? (uint32_t)KB : t.ksz;
    const uint64_t mask = t.mask;
    RegKey<KB> key;
    const uint64_t h = home_of<KB>(t, keys, j, key);
    uint64_t tp = NONE64;  // probe depth of the current target
    uint64_t p = 0;        // probe depth where the probe stopped
    bool empty_hit = false;
    uint32_t npt = 0;
    uint64_t wend = NONE64;
    auto mark = [&](uint64_t q) {
        atomicMin(&t.seg_min[(h + q) & mask], j);
        if (rs) atomicMin(const_cast<uint32_t*>(rs) + rsum_chunks(mask) + (((h + q) & mask) >> 5), j);
        if (npt < PT_MAX) sc.op_pt[(uint64_t)j * PT_MAX + npt] = (uint32_t)q;
        ++npt;
    };
    if (mask >= 7) {
        // 1. the probe
        bool stop = false;
        for (uint64_t wb = h & ~7ull; !stop; wb += 8) {
            const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
            const uint4 a = fp[0], b = fp[1];
            const uint32_t f8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int l = 0; l < 8; l++) {
                if (stop || wb + l < h) continue;
                const uint64_t q = wb + l - h;
                if (q > mask) {  // the whole table probed
                    p = q;
                    stop = true;
                    continue;
                }
                const uint32_t f = f8[l];
                const uint32_t st = st_of(f);
                if (st == ST_EMPTY) {
                    empty_hit = true;
                    p = q;
                    stop = true;
                } else if (st == ST_OCC) {
                    if (q > dist_of(f)) {  // Robin Hood exit (rayon_cpu.rs:298-302)
                        p = q;
                        stop = true;
                    } else if (dist_matches(f, q) && key.eq(t.keys + ((h + q) & mask) * ksz, ksz)) {
                        tp = q;
                        p = q;
                        stop = true;
                    }
                }
            }
        }
        uint64_t lim = (tp != NONE64 ? tp : 0) + dmax;
        if (lim > mask) lim = mask;
        if (empty_hit) {
            wend = p == 0 ? NONE64 : min(p - 1, lim);  // home slot EMPTY: nothing to watch
        } else {
            if (tp != NONE64) mark(tp);
            wend = min(p, lim);
            // 2. later copies of the key up to the bound (windows again)
            const uint64_t q0 = (tp != NONE64 ? tp : p) + 1;
            bool done = q0 > lim;
            if (rs) {
                // chunk by chunk: a chunk without an EMPTY slot whose largest
                // stored distance is below the depth reached holds no copy
                for (uint64_t q = q0; !done && q <= lim;) {
                    const uint64_t s0 = (h + q) & mask;
                    const uint64_t qe = min(q + (31 - (s0 & 31)), lim);  // this chunk's last depth in the window
                    const uint32_t sm = rs[s0 >> 5];
                    if (!(sm >> 31) && (uint64_t)(sm & 0x7FFFFFFFu) < q) {
                        wend = qe;
                        q = qe + 1;
                        continue;
                    }
                    for (; q <= qe; ++q) {
                        const uint64_t s = (h + q) & mask;
                        const uint32_t f = t.flags[s];
                        const uint32_t st = st_of(f);
                        if (st == ST_EMPTY) {
                            done = true;
                            break;
                        }
                        wend = q;
                        if (st == ST_OCC && dist_matches(f, q) && key.eq(t.keys + s * ksz, ksz)) mark(q);
                    }
                }
                done = true;
            }
            for (uint64_t wb = (h + q0) & ~7ull; !done; wb += 8) {
                const uint4* fp = reinterpret_cast<const uint4*>(t.flags + (wb & mask));
                const uint4 a = fp[0], b = fp[1];
                const uint32_t f8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    if (done || wb + l < h + q0) continue;
                    const uint64_t q = wb + l - h;
                    if (q > lim) {
                        done = true;
                        continue;
                    }
                    const uint32_t f = f8[l];
                    const uint32_t st = st_of(f);
                    if (st == ST_EMPTY) {
                        done = true;
                        continue;
                    }
                    wend = q;
                    if (st == ST_OCC && dist_matches(f, q) && key.eq(t.keys + ((h + q) & mask) * ksz, ksz)) mark(q);
                }
            }
        }
    } else {
        for (; p <= mask; ++p) {
            const uint64_t s = (h + p) & mask;
            const uint32_t f = t.flags[s];
            const uint32_t st = st_of(f);
            if (st == ST_EMPTY) {
                empty_hit = true;
                break;
            }
            if (st == ST_OCC) {
                if (p > dist_of(f)) break;  // Robin Hood exit (rayon_cpu.rs:298-302)
                if (dist_matches(f, p) && key.eq(t.keys + s * ksz, ksz)) {
                    tp = p;
                    break;
                }
            }
        }
        uint64_t lim = (tp != NONE64 ? tp : 0) + dmax;
        if (lim > mask) lim = mask;
        if (empty_hit) {
            wend = p == 0 ? NONE64 : min(p - 1, lim);  // home slot EMPTY: nothing to watch
        } else {
            if (tp != NONE64) mark(tp);
            wend = min(p, lim);
            for (uint64_t q = (tp != NONE64 ? tp : p) + 1; q <= lim; ++q) {
                const uint64_t s = (h + q) & mask;
                const uint32_t f = t.flags[s];
                const uint32_t st = st_of(f);
                if (st == ST_EMPTY) break;
                wend = q;
                if (st == ST_OCC && dist_matches(f, q) && key.eq(t.keys + s * ksz, ksz)) mark(q);
            }
        }
    }
    sc.op_slot[j] = tp != NONE64 ? ((h + tp) & mask) : NONE64;
    sc.op_word[j] = wend == NONE64 ? IDLE : (uint32_t)wend;
    sc.op_flag[j] = (uint8_t)min(npt, 255u);
}

// Phase 2 for op j: run unless an earlier op marked its window (read as
// aligned 4-slot groups of marks with capacity >= 4).
template <int KB>
__device__ __forceinline__ bool check_op(const TableView& t, const uint8_t* keys, uint32_t j, const OpScratch& sc,
                                         uint32_t& removed, const uint32_t* rs) {
    const uint64_t mask = t.mask;
    const uint32_t wend = sc.op_word[j];
    if (wend != IDLE) {
        RegKey<KB> key;
        const uint64_t h = home_of<KB>(t, keys, j, key);
        if (rs) {
            // a chunk's least mark first: slots only where it is below j and
            // the chunk is cut by the window's ends
            const uint32_t* cm = rs + rsum_chunks(mask);
            for (uint64_t q = 0; q <= wend;) {
                const uint64_t s0 = (h + q) & mask;
                const uint64_t qe = min(q + (31 - (s0 & 31)), (uint64_t)wend);
                if (cm[s0 >> 5] < j) {
                    if ((s0 & 31) == 0 && qe == q + 31) return false;
                    for (uint64_t x = q; x <= qe; ++x)
                        if (t.seg_min[(h + x) & mask] < j) return false;
                }
                q = qe + 1;
            }
        } else if (mask >= 3) {
            const uint64_t last = h + wend;
            for (uint64_t wb = h & ~3ull; wb <= last; wb += 4) {
                const uint4 m = *reinterpret_cast<const uint4*>(t.seg_min + (wb & mask));
                const uint32_t m4[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                for (int l = 0; l < 4; l++)
                    if (wb + l >= h && wb + l <= last && m4[l] < j) return false;
            }
        } else {
            for (uint64_t q = 0; q <= wend; ++q)
                if (t.seg_min[(h + q) & mask] < j) return false;
        }
    }
    const uint64_t ts = sc.op_slot[j];
    if (ts != NONE64) {
        t.flags[ts] = ST_TOMB;  // whole word 2: TOMBSTONE, dist 0 (rayon_cpu.rs:306-313)
        ++removed;
    }
    return true;
}

// Phase 3 for op j: clear its marks and its window word.
template <int KB>
__device__ __forceinline__ void reset_op(const TableView& t, const uint8_t* keys, uint32_t j, const OpScratch& sc,
                                         uint32_t* rs) {
    const uint64_t mask = t.mask;
    const uint32_t npt = sc.op_flag[j];
    const uint32_t wend = sc.op_word[j];
    sc.op_word[j] = IDLE;  // the word is the insert's inflow bound between calls
    if (npt == 0) return;
    RegKey<KB> key;
    const uint64_t h = home_of<KB>(t, keys, j, key);
    uint32_t* cm = rs ? rs + rsum_chunks(mask) : nullptr;
    if (npt <= PT_MAX) {
        for (uint32_t k = 0; k < npt; k++) {
            const uint64_t s = (h + sc.op_pt[(uint64_t)j * PT_MAX + k]) & mask;
            t.seg_min[s] = IDLE;
            if (cm) cm[s >> 5] = IDLE;
        }
    } else {
        for (uint64_t q = 0; q <= wend; ++q) {
            const uint64_t s = (h + q) & mask;
            if (t.seg_min[s] != IDLE) {
                t.seg_min[s] = IDLE;
                if (cm) cm[s >> 5] = IDLE;
            }
        }
    }
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rem_p1(TableView t, const uint8_t* __restrict__ keys, uint32_t n0,
                                                   uint32_t r, OpScratch sc, Ctl* ctl) {
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    if (blockIdx.x == 0 && threadIdx.x == 0) reset_next_round(ctl, r);
    const uint64_t dmax = *(volatile uint32_t*)&ctl->dmax;
    const uint32_t* rs = rsum_of(sc, ctl);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops.n; i += gridDim.x * blockDim.x)
        scan_op<KB>(t, keys, ops.op(i), dmax, sc, rs);
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rem_p2(TableView t, const uint8_t* __restrict__ keys, uint32_t n0,
                                                   uint32_t r, OpScratch sc, Ctl* ctl) {
    __shared__ AppendSmem s_app;
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    append_init(s_app);
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    uint32_t* out = pend_of(sc, r + 1);
    uint32_t* out_n = &ctl->npend[(r + 1) & 1];
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t iters = grid_iters(ops.n);
    const uint32_t* rs = rsum_of(sc, ctl);
    uint32_t removed = 0;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t i = i0 + it * stride;
        const bool valid = i < ops.n;
        uint32_t j = 0;
        bool ran = false;
        if (valid) {
            j = ops.op(i);
            ran = check_op<KB>(t, keys, j, sc, removed, rs);
        }
        block_append(out, out_n, j, valid && !ran, s_app);
    }
    block_add_count(ctl, removed, s_tmp);
    if (blockIdx.x == 0 && threadIdx.x == 0 && ops.n) atomicAdd(&ctl->rounds, 1u);
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rem_p3(TableView t, const uint8_t* __restrict__ keys, uint32_t n0,
                                                   uint32_t r, OpScratch sc, Ctl* ctl) {
    const RoundOps ops = round_ops(sc, ctl, r, n0);
    uint32_t* rs = rsum_of(sc, ctl);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops.n; i += gridDim.x * blockDim.x)
        reset_op<KB>(t, keys, ops.op(i), sc, rs);
}

template <int KB>
__device__ __forceinline__ void rem_tail_body(const TableView& t, const uint8_t* __restrict__ keys, uint32_t n0,
                                              uint32_t r0, const OpScratch& sc, Ctl* ctl, uint32_t limit) {
    __shared__ uint32_t s_n, s_next;
    if (threadIdx.x == 0) s_n = (r0 == 0) ? n0 : *(volatile uint32_t*)&ctl->npend[r0 & 1];
    __syncthreads();
    uint32_t n = s_n;
    if (n == 0 || n > limit) return;
    const uint64_t dmax = *(volatile uint32_t*)&ctl->dmax;
    uint32_t* rs = rsum_of(sc, ctl);
    uint32_t removed = 0, rounds = 0;
    uint32_t r = r0;
    bool stuck = false;
    for (;;) {
        const uint32_t* in = (r == 0) ? nullptr : pend_of(sc, r);
        uint32_t* out = pend_of(sc, r + 1);
        if (threadIdx.x == 0) s_next = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) scan_op<KB>(t, keys, in ? in[i] : i, dmax, sc, rs);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t j = in ? in[i] : i;
            if (!check_op<KB>(t, keys, j, sc, removed, rs)) out[atomicAdd(&s_next, 1u)] = j;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) reset_op<KB>(t, keys, in ? in[i] : i, sc, rs);
        __syncthreads();
        const uint32_t nn = s_next;
        ++r;
        ++rounds;
        if (nn == 0) break;
        if (nn >= n) {
            stuck = true;
            break;
        }
        n = nn;
        __syncthreads();
    }
    if (removed) atomicAdd(&ctl->count, (unsigned long long)removed);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (stuck) {
            atomicOr(&ctl->err, ERR_NO_PROGRESS);
        } else {
            ctl->npend[r0 & 1] = 0;
            ctl->npend[(r0 + 1) & 1] = 0;
        }
        atomicAdd(&ctl->rounds, rounds);
    }
}

template <int KB>
__global__ void __launch_bounds__(TAIL_THREADS) k_rem_tail(TableView t, const uint8_t* __restrict__ keys,
                                                           uint32_t n0, uint32_t r0, OpScratch sc, Ctl* ctl) {
    rem_tail_body<KB>(t, keys, n0, r0, sc, ctl, TAIL_MAX);
}

// ---- grouped rounds (batch waves): the removes of a wave, one launch per
// phase for all of them (see the grouped inserts in fm_insert.cu) -----------

__device__ __forceinline__ uint32_t grp_rem_pending(const GroupOp* ops, uint32_t o, uint32_t r) {
    const Ctl* c = ops[o].ctl;
    return r == 0 ? *(volatile const uint32_t*)&c->n0 : *(volatile const uint32_t*)&c->npend[r & 1];
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_grp_rem_p1(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r) {
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    const uint32_t total = group_prefix(nops, [&](uint32_t o) { return grp_rem_pending(ops, o, r); }, s_pre);
    if (blockIdx.x == 0)
        for (uint32_t o = threadIdx.x; o < nops; o += blockDim.x) reset_next_round(ops[o].ctl, r);
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t i = f - s_pre[o];
        const uint32_t j = r == 0 ? i : pend_of(g.sc, r)[i];
        scan_op<KB>(g.t, g.keys, j, *(volatile uint32_t*)&g.ctl->dmax, g.sc, rsum_of(g.sc, g.ctl));
    }
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_grp_rem_p2(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r) {
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    const uint32_t total = group_prefix(nops, [&](uint32_t o) { return grp_rem_pending(ops, o, r); }, s_pre);
    if (blockIdx.x == 0)
        for (uint32_t o = threadIdx.x; o < nops; o += blockDim.x)
            if (s_pre[o + 1] > s_pre[o]) atomicAdd(&ops[o].ctl->rounds, 1u);
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t i = f - s_pre[o];
        const uint32_t j = r == 0 ? i : pend_of(g.sc, r)[i];
        uint32_t removed = 0;
        const bool ran = check_op<KB>(g.t, g.keys, j, g.sc, removed, rsum_of(g.sc, g.ctl));
        append_peer(pend_of(g.sc, r + 1), &g.ctl->npend[(r + 1) & 1], j, !ran, o);
        add_peer(g.ctl, removed, o);
    }
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_grp_rem_p3(const GroupOp* __restrict__ ops, uint32_t nops, uint32_t r) {
    __shared__ uint32_t s_pre[GROUP_MAX + 1];
    const uint32_t total = group_prefix(nops, [&](uint32_t o) { return grp_rem_pending(ops, o, r); }, s_pre);
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const uint32_t o = group_find(s_pre, nops, f);
        const GroupOp& g = ops[o];
        const uint32_t i = f - s_pre[o];
        const uint32_t j = r == 0 ? i : pend_of(g.sc, r)[i];
        reset_op<KB>(g.t, g.keys, j, g.sc, rsum_of(g.sc, g.ctl));
    }
}

template <int KB>
__global__ void __launch_bounds__(TAIL_THREADS) k_grp_rem_tail(const GroupOp* __restrict__ ops, uint32_t r0) {
    const GroupOp& g = ops[blockIdx.x];
    const uint32_t n0 = *(volatile const uint32_t*)&g.ctl->n0;
    rem_tail_body<KB>(g.t, g.keys, n0, r0, g.sc, g.ctl, 0xFFFFFFFFu);
}

template <int KB>
void grp_rem_shape(const GroupOp* ops, uint32_t nops, uint64_t sum_n, int phase, uint32_t r0, uint32_t nrounds,
                   cudaStream_t s) {
    const unsigned g = grid_for(sum_n, 8);
    if (phase == GRP_BEGIN) {
        k_grp_setup<<<nops, 256, 0, s>>>(ops, 0);
        count_launches(1);
        return;
    }
    if (phase == GRP_END) {
        {
            KtScope kt(KC_REM_TAIL, s);
            k_grp_rem_tail<KB><<<nops, TAIL_THREADS, 0, s>>>(ops, r0);
        }
        k_grp_finish<<<(nops + 255) / 256, 256, 0, s>>>(ops, nops, 0);
        count_launches(2);
        return;
    }
    for (uint32_t r = r0; r < r0 + nrounds; r++) {
        {
            KtScope kt(KC_REM_MARK, s);
            k_grp_rem_p1<KB><<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
        {
            KtScope kt(KC_REM_CHECK, s);
            k_grp_rem_p2<KB><<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
        {
            KtScope kt(KC_REM_EXEC, s);
            k_grp_rem_p3<KB><<<g, RBLOCK, 0, s>>>(ops, nops, r);
        }
    }
    count_launches(3 * nrounds);
}

template <int KB>
void rounds_shape(const TableView& t, const uint8_t* keys, uint32_t n0, uint32_t r0, uint32_t nrounds,
                  uint32_t grid_ops, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    const unsigned g = grid_for(grid_ops, 8);
    for (uint32_t r = r0; r < r0 + nrounds; r++) {
        {
            KtScope kt(KC_REM_MARK, s);
            k_rem_p1<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, r, sc, ctl);
        }
        {
            KtScope kt(KC_REM_CHECK, s);
            k_rem_p2<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, r, sc, ctl);
        }
        {
            KtScope kt(KC_REM_EXEC, s);
            k_rem_p3<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, r, sc, ctl);
        }
    }
    count_launches(3 * nrounds);
}

// ---- direct remove: groups between EMPTY slots ------------------------------
//
// A remove's probe (rayon_cpu.rs:273-328) reads only [home, E], E the first
// EMPTY slot at or after its home, and writes at most one slot of it (the
// whole word TOMBSTONE).  Removes make no EMPTY slot, so E stays the same for
// the whole call, and ops with different E read and write disjoint slots.
// So the ops are grouped by E, without rounds:
//   find (a thread per op)  E, and the op's place in E's group
//        (atomicAdd on seg_cnt[E], kept in op_word); place 0 leads E.
//   exec (a thread per op)  an op alone at its E runs its probe at once; the
//        leader of an E with c >= 2 ops takes a segment of c words of pend[0]
//        (one atomic per warp on Ctl::big_ops), keeps its offset in seg_min[E]
//        and lists E for the group pass.
//   place (a thread per op)  each op of a group writes its index at its place
//        in its group's segment.
//   group (a lane per listed E)  reads the segment, orders it by index and
//        runs the ops one after another (up to RX_THREAD ops) or on the whole
//        warp in chunks of 32 (rx_group_run, up to RX_GMAX ops);
//   block (a block per larger group, up to RX_BMAX ops)  sorts the segment in
//        shared memory and runs it in chunks of 32 on warp 0 (rx_chunk32).
// A call where some op finds no EMPTY slot (its probe could go round the
// table) leaves every op to the rounds (Ctl::serial[0]); a group of more than
// RX_BMAX ops leaves its ops to them (pend[1], Ctl::npend[1]).  Every
// registration and list word is idle again when the five kernels end.

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rx_find(TableView t, const uint8_t* __restrict__ keys, uint32_t n0_arg,
                                                    OpScratch sc, Ctl* ctl) {
    const uint32_t n0 = n0_arg != CMP_N0_CTL ? n0_arg : *(volatile const uint32_t*)&ctl->n0;
    bool no_empty = false;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n0; j += gridDim.x * blockDim.x) {
        RegKey<KB> key;
        const uint64_t E = rx_first_empty(t, home_of<KB>(t, keys, j, key));
        sc.op_slot[j] = E;
        uint8_t lead = 0;
        uint32_t place = IDLE;
        if (E == NONE64) {
            no_empty = true;
        } else {
            place = atomicAdd(&t.seg_cnt[E], 1u);
            lead = place == 0u ? 1 : 0;
        }
        sc.op_word[j] = place;
        sc.op_flag[j] = lead;
    }
    if (no_empty) ctl->serial[0] = 1u;
}

template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rx_exec(TableView t, const uint8_t* __restrict__ keys, uint32_t n0_arg,
                                                    OpScratch sc, Ctl* ctl) {
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    const uint32_t n0 = n0_arg != CMP_N0_CTL ? n0_arg : *(volatile const uint32_t*)&ctl->n0;
    // with the count in the control block (a device-driven call) the ops of a
    // call that found no EMPTY slot go to pend[1] for the rounds launched
    // after this pass; otherwise the host runs every op from round 0
    const bool to_pend = n0_arg == CMP_N0_CTL;
    const bool serial = *(volatile uint32_t*)&ctl->serial[0] != 0;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t removed = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t iters = (n0 + stride - 1) / stride;
    for (uint32_t it = 0; it < iters; it++) {  // warp-uniform trip count
        const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x + it * stride;
        uint64_t E = NONE64;
        uint32_t cg = 0;  // the size of the group this op leads (0: none)
        if (j < n0 && serial && to_pend) sc.pend[1][atomicAdd(&ctl->npend[1], 1u)] = j;
        if (j < n0) {
            E = sc.op_slot[j];
            if (E != NONE64) {
                if (serial) {  // registrations back to idle; the rounds run every op
                    t.seg_cnt[E] = 0;
                    sc.op_word[j] = IDLE;
                } else {
                    const uint32_t c = t.seg_cnt[E];
                    if (c == 1) {
                        RegKey<KB> key;
                        removed += rx_probe<KB>(t, key, home_of<KB>(t, keys, j, key));
                        t.seg_cnt[E] = 0;
                        sc.op_word[j] = IDLE;
                    } else if (sc.op_flag[j]) {
                        cg = c;
                    }
                }
            }
        }
        // segments for the groups this warp leads: one atomic per warp
        uint32_t incl = cg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane >= o) incl += v;
        }
        const uint32_t tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint32_t wbase = 0;
        if (lane == 0 && tot) wbase = atomicAdd(&ctl->big_ops, tot);
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
        if (cg) t.seg_min[E] = wbase + incl - cg;
        append(sc.long_list, &ctl->nlong[0], j, cg != 0);
    }
    block_add_count(ctl, removed, s_tmp);
}

__global__ void __launch_bounds__(RBLOCK) k_rx_place(TableView t, uint32_t n0_arg, OpScratch sc, Ctl* ctl) {
    const uint32_t n0 = n0_arg != CMP_N0_CTL ? n0_arg : *(volatile const uint32_t*)&ctl->n0;
    if (*(volatile uint32_t*)&ctl->serial[0]) return;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n0; j += gridDim.x * blockDim.x) {
        const uint32_t place = sc.op_word[j];
        if (place == IDLE) continue;  // lone (already run) or no EMPTY slot
        const uint32_t at = t.seg_min[sc.op_slot[j]] + place;
        if (at < n0) sc.pend[0][at] = j;  // segments hold n0 words at most
        else atomicOr(&ctl->err, ERR_SCRATCH);
        sc.op_word[j] = IDLE;
    }
}

// The group pass: groups taken 32 at a time by a warp from a counter
// (Ctl::nlong[1], zero at the start of the call), one per lane.  A lane runs a
// group of at most RX_THREAD ops itself, one op after another in index order
// (each probe sees the ones before it); larger groups then run on the whole
// warp, one after another (rx_group_run), or go to the rounds above RX_GMAX.
template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rx_warp(TableView t, const uint8_t* __restrict__ keys, uint32_t n0_arg,
                                                    OpScratch sc, Ctl* ctl) {
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    __shared__ uint32_t s_grp[RBLOCK / 32][RX_GMAX];
    const uint32_t n0 = n0_arg != CMP_N0_CTL ? n0_arg : *(volatile const uint32_t*)&ctl->n0;
    const uint32_t n = *(volatile const uint32_t*)&ctl->nlong[0];
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t* grp = s_grp[threadIdx.x >> 5];
    uint32_t removed = 0;  // this lane's
    for (;;) {
        uint32_t i0 = 0;
        if (lane == 0) i0 = atomicAdd(&ctl->nlong[1], 32u);
        i0 = __shfl_sync(0xFFFFFFFFu, i0, 0);
        if (i0 >= n) break;
        const uint32_t i = i0 + lane;
        uint64_t E = NONE64;
        uint32_t c = 0, base = 0;
        bool bad = false;
        if (i < n) {
            E = sc.op_slot[sc.long_list[i]];
            c = t.seg_cnt[E];
            base = t.seg_min[E];
            bad = (uint64_t)base + c > n0;  // segments hold n0 words at most
            for (uint32_t q = 0; q < c && !bad; q++) {
                const uint32_t x = sc.pend[0][base + q];
                bad = x >= n0 || sc.op_slot[x] != E;  // a place this call did not fill
            }
            if (bad) atomicOr(&ctl->err, ERR_SCRATCH);  // the group is not run
        }
        if (!bad && c >= 2 && c <= RX_THREAD) {
            uint32_t ops[RX_THREAD];
            for (uint32_t q = 0; q < c; q++) {  // insertion sort: index order
                const uint32_t x = sc.pend[0][base + q];
                uint32_t k = q;
                while (k > 0 && ops[k - 1] > x) {
                    ops[k] = ops[k - 1];
                    --k;
                }
                ops[k] = x;
            }
            for (uint32_t q = 0; q < c; q++) {
                RegKey<KB> key;
                removed += rx_probe<KB>(t, key, home_of<KB>(t, keys, ops[q], key));
            }
        }
        // groups of up to RX_BMAX ops to the block pass (listed after the
        // groups in long_list; their registrations stay for it)
        const bool blk = !bad && c > RX_GMAX && c <= RX_BMAX;
        if (blk) sc.long_list[n + atomicAdd(&ctl->nbig, 1u)] = sc.long_list[i];
        // larger groups, one at a time on the whole warp
        for (uint32_t bm = __ballot_sync(0xFFFFFFFFu, !bad && !blk && c > RX_THREAD); bm; bm &= bm - 1) {
            const int L = __ffs(bm) - 1;
            const uint64_t EL = __shfl_sync(0xFFFFFFFFu, E, L);
            const uint32_t cL = __shfl_sync(0xFFFFFFFFu, c, L);
            const uint32_t bL = __shfl_sync(0xFFFFFFFFu, base, L);
            const uint32_t* seg = sc.pend[0] + bL;
            const bool over = cL > RX_GMAX;  // too many for a block: to the rounds
            uint32_t at = 0;
            if (over && lane == 0) at = atomicAdd(&ctl->npend[1], cL);
            at = __shfl_sync(0xFFFFFFFFu, at, 0);
            for (uint32_t q = lane; q < cL; q += 32) {
                if (over) sc.pend[1][at + q] = seg[q];
                else grp[q] = seg[q];
            }
            __syncwarp();
            const uint32_t r = rx_group_run<KB>(t, keys, EL, over ? 0u : cL, grp);
            if (lane == 0) removed += r;
        }
        if (i < n && !blk) {
            t.seg_min[E] = IDLE;
            t.seg_cnt[E] = 0;
        }
    }
    block_add_count(ctl, removed, s_tmp);
}

// The block pass: groups of RX_GMAX..RX_BMAX ops (listed by the group pass
// after its own entries, Ctl::nbig of them), taken one at a time per block
// from Ctl::big_next; each is sorted into index order in shared memory and
// run by warp 0 in chunks of 32 (rx_chunk32).
template <int KB>
__global__ void __launch_bounds__(RBLOCK) k_rx_big(TableView t, const uint8_t* __restrict__ keys, uint32_t n0_arg,
                                                   OpScratch sc, Ctl* ctl) {
    __shared__ uint32_t s_list[RX_BMAX];
    __shared__ uint32_t s_tmp[RBLOCK / 32];
    __shared__ uint32_t s_k;
    const uint32_t n0 = n0_arg != CMP_N0_CTL ? n0_arg : *(volatile const uint32_t*)&ctl->n0;
    const uint32_t n = *(volatile const uint32_t*)&ctl->nlong[0];
    const uint32_t nb = *(volatile const uint32_t*)&ctl->nbig;
    uint32_t removed = 0;
    for (;;) {
        if (threadIdx.x == 0) s_k = atomicAdd(&ctl->big_next, 1u);
        __syncthreads();
        const uint32_t k = s_k;
        __syncthreads();  // every thread has read s_k
        if (k >= nb) break;
        const uint64_t E = sc.op_slot[sc.long_list[n + k]];
        const uint32_t c = t.seg_cnt[E];
        const uint32_t base = t.seg_min[E];
        if (c > RX_BMAX || (uint64_t)base + c > n0) {  // not a group the group pass listed
            if (threadIdx.x == 0) atomicOr(&ctl->err, ERR_SCRATCH);
            continue;
        }
        for (uint32_t q = threadIdx.x; q < c; q += blockDim.x) {
            const uint32_t x = sc.pend[0][base + q];
            s_list[q] = x < n0 ? x : 0xFFFFFFFFu;  // out of range: flagged below
        }
        __syncthreads();
        block_sort_u32(s_list, c);
        // every entry valid and of this group (a sorted list of distinct ops:
        // the largest entry is in range)
        if (threadIdx.x < 32) {
            bool bad = s_list[c - 1] >= n0;
            for (uint32_t q = threadIdx.x; q < c && !bad; q += 32) bad = sc.op_slot[s_list[q]] != E;
            bad = __any_sync(0xFFFFFFFFu, bad);
            if (bad) {
                if (threadIdx.x == 0) atomicOr(&ctl->err, ERR_SCRATCH);
            } else {
                for (uint32_t q = 0; q < c; q += 32) {
                    const uint32_t r = rx_chunk32<KB>(t, keys, s_list + q, min(32u, c - q));
                    if (threadIdx.x == 0) removed += r;
                }
            }
            if (threadIdx.x == 0) {
                t.seg_min[E] = IDLE;
                t.seg_cnt[E] = 0;
            }
        }
        __syncthreads();
    }
    block_add_count(ctl, removed, s_tmp);
}

template <int KB>
void direct_shape(const TableView& t, const uint8_t* keys, uint32_t n0, uint32_t nmax, const OpScratch& sc, Ctl* ctl,
                  cudaStream_t s) {
    const unsigned g = grid_for(nmax, 8);
    {
        KtScope kt(KC_REM_MARK, s);
        k_rx_find<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, sc, ctl);
    }
    {
        KtScope kt(KC_REM_EXEC, s);
        k_rx_exec<KB><<<g, RBLOCK, 0, s>>>(t, keys, n0, sc, ctl);
    }
    {
        KtScope kt(KC_REM_GROUP, s);  // a lane per group, as many warps as can be resident
        k_rx_place<<<g, RBLOCK, 0, s>>>(t, n0, sc, ctl);
        k_rx_warp<KB><<<grid_for(nmax, 8), RBLOCK, 0, s>>>(t, keys, n0, sc, ctl);
        k_rx_big<KB><<<grid_for((uint64_t)nmax * 256 / (RX_GMAX + 1), 2), RBLOCK, 0, s>>>(t, keys, n0, sc, ctl);
    }
    count_launches(5);
}

}  // namespace

cudaError_t launch_rem_rounds(const TableView& t, Shape sh, const uint8_t* keys, uint32_t n0, uint32_t r0,
                              uint32_t nrounds, uint32_t grid_ops, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    switch (sh) {
        case SHAPE_8_8:
        case SHAPE_8_32: rounds_shape<8>(t, keys, n0, r0, nrounds, grid_ops, sc, ctl, s); break;
        case SHAPE_32_128:
        case SHAPE_32_64:
        case SHAPE_32_32: rounds_shape<32>(t, keys, n0, r0, nrounds, grid_ops, sc, ctl, s); break;
        default: rounds_shape<0>(t, keys, n0, r0, nrounds, grid_ops, sc, ctl, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_grp_rem(Shape sh, const GroupOp* ops, uint32_t nops, uint64_t sum_n, int phase, uint32_t r0,
                           uint32_t nrounds, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
    switch (sh) {
        case SHAPE_8_8:
        case SHAPE_8_32: grp_rem_shape<8>(ops, nops, sum_n, phase, r0, nrounds, s); break;
        case SHAPE_32_128:
        case SHAPE_32_64:
        case SHAPE_32_32: grp_rem_shape<32>(ops, nops, sum_n, phase, r0, nrounds, s); break;
        default: grp_rem_shape<0>(ops, nops, sum_n, phase, r0, nrounds, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_rem_direct(const TableView& t, Shape sh, const uint8_t* keys, uint32_t n0, const OpScratch& sc,
                              Ctl* ctl, cudaStream_t s) {
    switch (sh) {
        case SHAPE_8_8:
        case SHAPE_8_32: direct_shape<8>(t, keys, n0, n0, sc, ctl, s); break;
        case SHAPE_32_128:
        case SHAPE_32_64:
        case SHAPE_32_32: direct_shape<32>(t, keys, n0, n0, sc, ctl, s); break;
        default: direct_shape<0>(t, keys, n0, n0, sc, ctl, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_rem_direct_ctl(const TableView& t, Shape sh, const uint8_t* keys, uint32_t nmax,
                                  const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    switch (sh) {
        case SHAPE_8_8:
        case SHAPE_8_32: direct_shape<8>(t, keys, CMP_N0_CTL, nmax, sc, ctl, s); break;
        case SHAPE_32_128:
        case SHAPE_32_64:
        case SHAPE_32_32: direct_shape<32>(t, keys, CMP_N0_CTL, nmax, sc, ctl, s); break;
        default: direct_shape<0>(t, keys, CMP_N0_CTL, nmax, sc, ctl, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_rem_summary(const TableView& t, const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    // chunks are whole (capacity >= 32) and depths stay below the 28-bit
    // stored distance, so a depth compares exactly with the largest one
    if (!sc.rsum || t.mask < 31 || t.mask >= (1ull << 28)) return cudaSuccess;
    const uint64_t nch = rsum_chunks(t.mask);
    k_rem_sum<<<(unsigned)((nch + 255) / 256), 256, 0, s>>>(t, sc, ctl);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_rem_tail(const TableView& t, Shape sh, const uint8_t* keys, uint32_t n0, uint32_t r,
                            const OpScratch& sc, Ctl* ctl, cudaStream_t s) {
    KtScope kt(KC_REM_TAIL, s);
    switch (sh) {
        case SHAPE_8_8:
        case SHAPE_8_32: k_rem_tail<8><<<1, TAIL_THREADS, 0, s>>>(t, keys, n0, r, sc, ctl); break;
        case SHAPE_32_128:
        case SHAPE_32_64:
        case SHAPE_32_32: k_rem_tail<32><<<1, TAIL_THREADS, 0, s>>>(t, keys, n0, r, sc, ctl); break;
        default: k_rem_tail<0><<<1, TAIL_THREADS, 0, s>>>(t, keys, n0, r, sc, ctl); break;
    }
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace fm

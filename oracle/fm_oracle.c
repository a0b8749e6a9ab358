/*
 * fm_oracle.c -- CPU restatement of FlashMap's bulk semantics (TEST
 * INFRASTRUCTURE ONLY; see fm_oracle.h).
 *
 * The sequential functions restate src/rayon_cpu.rs of bajpainaman/flash-map
 * 0.5.0 with each bulk call applied one operation at a time in batch index
 * order.  With one thread every CAS in that file succeeds at the first try and
 * no slot is ever seen in the INSERTING state, so the CAS protocol reduces to
 * plain stores.  Line citations are to the reference files.
 */
#define _GNU_SOURCE
#include "fm_oracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

struct fmo_table {
    uint64_t capacity;
    uint64_t mask;
    uint32_t ksz, vsz, mode;
    uint32_t* flags;
    uint8_t* keys;
    uint8_t* vals;
    uint64_t len;
    int acct;
    int limit_hit;
    fmo_traffic traffic[3];
};

/* ---- flag word (src/rayon_cpu.rs:28-41) ---------------------------------- */
static inline uint32_t st_of(uint32_t f) { return f & 0xFu; }
static inline uint64_t dist_of(uint32_t f) { return (uint64_t)(f >> 4); }
/* make_flag truncates dist to u32 and shifts it left by 4 (rayon_cpu.rs:39-41). */
static inline uint32_t mk(uint32_t state, uint64_t dist) {
    return (((uint32_t)dist) << 4) | (state & 0xFu);
}

/* ---- hashes (src/hash.rs:30-86) ------------------------------------------ */
uint64_t fmo_identity_hash(const uint8_t* key, uint32_t ksz) {
    /* hash.rs:32-39: first min(8, len) bytes as a little-endian u64. */
    uint64_t h = 0;
    uint32_t n = ksz < 8 ? ksz : 8;
    for (uint32_t i = 0; i < n; i++) h |= (uint64_t)key[i] << (8 * i);
    return h;
}

uint64_t fmo_murmur3_hash(const uint8_t* key, uint32_t ksz) {
    /* hash.rs:43-77: per 8-byte chunk a two-round multiply/xorshift mix folded
     * by h = h*5 + 0x52dce729; the tail is folded only when it is non-zero or
     * the length is not a multiple of 8; then the length is xored in and the
     * 64-bit finaliser applied.  All arithmetic wraps modulo 2^64. */
    uint64_t h = 0x9e3779b97f4a7c15ull;
    uint32_t chunks = ksz / 8;
    for (uint32_t c = 0; c < chunks; c++) {
        uint64_t k = 0;
        for (uint32_t i = 0; i < 8; i++) k |= (uint64_t)key[c * 8 + i] << (8 * i);
        k *= 0xff51afd7ed558ccdull;
        k ^= k >> 33;
        k *= 0xc4ceb9fe1a85ec53ull;
        k ^= k >> 33;
        h ^= k;
        h = h * 5 + 0x52dce729ull;
    }
    uint64_t rem = 0;
    for (uint32_t i = chunks * 8; i < ksz; i++) rem |= (uint64_t)key[i] << (8 * (i - chunks * 8));
    if (rem != 0 || ksz % 8 != 0) {
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

uint64_t fmo_hash(const uint8_t* key, uint32_t ksz, uint32_t mode) {
    /* hash.rs:81-86 and HashStrategy::to_mode (hash.rs:22-27): 0 identity, 1 murmur3. */
    return mode == 0 ? fmo_identity_hash(key, ksz) : fmo_murmur3_hash(key, ksz);
}

/* ---- capacity / lifetime ------------------------------------------------- */
static uint64_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

int fmo_capacity_for(uint64_t req, int rule, uint64_t* out) {
    if (rule == 0) {
        if (req == 0) return FMO_ERR_ZERO_CAPACITY; /* gpu.rs:50-52 */
        *out = next_pow2(req);                     /* gpu.rs:54 */
    } else {
        *out = next_pow2(req < 16 ? 16 : req);     /* rayon_cpu.rs:64 */
    }
    return FMO_OK;
}

fmo_table* fmo_create(uint64_t cap, uint32_t ksz, uint32_t vsz, uint32_t mode) {
    if (cap == 0 || (cap & (cap - 1)) != 0) return NULL;
    fmo_table* t = (fmo_table*)calloc(1, sizeof(fmo_table));
    if (!t) return NULL;
    t->capacity = cap;
    t->mask = cap - 1;
    t->ksz = ksz;
    t->vsz = vsz;
    t->mode = mode;
    t->flags = (uint32_t*)calloc(cap, sizeof(uint32_t));
    t->keys = (uint8_t*)calloc(cap, ksz ? ksz : 1);
    t->vals = (uint8_t*)calloc(cap, vsz ? vsz : 1);
    if (!t->flags || !t->keys || !t->vals) {
        fmo_destroy(t);
        return NULL;
    }
    return t;
}

void fmo_destroy(fmo_table* t) {
    if (!t) return;
    free(t->flags);
    free(t->keys);
    free(t->vals);
    free(t);
}

uint64_t fmo_len(const fmo_table* t) { return t->len; }
uint64_t fmo_capacity(const fmo_table* t) { return t->capacity; }
uint32_t* fmo_flags(fmo_table* t) { return t->flags; }
uint8_t* fmo_keys(fmo_table* t) { return t->keys; }
uint8_t* fmo_values(fmo_table* t) { return t->vals; }
void fmo_set_len(fmo_table* t, uint64_t len) { t->len = len; }

/* ---- traffic accounting --------------------------------------------------
 * Distinct 32-byte sectors an operation must touch: the flag words of every
 * probed slot, keys only where a match is possible (a stored key can equal the
 * probing key only when its dist equals the current probe depth), values read
 * or written, and every displaced entry moved.  Reads and writes count apart. */
#define SET_CAP 4096
typedef struct sset {
    uint64_t v[SET_CAP];
    int n;
    int overflow;
} sset;

typedef struct acct_op {
    sset rd, wr;
} acct_op;

static acct_op g_acct; /* single-threaded oracle use only */

static void sset_add(sset* s, uint64_t id) {
    for (int i = 0; i < s->n; i++)
        if (s->v[i] == id) return;
    if (s->n < SET_CAP) s->v[s->n++] = id;
    else s->overflow++;
}

/* region tag in the top bits keeps flag/key/value sectors apart */
static void acct_range(fmo_table* t, sset* s, int region, uint64_t slot, uint32_t width) {
    if (!t->acct || width == 0) return;
    uint64_t b0 = slot * width, b1 = b0 + width - 1;
    for (uint64_t sec = b0 / 32; sec <= b1 / 32; sec++) sset_add(s, ((uint64_t)region << 60) | sec);
}
#define ACCT_FLAG_R(t, s) acct_range(t, &g_acct.rd, 0, s, 4)
#define ACCT_FLAG_W(t, s) acct_range(t, &g_acct.wr, 0, s, 4)
#define ACCT_KEY_R(t, s) acct_range(t, &g_acct.rd, 1, s, (t)->ksz)
#define ACCT_KEY_W(t, s) acct_range(t, &g_acct.wr, 1, s, (t)->ksz)
#define ACCT_VAL_R(t, s) acct_range(t, &g_acct.rd, 2, s, (t)->vsz)
#define ACCT_VAL_W(t, s) acct_range(t, &g_acct.wr, 2, s, (t)->vsz)

static void acct_begin(fmo_table* t) {
    if (!t->acct) return;
    g_acct.rd.n = g_acct.wr.n = 0;
}
static void acct_end(fmo_table* t, int kind, uint64_t in_bytes, uint64_t out_bytes) {
    if (!t->acct) return;
    fmo_traffic* tr = &t->traffic[kind];
    tr->ops++;
    tr->table_sectors_read += (uint64_t)g_acct.rd.n;
    tr->table_sectors_written += (uint64_t)g_acct.wr.n;
    tr->stream_bytes_in += in_bytes;
    tr->stream_bytes_out += out_bytes;
}

void fmo_traffic_enable(fmo_table* t, int on) { t->acct = on; }
void fmo_traffic_get(const fmo_table* t, int kind, fmo_traffic* out) { *out = t->traffic[kind]; }
void fmo_traffic_reset(fmo_table* t) { memset(t->traffic, 0, sizeof(t->traffic)); }

/* ---- sequential operations ---------------------------------------------- */

static inline const uint8_t* key_at(const fmo_table* t, uint64_t i) { return t->keys + i * t->ksz; }
static inline uint8_t* keyw_at(fmo_table* t, uint64_t i) { return t->keys + i * t->ksz; }
static inline uint8_t* val_at(fmo_table* t, uint64_t i) { return t->vals + i * t->vsz; }

/* One lookup: src/rayon_cpu.rs:85-122.  Returns the slot holding the key or
 * UINT64_MAX.  The Robin Hood exit (p > dist) is tested before the key compare
 * (rayon_cpu.rs:107-116); tombstones are skipped (rayon_cpu.rs:118-119). */
static uint64_t seq_find(fmo_table* t, const uint8_t* qk) {
    uint64_t slot = fmo_hash(qk, t->ksz, t->mode) & t->mask;
    uint64_t p = 0;
    while (p <= t->mask) {
        uint64_t idx = (slot + p) & t->mask;
        uint32_t f = t->flags[idx];
        ACCT_FLAG_R(t, idx);
        uint32_t st = st_of(f);
        uint64_t dist = dist_of(f);
        if (st == FMO_EMPTY) return UINT64_MAX;
        if (st == FMO_OCCUPIED) {
            if (p > dist) return UINT64_MAX;
            if (dist == p) ACCT_KEY_R(t, idx); /* only slots that can hold the key */
            if (memcmp(key_at(t, idx), qk, t->ksz) == 0) return idx;
        }
        p++;
    }
    return UINT64_MAX;
}

void fmo_bulk_get(fmo_table* t, const uint8_t* keys, uint64_t n, uint8_t* out_values,
                  uint8_t* out_found) {
    for (uint64_t i = 0; i < n; i++) {
        acct_begin(t);
        uint64_t s = seq_find(t, keys + i * t->ksz);
        uint8_t* ov = out_values ? out_values + i * t->vsz : NULL;
        if (s != UINT64_MAX) {
            ACCT_VAL_R(t, s);
            if (ov) memcpy(ov, val_at(t, s), t->vsz);
            if (out_found) out_found[i] = 1;
        } else {
            if (ov) memset(ov, 0, t->vsz); /* misses read as zero (gpu.rs:126-134) */
            if (out_found) out_found[i] = 0;
        }
        acct_end(t, 0, t->ksz, (uint64_t)t->vsz + 1);
    }
}

/* One insert: src/rayon_cpu.rs:153-265 run by a single thread.  Returns 1 when
 * a free (EMPTY or TOMBSTONE) slot was claimed, 0 for an in-place update, for an
 * evicted entry merged into an equal key further on, or for a drop when the
 * probe passes the capacity (rayon_cpu.rs:167-169). */
static int seq_insert_one(fmo_table* t, const uint8_t* key, const uint8_t* val, uint8_t* ck,
                          uint8_t* cv, uint8_t* tk, uint8_t* tv) {
    memcpy(ck, key, t->ksz);
    memcpy(cv, val, t->vsz);
    uint64_t home = fmo_hash(ck, t->ksz, t->mode) & t->mask;
    uint64_t p = 0;
    /* The reference's loop has no bound: on a table with no free slot (only
     * reachable through the uncounted insert) the walk can cycle forever.
     * Both this oracle and the GPU backend stop after 2*capacity+2 slots,
     * drop the carried entry and report ProbeLimit. */
    const uint64_t step_limit = 2 * t->capacity + 2;
    for (uint64_t step = 0;; ++step) {
        if (p > t->mask) return 0;
        if (step > step_limit) {
            t->limit_hit = 1;
            return 0;
        }
        uint64_t idx = (home + p) & t->mask;
        uint32_t f = t->flags[idx];
        ACCT_FLAG_R(t, idx);
        uint32_t st = st_of(f);
        uint64_t dist = dist_of(f);
        if (st == FMO_OCCUPIED) {
            if (dist == p) ACCT_KEY_R(t, idx);
            if (memcmp(key_at(t, idx), ck, t->ksz) == 0) {
                /* rayon_cpu.rs:178-182: update in place */
                memcpy(val_at(t, idx), cv, t->vsz);
                ACCT_VAL_W(t, idx);
                return 0;
            }
            if (p > dist) {
                /* rayon_cpu.rs:184-217: evict the resident and carry it on */
                ACCT_KEY_R(t, idx);
                ACCT_VAL_R(t, idx);
                memcpy(tk, key_at(t, idx), t->ksz);
                memcpy(tv, val_at(t, idx), t->vsz);
                memcpy(keyw_at(t, idx), ck, t->ksz);
                memcpy(val_at(t, idx), cv, t->vsz);
                t->flags[idx] = mk(FMO_OCCUPIED, p);
                ACCT_KEY_W(t, idx);
                ACCT_VAL_W(t, idx);
                ACCT_FLAG_W(t, idx);
                memcpy(ck, tk, t->ksz);
                memcpy(cv, tv, t->vsz);
                home = fmo_hash(ck, t->ksz, t->mode) & t->mask;
                p = dist + 1;
                continue;
            }
            p++;
            continue;
        }
        if (st == FMO_EMPTY || st == FMO_TOMBSTONE) {
            /* rayon_cpu.rs:228-251: claim the first free slot */
            memcpy(keyw_at(t, idx), ck, t->ksz);
            memcpy(val_at(t, idx), cv, t->vsz);
            t->flags[idx] = mk(FMO_OCCUPIED, p);
            ACCT_KEY_W(t, idx);
            ACCT_VAL_W(t, idx);
            ACCT_FLAG_W(t, idx);
            return 1;
        }
        p++; /* INSERTING never occurs sequentially; other states skip (rayon_cpu.rs:263) */
    }
}

static uint64_t seq_insert_all(fmo_table* t, const uint8_t* keys, const uint8_t* values,
                               uint64_t n) {
    uint32_t kb = t->ksz ? t->ksz : 1, vb = t->vsz ? t->vsz : 1;
    uint8_t* buf = (uint8_t*)malloc(2 * (size_t)kb + 2 * (size_t)vb);
    uint8_t *ck = buf, *tk = buf + kb, *cv = buf + 2 * kb, *tv = buf + 2 * kb + vb;
    uint64_t added = 0;
    for (uint64_t i = 0; i < n; i++) {
        acct_begin(t);
        added += (uint64_t)seq_insert_one(t, keys + i * t->ksz, values + i * t->vsz, ck, cv, tk, tv);
        acct_end(t, 1, (uint64_t)t->ksz + t->vsz, 0);
    }
    free(buf);
    return added;
}

int fmo_bulk_insert(fmo_table* t, const uint8_t* keys, const uint8_t* values, uint64_t n,
                    uint64_t* num_new) {
    *num_new = 0;
    if (n == 0) return FMO_OK; /* gpu.rs:194-196 */
    /* Precheck before any mutation: len + n > capacity * 1.0 (gpu.rs:198-206). */
    if (t->len + n > t->capacity) return FMO_ERR_TABLE_FULL;
    t->limit_hit = 0;
    uint64_t added = seq_insert_all(t, keys, values, n);
    t->len += added; /* rayon_cpu.rs:267-269 */
    *num_new = added;
    return t->limit_hit ? FMO_ERR_PROBE_LIMIT : FMO_OK;
}

int fmo_bulk_insert_uncounted(fmo_table* t, const uint8_t* keys, const uint8_t* values,
                              uint64_t n) {
    if (n == 0) return FMO_OK;
    t->limit_hit = 0;
    (void)seq_insert_all(t, keys, values, n);
    t->len += n; /* gpu.rs:670: assumes every key is new */
    return t->limit_hit ? FMO_ERR_PROBE_LIMIT : FMO_OK;
}

/* One remove: src/rayon_cpu.rs:276-323.  The first live match before a
 * terminator becomes the whole word TOMBSTONE (dist 0, rayon_cpu.rs:306-313). */
uint64_t fmo_bulk_remove(fmo_table* t, const uint8_t* keys, uint64_t n) {
    uint64_t removed = 0;
    for (uint64_t i = 0; i < n; i++) {
        acct_begin(t);
        uint64_t s = seq_find(t, keys + i * t->ksz);
        if (s != UINT64_MAX) {
            t->flags[s] = FMO_TOMBSTONE;
            ACCT_FLAG_W(t, s);
            removed++;
        }
        acct_end(t, 2, t->ksz, 0);
    }
    t->len -= removed; /* rayon_cpu.rs:325-327 */
    return removed;
}

void fmo_clear(fmo_table* t) {
    /* rayon_cpu.rs:347-353 / kernels.cu:319-326: flags reset, keys and values
     * left as they were. */
    memset(t->flags, 0, t->capacity * sizeof(uint32_t));
    t->len = 0;
}

uint64_t fmo_recount(fmo_table* t) {
    /* kernels.cu:328-337 + gpu.rs:677-712: count OCCUPIED slots, len := count */
    uint64_t c = 0;
    for (uint64_t i = 0; i < t->capacity; i++) c += st_of(t->flags[i]) == FMO_OCCUPIED;
    t->len = c;
    return c;
}

/* ---- multithreaded CAS restatement (timing baseline) --------------------
 * Mirrors rayon_cpu.rs: AtomicU32 flags, CAS to claim or evict, spin on
 * INSERTING, plain (racy) key/value writes published by a release store. */
typedef struct mt_job {
    fmo_table* t;
    const uint8_t* keys;
    const uint8_t* vals;
    uint8_t* out_vals;
    uint8_t* out_found;
    uint64_t n;
    _Atomic uint64_t next;
    _Atomic uint64_t count;
    int kind;
} mt_job;

#define MT_CHUNK 1024

static inline uint32_t aload(uint32_t* p) {
    return atomic_load_explicit((_Atomic uint32_t*)p, memory_order_acquire);
}
static inline int acas(uint32_t* p, uint32_t expect, uint32_t desired) {
    return atomic_compare_exchange_strong_explicit((_Atomic uint32_t*)p, &expect, desired,
                                                   memory_order_acq_rel, memory_order_relaxed);
}
static inline void astore(uint32_t* p, uint32_t v) {
    atomic_store_explicit((_Atomic uint32_t*)p, v, memory_order_release);
}

static uint64_t mt_find(fmo_table* t, const uint8_t* qk) {
    uint64_t slot = fmo_hash(qk, t->ksz, t->mode) & t->mask;
    uint64_t p = 0;
    while (p <= t->mask) {
        uint64_t idx = (slot + p) & t->mask;
        uint32_t f = aload(&t->flags[idx]);
        uint32_t st = st_of(f);
        uint64_t dist = dist_of(f);
        if (st == FMO_EMPTY) return UINT64_MAX;
        if (st == FMO_INSERTING) continue;
        if (st == FMO_OCCUPIED) {
            if (p > dist) return UINT64_MAX;
            if (memcmp(key_at(t, idx), qk, t->ksz) == 0) return idx;
        }
        p++;
    }
    return UINT64_MAX;
}

static int mt_insert_one(fmo_table* t, const uint8_t* key, const uint8_t* val, uint8_t* ck,
                         uint8_t* cv, uint8_t* tk, uint8_t* tv) {
    memcpy(ck, key, t->ksz);
    memcpy(cv, val, t->vsz);
    uint64_t home = fmo_hash(ck, t->ksz, t->mode) & t->mask;
    uint64_t p = 0;
    const uint64_t step_limit = 2 * t->capacity + 2;
    for (uint64_t step = 0;; ++step) {
        if (p > t->mask || step > step_limit) return 0;
        uint64_t idx = (home + p) & t->mask;
        uint32_t f = aload(&t->flags[idx]);
        uint32_t st = st_of(f);
        uint64_t dist = dist_of(f);
        if (st == FMO_OCCUPIED) {
            if (memcmp(key_at(t, idx), ck, t->ksz) == 0) {
                memcpy(val_at(t, idx), cv, t->vsz);
                return 0;
            }
            if (p > dist) {
                if (acas(&t->flags[idx], f, mk(FMO_INSERTING, p))) {
                    memcpy(tk, key_at(t, idx), t->ksz);
                    memcpy(tv, val_at(t, idx), t->vsz);
                    memcpy(keyw_at(t, idx), ck, t->ksz);
                    memcpy(val_at(t, idx), cv, t->vsz);
                    astore(&t->flags[idx], mk(FMO_OCCUPIED, p));
                    memcpy(ck, tk, t->ksz);
                    memcpy(cv, tv, t->vsz);
                    home = fmo_hash(ck, t->ksz, t->mode) & t->mask;
                    p = dist + 1;
                }
                continue;
            }
            p++;
            continue;
        }
        if (st == FMO_EMPTY || st == FMO_TOMBSTONE) {
            if (acas(&t->flags[idx], f, mk(FMO_INSERTING, p))) {
                memcpy(keyw_at(t, idx), ck, t->ksz);
                memcpy(val_at(t, idx), cv, t->vsz);
                astore(&t->flags[idx], mk(FMO_OCCUPIED, p));
                return 1;
            }
            continue;
        }
        if (st == FMO_INSERTING) continue;
        p++;
    }
}

static void* mt_worker(void* arg) {
    mt_job* j = (mt_job*)arg;
    fmo_table* t = j->t;
    uint32_t kb = t->ksz ? t->ksz : 1, vb = t->vsz ? t->vsz : 1;
    uint8_t* buf = (uint8_t*)malloc(2 * (size_t)kb + 2 * (size_t)vb);
    uint8_t *ck = buf, *tk = buf + kb, *cv = buf + 2 * kb, *tv = buf + 2 * kb + vb;
    uint64_t local = 0;
    for (;;) {
        uint64_t b = atomic_fetch_add(&j->next, MT_CHUNK);
        if (b >= j->n) break;
        uint64_t e = b + MT_CHUNK < j->n ? b + MT_CHUNK : j->n;
        for (uint64_t i = b; i < e; i++) {
            const uint8_t* k = j->keys + i * t->ksz;
            if (j->kind == 0) {
                uint64_t s = mt_find(t, k);
                if (s != UINT64_MAX) {
                    memcpy(j->out_vals + i * t->vsz, val_at(t, s), t->vsz);
                    j->out_found[i] = 1;
                } else {
                    memset(j->out_vals + i * t->vsz, 0, t->vsz);
                    j->out_found[i] = 0;
                }
            } else if (j->kind == 1) {
                local += (uint64_t)mt_insert_one(t, k, j->vals + i * t->vsz, ck, cv, tk, tv);
            } else {
                /* rayon_cpu.rs:298-318: CAS the matched flag to TOMBSTONE */
                uint64_t slot = fmo_hash(k, t->ksz, t->mode) & t->mask;
                uint64_t p = 0;
                while (p <= t->mask) {
                    uint64_t idx = (slot + p) & t->mask;
                    uint32_t f = aload(&t->flags[idx]);
                    uint32_t st = st_of(f);
                    if (st == FMO_EMPTY) break;
                    if (st == FMO_INSERTING) continue;
                    if (st == FMO_OCCUPIED) {
                        if (p > dist_of(f)) break;
                        if (memcmp(key_at(t, idx), k, t->ksz) == 0) {
                            if (acas(&t->flags[idx], f, FMO_TOMBSTONE)) local++;
                            break;
                        }
                    }
                    p++;
                }
            }
        }
    }
    atomic_fetch_add(&j->count, local);
    free(buf);
    return NULL;
}

static uint64_t mt_run(fmo_table* t, int kind, const uint8_t* keys, const uint8_t* vals,
                       uint64_t n, uint8_t* ov, uint8_t* of, int threads) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    mt_job j;
    j.t = t;
    j.keys = keys;
    j.vals = vals;
    j.out_vals = ov;
    j.out_found = of;
    j.n = n;
    j.kind = kind;
    atomic_init(&j.next, 0);
    atomic_init(&j.count, 0);
    pthread_t th[256];
    for (int i = 1; i < threads; i++) pthread_create(&th[i], NULL, mt_worker, &j);
    mt_worker(&j);
    for (int i = 1; i < threads; i++) pthread_join(th[i], NULL);
    return atomic_load(&j.count);
}

int fmo_mt_bulk_insert(fmo_table* t, const uint8_t* keys, const uint8_t* values, uint64_t n,
                       uint64_t* num_new, int threads) {
    *num_new = 0;
    if (n == 0) return FMO_OK;
    if (t->len + n > t->capacity) return FMO_ERR_TABLE_FULL;
    uint64_t added = mt_run(t, 1, keys, values, n, NULL, NULL, threads);
    t->len += added;
    *num_new = added;
    return FMO_OK;
}

void fmo_mt_bulk_get(fmo_table* t, const uint8_t* keys, uint64_t n, uint8_t* out_values,
                     uint8_t* out_found, int threads) {
    if (n == 0) return;
    (void)mt_run(t, 0, keys, NULL, n, out_values, out_found, threads);
}

uint64_t fmo_mt_bulk_remove(fmo_table* t, const uint8_t* keys, uint64_t n, int threads) {
    if (n == 0) return 0;
    uint64_t r = mt_run(t, 2, keys, NULL, n, NULL, NULL, threads);
    t->len -= r;
    return r;
}

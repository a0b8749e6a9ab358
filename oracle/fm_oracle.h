/*
 * fm_oracle.h -- CPU restatement of FlashMap's bulk semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * backend: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it.  The product library (libflashmap_b200.so) never links it.
 *
 * Two restatements live here:
 *   - the sequential oracle ("cpu-fallback" semantics): the reference's
 *     Rayon backend (src/rayon_cpu.rs:82-328) with every bulk call applied
 *     one operation at a time in batch index order, which is what a
 *     one-thread rayon pool does;
 *   - a multithreaded CAS restatement of the same file (the "rayon" stand-in),
 *     used only as a timed CPU baseline: like the reference it is racy and its
 *     layout is not deterministic under in-batch conflicts.
 */
#ifndef FM_ORACLE_H
#define FM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flag word: (dist << 4) | state  (src/rayon_cpu.rs:23-41, src/kernels.cu:23-30) */
#define FMO_EMPTY 0u
#define FMO_OCCUPIED 1u
#define FMO_TOMBSTONE 2u
#define FMO_INSERTING 3u

#define FMO_OK 0
#define FMO_ERR_TABLE_FULL 5
#define FMO_ERR_ZERO_CAPACITY 6
#define FMO_ERR_PROBE_LIMIT 9

typedef struct fmo_table fmo_table;

/* Per-op-type algorithmic traffic, in 32-byte sectors (reads and writes of the
 * table counted separately) plus streamed input/output bytes. */
typedef struct fmo_traffic {
    uint64_t ops;
    uint64_t table_sectors_read;
    uint64_t table_sectors_written;
    uint64_t stream_bytes_in;
    uint64_t stream_bytes_out;
} fmo_traffic;

/* Capacity rules: rule 0 = src/gpu.rs:50-54 (0 -> ZeroCapacity, else
 * next_power_of_two); rule 1 = src/rayon_cpu.rs:64 (max(16).next_power_of_two). */
int fmo_capacity_for(uint64_t requested, int rule, uint64_t* out_capacity);

fmo_table* fmo_create(uint64_t capacity_pow2, uint32_t key_size, uint32_t value_size,
                      uint32_t hash_mode);
void fmo_destroy(fmo_table* t);

uint64_t fmo_hash(const uint8_t* key, uint32_t key_size, uint32_t mode);
uint64_t fmo_identity_hash(const uint8_t* key, uint32_t key_size);
uint64_t fmo_murmur3_hash(const uint8_t* key, uint32_t key_size);

/* Sequential bulk operations (index order). */
int fmo_bulk_insert(fmo_table* t, const uint8_t* keys, const uint8_t* values, uint64_t n,
                    uint64_t* num_new);
void fmo_bulk_get(fmo_table* t, const uint8_t* keys, uint64_t n, uint8_t* out_values,
                  uint8_t* out_found);
uint64_t fmo_bulk_remove(fmo_table* t, const uint8_t* keys, uint64_t n);
void fmo_clear(fmo_table* t);
/* Device-path insert without the load-factor precheck: len += n (src/gpu.rs:618-672). */
int fmo_bulk_insert_uncounted(fmo_table* t, const uint8_t* keys, const uint8_t* values,
                              uint64_t n);
uint64_t fmo_recount(fmo_table* t);

uint64_t fmo_len(const fmo_table* t);
uint64_t fmo_capacity(const fmo_table* t);

/* Raw state access, for layout comparisons and for uploading prefilled tables. */
uint32_t* fmo_flags(fmo_table* t);
uint8_t* fmo_keys(fmo_table* t);
uint8_t* fmo_values(fmo_table* t);
void fmo_set_len(fmo_table* t, uint64_t len);

/* Traffic accounting: kind 0 = get, 1 = insert, 2 = remove. */
void fmo_traffic_enable(fmo_table* t, int on);
void fmo_traffic_get(const fmo_table* t, int kind, fmo_traffic* out);
void fmo_traffic_reset(fmo_table* t);

/* Multithreaded CAS restatement of src/rayon_cpu.rs (timing baseline only). */
int fmo_mt_bulk_insert(fmo_table* t, const uint8_t* keys, const uint8_t* values, uint64_t n,
                       uint64_t* num_new, int threads);
void fmo_mt_bulk_get(fmo_table* t, const uint8_t* keys, uint64_t n, uint8_t* out_values,
                     uint8_t* out_found, int threads);
uint64_t fmo_mt_bulk_remove(fmo_table* t, const uint8_t* keys, uint64_t n, int threads);

#ifdef __cplusplus
}
#endif
#endif

/*
 * flashmap_b200.h -- C ABI of the FlashMap B200 backend (libflashmap_b200.so).
 *
 * This ABI replaces the reference's src/gpu.rs (bajpainaman/flash-map 0.5.0):
 * each entry point below is what a thin Rust `GpuFlashMap<K, V>` shim binds so
 * that src/lib.rs (FlashMap / FlashMapBuilder) and src/async_map.rs
 * (AsyncFlashMap) stay unchanged.  Citations are file:line in the reference.
 *
 * Conventions
 *  - Every call returns an fm_status; 0 is success.  A thread-local message
 *    for the last failure is available from fm_last_error().
 *  - Keys and values are fixed-size byte records (K = key_size bytes,
 *    V = value_size bytes), laid out structure-of-arrays: n keys back to back,
 *    n values back to back.  A Rust (K, V) tuple has no C layout, so the shim
 *    splits pairs exactly as gpu.rs:212-217 does.
 *  - Host-pointer entry points copy inputs to the GPU, run, copy results back
 *    and return when the results are in place (gpu.rs's synchronous model).
 *  - *_device entry points take raw device pointers (cudarc CudaSlice device
 *    pointers) and a CUDA stream (cudaStream_t / CUstream cast to void*; NULL =
 *    the legacy default stream).  Work is ordered on that stream.
 *  - Results are bit-exact with the reference's sequential semantics
 *    (src/rayon_cpu.rs:82-328 applied in batch index order): in-batch
 *    duplicate keys resolve to the later position, tombstones are reused by
 *    inserts, and gets stop at the Robin Hood exit.
 *  - Thread safety: fm_bulk_get* may run concurrently on one table (the
 *    AsyncFlashMap read lock, async_map.rs:48-61).  Mutating calls (insert,
 *    remove, clear, recount) must be exclusive on a table (`&mut self`).
 */
#ifndef FLASHMAP_B200_H
#define FLASHMAP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1-6 map one to one onto FlashMapError (src/error.rs:5-27). */
typedef enum fm_status {
    FM_OK = 0,
    FM_ERR_CUDA_INIT = 1,       /* FlashMapError::CudaInit */
    FM_ERR_GPU_ALLOC = 2,       /* FlashMapError::GpuAlloc */
    FM_ERR_KERNEL_LAUNCH = 3,   /* FlashMapError::KernelLaunch */
    FM_ERR_TRANSFER = 4,        /* FlashMapError::Transfer */
    FM_ERR_TABLE_FULL = 5,      /* FlashMapError::TableFull: occupied = fm_len(),
                                   capacity = fm_capacity() */
    FM_ERR_ZERO_CAPACITY = 6,   /* FlashMapError::ZeroCapacity */
    FM_ERR_INVALID_ARG = 7,     /* -> KernelLaunch with message (unsupported size, NULL) */
    FM_ERR_DEVICE_TIMEOUT = 8,  /* -> KernelLaunch with message (bounded device wait ran out) */
    FM_ERR_PROBE_LIMIT = 9      /* -> KernelLaunch with message (round limit exceeded) */
} fm_status;

/* HashStrategy::to_mode (src/hash.rs:22-27). */
#define FM_HASH_IDENTITY 0u
#define FM_HASH_MURMUR3 1u

typedef struct fm_table fm_table;

/* GpuFlashMap::new (gpu.rs:45-105).  capacity 0 -> FM_ERR_ZERO_CAPACITY;
 * otherwise rounded up to the next power of two (gpu.rs:54).  Allocates the
 * zeroed SoA table on `device_id` (the CUDA primary context). */
int fm_create(uint64_t capacity, uint32_t key_size, uint32_t value_size, uint32_t hash_mode,
              int device_id, fm_table** out);

/* Drop for GpuFlashMap: frees the table and every buffer the library owns. */
void fm_destroy(fm_table* t);

/* GpuFlashMap::bulk_get (gpu.rs:111-191).  out_values receives n*V bytes
 * (zeros for misses), out_found n bytes (1 = found, 0 = miss). */
int fm_bulk_get(fm_table* t, const void* keys, uint64_t n, void* out_values, uint8_t* out_found);

/* GpuFlashMap::bulk_insert (gpu.rs:193-273).  Precheck len + n > capacity ->
 * FM_ERR_TABLE_FULL before any mutation (gpu.rs:198-206).  *num_new = number
 * of keys not present before (updates do not count). */
int fm_bulk_insert(fm_table* t, const void* keys, const void* values, uint64_t n, uint64_t* num_new);

/* GpuFlashMap::bulk_remove (gpu.rs:275-332).  *num_removed = keys tombstoned. */
int fm_bulk_remove(fm_table* t, const void* keys, uint64_t n, uint64_t* num_removed);

/* len / capacity / load_factor (gpu.rs:334-348).  len is a host-side count. */
uint64_t fm_len(const fm_table* t);
uint64_t fm_capacity(const fm_table* t);
double fm_load_factor(const fm_table* t);

/* GpuFlashMap::clear (gpu.rs:350-374): every slot EMPTY, len = 0. */
int fm_clear(fm_table* t);

/* GpuFlashMap::device (gpu.rs:381-383): the CUDA device ordinal. */
int fm_device(const fm_table* t);

/* GpuFlashMap::bulk_get_device (gpu.rs:422-478).  Outputs are caller-owned
 * device buffers (n*V and n bytes); misses are written as zeros. */
int fm_bulk_get_device(fm_table* t, const void* d_keys, uint64_t n, void* d_out_values,
                       uint8_t* d_out_found, void* stream);

/* GpuFlashMap::bulk_get_values_device (gpu.rs:484-536): no found mask;
 * misses are written as zeros. */
int fm_bulk_get_values_device(fm_table* t, const void* d_keys, uint64_t n, void* d_out_values,
                              void* stream);

/* GpuFlashMap::bulk_insert_device (gpu.rs:541-611): precheck, then a 4-byte
 * class readback of the new-key count. */
int fm_bulk_insert_device(fm_table* t, const void* d_keys, const void* d_values, uint64_t n,
                          uint64_t* num_new, void* stream);

/* GpuFlashMap::bulk_insert_device_uncounted (gpu.rs:618-672): no precheck,
 * len += n; call fm_recount for the exact count. */
int fm_bulk_insert_device_uncounted(fm_table* t, const void* d_keys, const void* d_values, uint64_t n,
                                    void* stream);

/* Device-pointer counterpart of bulk_remove (gpu.rs:275-332) for pipelines
 * that keep keys on the GPU. */
int fm_bulk_remove_device(fm_table* t, const void* d_keys, uint64_t n, uint64_t* num_removed,
                          void* stream);

/* Allocation-free insert.  No counterpart in the reference: an addition for
 * callers that must not allocate device memory once they are running -- a
 * serving process that sizes all its device memory up front under a fixed
 * budget, or one whose caching allocator (PyTorch's, for instance) holds the
 * free memory, so that a cudaMalloc made by this library at insert time could
 * fail, and a cudaFree would synchronize the whole device and stall the
 * caller's other streams.  Same semantics and arguments as
 * fm_bulk_insert_device, but it calls no cudaMalloc, cudaFree or other
 * allocating routine: its per-call scratch is a fixed device array inside the
 * library (about 2.5 MB, held by every device that loads the library until
 * the process exits), so a call takes at most FM_NOALLOC_MAX_OPS keys (larger
 * batches fail with FM_ERR_INVALID_ARG; split them).
 * Call it from an ordinary host thread: it launches kernels, copies control
 * words and waits on `stream` like fm_bulk_insert_device does, so it cannot
 * run inside a CUDA host function (cudaLaunchHostFunc), where CUDA calls are
 * not allowed.  The first call on a device also sets the array up (looks up
 * its device address, marks its per-op words idle, synchronizes the device);
 * make that first call before any stream capture on that device.  All calls
 * share the one array: calls whose GPU work overlaps (on any table of the same
 * device) race on it, so keep them ordered on one stream.  Near a full table,
 * where the parallel rounds of an insert stop making progress, this entry
 * point finishes the remaining keys one at a time on a single thread block
 * (fm_bulk_insert_device spreads that work over the GPU), so it is much slower
 * there. */
#define FM_NOALLOC_MAX_OPS 65536u
int fm_bulk_insert_device_noalloc(fm_table* t, const void* d_keys, const void* d_values, uint64_t n,
                                  uint64_t* num_new, void* stream);

/* GpuFlashMap::recount (gpu.rs:677-712): counts OCCUPIED slots, len := count. */
int fm_recount(fm_table* t, uint64_t* out);

/* Message of the last failed call on this thread ("" if none). */
const char* fm_last_error(void);

/* Instrumentation (no counterpart in gpu.rs): number of kernels this library
 * has launched in the process so far, across all tables. */
uint64_t fm_launch_count(void);

/* Host-side failure injection for tests of the error paths (no counterpart in
 * gpu.rs; the reference's error variants are src/error.rs:5-27).  Arms one
 * fault for the whole process: the `after`-th next pass (0 = the next one)
 * through `site` fails as if the CUDA call made there had returned an error,
 * the call reports the matching status, and the fault disarms.  The failing
 * CUDA call is not made, so nothing fails on the GPU.  FM_FAULT_NONE disarms.
 * After a failed mutating call the table holds the host pieces that completed
 * (len counts them) and possibly part of the failing piece; fm_recount gives
 * the exact count. */
#define FM_FAULT_NONE 0u
#define FM_FAULT_ALLOC 1u     /* a device allocation (table, scratch, staging) -> FM_ERR_GPU_ALLOC */
#define FM_FAULT_TRANSFER 2u  /* a host<->device copy of the host-pointer calls -> FM_ERR_TRANSFER */
#define FM_FAULT_ROUND 3u     /* the readback after a pass of insert/remove rounds -> FM_ERR_KERNEL_LAUNCH */
int fm_inject_fault(uint32_t site, uint32_t after);

/* Per-kernel device timing (no counterpart in gpu.rs).  While on, every call
 * on the table records a CUDA event pair around each kernel it launches;
 * fm_kernel_times waits for the recorded launches and returns, per kernel
 * class (index < FM_KERNEL_CLASSES, named by fm_kernel_class_name), the summed
 * device milliseconds and the launch count since the last reset.  Off by
 * default: no events are recorded then. */
#define FM_KERNEL_CLASSES 13u
int fm_kernel_timing(fm_table* t, int on);
int fm_kernel_times(fm_table* t, double* total_ms, uint64_t* launches, uint32_t n);
int fm_kernel_times_reset(fm_table* t);
const char* fm_kernel_class_name(uint32_t cls);

/* Batched form (no counterpart in gpu.rs).
 * A queue of bulk operations over any number of tables of one device, with
 * device-resident keys, values and outputs, executed with the result of
 * calling fm_bulk_get_device / fm_bulk_insert_device / fm_bulk_remove_device
 * one by one in queue order (each insert's TableFull precheck sees the
 * table's count after the ops before it).  Batches whose tables all have
 * compile-time record sizes and whose buffers are 16-byte aligned run every
 * op as device-driven kernels (counts read from the device, no host step
 * between ops) on 8 stream lanes forked from the caller's stream and joined
 * back before the results are copied out: a table's inserts and removes in
 * order on its lane, its lookups between two writes at once (on other lanes
 * when the batch has fewer tables than lanes), each lane waiting for the
 * steps of other lanes it depends on through events.  With the environment
 * variable FLASHMAP_BATCH_MODE=queue set when the batch is created, they run
 * instead through one persistent kernel per record shape that drains the
 * ops' phases (large ops run as the same device-driven kernels between its
 * launches).  Other batches run as waves of independent ops with grouped
 * kernels, on the same lanes.  Without a graph, fm_batch_run drives any
 * rounds (a remove's fallback, a wave's inserts and removes) from the host
 * (a small readback per two rounds, as the plain calls do) and records how
 * many each needed; fm_batch_capture records the whole batch into a CUDA
 * graph with those round counts and no host synchronisation; later
 * fm_batch_run calls replay it.  A replay whose data needs more rounds than
 * recorded still gives the same results, more slowly -- run the batch
 * eagerly once on representative data before capturing.  Between
 * fm_batch_run and fm_batch_wait the batch's tables must not be used by other
 * calls, and no op of the batch may read or write a buffer that another op
 * of it writes (lookups of one table may run at the same time).  Per-op
 * results (new /
 * removed key counts) and status codes (FM_OK, FM_ERR_TABLE_FULL,
 * FM_ERR_PROBE_LIMIT, ...) are written back into the op array by
 * fm_batch_wait, which also updates each table's len. */
#define FM_OP_GET 0u
#define FM_OP_INSERT 1u
#define FM_OP_REMOVE 2u
typedef struct fm_op {
    fm_table* table;
    uint32_t kind;          /* FM_OP_GET / FM_OP_INSERT / FM_OP_REMOVE */
    uint64_t n;             /* keys */
    const void* d_keys;     /* n * K bytes, device */
    const void* d_values;   /* insert: n * V bytes, device */
    void* d_out_values;     /* get: n * V bytes, device (NULL: not wanted) */
    uint8_t* d_out_found;   /* get: n bytes, device (NULL: not wanted) */
    uint64_t result;        /* out: new keys (insert) / removed keys (remove) */
    int status;             /* out: FM_OK or the op's error code */
} fm_op;
typedef struct fm_batch fm_batch;
int fm_batch_create(const fm_op* ops, uint32_t nops, fm_batch** out);
int fm_batch_capture(fm_batch* b, void* stream);
int fm_batch_run(fm_batch* b, void* stream);
int fm_batch_wait(fm_batch* b, fm_op* ops);
uint32_t fm_batch_waves(const fm_batch* b);
/* Instrumentation (no counterpart in the reference).  fm_batch_profile(b, 1)
 * before fm_batch_capture (or for eager runs) makes the persistent launches
 * of a queue-mode batch record, per phase, device times (globaltimer ns);
 * after fm_batch_wait, fm_batch_phase_times writes up to max_rows rows of 8
 * words: step, phase kind (0 get, 1 begin, 2-5 insert find / flow / exec /
 * warp, 6-7 remove find / exec, 8 end, 9 insert block pass), op index, units, first unit start,
 * last unit end, summed dependency waits, summed unit run times.  A wave-mode
 * batch refuses profiling (FM_ERR_INVALID_ARG). */
int fm_batch_profile(fm_batch* b, int on);
int fm_batch_phase_times(fm_batch* b, uint64_t* rows, uint32_t max_rows, uint32_t* nrows);
void fm_batch_destroy(fm_batch* b);

/* Device-side copy of a whole table (no counterpart in gpu.rs): dst takes
 * src's slots, len and persistent probe facts; both must have the same
 * capacity and record sizes.  Stream-ordered on `stream`.  Keeps a checkpoint
 * of a table on the GPU to roll back to. */
int fm_copy(fm_table* dst, const fm_table* src, void* stream);

/* Lookup autotuner (no counterpart in gpu.rs).  Times every lookup kernel
 * configuration -- lanes per query (1, 4, 8, 16, 32) x resident blocks per SM
 * (8, 16, 32, 64) -- per compile-time record shape (8/8, 32/128, 32/64, 32/32,
 * 8/32) and load bucket (< 0.6, < 0.8, >= 0.8) on sample tables of 2^20 slots,
 * and makes the fastest the configuration of every later lookup (plain and
 * batched) in the process.  With cache_path, a file of earlier results is
 * loaded instead when it exists, and new results are written to it. */
int fm_autotune(int device, const char* cache_path);
int fm_tuned_get_config(uint32_t key_size, uint32_t value_size, double load, int* lanes, int* blocks_per_sm);

/* Raw table access for layout checks and for loading a prefilled table:
 * flags (capacity u32), keys (capacity*K bytes), values (capacity*V bytes),
 * all host pointers; any may be NULL to skip it. */
int fm_snapshot(fm_table* t, uint32_t* flags, void* keys, void* values);
int fm_load(fm_table* t, const uint32_t* flags, const void* keys, const void* values, uint64_t len);

#ifdef __cplusplus
}
#endif
#endif /* FLASHMAP_B200_H */

// fm_internal.h -- host-side interface between the C ABI layer (fm_capi.cu)
// and the kernel launchers (fm_get.cu, fm_insert.cu, fm_remove.cu).  Not part
// of the public ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fm_device.cuh"

namespace fm {

// Control block in device memory, one per table, reused by every mutating
// call (mutating calls are exclusive per table).  Round r reads its pending
// count from npend[r & 1] (round 0: the call size) and its op list from
// OpScratch::pend[r & 1] (round 0: the identity), and appends the ops that
// did not run to pend[(r + 1) & 1].  The first CTL_CALL_BYTES bytes are
// zeroed at the start of every call.
// Counters that every block of a grid adds to are spread over COUNT_PARTS
// slots, each in its own 32-byte sector, so the atomics do not queue on one
// address; the host sums them.
constexpr int COUNT_PARTS = 32;

struct Ctl {
    uint32_t npend[2];       // pending ops per round parity
    uint32_t serial[2];      // 1: a round found no free slot / a flow wrapping the table
    uint32_t err;            // device-side error bits
    uint32_t rounds;         // rounds run by the call (statistics)
    uint32_t nlong[2];       // inserts deferred to the warp-per-op pass, per round parity
    uint32_t n0;             // grouped (batch) calls: the call's op count after the precheck
    uint32_t tail_handoff;   // insert tail: 1 + the round it left pending for the host (0: none)
    uint32_t rsum_on;        // remove: the chunk summaries (OpScratch::rsum) are built for this call
    uint32_t nbig;           // batch queue inserts: components listed for the block pass (pend[0] pairs)
    uint32_t big_next;       //   the next of them to take
    uint32_t big_ops;        //   op indices they hold (pend[1])
    uint32_t exec_next;      // direct insert exec pass: the next op a warp takes
    uint32_t pad_[7];        // count_part on a 32-byte boundary
    unsigned long long count;  // new keys (insert) / removed keys (remove), single-block kernels
    unsigned long long count_part[COUNT_PARTS][4];  // the same from grid kernels, [i][0] used
    // Persistent table facts (survive across calls, reset by clear):
    uint32_t dmax;           // largest probe distance ever stored since clear
    uint32_t tomb_claimed;   // 1 once an insert reused a tombstone since clear
    unsigned long long occupied;  // recount result
    __host__ __device__ unsigned long long total_count() const {
        unsigned long long s = count;
        for (int i = 0; i < COUNT_PARTS; i++) s += count_part[i][0];
        return s;
    }
};
constexpr size_t CTL_CALL_BYTES = 96 + 32 * COUNT_PARTS;  // npend .. count_part
static_assert(offsetof(Ctl, count_part) % 32 == 0, "count parts in their own sectors");
static_assert(offsetof(Ctl, dmax) == CTL_CALL_BYTES, "Ctl layout");

// Op status codes written by device code (the FM_* values of the C ABI).
constexpr int STATUS_OK = 0;
constexpr int STATUS_KERNEL = 3;       // FM_ERR_KERNEL_LAUNCH
constexpr int STATUS_TABLE_FULL = 5;   // FM_ERR_TABLE_FULL
constexpr int STATUS_PROBE_LIMIT = 9;  // FM_ERR_PROBE_LIMIT

// Device-side error bits (Ctl::err).
constexpr uint32_t ERR_WALK_LIMIT = 1u;   // an insert walk passed 2*capacity+2 slots (full table)
constexpr uint32_t ERR_SCRATCH = 2u;      // a segment registration did not belong to this call
constexpr uint32_t ERR_NO_PROGRESS = 4u;  // a tail round ran no op (never expected)

// Per-op scratch for the round-based insert and remove (op index space).
struct OpScratch {
    uint32_t* pend[2];   // pending op indices, by round parity
    uint64_t* op_slot;   // insert: terminating free slot F; remove: target slot
    uint32_t* op_word;   // insert: inflow lower bound; remove: window length (idle 0xFFFFFFFF)
    uint8_t* op_flag;    // insert: leader bit; remove: potential-target count
    uint32_t* op_pt;     // remove: up to PT_MAX potential-target distances per op
    uint32_t* long_list; // insert: ops of this round deferred to the warp-per-op pass
    uint8_t* comp;       // insert: component buffer (cmp_bytes of the table; null: none)
    uint32_t* rsum;      // remove: per 32-slot chunk, a metadata summary then the least mark
                         //   (rsum_words of the table; marks IDLE between calls; null: none)
    uint64_t cap_ops;
};

// Remove chunk summaries: for each chunk of 32 slots, (has an EMPTY slot) << 31
// | largest stored distance, then the least op index marking a slot of it.
__host__ __device__ inline uint64_t rsum_chunks(uint64_t mask) { return (mask + 32) >> 5; }
__host__ __device__ inline uint64_t rsum_words(uint64_t mask) { return 2 * rsum_chunks(mask); }

// Component buffer of the one-at-a-time insert path: a 256-byte header, then
// 32 bytes per chunk of CMP_CHUNK slots.  CMP_N0_CTL as a call's op count:
// read it from the control block (grouped calls).
constexpr uint64_t CMP_CHUNK = 8192;
__host__ __device__ inline uint64_t cmp_chunks(uint64_t mask) { return (mask + CMP_CHUNK) / CMP_CHUNK; }
__host__ __device__ inline uint64_t cmp_bytes(uint64_t mask) { return 256 + cmp_chunks(mask) * 32; }
constexpr uint32_t CMP_N0_CTL = 0xFFFFFFFFu;
constexpr int PT_MAX = 4;

enum Shape { SHAPE_8_8 = 0, SHAPE_32_128, SHAPE_32_64, SHAPE_32_32, SHAPE_8_32, SHAPE_GENERIC };
Shape pick_shape(uint32_t ksz, uint32_t vsz);
constexpr uint32_t GENERIC_MAX_KV = 256;  // byte limit of the run-time-size path (kernels.cu:32)

// Single-CTA tail: rounds with at most this many pending ops run inside one
// block with block-level barriers between phases.
constexpr uint32_t TAIL_MAX = 256;
constexpr int TAIL_THREADS = 512;

// Launchers.  All are stream-ordered and return the launch error.
cudaError_t launch_get(const TableView& t, Shape sh, const uint8_t* qkeys, uint64_t n, uint8_t* out_vals,
                       uint8_t* out_found, cudaStream_t s);
// Grid-wide rounds r0 .. r0+nrounds-1 of an insert call of n0 ops; `grid_ops`
// bounds the pending count of every launched round (sizes the grids).
cudaError_t launch_ins_rounds(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                              uint32_t r0, uint32_t nrounds, uint32_t grid_ops, const OpScratch& sc, Ctl* ctl,
                              cudaStream_t s);
// A whole insert call of n0 ops without rounds (compile-time record shapes,
// a table with a component buffer): ops alone at their first free slot run
// at once, the ops that share free slots (components) run in index order on
// a warp each.  On return (stream-ordered) Ctl::serial[0] set means nothing
// ran and every op is left to launch_ins_comp at round 0; otherwise
// Ctl::npend[1] ops (components too large for a warp) are left in pend[1]
// for launch_ins_comp at round 1.
cudaError_t launch_ins_direct(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                              const OpScratch& sc, Ctl* ctl, double load, cudaStream_t s);
// The same passes with the op count read from Ctl::n0 (a grouped call after
// its precheck; nmax bounds it and sizes the grids) and no host step after
// them: a call that found no free slot lists every op in pend[1], so
// launch_ins_comp at round 1 with CMP_N0_CTL completes the call either way.
cudaError_t launch_ins_direct_ctl(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals,
                                  uint32_t nmax, const OpScratch& sc, Ctl* ctl, double load, cudaStream_t s);
// Runs every remaining round starting at r in one block if the pending count
// is at most TAIL_MAX; otherwise returns without touching anything.  With
// handoff, rounds that stop progressing are left pending for the host
// (Ctl::tail_handoff) instead of run one at a time in the block.
cudaError_t launch_ins_tail(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                            uint32_t r, const OpScratch& sc, Ctl* ctl, cudaStream_t s, bool handoff = false);
// Applies round r's pending ops one at a time in index order (a round that
// found the table full, with more than TAIL_MAX ops pending).
cudaError_t launch_ins_serial(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                              uint32_t r, const OpScratch& sc, Ctl* ctl, cudaStream_t s);
// The same over the whole GPU: round r's pending ops (at most npend) split
// into components that touch disjoint slots, each run in index order on one
// block.  n0 may be CMP_N0_CTL (grouped calls; npend then also bounds the
// call size).  Without a component buffer (sc.comp null) it is
// launch_ins_serial.
cudaError_t launch_ins_comp(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals, uint32_t n0,
                            uint32_t r, uint32_t npend, const OpScratch& sc, Ctl* ctl, cudaStream_t s);
// A whole remove call of n0 ops without rounds: ops grouped by the first
// EMPTY slot at or after their home, lone ops run at once, each group in
// index order on one warp.  On return (stream-ordered) Ctl::serial[0] set
// means nothing ran (an op found no EMPTY slot) and every op is left to the
// rounds from round 0; otherwise Ctl::npend[1] ops (groups too large for a
// warp) are left in pend[1] for the rounds from round 1.
cudaError_t launch_rem_direct(const TableView& t, Shape sh, const uint8_t* keys, uint32_t n0, const OpScratch& sc,
                              Ctl* ctl, cudaStream_t s);
// The same with the op count read from Ctl::n0 (nmax bounds it and sizes the
// grids) and no host step after it: a call that found no EMPTY slot lists
// every op in pend[1], so the rounds from round 1 complete the call either way.
cudaError_t launch_rem_direct_ctl(const TableView& t, Shape sh, const uint8_t* keys, uint32_t nmax,
                                  const OpScratch& sc, Ctl* ctl, cudaStream_t s);
cudaError_t launch_rem_rounds(const TableView& t, Shape sh, const uint8_t* keys, uint32_t n0, uint32_t r0,
                              uint32_t nrounds, uint32_t grid_ops, const OpScratch& sc, Ctl* ctl, cudaStream_t s);
cudaError_t launch_rem_tail(const TableView& t, Shape sh, const uint8_t* keys, uint32_t n0, uint32_t r,
                            const OpScratch& sc, Ctl* ctl, cudaStream_t s);
// Builds the chunk summaries of a remove call (after its control block is
// reset) when the table's largest stored distance makes the windows long;
// the call's kernels then skip chunks that cannot matter.
cudaError_t launch_rem_summary(const TableView& t, const OpScratch& sc, Ctl* ctl, cudaStream_t s);
cudaError_t launch_count(const TableView& t, Ctl* ctl, cudaStream_t s);
int num_sms();
unsigned long long launch_count();

// ---- grouped (batch) execution ---------------------------------------------
//
// A batch wave runs many bulk operations on distinct tables with one launch
// per phase: every thread maps a flat item index to (op, item) through a
// prefix of the ops' item counts.  GROUP_MAX bounds the ops of one launch.
constexpr uint32_t GROUP_MAX = 1024;

// One get of a wave.
struct GroupGet {
    TableView t;
    const uint8_t* keys;
    uint8_t* out_vals;   // may be null (values not wanted)
    uint8_t* out_found;  // may be null
};

// One insert or remove of a wave, on its table's control block and scratch.
struct GroupOp {
    TableView t;
    const uint8_t* keys;
    const uint8_t* vals;        // insert values
    OpScratch sc;
    Ctl* ctl;
    unsigned long long* len;    // the table's element count within the batch
    unsigned long long* result; // new keys / removed keys
    int* status;                // FM status of the op
    uint32_t n;                 // requested ops
    uint32_t counted;           // insert: precheck and count (1)
};

// Lookup kernel configuration: lanes per query (1: one thread per query with
// 8-slot windows; 4..32: a tile) and resident blocks per SM for the grid.
struct GetCfg {
    int lanes = 1;          // lanes per query
    int blocks_per_sm = 64;
    int qpt = 1;            // one lane per query: queries per thread probed in lockstep (1, 2 or 4)
};
cudaError_t launch_get_cfg(const TableView& t, Shape sh, const uint8_t* qkeys, uint64_t n, uint8_t* out_vals,
                           uint8_t* out_found, GetCfg cfg, cudaStream_t s);
// The tuned configuration for a table (defaults when none was measured).
GetCfg tuned_get_cfg(Shape sh, double load);
void set_tuned_get_cfg(Shape sh, int load_bucket, GetCfg cfg);
constexpr int LOAD_BUCKETS = 3;  // load < 0.6, < 0.8, >= 0.8
inline int load_bucket(double load) { return load < 0.6 ? 0 : (load < 0.8 ? 1 : 2); }

// Direct insert configuration: lanes per entry of the warp pass (8, 16 or 32).
struct InsCfg {
    int tile = 32;
};
InsCfg tuned_ins_cfg(Shape sh, double load);  // defaults when none was measured
void set_tuned_ins_cfg(Shape sh, int load_bucket, InsCfg cfg);

// Fills `bytes` (a multiple of 8) with seeded pseudo-random words.
cudaError_t launch_fill_random(void* out, uint64_t bytes, uint64_t seed, cudaStream_t s);

// Grouped launchers (all ops of one call share the shape).  `prefix` holds
// the nops+1 exclusive prefix sums of the gets' sizes (device memory).
cudaError_t launch_grp_get(Shape sh, const GroupGet* ops, const uint64_t* prefix, uint32_t nops, uint64_t total,
                           GetCfg cfg, cudaStream_t s);
// A grouped insert / remove call in three stream-ordered phases: GRP_BEGIN
// (control reset, precheck against the table's count in the batch),
// GRP_ROUNDS (grid rounds r0 .. r0+nrounds-1, each a no-op for ops with
// nothing pending), GRP_END (block-per-op tail that finishes every op from
// round r0 -- fast when at most TAIL_MAX ops are left -- and the result
// write-back).  sum_n (the ops' total size) sizes the grids.
// GRP_SERIAL (inserts): every op's ops pending at round r0 one at a time in
// index order, one block per op (for rounds that stopped making progress).
enum { GRP_BEGIN = 0, GRP_ROUNDS = 1, GRP_END = 2, GRP_SERIAL = 3 };
// ---- persistent batch (one launch per record shape drains a queue) --------
//
// Every op of a batch is a chain of phases; each phase has `units` work units
// (one block each); the phases of all ops are listed in an order where every
// phase follows the one it waits for (`dep`: the previous phase of its op, or
// the last phase of the previous op on its table; -1: none).  `base` is the
// first global unit of the phase (the prefix of the units before it).
enum QPhaseKind : uint32_t {
    QP_GET = 0,  // lookups
    QP_BEGIN,    // control block reset; inserts: the TableFull precheck
    QP_IFIND,    // direct insert: find, flow, exec, warp passes
    QP_IFLOW,
    QP_IEXEC,
    QP_IWARP,
    QP_RFIND,    // direct remove: find, exec
    QP_REXEC,
    QP_END,      // leftovers in index order, result write-back
    QP_IBIG,     // direct insert: components too large for a warp, a block each
};
struct QPhase {
    uint64_t base;
    uint32_t units;
    uint32_t per;  // items (queries / ops) per unit
    uint32_t op;
    uint32_t kind;
    int32_t dep;
};
// One op of the queue (device descriptor).
struct QOp {
    TableView t;
    const uint8_t* keys;
    const uint8_t* vals;         // inserts
    uint8_t* out_vals;           // gets (may be null)
    uint8_t* out_found;          // gets (may be null)
    OpScratch sc;
    Ctl* ctl;
    unsigned long long* len;     // the table's count within the batch
    unsigned long long* result;  // new / removed keys
    int* status;
    uint32_t n;
    uint32_t kind;               // 0 get, 1 insert, 2 remove
    uint32_t counted;
    uint32_t pad_;
};
struct QState {
    unsigned long long next;  // the next unit to hand out
    uint32_t err;             // 1: a dependency wait ran out
    uint32_t pad_;
};
// Per-phase device timing of a persistent launch (globaltimer ns): first
// unit start, last unit end, summed dependency waits and summed unit run
// times.  Instrumentation, recorded only when the launch is given a buffer.
struct QProf {
    unsigned long long t0, t1, wait, busy;
};
// Items per unit and units of each phase kind for an op of n keys: small
// ops get small units, so that one op's phase still spreads over the SMs.
uint32_t queue_per(uint32_t kind, uint32_t n);
uint32_t queue_units(uint32_t kind, uint32_t n);
// One persistent launch over phases [0, nph) of ops of one record shape;
// `done` holds nph zeroed counters and `st` a zeroed QState.
cudaError_t launch_queue(Shape sh, const QPhase* ph, uint32_t nph, uint64_t total_units, const QOp* ops,
                         uint32_t* done, QState* st, QProf* prof, cudaStream_t s);

cudaError_t launch_grp_ins(Shape sh, const GroupOp* ops, uint32_t nops, uint64_t sum_n, int phase, uint32_t r0,
                           uint32_t nrounds, cudaStream_t s);
cudaError_t launch_grp_rem(Shape sh, const GroupOp* ops, uint32_t nops, uint64_t sum_n, int phase, uint32_t r0,
                           uint32_t nrounds, cudaStream_t s);
// *out = the largest pending count of round r over the ops (insert or remove).
cudaError_t launch_grp_pending(const GroupOp* ops, uint32_t nops, uint32_t r, uint32_t* out, cudaStream_t s);
// out[o] = the pending count of round r of op o.
cudaError_t launch_grp_pending_each(const GroupOp* ops, uint32_t nops, uint32_t r, uint32_t* out, cudaStream_t s);

// Optional device timing per kernel class: while a table's timing is on, the
// library records a CUDA event pair around each launch made for it on the
// calling thread (no events otherwise).
enum KernelClass : int {
    KC_GET = 0,     // k_get_thread / k_get
    KC_INS_FIND,    // k_dx_find / k_ins_p1: first free slot, registration
    KC_INS_WALK,    // k_dx_flow / k_ins_p2: flows over the free slots
    KC_INS_EXEC,    // k_dx_exec / k_ins_p3: thread-per-op execution
    KC_INS_LONG,    // k_dx_warp / k_ins_p4: warp-per-op execution (long walks, components)
    KC_INS_TAIL,    // k_ins_tail: remaining rounds in one block
    KC_INS_SERIAL,  // k_ins_serial
    KC_REM_MARK,    // k_rx_find / k_rem_p1
    KC_REM_CHECK,   // k_rem_p2
    KC_REM_EXEC,    // k_rx_exec / k_rem_p3
    KC_REM_TAIL,    // k_rem_tail
    KC_COUNT_OCC,   // k_count
    KC_REM_GROUP,   // k_rx_warp: a warp per group of removes
    KC_N
};
void kt_mark(int cls, bool begin, cudaStream_t s);
bool kt_active();  // per-kernel timing is on for the calling thread's current call
struct KtScope {
    int c;
    cudaStream_t s;
    KtScope(int c_, cudaStream_t s_) : c(c_), s(s_) { kt_mark(c, true, s); }
    ~KtScope() { kt_mark(c, false, s); }
};
void count_launches(unsigned n);
unsigned grid_for(uint64_t threads, unsigned per_sm);

}  // namespace fm

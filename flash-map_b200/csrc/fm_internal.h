// fm_internal.h -- host-side interface between the C ABI layer (fm_capi.cu)
// and the kernel launchers (fm_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fm_device.cuh"

namespace fm {

// Per-call control block in device memory (one per table, reused by every
// mutating call, which are exclusive per table).
struct Ctl {
    uint32_t npend_next;     // ops still pending after this round
    uint32_t gmin;           // smallest pending op index (serial mode)
    uint32_t serial;         // 1: this round runs only the smallest pending op
    uint32_t err;            // device-side error bits
    unsigned long long count;  // new keys (insert) / removed keys (remove)
    // Persistent table facts (survive across calls, reset by clear):
    uint32_t dmax;           // largest probe distance ever stored since clear
    uint32_t tomb_claimed;   // 1 once an insert reused a tombstone since clear
    unsigned long long occupied;  // recount result
};

// Device-side error bits (Ctl::err).
constexpr uint32_t ERR_WALK_LIMIT = 1u;  // an insert walk passed 2*capacity+2 slots (full table)
constexpr uint32_t ERR_SCRATCH = 2u;     // a segment registration did not belong to this call

// Per-op scratch for the round-based insert and remove (op index space).
struct OpScratch {
    uint32_t* pend_a;    // pending op indices (this round)
    uint32_t* pend_b;    // pending op indices (next round)
    uint64_t* op_slot;   // insert: terminating free slot F; remove: target slot
    uint32_t* op_word;   // insert: inflow lower bound; remove: window length
    uint8_t* op_flag;    // insert: leader bit; remove: potential-target count
    uint32_t* op_pt;     // remove: up to PT_MAX potential-target distances per op
    uint64_t cap_ops;
};
constexpr int PT_MAX = 4;

enum Shape { SHAPE_8_8 = 0, SHAPE_32_128, SHAPE_32_64, SHAPE_32_32, SHAPE_8_32, SHAPE_GENERIC };
Shape pick_shape(uint32_t ksz, uint32_t vsz);
constexpr uint32_t GENERIC_MAX_KV = 256;  // byte limit of the run-time-size path (kernels.cu:32)

// Launchers.  All are stream-ordered and return the launch error.
cudaError_t launch_get(const TableView& t, Shape sh, const uint8_t* qkeys, uint64_t n, uint8_t* out_vals,
                       uint8_t* out_found, cudaStream_t s);
cudaError_t launch_iota(uint32_t* p, uint64_t n, cudaStream_t s);
cudaError_t launch_ins_round(const TableView& t, Shape sh, const uint8_t* keys, const uint8_t* vals,
                             const uint32_t* pend, uint32_t npend, uint32_t nops, uint32_t* pend_next,
                             const OpScratch& sc, Ctl* ctl, cudaStream_t s);
cudaError_t launch_rem_round(const TableView& t, Shape sh, const uint8_t* keys, const uint32_t* pend,
                             uint32_t npend, uint32_t* pend_next, const OpScratch& sc, Ctl* ctl,
                             cudaStream_t s);
cudaError_t launch_count(const TableView& t, Ctl* ctl, cudaStream_t s);
int num_sms();
unsigned long long launch_count();

}  // namespace fm

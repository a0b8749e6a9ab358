/*
 * ref_host_shim.h -- lets the reference's src/kernels.cu compile as plain host
 * C++ so its hash functions and its thread-per-key insert kernel can be run on
 * the CPU as a checker for the oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * Every simulated thread runs to completion before the next one starts, so
 * the CAS calls of the insert kernel always see the value they expect: the
 * run is the reference kernel's own code under single-threaded semantics.
 * The warp intrinsics below exist only so the query kernels compile; the
 * harness never calls those kernels.
 */
#pragma once
#include <cstdint>

#define __device__
#define __global__
#define __forceinline__ inline
#define __restrict__ __restrict

struct uint4 { unsigned int x, y, z, w; };
struct ref_dim3 { unsigned int x, y, z; };

static thread_local ref_dim3 blockIdx, threadIdx, blockDim;

inline unsigned int atomicCAS(unsigned int* a, unsigned int cmp, unsigned int val) {
    unsigned int old = *a;
    if (old == cmp) *a = val;
    return old;
}
inline unsigned int atomicAdd(unsigned int* a, unsigned int v) {
    unsigned int old = *a;
    *a = old + v;
    return old;
}
inline void __threadfence() {}
template <class T> inline T __ldg(const T* p) { return *p; }
inline unsigned int __ballot_sync(unsigned int, unsigned int) { return 0u; }
template <class T> inline T __shfl_sync(unsigned int, T v, int) { return v; }
inline int __ffs(unsigned int x) { return __builtin_ffs((int)x); }

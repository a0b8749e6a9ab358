/*
 * ref_host_harness.cpp -- C entry points over the reference's own
 * src/kernels.cu compiled for the host (see ref_host_shim.h).  Built by
 * `make ref` into _ref/ only when the reference tree is present.
 * TEST INFRASTRUCTURE ONLY: used to pin the oracle, never by the product.
 */
#include "ref_host_shim.h"
#include REF_KERNELS

extern "C" {

uint64_t ref_identity_hash(const unsigned char* k, unsigned int ksz) {
    return fm_identity_hash(k, ksz);
}

uint64_t ref_murmur3_hash(const unsigned char* k, unsigned int ksz) {
    return fm_murmur3_hash(k, ksz);
}

/* flashmap_bulk_insert (kernels.cu:224-313) launched as gpu.rs:238-243 does
 * (256 threads per block), with the simulated threads run one after another
 * in thread-index order. */
unsigned int ref_seq_bulk_insert(unsigned char* keys, unsigned int* flags, unsigned char* values,
                                 const unsigned char* in_keys, const unsigned char* in_values,
                                 unsigned long long capacity_mask, unsigned int key_size,
                                 unsigned int value_size, unsigned int n, unsigned int hash_mode) {
    unsigned int count = 0;
    blockDim = {256u, 1u, 1u};
    for (unsigned int tid = 0; tid < n; ++tid) {
        blockIdx = {tid / 256u, 0u, 0u};
        threadIdx = {tid % 256u, 0u, 0u};
        flashmap_bulk_insert(keys, flags, values, in_keys, in_values, capacity_mask, key_size,
                             value_size, n, hash_mode, &count);
    }
    return count;
}

void ref_clear(unsigned int* flags, unsigned long long capacity) {
    blockDim = {256u, 1u, 1u};
    for (unsigned long long tid = 0; tid < capacity; ++tid) {
        blockIdx = {(unsigned int)(tid / 256u), 0u, 0u};
        threadIdx = {(unsigned int)(tid % 256u), 0u, 0u};
        flashmap_clear(flags, capacity);
    }
}

unsigned int ref_count(const unsigned int* flags, unsigned long long capacity) {
    unsigned int count = 0;
    blockDim = {256u, 1u, 1u};
    for (unsigned long long tid = 0; tid < capacity; ++tid) {
        blockIdx = {(unsigned int)(tid / 256u), 0u, 0u};
        threadIdx = {(unsigned int)(tid % 256u), 0u, 0u};
        flashmap_count(flags, capacity, &count);
    }
    return count;
}

}  // extern "C"

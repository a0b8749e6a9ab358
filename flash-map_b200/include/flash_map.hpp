// flash_map.hpp -- C++ host API of the FlashMap B200 backend (header-only).
//
// Mirrors the reference's public Rust API for the GPU path
// (bajpainaman/flash-map 0.5.0: FlashMap / FlashMapBuilder in src/lib.rs:94-450,
// HashStrategy in src/hash.rs:2-27, FlashMapError in src/error.rs:3-40) over the
// C ABI of libflashmap_b200.so (include/flashmap_b200.h).  Rust's
// `Result<T, FlashMapError>` becomes a return value or a thrown FlashMapError
// subclass; `Vec<Option<V>>` becomes std::vector<std::optional<V>>.  K and V
// are trivially copyable fixed-size types (bytemuck::Pod).
#pragma once

#include <cstdint>
#include <cstring>
#include <optional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/flashmap_b200.h"

namespace flash_map {

enum class HashStrategy : uint32_t { Identity = FM_HASH_IDENTITY, Murmur3 = FM_HASH_MURMUR3 };

// ---- FlashMapError (src/error.rs) -----------------------------------------
struct FlashMapError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CudaInit : FlashMapError {
    explicit CudaInit(const std::string& m) : FlashMapError("CUDA initialization failed: " + m) {}
};
struct GpuAlloc : FlashMapError {
    explicit GpuAlloc(const std::string& m) : FlashMapError("GPU memory allocation failed: " + m) {}
};
struct KernelLaunch : FlashMapError {
    explicit KernelLaunch(const std::string& m) : FlashMapError("kernel launch failed: " + m) {}
};
struct Transfer : FlashMapError {
    explicit Transfer(const std::string& m) : FlashMapError("host-device transfer failed: " + m) {}
};
struct TableFull : FlashMapError {
    size_t occupied, capacity;
    double load_factor;
    TableFull(size_t occ, size_t cap)
        : FlashMapError("table full: " + std::to_string(occ) + " occupied of " + std::to_string(cap) + " capacity"),
          occupied(occ),
          capacity(cap),
          load_factor((double)occ / (double)cap * 100.0) {}
};
struct ZeroCapacity : FlashMapError {
    ZeroCapacity() : FlashMapError("capacity must be positive") {}
};
struct NoBackend : FlashMapError {
    explicit NoBackend(const std::string& m) : FlashMapError(m) {}
};

namespace detail {
inline void check(int rc, const fm_table* t) {
    if (rc == FM_OK) return;
    const std::string msg = fm_last_error();
    switch (rc) {
        case FM_ERR_CUDA_INIT: throw CudaInit(msg);
        case FM_ERR_GPU_ALLOC: throw GpuAlloc(msg);
        case FM_ERR_TRANSFER: throw Transfer(msg);
        case FM_ERR_TABLE_FULL: throw TableFull(fm_len(t), fm_capacity(t));
        case FM_ERR_ZERO_CAPACITY: throw ZeroCapacity();
        default: throw KernelLaunch(msg);
    }
}
}  // namespace detail

template <class K, class V>
class FlashMap {
    static_assert(std::is_trivially_copyable<K>::value && std::is_trivially_copyable<V>::value,
                  "keys and values must be plain old data");

   public:
    // FlashMap::with_capacity (lib.rs:110-112): Identity hash, device 0.
    static FlashMap with_capacity(size_t capacity) { return FlashMap(capacity, HashStrategy::Identity, 0); }

    FlashMap(size_t capacity, HashStrategy hash, int device_id) {
        fm_table* t = nullptr;
        detail::check(fm_create(capacity, sizeof(K), sizeof(V), (uint32_t)hash, device_id, &t), nullptr);
        t_ = t;
    }
    FlashMap(const FlashMap&) = delete;
    FlashMap& operator=(const FlashMap&) = delete;
    FlashMap(FlashMap&& o) noexcept : t_(std::exchange(o.t_, nullptr)) {}
    FlashMap& operator=(FlashMap&& o) noexcept {
        if (this != &o) {
            if (t_) fm_destroy(t_);
            t_ = std::exchange(o.t_, nullptr);
        }
        return *this;
    }
    ~FlashMap() {
        if (t_) fm_destroy(t_);
    }

    // bulk_get (lib.rs:124-131)
    std::vector<std::optional<V>> bulk_get(const std::vector<K>& keys) const {
        std::vector<std::optional<V>> out(keys.size());
        if (keys.empty()) return out;
        std::vector<V> vals(keys.size());
        std::vector<uint8_t> found(keys.size());
        detail::check(fm_bulk_get(t_, keys.data(), keys.size(), vals.data(), found.data()), t_);
        for (size_t i = 0; i < keys.size(); i++)
            if (found[i]) out[i] = vals[i];
        return out;
    }

    // bulk_insert (lib.rs:143-150): returns the number of new keys.
    size_t bulk_insert(const std::vector<std::pair<K, V>>& pairs) {
        if (pairs.empty()) return 0;
        std::vector<K> ks(pairs.size());
        std::vector<V> vs(pairs.size());
        for (size_t i = 0; i < pairs.size(); i++) {  // SoA split (gpu.rs:212-217)
            ks[i] = pairs[i].first;
            vs[i] = pairs[i].second;
        }
        uint64_t added = 0;
        detail::check(fm_bulk_insert(t_, ks.data(), vs.data(), pairs.size(), &added), t_);
        return (size_t)added;
    }

    // bulk_remove (lib.rs:155-162)
    size_t bulk_remove(const std::vector<K>& keys) {
        if (keys.empty()) return 0;
        uint64_t removed = 0;
        detail::check(fm_bulk_remove(t_, keys.data(), keys.size(), &removed), t_);
        return (size_t)removed;
    }

    size_t len() const { return (size_t)fm_len(t_); }
    bool is_empty() const { return len() == 0; }
    size_t capacity() const { return (size_t)fm_capacity(t_); }
    double load_factor() const { return fm_load_factor(t_); }
    void clear() { detail::check(fm_clear(t_), t_); }
    int device() const { return fm_device(t_); }

    // Device-resident API (lib.rs:213-350): raw device pointers + stream.
    void bulk_get_device(const void* d_keys, size_t count, void* d_values, uint8_t* d_found,
                         void* stream = nullptr) const {
        detail::check(fm_bulk_get_device(t_, d_keys, count, d_values, d_found, stream), t_);
    }
    void bulk_get_values_device(const void* d_keys, size_t count, void* d_values, void* stream = nullptr) const {
        detail::check(fm_bulk_get_values_device(t_, d_keys, count, d_values, stream), t_);
    }
    size_t bulk_insert_device(const void* d_keys, const void* d_values, size_t count, void* stream = nullptr) {
        uint64_t added = 0;
        detail::check(fm_bulk_insert_device(t_, d_keys, d_values, count, &added, stream), t_);
        return (size_t)added;
    }
    void bulk_insert_device_uncounted(const void* d_keys, const void* d_values, size_t count,
                                      void* stream = nullptr) {
        detail::check(fm_bulk_insert_device_uncounted(t_, d_keys, d_values, count, stream), t_);
    }
    size_t recount() {
        uint64_t c = 0;
        detail::check(fm_recount(t_, &c), t_);
        return (size_t)c;
    }

    // Debug formatting (lib.rs:353-370)
    std::string debug_string() const {
        char buf[160];
        snprintf(buf, sizeof buf, "FlashMap { backend: \"GPU\", len: %zu, capacity: %zu, load_factor: \"%.1f%%\" }",
                 len(), capacity(), load_factor() * 100.0);
        return buf;
    }

   private:
    fm_table* t_ = nullptr;
};

// FlashMapBuilder (lib.rs:376-449) for the GPU backend.
class FlashMapBuilder {
   public:
    explicit FlashMapBuilder(size_t capacity) : capacity_(capacity) {}
    FlashMapBuilder& hash_strategy(HashStrategy s) {
        hash_ = s;
        return *this;
    }
    FlashMapBuilder& device_id(int d) {
        device_ = d;
        return *this;
    }
    FlashMapBuilder& force_cpu() {
        force_cpu_ = true;
        return *this;
    }
    template <class K, class V>
    FlashMap<K, V> build() const {
        // The CPU backend is the reference crate's Rayon code; this library is
        // only the GPU backend and never substitutes a CPU path.
        if (force_cpu_) throw NoBackend("force_cpu: this library provides only the GPU backend");
        return FlashMap<K, V>(capacity_, hash_, device_);
    }

   private:
    size_t capacity_;
    HashStrategy hash_ = HashStrategy::Identity;
    int device_ = 0;
    bool force_cpu_ = false;
};

}  // namespace flash_map

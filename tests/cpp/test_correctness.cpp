// C++ port of the reference's integration tests (tests/correctness.rs:1-392)
// through the C++ host API (flash-map_b200/include/flash_map.hpp) on the GPU.
// Exit code 0 = all passed.  Run by tests/test_cpp_api.py (marked gpu).
#include <array>
#include <cstdio>
#include <cstdlib>

#include "../../flash-map_b200/include/flash_map.hpp"

using namespace flash_map;
using K8 = std::array<uint8_t, 8>;

static int failures = 0;
#define CHECK(c)                                                          \
    do {                                                                  \
        if (!(c)) {                                                       \
            std::fprintf(stderr, "%s:%d: CHECK failed: %s\n", __FILE__, __LINE__, #c); \
            ++failures;                                                   \
        }                                                                 \
    } while (0)

static K8 le(uint64_t v) {
    K8 k;
    std::memcpy(k.data(), &v, 8);
    return k;
}

static std::vector<std::pair<K8, K8>> pairs(uint64_t a, uint64_t b, uint64_t mul, uint64_t add = 0) {
    std::vector<std::pair<K8, K8>> p;
    for (uint64_t i = a; i < b; i++) p.push_back({le(i), le(i * mul + add)});
    return p;
}
static std::vector<K8> keys(uint64_t a, uint64_t b) {
    std::vector<K8> k;
    for (uint64_t i = a; i < b; i++) k.push_back(le(i));
    return k;
}

static void insert_and_get() {  // correctness.rs:4-22
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    CHECK(m.bulk_insert(pairs(0, 100, 100)) == 100);
    CHECK(m.len() == 100);
    auto r = m.bulk_get(keys(0, 100));
    for (uint64_t i = 0; i < 100; i++) CHECK(r[i] && *r[i] == le(i * 100));
}

static void get_missing_keys() {  // :25-39
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    m.bulk_insert(pairs(0, 10, 1));
    for (auto& r : m.bulk_get(keys(100, 110))) CHECK(!r);
}

static void update_existing_keys() {  // :42-65
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    CHECK(m.bulk_insert(pairs(0, 10, 1)) == 10);
    CHECK(m.bulk_insert(pairs(0, 10, 1, 1000)) == 0);
    CHECK(m.len() == 10);
    auto r = m.bulk_get(keys(0, 10));
    for (uint64_t i = 0; i < 10; i++) CHECK(r[i] && *r[i] == le(i + 1000));
}

static void remove_keys() {  // :68-95
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    m.bulk_insert(pairs(0, 100, 1));
    CHECK(m.bulk_remove(keys(0, 50)) == 50);
    CHECK(m.len() == 50);
    for (auto& r : m.bulk_get(keys(0, 50))) CHECK(!r);
    for (auto& r : m.bulk_get(keys(50, 100))) CHECK(r.has_value());
}

static void insert_after_remove_reuses_tombstones() {  // :98-124
    auto m = FlashMap<K8, K8>::with_capacity(64);
    m.bulk_insert(pairs(0, 10, 1));
    m.bulk_remove(keys(0, 10));
    CHECK(m.len() == 0);
    CHECK(m.bulk_insert(pairs(100, 110, 2)) == 10);
    auto r = m.bulk_get(keys(100, 110));
    for (uint64_t i = 0; i < 10; i++) CHECK(r[i] && *r[i] == le((100 + i) * 2));
}

static void clear_resets_map() {  // :127-145
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    m.bulk_insert(pairs(0, 100, 1));
    m.clear();
    CHECK(m.len() == 0 && m.is_empty());
    for (auto& r : m.bulk_get(keys(0, 100))) CHECK(!r);
}

static void murmur3_hash_strategy() {  // :148-164
    auto m = FlashMapBuilder(1024).hash_strategy(HashStrategy::Murmur3).build<K8, K8>();
    m.bulk_insert(pairs(0, 100, 7));
    auto r = m.bulk_get(keys(0, 100));
    for (uint64_t i = 0; i < 100; i++) CHECK(r[i] && *r[i] == le(i * 7));
}

static void large_keys_and_values() {  // :167-191
    using K32 = std::array<uint8_t, 32>;
    using V64 = std::array<uint8_t, 64>;
    auto m = FlashMap<K32, V64>::with_capacity(4096);
    std::vector<std::pair<K32, V64>> p;
    std::vector<K32> ks;
    for (uint64_t i = 0; i < 500; i++) {
        K32 k{};
        V64 v{};
        uint64_t x = i * 42;
        std::memcpy(k.data(), &i, 8);
        std::memcpy(v.data(), &x, 8);
        p.push_back({k, v});
        ks.push_back(k);
    }
    m.bulk_insert(p);
    CHECK(m.len() == 500);
    auto r = m.bulk_get(ks);
    for (size_t i = 0; i < 500; i++) CHECK(r[i] && *r[i] == p[i].second);
}

static void load_factor_and_capacity() {  // :194-199
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    CHECK(m.load_factor() == 0.0);
    CHECK(m.capacity() >= 1024);
    CHECK((m.capacity() & (m.capacity() - 1)) == 0);
}

static void empty_operations_are_no_ops() {  // :202-211
    auto m = FlashMap<K8, K8>::with_capacity(64);
    CHECK(m.bulk_insert({}) == 0);
    CHECK(m.bulk_get({}).empty());
    CHECK(m.bulk_remove({}) == 0);
}

static void table_full_error() {  // :214-227
    auto m = FlashMap<K8, K8>::with_capacity(16);
    m.bulk_insert(pairs(0, 16, 1));
    bool threw = false;
    try {
        m.bulk_insert({{le(99), le(99)}});
    } catch (const TableFull& e) {
        threw = e.occupied == 16 && e.capacity == 16;
    }
    CHECK(threw);
}

static void debug_formatting() {  // :230-236
    auto m = FlashMap<K8, K8>::with_capacity(256);
    auto s = m.debug_string();
    CHECK(s.find("FlashMap") != std::string::npos && s.find("len") != std::string::npos &&
          s.find("capacity") != std::string::npos);
}

static void u64_key_value_types() {  // :239-250
    auto m = FlashMap<uint64_t, uint64_t>::with_capacity(1024);
    std::vector<std::pair<uint64_t, uint64_t>> p;
    std::vector<uint64_t> k;
    for (uint64_t i = 0; i < 50; i++) {
        p.push_back({i, i * i});
        k.push_back(i);
    }
    m.bulk_insert(p);
    auto r = m.bulk_get(k);
    for (uint64_t i = 0; i < 50; i++) CHECK(r[i] && *r[i] == i * i);
}

static void robin_hood_high_load_correctness() {  // :257-285
    for (int pct : {80, 90, 95}) {
        const uint64_t n = 1024 * pct / 100;
        auto m = FlashMap<K8, K8>::with_capacity(1024);
        CHECK(m.bulk_insert(pairs(0, n, 7)) == n);
        CHECK(m.len() == n);
        auto r = m.bulk_get(keys(0, n));
        for (uint64_t i = 0; i < n; i++) CHECK(r[i] && *r[i] == le(i * 7));
    }
}

static void robin_hood_miss_exits_early() {  // :288-309
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    m.bulk_insert(pairs(0, 1024 * 90 / 100, 1));
    for (auto& r : m.bulk_get(keys(10000, 10500))) CHECK(!r);
}

static void robin_hood_insert_remove_reinsert() {  // :312-362
    const uint64_t n = 512 * 80 / 100;
    auto m = FlashMap<K8, K8>::with_capacity(512);
    m.bulk_insert(pairs(0, n, 1));
    CHECK(m.bulk_remove(keys(0, n / 2)) == n / 2);
    CHECK(m.bulk_insert(pairs(10000, 10000 + n / 2, 3)) == n / 2);
    auto r = m.bulk_get(keys(n / 2, n));
    for (uint64_t i = 0; i < n - n / 2; i++) CHECK(r[i] && *r[i] == le(n / 2 + i));
    r = m.bulk_get(keys(10000, 10000 + n / 2));
    for (uint64_t i = 0; i < n / 2; i++) CHECK(r[i] && *r[i] == le((10000 + i) * 3));
}

static void robin_hood_update_at_high_load() {  // :365-392
    const uint64_t n = 1024 * 45 / 100;
    auto m = FlashMap<K8, K8>::with_capacity(1024);
    m.bulk_insert(pairs(0, n, 1));
    CHECK(m.bulk_insert(pairs(0, n, 1, 999)) == 0);
    CHECK(m.len() == n);
    auto r = m.bulk_get(keys(0, n));
    for (uint64_t i = 0; i < n; i++) CHECK(r[i] && *r[i] == le(i + 999));
}

static void zero_capacity_and_force_cpu() {  // gpu.rs:50-52; lib.rs:407-411
    bool z = false, nb = false;
    try {
        FlashMap<K8, K8>::with_capacity(0);
    } catch (const ZeroCapacity&) {
        z = true;
    }
    try {
        FlashMapBuilder(64).force_cpu().build<K8, K8>();
    } catch (const NoBackend&) {
        nb = true;
    }
    CHECK(z && nb);
}

int main() {
    insert_and_get();
    get_missing_keys();
    update_existing_keys();
    remove_keys();
    insert_after_remove_reuses_tombstones();
    clear_resets_map();
    murmur3_hash_strategy();
    large_keys_and_values();
    load_factor_and_capacity();
    empty_operations_are_no_ops();
    table_full_error();
    debug_formatting();
    u64_key_value_types();
    robin_hood_high_load_correctness();
    robin_hood_miss_exits_early();
    robin_hood_insert_remove_reinsert();
    robin_hood_update_at_high_load();
    zero_capacity_and_force_cpu();
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "ok", failures);
    return failures ? 1 : 0;
}

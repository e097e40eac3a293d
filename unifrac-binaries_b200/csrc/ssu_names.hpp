// Flat open-addressing map from name (string_view) to index, for the
// per-call table/tree name matching on the host.  One allocation, linear
// probing, FNV-1a hashing; keys are views that must outlive the map.
#pragma once

#include <cstdint>
#include <string_view>
#include <vector>

namespace ssu {

class NameMap {
  public:
    explicit NameMap(size_t expected) {
        size_t cap = 16;
        while (cap < expected * 2 + 1) cap <<= 1;
        keys_.assign(cap, std::string_view());
        vals_.assign(cap, kEmpty);
        mask_ = cap - 1;
    }

    // Insert or overwrite (the last index for a repeated name wins, as a
    // std::unordered_map assignment would); true when the key is new.
    bool set(std::string_view key, uint32_t value) {
        size_t i = hash(key) & mask_;
        while (vals_[i] != kEmpty && keys_[i] != key) i = (i + 1) & mask_;
        const bool fresh = vals_[i] == kEmpty;
        keys_[i] = key;
        vals_[i] = value;
        return fresh;
    }

    // Index of `key`, or -1.
    int64_t find(std::string_view key) const {
        size_t i = hash(key) & mask_;
        while (vals_[i] != kEmpty) {
            if (keys_[i] == key) return vals_[i];
            i = (i + 1) & mask_;
        }
        return -1;
    }

  private:
    static constexpr uint32_t kEmpty = 0xFFFFFFFFu;
    static size_t hash(std::string_view s) {
        uint64_t h = 1469598103934665603ull;
        for (unsigned char c : s) {
            h ^= c;
            h *= 1099511628211ull;
        }
        return static_cast<size_t>(h ^ (h >> 29));
    }
    std::vector<std::string_view> keys_;
    std::vector<uint32_t> vals_;
    size_t mask_ = 0;
};

}  // namespace ssu

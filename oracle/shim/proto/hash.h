// Test infrastructure (oracle): clean-room FNV hasher with the interface SoL uses
// (combine(value) chained, conversion to an integer).  32-bit FNV-1a over the
// object bytes of each combined value, as sol_b200::pixel_seed defines it.
#pragma once

#include <cstdint>
#include <cstring>
#include <type_traits>

namespace proto::fnv {

class Hasher {
public:
    Hasher() : h_(2166136261u) {}

    template <typename T>
    Hasher& combine(const T& value) {
        static_assert(std::is_trivially_copyable_v<T>, "hashable values are plain data");
        unsigned char bytes[sizeof(T)];
        std::memcpy(bytes, &value, sizeof(T));
        for (size_t i = 0; i < sizeof(T); ++i) { h_ ^= bytes[i]; h_ *= 16777619u; }
        return *this;
    }

    operator uint32_t() const { return h_; }

private:
    uint32_t h_;
};

} // namespace proto::fnv

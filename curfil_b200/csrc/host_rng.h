// Host random numbers of the reference's training driver.
//
// Sampler (random_tree.h:1009-1063) is an mt19937 seeded with the sampler's seed and a uniform
// integer distribution on [lo, hi]; RandomSource (random_tree.h:1129-1156) hands every new sampler
// the next seed. The integer distribution is Boost.Random's uniform_int bucket-rejection method
// (engine range 2^32-1 split into equal buckets; draws past the last whole bucket are redrawn).
#pragma once

#include <cstdint>
#include <random>

namespace cf {

inline int32_t uniform_int_draw(std::mt19937& eng, int32_t lo, int32_t hi) {
    const uint32_t range = static_cast<uint32_t>(hi) - static_cast<uint32_t>(lo);
    const uint32_t brange = 0xFFFFFFFFu;
    if (range == 0) return lo;
    if (range == brange) return static_cast<int32_t>(static_cast<uint32_t>(eng()) + static_cast<uint32_t>(lo));
    uint32_t bucket = brange / (range + 1u);
    if (brange % (range + 1u) == range) ++bucket;
    for (;;) {
        const uint32_t r = static_cast<uint32_t>(eng()) / bucket;
        if (r <= range) return static_cast<int32_t>(r + static_cast<uint32_t>(lo));
    }
}

struct Sampler {
    std::mt19937 eng;
    int32_t lo, hi;
    Sampler(int seed, int lo_, int hi_) : eng(static_cast<uint32_t>(seed)), lo(lo_), hi(hi_) {}
    int32_t next() { return uniform_int_draw(eng, lo, hi); }
};

// RandomSource over an external seed counter.
struct RandomSource {
    int32_t* counter;
    explicit RandomSource(int32_t* c) : counter(c) {}
    Sampler uniform(int upper_exclusive) { return Sampler((*counter)++, 0, upper_exclusive - 1); }
    Sampler uniform(int lo, int hi) { return Sampler((*counter)++, lo, hi); }
};

}  // namespace cf

// splitmix.h -- the seeded generator of the sphere packings (host and GPU
// packing generators draw the same spheres from it).
#pragma once

#include <stdint.h>

namespace mlbm {

struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform float in [0, 1) with 24 random bits
  float uniform() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
};

}  // namespace mlbm

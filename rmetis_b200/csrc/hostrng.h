// Host pseudo-random numbers for seed choices: xoshiro256++ (Blackman &
// Vigna) seeded by SplitMix64, with a widening-multiply rejection sampler for
// uniform integers below a bound.
#pragma once

#include <stdint.h>

namespace rmb {

class HostRng {
 public:
  explicit HostRng(uint64_t seed) {
    for (int i = 0; i < 4; ++i) {
      seed += 0x9e3779b97f4a7c15ULL;
      uint64_t z = seed;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s_[i] = z ^ (z >> 31);
    }
  }
  uint64_t next() {
    const uint64_t r = rotl(s_[0] + s_[3], 23) + s_[0];
    const uint64_t t = s_[1] << 17;
    s_[2] ^= s_[0];
    s_[3] ^= s_[1];
    s_[1] ^= s_[2];
    s_[0] ^= s_[3];
    s_[2] ^= t;
    s_[3] = rotl(s_[3], 45);
    return r;
  }
  // Uniform in [0, bound), bound > 0.
  uint64_t below(uint64_t bound) {
    const uint64_t zone = (bound << __builtin_clzll(bound)) - 1;
    for (;;) {
      const unsigned __int128 m = (unsigned __int128)next() * bound;
      if ((uint64_t)m <= zone) return (uint64_t)(m >> 64);
    }
  }

 private:
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t s_[4];
};

}  // namespace rmb

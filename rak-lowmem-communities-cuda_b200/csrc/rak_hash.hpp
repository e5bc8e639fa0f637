// rak_hash.hpp -- counter-based random numbers shared by the host and device graph generators,
// so a graph generated on either side is bit-identical for the same seed.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define RAK_HD __host__ __device__ __forceinline__
#else
#define RAK_HD inline
#endif

namespace rak {

// SplitMix64 finaliser (Steele, Lea & Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014): a bijective 64-bit mixer used here as a counter-based generator.
RAK_HD uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Random 64-bit word number `i` of stream `stream` under `seed`.
RAK_HD uint64_t rand64(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ (stream * 0xD6E8FEB86659FD93ull)) + i);
}

// Uniform float in [0,1) with 24 random bits (exactly representable).
RAK_HD float unit24(uint64_t h) { return float(h >> 40) * (1.0f / 16777216.0f); }

}  // namespace rak

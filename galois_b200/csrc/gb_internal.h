// Internal declarations shared by the host (.cpp) and device (.cu) parts of
// libgb.  Nothing here is part of the C ABI.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/gb.h"

namespace gb {

// Thread-local last-error message; every failing entry point sets it.
void set_error(const char* fmt, ...);
void clear_error();

// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014).  Used as a counter-based generator:
// stream value i of seed s is mix(mix(s ^ tag) + i * golden).
#if defined(__CUDACC__)
#define GB_HD __host__ __device__ __forceinline__
#else
#define GB_HD inline
#endif
GB_HD uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
GB_HD uint64_t stream_key(uint64_t seed, uint64_t tag) {
  return mix64(seed ^ (tag * 0xD1B54A32D192ED03ull));
}
GB_HD uint64_t rand_at(uint64_t key, uint64_t i) {
  return mix64(key + i * 0x9E3779B97F4A7C15ull);
}

// Stream tags (distinct generator streams derived from one seed).
enum : uint64_t {
  kTagRmat = 1,
  kTagPerm = 2,
  kTagWeightU32 = 3,
  kTagWeightF32 = 4,
  kTagEr = 5,
};

// gr2randomweightgr's weights (host_graph.cpp): argument check, then the
// draws of a default std::mt19937 in arc order into out[m] (uint32 for
// edge_bytes 4, float for -4).
int check_reference_weights(int min_value, int max_value, int edge_bytes, const char* what);
void draw_reference_weights(uint64_t m, int min_value, int max_value, int edge_bytes, void* out);

}  // namespace gb

#define GB_FAIL(code, ...)        \
  do {                            \
    ::gb::set_error(__VA_ARGS__); \
    return (code);                \
  } while (0)

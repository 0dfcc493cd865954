// Internal helpers shared by the host and device translation units.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/hc.h"

// Functions shared by host and device code (the graph generators).
#ifdef __CUDACC__
#define HC_HD __host__ __device__
#else
#define HC_HD
#endif

namespace hc {

// Records a printf-style message as this thread's last error and returns `s`.
hc_status fail(hc_status s, const char *fmt, ...);
void clear_error();
// Counts kernel launches made by the library (hc_kernel_launches).
void count_launch(int n = 1);

// Counter-based 64-bit mixer (SplitMix64 finaliser, Steele/Lea/Flood 2014).
// Graph generation draws every random number from (seed, stream, counter), so
// the output does not depend on the number of threads that produced it.
HC_HD inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
HC_HD inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
    return mix64(mix64(seed ^ (stream * 0x9e3779b97f4a7c15ULL)) + i);
}

}  // namespace hc

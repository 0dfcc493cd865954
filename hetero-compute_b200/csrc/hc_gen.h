// Edge streams of the synthetic graph generators, shared by the host builder
// (hc_host.cpp) and the device builder (hc_build.cu) so that both produce the
// same graph: counter-based random numbers, an invertible id permutation,
// R-MAT and uniform endpoint pairs, and edge weights.
#pragma once

#include <cstring>
#include <random>

#include "hc_common.h"

namespace hc {

enum Stream : uint64_t { kRmat = 1, kWeight = 2, kPerm = 3, kUniform = 4 };

// Bijection on [0, 2^bits): rounds of odd multiply + add and xorshift, all
// invertible modulo 2^bits.  Stands in for the shuffle of
// src/gapbs/generator.h:53-63 (which needs a serial mt19937 walk).
struct Permutation {
    uint32_t mask;
    int shift;
    uint32_t mul[4], add[4];
    HC_HD Permutation(int bits, uint64_t seed) {
        mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
        shift = bits / 2 + 1;
        for (int r = 0; r < 4; r++) {
            uint64_t k = draw(seed, kPerm, r);
            mul[r] = (uint32_t)k | 1u;
            add[r] = (uint32_t)(k >> 32);
        }
    }
    HC_HD uint32_t operator()(uint32_t x) const {
        for (int r = 0; r < 4; r++) {
            x = (x * mul[r] + add[r]) & mask;
            x ^= x >> shift;
        }
        return x & mask;
    }
};

// Endpoint pair e of an R-MAT edge list (src/gapbs/generator.h:82-115).
struct RmatPairs {
    int scale;
    uint64_t seed;
    Permutation perm;
    HC_HD RmatPairs(int s, uint64_t sd) : scale(s), seed(sd), perm(s, sd) {}
    HC_HD void operator()(int64_t e, uint32_t &src, uint32_t &dst) const {
        const float A = 0.57f, B = 0.19f, C = 0.19f;
        const float inv24 = 1.0f / 16777216.0f;
        uint32_t s = 0, d = 0;
        const int words = (scale + 1) / 2;
        for (int k = 0; k < words; k++) {
            uint64_t h = draw(seed, kRmat, (uint64_t)e * (uint64_t)words + k);
            for (int half = 0; half < 2; half++) {
                if (2 * k + half >= scale) break;
                float r = (float)((half ? (h >> 8) : (h >> 40)) & 0xffffffu) * inv24;
                s <<= 1;
                d <<= 1;
                if (r < A + B) {
                    if (r > A) d++;
                } else {
                    s++;
                    if (r > A + B + C) d++;
                }
            }
        }
        src = perm(s);
        dst = perm(d);
    }
};

// Uniform endpoints (src/gapbs/generator.h:65-80).
struct UniformPairs {
    int scale;
    uint64_t seed;
    HC_HD void operator()(int64_t e, uint32_t &src, uint32_t &dst) const {
        uint64_t h = draw(seed, kUniform, (uint64_t)e);
        uint32_t mask = (uint32_t)((1ull << scale) - 1);
        src = (uint32_t)h & mask;
        dst = (uint32_t)(h >> 32) & mask;
    }
};

HC_HD inline uint32_t weight_bits(hc_wtype wt, uint64_t seed, int64_t e) {
    uint64_t h = draw(seed, kWeight, (uint64_t)e);
    if (wt == HC_W_I32) return (uint32_t)(1 + (h % 255));  // uniform [1,255]
    if (wt == HC_W_F32) {
        float f = (float)((h >> 40) + 1) * (1.0f / 16777216.0f);  // uniform (0,1]
        uint32_t b;
        memcpy(&b, &f, 4);
        return b;  // positive floats order like their bit patterns
    }
    return 0;
}

// SourcePicker (src/graph.cuh:106-141): mt19937 seeded 37525, uniform over
// [0, N-1], rejecting degree-0 vertices and degree-1 vertices whose only edge
// is a self-loop (`self_only(v)`).  const_source >= 0 repeats that vertex.
template <class SelfOnly>
hc_status pick_sources_impl(const int64_t *index, int32_t num_nodes, int32_t count, int32_t const_source,
                            int32_t *out, SelfOnly &&self_only) {
    if (const_source >= 0) {
        for (int32_t i = 0; i < count; i++) out[i] = const_source;
        return HC_OK;
    }
    bool any = false;
    for (int32_t v = 0; v < num_nodes && !any; v++) {
        const int64_t d = index[v + 1] - index[v];
        any = d > 1 || (d == 1 && !self_only(v));
    }
    if (!any) return fail(HC_ERR_INVALID_ARG, "pick sources: graph has no eligible source");
    std::mt19937 rng(37525);
    std::uniform_int_distribution<int32_t> udist(0, num_nodes - 1);
    for (int32_t i = 0; i < count; i++) {
        int32_t s;
        for (;;) {
            s = udist(rng);
            const int64_t d = index[s + 1] - index[s];
            if (d == 0) continue;
            if (d == 1 && self_only(s)) continue;
            break;
        }
        out[i] = s;
    }
    return HC_OK;
}

}  // namespace hc

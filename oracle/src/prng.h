// Oracle (test infrastructure only): the PrngState interface of the reference,
// raymond/bridge/PrngState.hpp:5-23 and raymond/device/PrngState.metal:20-93,
// with two bodies:
//   * TEA: the reference's own generator (Zafar, Olano, Curtis: "GPU random
//     numbers via the Tiny Encryption Algorithm"), 6 rounds, 16-bit dimension
//     counter, float = (tea >> 9 | 0x3f800000) - 1, int = tea % max.
//   * PCG32 (O'Neill, pcg-random.org, pcg32_srandom_r / pcg32_random_r): one
//     stream per path, same float/int conversions as the TEA body.
#pragma once
#include <cstdint>
#include "vec.h"

namespace orc {

// PrngState.metal:20-30
inline uint32_t sample_tea_32(uint32_t v0, uint32_t v1, int rounds = 6) {
    uint32_t sum = 0;
    for (int i = 0; i < rounds; ++i) {
        sum += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v1;
}

// PrngState.metal:49-56
inline float u32_to_unit_float(uint32_t r) { return uint_as_float((r >> 9) | 0x3f800000u) - 1.0f; }

constexpr uint64_t PCG_MULT = 6364136223846793005ull;

struct PrngState {
    int mode = 0;          // 0 = PCG32, 1 = TEA
    uint32_t seed = 0;     // TEA
    uint16_t index = 0;    // TEA dimension counter (uint16_t, PrngState.hpp:7)
    uint64_t state = 0;    // PCG32
    uint64_t inc = 1;      // PCG32

    // PrngState.metal:58-61
    static PrngState tea(uint32_t a, uint32_t b) {
        PrngState p;
        p.mode = 1;
        p.seed = sample_tea_32(a, b);
        p.index = 0;
        return p;
    }
    // pcg32_srandom_r(initstate, initseq)
    static PrngState pcg(uint64_t initstate, uint64_t initseq) {
        PrngState p;
        p.mode = 0;
        p.state = 0;
        p.inc = (initseq << 1u) | 1u;
        p.next32();
        p.state += initstate;
        p.next32();
        return p;
    }
    uint32_t next32() {
        if (mode == 1) return sample_tea_32(seed, index++);
        uint64_t old = state;
        state = old * PCG_MULT + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
    }
    // PrngState.metal:63-77
    float sample() { return u32_to_unit_float(next32()); }
    float2 sample2d() {
        float a = sample();
        float b = sample();
        return {a, b};
    }
    float3 sample3d() {
        float a = sample();
        float b = sample();
        float c = sample();
        return {a, b, c};
    }
    int sampleInt(int max) { return (int)(next32() % (uint32_t)max); }
};

}  // namespace orc

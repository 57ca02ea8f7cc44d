// The reference's PrngState interface (raymond/bridge/PrngState.hpp:5-23,
// raymond/device/PrngState.metal:20-93) with two bodies selected per render:
//   TEA   — the reference generator: seed = tea(a, b), 16-bit dimension counter;
//   PCG32 — one PCG32 stream per path (O'Neill), same float / int mapping.
// In path state it occupies one uint2: TEA (seed, index) or the PCG32 state;
// the PCG32 increment is rebuilt from the path's sequence number on load.
#pragma once
#include "rt_math.cuh"

namespace rmd {

constexpr uint32_t RNG_PCG32 = 0;
constexpr uint32_t RNG_TEA = 1;
constexpr uint64_t PCG_MULT = 6364136223846793005ull;

// PrngState.metal:20-30
RMD_HD uint32_t sample_tea_32(uint32_t v0, uint32_t v1) {
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        sum += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v1;
}
// PrngState.metal:49-56
RMD_HD float unit_float(uint32_t r) { return __uint_as_float((r >> 9) | 0x3f800000u) - 1.0f; }

struct PrngState {
    uint32_t mode;
    uint32_t seed;    // TEA
    uint32_t index;   // TEA (wraps at 16 bits like the reference's uint16_t)
    uint64_t state;   // PCG32
    uint64_t inc;     // PCG32

    RMD_HD static PrngState tea(uint32_t a, uint32_t b) {
        PrngState p;
        p.mode = RNG_TEA;
        p.seed = sample_tea_32(a, b);
        p.index = 0;
        p.state = 0;
        p.inc = 1;
        return p;
    }
    // pcg32_srandom_r(initstate, initseq)
    RMD_HD static PrngState pcg(uint64_t initstate, uint64_t initseq) {
        PrngState p;
        p.mode = RNG_PCG32;
        p.seed = 0;
        p.index = 0;
        p.state = 0;
        p.inc = (initseq << 1) | 1ull;
        p.next32();
        p.state += initstate;
        p.next32();
        return p;
    }
    RMD_HD uint32_t next32() {
        if (mode == RNG_TEA) {
            uint32_t r = sample_tea_32(seed, index & 0xffffu);
            index = (index + 1) & 0xffffu;
            return r;
        }
        uint64_t old = state;
        state = old * PCG_MULT + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
    }
    RMD_HD float sample() { return unit_float(next32()); }
    RMD_HD float2 sample2d() {
        float a = sample();
        float b = sample();
        return make_float2(a, b);
    }
    RMD_HD float3 sample3d() {
        float a = sample();
        float b = sample();
        float c = sample();
        return make_float3(a, b, c);
    }
    RMD_HD int sampleInt(int max) { return (int)(next32() % (uint32_t)max); }

    // packed path-state form
    RMD_HD uint2 pack() const {
        if (mode == RNG_TEA) return make_uint2(seed, index);
        return make_uint2((uint32_t)state, (uint32_t)(state >> 32));
    }
    RMD_HD static PrngState unpack(uint32_t mode, uint2 v, uint64_t seq) {
        PrngState p;
        p.mode = mode;
        p.seed = v.x;
        p.index = v.y;
        p.state = (uint64_t)v.x | ((uint64_t)v.y << 32);
        p.inc = (seq << 1) | 1ull;
        return p;
    }
};

}  // namespace rmd

// Device random streams.
//
// * Xoshiro: the reference's per-point stream, xoshiro256++ seeded through
//   splitmix64 (include/wos/prng.hpp:7-45, src/prng.cpp:6-15,
//   include/wos/hash.hpp:7-12).  Bit-exact with the host reference; used by
//   the PLAIN_FP64 walks and the 3D inside test.
// * Philox: counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
//   "Parallel random numbers: as easy as 1, 2, 3", SC'11) keyed by the
//   reference's per-point seed and counted by (walk index, block index), so
//   every walk of every point has its own stream whatever lane runs it.  Used
//   by the FAST walks and by the adjoint replay.
#pragma once
#include <cstdint>

namespace wosb {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

// Stream tags XOR-ed into the point seed (include/wos/runner.hpp:182, 208, 211).
constexpr uint64_t kInsideStream = 0x243F6A8885A308D3ULL;
constexpr uint64_t kWalkStream = 0x13198A2E03707344ULL;
constexpr uint64_t kSourceStream = 0xA4093822299F31D0ULL;
// Tag of the counter-based fast streams (not in the reference).
constexpr uint64_t kFastStream = 0x082EFA98EC4E6C89ULL;

// Per-point seed of a global linear index (include/wos/runner.hpp:163-168).
__host__ __device__ __forceinline__ uint64_t point_seed(uint64_t seed, uint64_t linear) {
    return splitmix64(seed ^ splitmix64(linear));
}

struct Xoshiro {
    uint64_t s0, s1, s2, s3;

    __device__ __forceinline__ explicit Xoshiro(uint64_t seed) {
        s0 = splitmix64(seed);
        s1 = splitmix64(seed + 0x9E3779B97F4A7C15ULL);
        s2 = splitmix64(seed + 0x3C6EF372FE94F82AULL);
        s3 = splitmix64(seed + 0xDAA66D2C7DDF743FULL);
        if (!(s0 | s1 | s2 | s3)) s0 = 1;
    }

    __device__ __forceinline__ static uint64_t rotl(uint64_t x, int k) {
        return (x << k) | (x >> (64 - k));
    }

    __device__ __forceinline__ uint64_t u64() {
        const uint64_t out = rotl(s0 + s3, 23) + s0;
        const uint64_t t = s1 << 17;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = rotl(s3, 45);
        return out;
    }

    // [0, 1) from the top 53 bits (prng.hpp:27-29)
    __device__ __forceinline__ double unit() {
        return static_cast<double>(u64() >> 11) * (1.0 / 9007199254740992.0);
    }

    // (0, 1): redraw an exact zero (prng.hpp:31-37).  Zero has probability
    // 2^-53 per draw; the loop is bounded for the device.
    __device__ __forceinline__ double unit_open() {
        double v = unit();
        for (int i = 0; i < 64 && v == 0.0; ++i) v = unit();
        return v;
    }

    // FP64 draws for samplers that always work in double (same as above)
    __device__ __forceinline__ double unit64() { return unit(); }
    __device__ __forceinline__ double unit64_open() { return unit_open(); }
};

// Philox4x32-10 block function.
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = M0 * ctr.x, hi0 = __umulhi(M0, ctr.x);
        const uint32_t lo1 = M1 * ctr.z, hi1 = __umulhi(M1, ctr.z);
        ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
        key.x += W0;
        key.y += W1;
    }
    return ctr;
}

// One walk's stream under the point's key: counter (block, walk, tag, step).
// begin_step(s) starts step s at a fresh block, so every lane of a warp runs
// the Philox rounds at that one point of the step instead of wherever its
// four-value buffer happens to run dry; draws past the first four of a step
// take the step's next blocks.  Values left over at the end of a step are
// dropped.
struct PhiloxStream {
    uint2 key;
    uint32_t walk;
    uint32_t block;
    uint32_t base;  // first block of every step (the tag's range)
    uint32_t step;
    uint32_t b0, b1, b2, b3;
    int left;

    // The key of a point's streams (the same for all of its walks).
    static __device__ __forceinline__ uint2 key_of(uint64_t point_seed_value) {
        const uint64_t k = splitmix64(point_seed_value ^ kFastStream);
        return make_uint2(static_cast<uint32_t>(k), static_cast<uint32_t>(k >> 32));
    }

    __device__ __forceinline__ PhiloxStream(uint64_t point_seed_value, uint32_t walk_index,
                                            uint32_t tag = 0)
        : PhiloxStream(key_of(point_seed_value), walk_index, tag) {}

    __device__ __forceinline__ PhiloxStream(uint2 point_key, uint32_t walk_index,
                                            uint32_t tag = 0) {
        key = point_key;
        walk = walk_index;
        block = tag << 24;  // disjoint block ranges per tag (2^24 blocks each)
        base = block;
        step = 0;
        left = 0;
        b0 = b1 = b2 = b3 = 0;
    }

    __device__ __forceinline__ void begin_step(uint32_t s) {
        step = s;
        block = base;
        const uint4 r = philox4x32_10(make_uint4(block++, walk, 0x5A17u, step), key);
        b0 = r.x;
        b1 = r.y;
        b2 = r.z;
        b3 = r.w;
        left = 4;
    }

    __device__ __forceinline__ uint32_t next_u32() {
        if (left == 0) {
            const uint4 r = philox4x32_10(make_uint4(block++, walk, 0x5A17u, step), key);
            b0 = r.x;
            b1 = r.y;
            b2 = r.z;
            b3 = r.w;
            left = 4;
        }
        const uint32_t v = b0;
        b0 = b1;
        b1 = b2;
        b2 = b3;
        --left;
        return v;
    }

    // (0, 1): midpoints of the 2^24-point grid, so log and division are safe.
    __device__ __forceinline__ float uniform_f() {
        return (static_cast<float>(next_u32() >> 8) + 0.5f) * (1.0f / 16777216.0f);
    }

    // (0, 1) in double from two draws (53 bits).
    __device__ __forceinline__ double uniform_d() {
        const uint64_t hi = next_u32();
        const uint64_t lo = next_u32();
        const uint64_t bits = ((hi << 32) | lo) >> 11;
        return (static_cast<double>(bits) + 0.5) * (1.0 / 9007199254740992.0);
    }
};

}  // namespace wosb

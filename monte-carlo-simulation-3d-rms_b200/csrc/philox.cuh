// philox.cuh -- the engine's counter-based random stream (host and device).
//
// Replaces cuRAND's curandStatePhilox4_32_10_t of the reference
// (hpc_code/lib/main.cu:58-61 curand_init(seed, idx, 0); draws at
// main.cu:118-120, 140, 144, 282).  Generator: Philox4x32-10 of Salmon,
// Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
// Stream of walker w under seed s:
//   key      = (s_lo, s_hi)
//   block b  = Philox4x32-10(counter = (b_lo, b_hi, w_lo, w_hi), key): 4 words
//   double   = next two words (lo, hi): m = ((hi:lo) >> 12), u = (2m+1) 2^-53
//   float    = next word x:             u = (2(x >> 9) + 1) 2^-24
// Both maps are exact and land strictly inside (0, 1).  Doubles start on an
// even word, so a block is two doubles or four floats.  The stream is a pure
// function of (seed, walker, draw index): any walker can be replayed alone.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define RMS_HD __host__ __device__ __forceinline__
#else
#define RMS_HD inline
#endif

namespace rms {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

RMS_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

struct U4 {
    uint32_t x, y, z, w;
};

// Philox4x32-10: ten rounds of two 32x32 multiplies and the round's
// permutation, bumping the key by the Weyl constants between rounds.
RMS_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += kPhiloxW0; k1 += kPhiloxW1; }
        const uint32_t hi0 = mulhi32(kPhiloxM0, c.x), lo0 = kPhiloxM0 * c.x;
        const uint32_t hi1 = mulhi32(kPhiloxM1, c.z), lo1 = kPhiloxM1 * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    }
    return c;
}

RMS_HD double u53_to_double(uint32_t lo, uint32_t hi) {
    const uint64_t m = ((((uint64_t)hi) << 32) | lo) >> 12;
    return (double)(2 * m + 1) * 0x1p-53;
}

RMS_HD float u32_to_float(uint32_t x) {
#if defined(__CUDA_ARCH__)
    // the same value from the bits: 1 + k 2^-23 (k = x >> 9) minus
    // (1 - 2^-24) is (2k + 1) 2^-24, and the subtraction is exact (Sterbenz:
    // both operands lie within a factor of two of each other)
    return __uint_as_float(0x3f800000u | (x >> 9)) - (1.0f - 0x1p-24f);
#else
    return (float)(2u * (x >> 9) + 1u) * 0x1p-24f;
#endif
}

// Walker stream drawing doubles: holds the unread half of the last block in
// registers (no indexed arrays, so nothing spills to local memory).
struct DoubleStream {
    uint32_t k0, k1, w0, w1;
    uint64_t block;
    double spare;
    bool has_spare;

    RMS_HD void init(uint64_t seed, uint64_t walker) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        w0 = (uint32_t)walker; w1 = (uint32_t)(walker >> 32);
        block = 0; spare = 0.0; has_spare = false;
    }
    RMS_HD double next() {
        if (has_spare) { has_spare = false; return spare; }
        const U4 r = philox4x32_10(U4{(uint32_t)block, (uint32_t)(block >> 32), w0, w1}, k0, k1);
        ++block;
        spare = u53_to_double(r.z, r.w);
        has_spare = true;
        return u53_to_double(r.x, r.y);
    }
};

// Walker stream drawing floats: four per block, served oldest first.
struct FloatStream {
    uint32_t k0, k1, w0, w1;
    uint64_t block;
    uint32_t q1, q2, q3;   // unread words, next first
    int left;

    RMS_HD void init(uint64_t seed, uint64_t walker) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        w0 = (uint32_t)walker; w1 = (uint32_t)(walker >> 32);
        block = 0; q1 = q2 = q3 = 0; left = 0;
    }
    RMS_HD uint32_t next_word() {
        if (left == 0) {
            const U4 r = philox4x32_10(U4{(uint32_t)block, (uint32_t)(block >> 32), w0, w1}, k0, k1);
            ++block;
            q1 = r.y; q2 = r.z; q3 = r.w; left = 3;
            return r.x;
        }
        const uint32_t x = q1;
        q1 = q2; q2 = q3; --left;
        return x;
    }
    RMS_HD float next() { return u32_to_float(next_word()); }
};

// Streams of the split-precision walk.  Three counter domains per walker
// (counter word 1 = domain):
//   kDomDir  block k = the direction uniforms of steps 3k, 3k+1 and 3k+2: the
//            block's 128 bits (x the most significant word) cut into six 21-bit
//            fields from the top, fields 2j and 2j+1 for step 3k+j, each field f
//            read as u = (2f + 1) 2^-22 (dir_fields, u21_to_float; the two low
//            bits are unused): a pure function of the step index, so the lanes
//            of a warp generate blocks in lock step however many other draws
//            each lane made;
//   kDomInit sequential words for the rejection-sampled start position;
//   kDomPerm sequential words for partial-permeation draws;
//   kDomForce sequential words of the adjoint's forced-decision choice
// (the last three read as floats, u32_to_float).
// counter = (k, domain, walker_lo, walker_hi), key = (seed_lo, seed_hi).
constexpr uint32_t kDomDir = 0u;
constexpr uint32_t kDomInit = 1u;
constexpr uint32_t kDomPerm = 2u;
constexpr uint32_t kDomForce = 3u;

RMS_HD U4 dir_block(uint32_t k, uint32_t k0, uint32_t k1, uint32_t w0, uint32_t w1) {
    return philox4x32_10(U4{k, kDomDir, w0, w1}, k0, k1);
}

// A 21-bit field f as the uniform (2f + 1) 2^-22, in (0, 1).
RMS_HD float u21_to_float(uint32_t f) {
#if defined(__CUDA_ARCH__)
    // 1 + f 2^-21 from the bits, minus (1 - 2^-22): exact (Sterbenz)
    return __uint_as_float(0x3f800000u | ((f & 0x1fffffu) << 2)) - (1.0f - 0x1p-22f);
#else
    return (float)(2u * (f & 0x1fffffu) + 1u) * 0x1p-22f;
#endif
}

// The six direction uniforms of a kDomDir block: u[2j], u[2j+1] for step 3k+j.
RMS_HD void dir_fields(const U4& b, float u[6]) {
    u[0] = u21_to_float(b.x >> 11);
    u[1] = u21_to_float((b.x << 10) | (b.y >> 22));
    u[2] = u21_to_float(b.y >> 1);
    u[3] = u21_to_float((b.y << 20) | (b.z >> 12));
    u[4] = u21_to_float((b.z << 9) | (b.w >> 23));
    u[5] = u21_to_float(b.w >> 2);
}

// Sequential floats of one counter domain.
struct DomainStream {
    uint32_t k0, k1, w0, w1, dom, block;
    uint32_t q1, q2, q3;
    int left;

    RMS_HD void init(uint64_t seed, uint64_t walker, uint32_t domain) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        w0 = (uint32_t)walker; w1 = (uint32_t)(walker >> 32);
        dom = domain; block = 0; q1 = q2 = q3 = 0; left = 0;
    }
    RMS_HD uint32_t next_word() {
        if (left == 0) {
            const U4 r = philox4x32_10(U4{block, dom, w0, w1}, k0, k1);
            ++block;
            q1 = r.y; q2 = r.z; q3 = r.w; left = 3;
            return r.x;
        }
        const uint32_t x = q1;
        q1 = q2; q2 = q3; --left;
        return x;
    }
    RMS_HD float next() { return u32_to_float(next_word()); }
};

}  // namespace rms

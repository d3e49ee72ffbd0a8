/*
 * oracle/philox_stream.h -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * The project's counter-based random stream, restated in plain C for the CPU
 * oracle and for the host shim that compiles the reference simulator for the
 * CPU.  The product carries its own, independent implementation of the same
 * stream (monte-carlo-simulation-3d-rms_b200/csrc/philox.cuh); the tests check
 * both against the published Philox4x32-10 known-answer vectors and against
 * each other.
 *
 * Generator: Philox4x32-10, J. K. Salmon, M. A. Moraes, R. O. Dror,
 * D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11.
 * It replaces cuRAND's curandStatePhilox4_32_10_t in the reference
 * (hpc_code/lib/main.cu:58-61 curand_init(seed, idx, 0, ...); draws at
 * main.cu:118-120, 140, 144, 282).  cuRAND's own bit mapping is NOT
 * reproduced; the stream below is this project's own definition:
 *
 *   key     = (seed & 0xffffffff, seed >> 32)
 *   block b = Philox4x32-10(ctr = (b_lo, b_hi, walker_lo, walker_hi), key)
 *             -> words 4b, 4b+1, 4b+2, 4b+3 of the walker's stream
 *   double  : takes the next two words (lo, hi) of the stream,
 *             m = (((uint64)hi << 32) | lo) >> 12          (52 bits)
 *             u = (2m + 1) * 2^-53                  in (0, 1), exact
 *   float   : takes the next word x,
 *             u = (2(x >> 9) + 1) * 2^-24           in (0, 1), exact
 *
 * A double always starts on an even word, so one Philox block yields two
 * doubles or four floats.
 */
#ifndef RMS_ORACLE_PHILOX_STREAM_H
#define RMS_ORACLE_PHILOX_STREAM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_PHILOX_M0 0xD2511F53u
#define OR_PHILOX_M1 0xCD9E8D57u
#define OR_PHILOX_W0 0x9E3779B9u
#define OR_PHILOX_W1 0xBB67AE85u

/* One Philox4x32 round: two 32x32->64 products, then the S-box permutation
 * of Salmon et al. (their eq. for Philox4x32). */
static inline void or_philox_round(uint32_t c[4], const uint32_t k[2]) {
    uint64_t p0 = (uint64_t)OR_PHILOX_M0 * c[0];
    uint64_t p1 = (uint64_t)OR_PHILOX_M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k[0];
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c[3] ^ k[1];
    uint32_t n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
}

/* Philox4x32 with R rounds (10 for Philox4x32-10). */
static inline void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2],
                                 int rounds, uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    for (int r = 0; r < rounds; ++r) {
        if (r) { k[0] += OR_PHILOX_W0; k[1] += OR_PHILOX_W1; }
        or_philox_round(c, k);
    }
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
}

/* Sequential per-walker stream. */
typedef struct or_stream {
    uint32_t key[2];
    uint64_t walker;
    uint64_t block;    /* next block to generate */
    uint32_t buf[4];
    int pos;           /* next unread word in buf; 4 = empty */
} or_stream;

static inline void or_stream_init(or_stream* s, uint64_t seed, uint64_t walker) {
    s->key[0] = (uint32_t)seed;
    s->key[1] = (uint32_t)(seed >> 32);
    s->walker = walker;
    s->block = 0;
    s->pos = 4;
    s->buf[0] = s->buf[1] = s->buf[2] = s->buf[3] = 0;
}

static inline uint32_t or_stream_word(or_stream* s) {
    if (s->pos >= 4) {
        uint32_t ctr[4] = {(uint32_t)s->block, (uint32_t)(s->block >> 32),
                           (uint32_t)s->walker, (uint32_t)(s->walker >> 32)};
        or_philox4x32(ctr, s->key, 10, s->buf);
        s->block++;
        s->pos = 0;
    }
    return s->buf[s->pos++];
}

static inline double or_u53_to_double(uint32_t lo, uint32_t hi) {
    uint64_t m = ((((uint64_t)hi) << 32) | lo) >> 12;
    return (double)(2 * m + 1) * 0x1p-53;
}

static inline float or_u32_to_float(uint32_t x) {
    return (float)(2u * (x >> 9) + 1u) * 0x1p-24f;
}

/* Uniform double in (0,1): always two words starting at an even word. */
static inline double or_stream_double(or_stream* s) {
    if (s->pos & 1) s->pos++;       /* align to an even word */
    uint32_t lo = or_stream_word(s);
    uint32_t hi = or_stream_word(s);
    return or_u53_to_double(lo, hi);
}

static inline float or_stream_float(or_stream* s) {
    return or_u32_to_float(or_stream_word(s));
}

/* Streams of the engine's split-precision walk: Philox counter
 * (k, domain, walker_lo, walker_hi).  Domain 0: block k holds the direction
 * uniforms of steps 3k, 3k+1, 3k+2: its 128 bits (word 0 the most
 * significant) cut into six 21-bit fields from the top, fields 2j and 2j+1
 * for step 3k+j, a field f read as (2f + 1) 2^-22.  Domain 1: start
 * positions, sequential.  Domain 2: partial-permeation draws, sequential.
 * Domain 3: the adjoint's choice of the permeation decision it forces,
 * sequential (words read as floats, or_u32_to_float). */
#define OR_DOM_DIR 0u
#define OR_DOM_INIT 1u
#define OR_DOM_PERM 2u
#define OR_DOM_FORCE 3u

static inline float or_u21_to_float(uint32_t f) {
    return (float)(2u * (f & 0x1fffffu) + 1u) * 0x1p-22f;
}

static inline void or_dir_uniforms(uint64_t seed, uint64_t walker, uint32_t step, float* u1, float* u2) {
    uint32_t ctr[4] = {step / 3u, OR_DOM_DIR, (uint32_t)walker, (uint32_t)(walker >> 32)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t b[4];
    or_philox4x32(ctr, key, 10, b);
    const uint32_t f[6] = {b[0] >> 11, (b[0] << 10) | (b[1] >> 22), b[1] >> 1, (b[1] << 20) | (b[2] >> 12),
                           (b[2] << 9) | (b[3] >> 23), b[3] >> 2};
    const unsigned j = step % 3u;
    *u1 = or_u21_to_float(f[2 * j]);
    *u2 = or_u21_to_float(f[2 * j + 1]);
}

typedef struct or_dstream {
    uint32_t key[2];
    uint64_t walker;
    uint32_t dom, block;
    uint32_t buf[4];
    int pos;
} or_dstream;

static inline void or_dstream_init(or_dstream* s, uint64_t seed, uint64_t walker, uint32_t dom) {
    s->key[0] = (uint32_t)seed; s->key[1] = (uint32_t)(seed >> 32);
    s->walker = walker; s->dom = dom; s->block = 0; s->pos = 4;
}

static inline float or_dstream_float(or_dstream* s) {
    if (s->pos >= 4) {
        uint32_t ctr[4] = {s->block, s->dom, (uint32_t)s->walker, (uint32_t)(s->walker >> 32)};
        or_philox4x32(ctr, s->key, 10, s->buf);
        s->block++;
        s->pos = 0;
    }
    return or_u32_to_float(s->buf[s->pos++]);
}

#ifdef __cplusplus
}
#endif
#endif

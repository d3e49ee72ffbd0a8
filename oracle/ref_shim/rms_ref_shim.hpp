/*
 * oracle/ref_shim/rms_ref_shim.hpp -- TEST INFRASTRUCTURE (the oracle).
 *
 * Host stand-ins for the few CUDA, cuRAND and Thrust names used by the
 * reference simulator (hpc_code/lib/main.cu, hpc_code/lib/main_PGSE.cu), so
 * that its unmodified source text compiles with g++ and runs on the CPU.
 * oracle/Makefile streams each source file through one sed expression that
 * rewrites the kernel-launch syntax `f<<<grid, block>>>(args)` into
 * `_shim_launch(grid, block, f, args)`; nothing else in the text is changed
 * and no copy of it is stored.
 *
 *  - __global__/__device__ vanish; threadIdx/blockIdx/blockDim/gridDim are
 *    thread-local host variables set by _shim_launch (blocks and threads run
 *    in order, one OS thread) or by the OpenMP harness in ref_harness.cpp.
 *  - curandStatePhilox4_32_10_t / curand_init / curand_uniform_double are the
 *    project's Philox4x32-10 stream (oracle/philox_stream.h); cuRAND itself
 *    is not reproduced.
 *  - atomicCAS is a real host atomic compare-and-swap, so the reference's
 *    FP64 CAS loop (main.cu:40-56) keeps its meaning.
 *  - thrust::host_vector / device_vector are std::vector with the members the
 *    reference calls (.data().get(), begin/end, operator[]).
 *  - fopen("/dev/random") (main.cu:492-496) is answered from the environment
 *    variable RMS_REF_SEED when it is set, so a run can be seed-pinned.
 */
#ifndef RMS_REF_SHIM_HPP
#define RMS_REF_SHIM_HPP

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <vector>
#include <algorithm>
#include "../philox_stream.h"

#define __global__
#define __device__
#define __host__

struct _shim_dim3 { unsigned x, y, z; };
extern thread_local _shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

/* ---- cuRAND device API, restated on the project's stream ---- */
typedef or_stream curandStatePhilox4_32_10_t;

static inline void curand_init(unsigned long long seed, unsigned long long subsequence,
                               unsigned long long offset, curandStatePhilox4_32_10_t* state) {
    or_stream_init(state, (uint64_t)seed, (uint64_t)subsequence);
    for (unsigned long long i = 0; i < offset; ++i) (void)or_stream_word(state);
}

static inline double curand_uniform_double(curandStatePhilox4_32_10_t* state) {
    return or_stream_double(state);
}

/* ---- device intrinsics ---- */
static inline unsigned long long atomicCAS(unsigned long long* address,
                                           unsigned long long compare,
                                           unsigned long long val) {
    unsigned long long expected = compare;
    __atomic_compare_exchange_n(address, &expected, val, false,
                                __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return expected;   /* the old value, as atomicCAS returns */
}
static inline long long __double_as_longlong(double d) {
    long long r; std::memcpy(&r, &d, sizeof r); return r;
}
static inline double __longlong_as_double(long long l) {
    double r; std::memcpy(&r, &l, sizeof r); return r;
}
static inline int cudaDeviceSynchronize() { return 0; }

/* ---- launch: every block, every thread, in order ---- */
template <class F, class... A>
static inline void _shim_launch(int grid, int block, F fn, A... args) {
    _shim_dim3 saved_t = threadIdx, saved_b = blockIdx, saved_bd = blockDim, saved_gd = gridDim;
    blockDim = _shim_dim3{(unsigned)block, 1, 1};
    gridDim = _shim_dim3{(unsigned)grid, 1, 1};
    for (int b = 0; b < grid; ++b) {
        blockIdx = _shim_dim3{(unsigned)b, 0, 0};
        for (int t = 0; t < block; ++t) {
            threadIdx = _shim_dim3{(unsigned)t, 0, 0};
            fn(args...);
        }
    }
    threadIdx = saved_t; blockIdx = saved_b; blockDim = saved_bd; gridDim = saved_gd;
}

/* ---- Thrust containers used by the reference host code ---- */
namespace thrust {
template <class T> struct _shim_ptr {
    T* p;
    T* get() const { return p; }
};
template <class T> struct host_vector : std::vector<T> {
    host_vector() {}
    explicit host_vector(size_t n) : std::vector<T>(n) {}
};
template <class T> struct device_vector : std::vector<T> {
    explicit device_vector(size_t n) : std::vector<T>(n) {}
    device_vector(const host_vector<T>& h) : std::vector<T>(h.begin(), h.end()) {}
    _shim_ptr<T> data() { return _shim_ptr<T>{std::vector<T>::data()}; }
};
template <class I, class O> static inline O copy(I first, I last, O out) {
    return std::copy(first, last, out);
}
template <class T> static inline T* raw_pointer_cast(T* p) { return p; }
}  // namespace thrust

/* ---- seed pinning: fopen("/dev/random") reads RMS_REF_SEED when set ---- */
static inline FILE* _shim_fopen(const char* path, const char* mode) {
    const char* pinned = std::getenv("RMS_REF_SEED");
    if (pinned && std::strcmp(path, "/dev/random") == 0) {
        static thread_local unsigned long long seed_bytes;
        seed_bytes = std::strtoull(pinned, nullptr, 0);
        return fmemopen(&seed_bytes, sizeof seed_bytes, "r");
    }
    return std::fopen(path, mode);
}
#define fopen _shim_fopen

#endif

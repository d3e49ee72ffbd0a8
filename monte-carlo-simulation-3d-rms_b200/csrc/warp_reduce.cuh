// warp_reduce.cuh -- cross-walker FP64 sums inside one warp.
//
// The reference adds every walker's record into the same global addresses
// with an FP64 compare-and-swap loop (hpc_code/lib/main.cu:40-56, 344-378):
// 23+Nbvec contended atomics per walker per record.  Here a warp first sums
// its 32 walkers with register shuffles, in a fixed order, and one lane per
// value adds the warp total into that warp's private accumulator row -- no
// atomics, and a repeatable result for a fixed launch shape.
#pragma once
#include <cuda_runtime.h>

namespace rms {

constexpr unsigned kFullMask = 0xffffffffu;

// Sum over the warp; every lane receives the total (butterfly, fixed order).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFullMask, v, off);
    return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFullMask, v, off);
    return v;
}

// Reduce-scatter of 32 values held by every lane: on return lane l holds the
// warp-wide sum of v[l].  Each halving level exchanges half of the remaining
// values (16 + 8 + 4 + 2 + 1 = 31 shuffles instead of 32 x 5).
__device__ __forceinline__ double warp_reduce_scatter32(double (&v)[32], int lane) {
#pragma unroll
    for (int half = 16; half > 0; half >>= 1) {
        const bool upper = (lane & half) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const double send = upper ? v[k] : v[k + half];
            const double keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(kFullMask, send, half);
        }
    }
    return v[0];
}

// Reduce-scatter of 16 values: on return lanes l and l ^ 16 both hold the
// warp-wide sum of v[l & 15] (8 + 4 + 2 + 1 halving shuffles, then one
// butterfly across the half-warps).  Half the registers of the 32-value form.
__device__ __forceinline__ double warp_reduce_scatter16(double (&v)[16], int lane) {
#pragma unroll
    for (int half = 8; half > 0; half >>= 1) {
        const bool upper = (lane & half) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const double send = upper ? v[k] : v[k + half];
            const double keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(kFullMask, send, half);
        }
    }
    return v[0] + __shfl_xor_sync(kFullMask, v[0], 16);
}

}  // namespace rms

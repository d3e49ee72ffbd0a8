// split_lattice.cuh -- the padded, packed label lattice of the split walk
// (rms_walk_split.cu) and the pieces of the walk shared with the adjoint
// (rms_adjoint.cu): cell decoding and the origin mirror at a domain wall.
#pragma once
#include <cstdint>

namespace rms {

// Lattice cell: label in the low bits, free-flight flag in the top bit
// (BITS = 4: 3 + 1 bits, two voxels per byte, voxel v in bits 4(v % 2);
// BITS = 8: 7 + 1).
template <int BITS>
__device__ __forceinline__ unsigned cell_at(const uint8_t* __restrict__ lat, unsigned lin) {
    if (BITS == 4) return (__ldg(lat + (lin >> 1)) >> ((lin & 1u) * 4u)) & 15u;
    return __ldg(lat + lin);
}

template <int BITS> __host__ __device__ constexpr unsigned label_mask() { return BITS == 4 ? 7u : 127u; }
template <int BITS> __host__ __device__ constexpr unsigned flight_bit() { return BITS == 4 ? 8u : 128u; }

template <int BITS>
__device__ __forceinline__ int label_at(const uint8_t* __restrict__ lat, unsigned lin) {
    return (int)(cell_at<BITS>(lat, lin) & label_mask<BITS>());
}

template <int BITS> __host__ __device__ constexpr int wall_code() { return (int)label_mask<BITS>(); }

// Origin image after a mirror wall: x -> -x (lo) or x -> 2N - x (hi), on the
// split form x = I + F, F in [0, 1).
__device__ __forceinline__ void mirror_origin(int& I, float& F, bool hi, int n) {
    const int base = hi ? 2 * n : 0;
    if (F > 0.0f) { I = base - I - 1; F = 1.0f - F; }
    else { I = base - I; }
}

}  // namespace rms

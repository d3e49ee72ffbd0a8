// rms_geometry.cu -- synthetic lattices built on the GPU.
//
// One tube along z with a per-slice centre and radius: the caliber variation
// and undulation of an axon (analysis/visualizeaxon.m:28-67 applies the same
// two transforms to segmented axons).  Voxel (i, j, k) is `inside` when
// ((i + 0.5) res - cx[k])^2 + ((j + 0.5) res - cy[k])^2 < r2[k], with every
// operation rounded on its own (no fused multiply-add), so the lattice equals
// the one numpy builds from the same per-slice tables bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

namespace rms {
namespace {

__global__ void tube_kernel(uint8_t* __restrict__ out, int n1, int n2, int n3, double res,
                            const double* __restrict__ r2, const double* __restrict__ cx,
                            const double* __restrict__ cy, uint8_t inside, uint8_t outside) {
    const size_t n = (size_t)n1 * n2 * n3;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(v % (size_t)n3);
        const size_t ij = v / (size_t)n3;
        const int j = (int)(ij % (size_t)n2), i = (int)(ij / (size_t)n2);
        const double x = __dmul_rn((double)i + 0.5, res), y = __dmul_rn((double)j + 0.5, res);
        const double dx = __dsub_rn(x, cx[k]), dy = __dsub_rn(y, cy[k]);
        const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        out[v] = d2 < r2[k] ? inside : outside;
    }
}

}  // namespace

int build_tube_lattice(uint8_t* d_out, int n1, int n2, int n3, double res, const double* d_r2, const double* d_cx,
                       const double* d_cy, uint8_t inside, uint8_t outside, void* stream) {
    const size_t n = (size_t)n1 * n2 * n3;
    size_t grid = (n + 255) / 256;
    if (grid > 65536) grid = 65536;
    tube_kernel<<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(d_out, n1, n2, n3, res, d_r2, d_cx, d_cy, inside,
                                                                   outside);
    return (int)cudaGetLastError();
}

}  // namespace rms

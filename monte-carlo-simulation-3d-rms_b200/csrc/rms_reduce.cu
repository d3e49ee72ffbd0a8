// rms_reduce.cu -- ordered sum of the per-warp accumulator rows.
//
// Each warp of a walk launch owns one FP64 row block (rms_walk_*.cu); the
// job's totals are their sum.  Column i is summed by one thread over the
// rows in slot order with eight interleaved partial sums (slot k goes to
// partial k % 8), then the partials are added in order: a fixed association,
// so a rerun with the same launch shape reproduces every bit.
// Replaces the contended FP64 CAS atomics of hpc_code/lib/main.cu:40-56.
#include <cuda_runtime.h>
#include "rms_internal.h"

namespace rms {
namespace {

__global__ void reduce_slots_kernel(const double* __restrict__ slots, int nslots, size_t row,
                                    double* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < row; i += stride) {
        double p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int k = 0;
        for (; k + 8 <= nslots; k += 8) {
#pragma unroll
            for (int u = 0; u < 8; ++u) p[u] += __ldcs(slots + (size_t)(k + u) * row + i);
        }
        for (int u = 0; k < nslots; ++k, ++u) p[u] += __ldcs(slots + (size_t)k * row + i);
        out[i] = ((p[0] + p[1]) + (p[2] + p[3])) + ((p[4] + p[5]) + (p[6] + p[7]));
    }
}

}  // namespace

int launch_reduce_slots(const double* slots, int nslots, size_t row, double* out, void* stream) {
    if (row == 0) return 0;
    const int block = 256;
    size_t grid = (row + block - 1) / block;
    if (grid > 4096) grid = 4096;
    reduce_slots_kernel<<<(unsigned)grid, block, 0, (cudaStream_t)stream>>>(slots, nslots, row, out);
    return (int)cudaGetLastError();
}

const char* cuda_error_string(int code) { return cudaGetErrorString((cudaError_t)code); }

}  // namespace rms

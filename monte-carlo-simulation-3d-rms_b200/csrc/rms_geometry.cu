// rms_geometry.cu -- lattices on the GPU: synthetic tubes, and the check of
// a lattice that is already in device memory.
//
// One tube along z with a per-slice centre and radius: the caliber variation
// and undulation of an axon (analysis/visualizeaxon.m:28-67 applies the same
// two transforms to segmented axons).  Voxel (i, j, k) is `inside` when
// ((i + 0.5) res - cx[k])^2 + ((j + 0.5) res - cy[k])^2 < r2[k], with every
// operation rounded on its own (no fused multiply-add), so the lattice equals
// the one numpy builds from the same per-slice tables bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
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

// A lattice in device memory, checked as validate_lattice checks a host one: counts[0] = voxels with a label >= nc, counts[1] = labelled voxels.
// 16-byte loads over the aligned middle, byte loads at the two ends.
__global__ void check_labels_kernel(const uint8_t* __restrict__ lab, size_t n, unsigned nc,
                                    unsigned long long* counts) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nthr = (size_t)gridDim.x * blockDim.x;
    const size_t mis = (size_t)((16u - ((uintptr_t)lab & 15u)) & 15u);
    const size_t head = mis < n ? mis : n;
    const size_t nvec = (n - head) / 16;
    const unsigned ncr = nc * 0x01010101u;
    unsigned bad = 0, labelled = 0;
    auto one = [&](unsigned v) { bad += v >= nc; labelled += v != 0; };
    if (tid < head) one(lab[tid]);
    const uint4* vec = reinterpret_cast<const uint4*>(lab + head);
    for (size_t i = tid; i < nvec; i += nthr) {
        const uint4 q = __ldg(vec + i);
        const unsigned w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            bad += __popc(__vcmpgeu4(w[k], ncr)) >> 3;     // 0xff per byte >= nc
            labelled += 4 - (__popc(__vcmpeq4(w[k], 0u)) >> 3);
        }
    }
    for (size_t i = head + nvec * 16 + tid; i < n; i += nthr) one(lab[i]);
    for (int o = 16; o > 0; o >>= 1) {
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
        labelled += __shfl_xor_sync(0xffffffffu, labelled, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(counts, (unsigned long long)bad);
        if (labelled) atomicAdd(counts + 1, (unsigned long long)labelled);
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

int check_labels(const uint8_t* d_labels, size_t n, unsigned nc, unsigned long long* d_counts, int sms,
                 void* stream) {
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(4 * (int64_t)sms, (int64_t)(n / 4096) + 1));
    check_labels_kernel<<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(d_labels, n, nc, d_counts);
    return (int)cudaGetLastError();
}

}  // namespace rms

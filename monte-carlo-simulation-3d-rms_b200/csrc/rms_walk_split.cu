// rms_walk_split.cu -- the split-precision walk (RMS_PREC_SPLIT).
//
// The same walk as the reference kernel `propagate` (hpc_code/lib/main.cu:
// 63-384, main_PGSE.cu:65-410) -- fixed-length isotropic steps, at most nite
// sub-segments, voxel-face reflection or Bernoulli(Pij) permeation, mirror
// walls, T2 weighting, moments and signal at the same records -- in the
// arithmetic a B200 issues fastest:
//
//  - position = int32 voxel index + FP32 offset inside the voxel, so FP32
//    keeps ~1e-7 voxel resolution anywhere in a 2048-voxel lattice; a walker
//    that crosses or reflects at a face is put exactly on it (offset 0 or 1);
//  - FP32 uniforms (one Philox4x32-10 block per two steps), sincospif for the
//    azimuth, one reciprocal per axis per step for the face distances;
//  - labels packed 2 bits per voxel when Nc <= 4 (a 256x256x2048 lattice is
//    33.5 MB and stays in the 126 MB L2), else one byte per voxel;
//  - per-walker sums that grow over the walk (T2 exponent, PGSE displacement
//    sums) are carried in FP32 for at most 32 steps and folded into FP64;
//  - cross-walker sums: FP32 products per walker, warp reduce-scatter in
//    FP64, per-warp FP64 rows, ordered FP64 reduction (rms_reduce.cu).
//
// Random stream: the same Philox4x32-10 stream as the FP64 walk, read as
// floats (one word each); draw order per walker: 3 per initial-position try,
// 2 per step, 1 per partial-permeation face.
#include <cuda_runtime.h>
#include <math.h>

#include "philox.cuh"
#include "rms_internal.h"
#include "warp_reduce.cuh"

namespace rms {
namespace {

constexpr int kSplitBlockMax = 512;

__device__ __forceinline__ unsigned lin3(int i, int j, int k, int n2, int n3) {
    return ((unsigned)i * (unsigned)n2 + (unsigned)j) * (unsigned)n3 + (unsigned)k;
}

template <int BITS>
__device__ __forceinline__ int label_at(const uint8_t* __restrict__ lat, unsigned lin) {
    if (BITS == 2) {
        const unsigned byte = __ldg(lat + (lin >> 2));
        return (int)((byte >> ((lin & 3u) * 2u)) & 3u);
    } else {
        return (int)__ldg(lat + lin);
    }
}

// Distance along the ray to the face the walker moves towards, on one axis
// (clamped at 0 for an offset a rounding step outside [0, 1]).
__device__ __forceinline__ float face_dist(float f, float v, float inv_abs_v) {
    const float d = (v > 0.0f) ? (1.0f - f) : f;
    return (v == 0.0f) ? INFINITY : fmaxf(d, 0.0f) * inv_abs_v;
}

// Origin image after a mirror wall: x -> -x (lo) or x -> 2N - x (hi), on the
// split form x = I + F, F in [0, 1).
__device__ __forceinline__ void mirror_origin(int& I, float& F, bool hi, int n) {
    const int base = hi ? 2 * n : 0;
    if (F > 0.0f) { I = base - I - 1; F = 1.0f - F; }
    else { I = base - I; }
}

template <int NCMAX, int BITS>
__global__ void __launch_bounds__(256) walk_split_kernel(const WalkArgs a, const uint8_t* __restrict__ lat) {
    __shared__ float s_step[NCMAX], s_istep[NCMAX], s_k[NCMAX], s_pij[NCMAX * NCMAX];
    for (int i = threadIdx.x; i < NCMAX * NCMAX; i += blockDim.x) {
        s_pij[i] = (i < a.nc * a.nc) ? a.pijf[i] : 0.0f;
        if (i < NCMAX) {
            const float st = (i < a.nc) ? a.stepf[i] : 0.0f;
            s_step[i] = st;
            s_istep[i] = st > 0.0f ? 1.0f / st : 0.0f;
            // T2 exponent per voxel of path: (1/step) * (1/T2 in steps)
            s_k[i] = st > 0.0f ? (1.0f / st) * ((i < a.nc) ? a.t2invf[i] : 0.0f) : 0.0f;
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    const int warp_global = gtid >> 5;
    const int nwarps = nthr >> 5;
    const int64_t ntiles = (a.walker_end - a.walker_begin + 31) / 32;
    const bool pgse = (a.mode == 1);
    const bool mirror = (a.boundary == 0);
    const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
    const unsigned stride0 = (unsigned)n2 * (unsigned)n3, stride1 = (unsigned)n3;
    const float res = (float)a.res;
    double* slot = a.slots + (size_t)warp_global * a.timepoints * a.nvals;
    double* sig_slot = pgse ? a.sig_slots + (size_t)warp_global * a.ngrad_pad : nullptr;

    for (int64_t tile = warp_global; tile < ntiles; tile += nwarps) {
        const int64_t w = a.walker_begin + tile * 32 + lane;
        bool active = w < a.walker_end;
        FloatStream rng;
        rng.init(a.seed, (uint64_t)w);

        // initial position: uniform in the labelled voxels (rejection sampling)
        int g0 = 0, g1 = 0, g2 = 0;
        float f0 = 0.5f, f1 = 0.5f, f2 = 0.5f;
        if (active) {
            long long tries = 0;
            for (;;) {
                const float x0 = rng.next() * (float)n1;
                const float x1 = rng.next() * (float)n2;
                const float x2 = rng.next() * (float)n3;
                g0 = min((int)x0, n1 - 1); g1 = min((int)x1, n2 - 1); g2 = min((int)x2, n3 - 1);
                f0 = x0 - (float)g0; f1 = x1 - (float)g1; f2 = x2 - (float)g2;
                if (label_at<BITS>(lat, lin3(g0, g1, g2, n2, n3)) != 0) break;
                if (++tries >= kInitTryCap) { atomicOr(a.err, kErrInitCap); active = false; break; }
            }
        }
        unsigned lin = lin3(g0, g1, g2, n2, n3);
        int ai = active ? label_at<BITS>(lat, lin) : 0;
        // origin image (I + F per axis); displacement = (g - I) + (f - F)
        int I0 = g0, I1 = g1, I2 = g2;
        float F0 = f0, F1 = f1, F2 = f2;

        double w64 = 0.0;          // T2 exponent, folded
        float w32 = 0.0f;          // T2 exponent since the last fold
        double P0 = 0.0, P1 = 0.0, P2 = 0.0;   // PGSE displacement sums (voxels), folded
        float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
        int evi = 0;
        int next_ev = (pgse && a.nevents > 0) ? a.ev_step[0] : -1;
        if (pgse)
            for (int k = 0; k < a.npairs * 3; ++k) a.vscr[(size_t)k * nthr + gtid] = 0.0;

        for (int i = 0; i < a.tn; ++i) {
            if (active) {
                const float u1 = rng.next();
                const float u2 = rng.next();
                const float cz = 1.0f - 2.0f * u1;
                const float sz = 2.0f * sqrtf(u1 * (1.0f - u1));
                float sp, cp;
                sincospif(2.0f * u2, &sp, &cp);
                float v0 = sz * cp, v1 = sz * sp, v2 = cz;
                const float iv0 = __frcp_rn(fabsf(v0)), iv1 = __frcp_rn(fabsf(v1)), iv2 = __frcp_rn(fabsf(v2));
                float fstep = 1.0f;
                unsigned flo = 0u, fhi = 0u;
                for (int j = 0; (j < a.nite) && (fstep > 0.0f); ++j) {
                    const float t0 = face_dist(f0, v0, iv0);
                    const float t1 = face_dist(f1, v1, iv1);
                    const float t2 = face_dist(f2, v2, iv2);
                    float tmin = t0;
                    int hit = 0;
                    if (t1 < tmin) { tmin = t1; hit = 1; }
                    if (t2 < tmin) { tmin = t2; hit = 2; }
                    const float st = s_step[ai];
                    const float rem = fstep * st;
                    if (!(rem >= tmin)) {
                        // the step ends inside the voxel
                        f0 = fmaf(rem, v0, f0); f1 = fmaf(rem, v1, f1); f2 = fmaf(rem, v2, f2);
                        w32 = fmaf(rem, s_k[ai], w32);
                        fstep = 0.0f;
                        break;
                    }
                    // move onto the face
                    f0 = fmaf(tmin, v0, f0); f1 = fmaf(tmin, v1, f1); f2 = fmaf(tmin, v2, f2);
                    w32 = fmaf(tmin, s_k[ai], w32);
                    fstep = fmaxf(fstep - tmin * s_istep[ai], 0.0f);
                    const float vh = hit == 0 ? v0 : (hit == 1 ? v1 : v2);
                    const bool up = vh >= 0.0f;
                    if (hit == 0) f0 = up ? 1.0f : 0.0f;
                    else if (hit == 1) f1 = up ? 1.0f : 0.0f;
                    else f2 = up ? 1.0f : 0.0f;
                    const int gh = hit == 0 ? g0 : (hit == 1 ? g1 : g2);
                    const int nh = hit == 0 ? n1 : (hit == 1 ? n2 : n3);
                    int gj = up ? gh + 1 : gh - 1;
                    const int wall = (gj >= nh) ? 1 : ((gj < 0) ? -1 : 0);
                    if (wall != 0 && mirror) {
                        if (wall > 0) fhi |= 1u << hit; else flo |= 1u << hit;
                        if (hit == 0) v0 = -v0; else if (hit == 1) v1 = -v1; else v2 = -v2;
                        continue;
                    }
                    const unsigned st_h = hit == 0 ? stride0 : (hit == 1 ? stride1 : 1u);
                    unsigned lj;
                    if (wall == 0) {
                        lj = up ? lin + st_h : lin - st_h;
                    } else {
                        gj = (wall > 0) ? 0 : nh - 1;   // periodic neighbour
                        lj = (wall > 0) ? lin - (unsigned)(nh - 1) * st_h : lin + (unsigned)(nh - 1) * st_h;
                    }
                    const int aj = label_at<BITS>(lat, lj);
                    const float P = s_pij[ai * a.nc + aj];
                    bool cross;
                    if (P > 0.999999f) cross = true;
                    else if (P < 0.000001f) cross = false;
                    else cross = rng.next() < P;
                    if (cross) {
                        ai = aj;
                        lin = lj;
                        const float fin = up ? 0.0f : 1.0f;
                        if (hit == 0) { g0 = gj; f0 = fin; }
                        else if (hit == 1) { g1 = gj; f1 = fin; }
                        else { g2 = gj; f2 = fin; }
                        if (wall != 0) {
                            // periodic: shift the origin with the walker
                            const int sh = (wall > 0) ? -nh : nh;
                            if (hit == 0) I0 += sh; else if (hit == 1) I1 += sh; else I2 += sh;
                        }
                    } else {
                        if (hit == 0) v0 = -v0; else if (hit == 1) v1 = -v1; else v2 = -v2;
                    }
                }
                // mirror the origin for each wall hit this step (main.cu:302-310)
                if (flo | fhi) {
                    if (flo & 1u) mirror_origin(I0, F0, false, n1);
                    if (fhi & 1u) mirror_origin(I0, F0, true, n1);
                    if (flo & 2u) mirror_origin(I1, F1, false, n2);
                    if (fhi & 2u) mirror_origin(I1, F1, true, n2);
                    if (flo & 4u) mirror_origin(I2, F2, false, n3);
                    if (fhi & 4u) mirror_origin(I2, F2, true, n3);
                }
            }

            if (pgse) {
                // displacement sums (voxels) over the lobes
                p0 += (float)(g0 - I0) + (f0 - F0);
                p1 += (float)(g1 - I1) + (f1 - F1);
                p2 += (float)(g2 - I2) + (f2 - F2);
                const bool event = (i + 1 == next_ev);
                if (event || (i & 31) == 31) {
                    P0 += (double)p0; P1 += (double)p1; P2 += (double)p2;
                    p0 = p1 = p2 = 0.0f;
                }
                if (event) {
                    do {
                        const double cf = a.ev_coef[evi];
                        double* vv = a.vscr + (size_t)(a.ev_pair[evi] * 3) * nthr + gtid;
                        vv[0] += cf * P0;
                        vv[nthr] += cf * P1;
                        vv[2 * (size_t)nthr] += cf * P2;
                        ++evi;
                    } while (evi < a.nevents && a.ev_step[evi] == i + 1);
                    next_ev = (evi < a.nevents) ? a.ev_step[evi] : -1;
                }
                if (i == a.tn - 1) {
                    // final T2-weighted signal: phase_j = |g| (g_hat . V) res dt
                    const double s0 = active ? exp(-(w64 + (double)w32)) : 0.0;
                    const double scale = a.res * a.dt;
                    for (int base = 0; base < a.ngrad; base += 32) {
                        double mine = 0.0;
                        const int cnt = min(32, a.ngrad - base);
                        for (int k = 0; k < cnt; ++k) {
                            const int jg = base + k;
                            const double* vv = a.vscr + (size_t)(a.gpair[jg] * 3) * nthr + gtid;
                            const double* g = a.grad + 6 * jg;
                            const double phase =
                                g[2] * (vv[0] * g[3] + vv[nthr] * g[4] + vv[2 * (size_t)nthr] * g[5]) * scale;
                            const double r = warp_sum(s0 * cos(phase));
                            if (lane == k) mine = r;
                        }
                        if (lane < cnt) sig_slot[base + lane] += mine;
                    }
                }
            }

            if ((i % a.tstep) == 0) {
                const int tidx = i / a.tstep;
                if (tidx < a.timepoints) {
                    w64 += (double)w32;
                    w32 = 0.0f;
                    const float s0 = active ? (float)exp(-w64) : 0.0f;
                    const float dx = ((float)(g0 - I0) + (f0 - F0)) * res;
                    const float dy = ((float)(g1 - I1) + (f1 - F1)) * res;
                    const float dz = ((float)(g2 - I2) + (f2 - F2)) * res;
                    const float xx = dx * dx, yy = dy * dy, zz = dz * dz;
                    const float sxx = s0 * xx, syy = s0 * yy, szz = s0 * zz;
                    double* row = slot + (size_t)tidx * a.nvals;
                    // two rounds of 16 values: [sig0, dx2 x6, dx4 0..8], [dx4 9..14, counts]
                    double r;
                    {
                        double v[16];
                        v[0] = s0;
                        v[1] = sxx;  v[2] = s0 * dx * dy;  v[3] = s0 * dx * dz;
                        v[4] = syy;  v[5] = s0 * dy * dz;  v[6] = szz;
                        v[7] = sxx * xx;        v[8] = sxx * dx * dy;   v[9] = sxx * dx * dz;
                        v[10] = sxx * yy;       v[11] = sxx * dy * dz;  v[12] = sxx * zz;
                        v[13] = syy * dx * dy;  v[14] = syy * dx * dz;  v[15] = szz * dx * dy;
                        r = warp_reduce_scatter16(v, lane);
                    }
                    {
                        double v[16];
                        v[0] = szz * dx * dz;  v[1] = syy * yy;       v[2] = syy * dy * dz;
                        v[3] = syy * zz;       v[4] = szz * dy * dz;  v[5] = szz * zz;
#pragma unroll
                        for (int c = 0; c < 10; ++c) v[6 + c] = (active && ai == c) ? 1.0 : 0.0;
                        const double rb = warp_reduce_scatter16(v, lane);
                        if (lane >= 16) r = rb;
                    }
                    row[lane] += r;
                    if (!pgse) {
                        for (int base = 0; base < a.nbvec; base += 32) {
                            double mine = 0.0;
                            const int cnt = min(32, a.nbvec - base);
                            for (int k = 0; k < cnt; ++k) {
                                const int jb = base + k;
                                const float q = (float)a.qtab[(size_t)tidx * a.nbvec + jb];
                                const float qx = q * (dx * (float)a.bvec[jb * 3 + 0] + dy * (float)a.bvec[jb * 3 + 1] +
                                                      dz * (float)a.bvec[jb * 3 + 2]);
                                const double rr = warp_sum((double)(s0 * cosf(qx)));
                                if (lane == k) mine = rr;
                            }
                            if (lane < cnt) row[kRowHead + base + lane] += mine;
                        }
                    }
                }
            }
        }
    }
}

__global__ void pack2_kernel(const uint8_t* __restrict__ labels, size_t n, uint8_t* __restrict__ out) {
    const size_t nb = (n + 3) / 4;
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (size_t)gridDim.x * blockDim.x) {
        unsigned v = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const size_t i = 4 * b + k;
            if (i < n) v |= (unsigned)(labels[i] & 3u) << (2 * k);
        }
        out[b] = (uint8_t)v;
    }
}

template <int NCMAX, int BITS>
int launch_t(const WalkArgs& a, const uint8_t* lat, int grid, int block, void* stream) {
    walk_split_kernel<NCMAX, BITS><<<grid, block, 0, (cudaStream_t)stream>>>(a, lat);
    return (int)cudaGetLastError();
}

}  // namespace

int pack_labels_2bit(const uint8_t* labels, size_t n, uint8_t* out, void* stream) {
    const size_t nb = (n + 3) / 4;
    size_t grid = (nb + 255) / 256;
    if (grid > 8192) grid = 8192;
    pack2_kernel<<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(labels, n, out);
    return (int)cudaGetLastError();
}

int launch_walk_split(const WalkArgs& a, const uint8_t* lattice, int lattice_bits, int grid, int block,
                      void* stream) {
    if (block > 256 || block % 32) return (int)cudaErrorInvalidValue;
    if (lattice_bits == 2) return a.nc <= 4 ? launch_t<4, 2>(a, lattice, grid, block, stream)
                                            : (int)cudaErrorInvalidValue;
    return a.nc <= 4 ? launch_t<4, 8>(a, lattice, grid, block, stream)
                     : launch_t<8, 8>(a, lattice, grid, block, stream);
}

int walk_split_blocks_per_sm(int nc, int block) {
    int n = 0;
    cudaError_t e;
    if (nc <= 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, walk_split_kernel<4, 2>, block, 0);
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, walk_split_kernel<8, 8>, block, 0);
    return e == cudaSuccess ? n : -1;
}

}  // namespace rms

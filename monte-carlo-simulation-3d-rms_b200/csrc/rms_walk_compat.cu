// rms_walk_compat.cu -- the FP64, reference-compatible walk (RMS_PREC_COMPAT).
//
// Same per-walker algorithm as the reference kernel `propagate`
// (hpc_code/lib/main.cu:63-384 narrow pulse, main_PGSE.cu:65-410 PGSE): FP64
// positions, FP64 uniforms in the same draw order, the same sub-segment rule,
// mirror walls and Pij decisions, so a walker's voxel and event sequence is
// the CPU oracle's.  This file is compiled with -fmad=false: every product and
// sum is rounded like the reference's own expressions.
//
// What differs from the reference, by design:
//  - cross-walker sums: warp shuffles into per-warp FP64 rows, then one
//    ordered reduction (no CAS atomics, repeatable);
//  - PGSE phase: per walker the displacement sums over each gradient's two
//    lobes are formed from running prefix sums at the lobe edges, instead of
//    an O(Ngrad) update every step into a 16 KB local array
//    (main_PGSE.cu:99-100, 340-346).  phase_j = |g| (g_hat . V_j) dt with
//    V_j = sum_{lobe 1} dx - sum_{lobe 2} dx is the same sum, reassociated;
//  - walls: periodic as an option beside the reference's mirror;
//  - persistent grid: each warp walks 32 walkers at a time, tiles strided by
//    the number of warps in the grid.
#include <cuda_runtime.h>
#include <math.h>

#include "philox.cuh"
#include "rms_internal.h"
#include "warp_reduce.cuh"

namespace rms {
namespace {

constexpr double kRefPi = 3.14159265;  // main.cu:34 (the reference's truncated pi)
constexpr int kBlock = 128;

template <int NCMAX>
__device__ __forceinline__ void add_residence(double (&tc)[NCMAX], int c, double x) {
#pragma unroll
    for (int k = 0; k < NCMAX; ++k)
        if (k == c) tc[k] = tc[k] + x;
}

__device__ __forceinline__ unsigned lin3(int i, int j, int k, int n2, int n3) {
    return ((unsigned)i * (unsigned)n2 + (unsigned)j) * (unsigned)n3 + (unsigned)k;
}

// Nearest face along the ray on one axis (main.cu:200-219).
__device__ __forceinline__ void face(int axis, double v, double x, int g, double& tmin, int& hit) {
    double tmp;
    if (v > 0.0) {
        tmp = (double)g + 1.0 - x;
    } else if (v < 0.0) {
        tmp = (double)g - x;
    } else {
        tmp = 2.0;
    }
    double tt;
    if (fabs(tmp) > fabs(v)) {
        tt = 2.0;
    } else {
        const double q = tmp / v;
        tt = (0.0 < q) ? q : 0.0;  // std::max(0.0, q)
    }
    if (tt < tmin) { tmin = tt; hit = axis; }
}

template <int NCMAX, bool TRACE>
__global__ void __launch_bounds__(kBlock) walk_compat_kernel(const WalkArgs a) {
    __shared__ double s_step[NCMAX], s_t2[NCMAX], s_pij[NCMAX * NCMAX];
    for (int i = threadIdx.x; i < NCMAX * NCMAX; i += blockDim.x) {
        s_pij[i] = (i < a.nc * a.nc) ? a.pij[i] : 0.0;
        if (i < NCMAX) {
            s_step[i] = (i < a.nc) ? a.step[i] : 0.0;
            s_t2[i] = (i < a.nc) ? a.t2[i] : 1.0;
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    const int warp_global = gtid >> 5;
    const int nwarps = nthr >> 5;
    const int64_t nwalk = a.walker_end - a.walker_begin;
    const int64_t ntiles = (nwalk + 31) / 32;
    const bool pgse = (a.mode == 1);
    const bool mirror = (a.boundary == 0);
    double* slot = a.slots + (size_t)warp_global * a.timepoints * a.nvals;
    double* sig_slot = pgse ? a.sig_slots + (size_t)warp_global * a.ngrad_pad : nullptr;

    for (int64_t tile = warp_global; tile < ntiles; tile += nwarps) {
        const int64_t w = a.walker_begin + tile * 32 + lane;
        bool active = w < a.walker_end;
        DoubleStream rng;
        rng.init(a.seed, (uint64_t)w);

        // initial position: rejection sampling in the box (main.cu:117-125)
        double xi0 = 0.0, xi1 = 0.0, xi2 = 0.0;
        int g0 = 0, g1 = 0, g2 = 0;
        if (active) {
            long long tries = 0;
            for (;;) {
                xi0 = rng.next() * (double)a.n1;
                xi1 = rng.next() * (double)a.n2;
                xi2 = rng.next() * (double)a.n3;
                g0 = (int)floor(xi0); g1 = (int)floor(xi1); g2 = (int)floor(xi2);
                if (__ldg(a.labels + lin3(g0, g1, g2, a.n2, a.n3)) != 0) break;
                if (++tries >= kInitTryCap) { atomicOr(a.err, kErrInitCap); active = false; break; }
            }
        }
        // main.cu:129-132
        double xt0 = xi0, xt1 = xi1, xt2 = xi2;
        g0 = (int)floor(xt0); g1 = (int)floor(xt1); g2 = (int)floor(xt2);
        int ai = active ? (int)__ldg(a.labels + lin3(g0, g1, g2, a.n2, a.n3)) : 0;
        if (TRACE && active && w < a.trace_n) a.tr_init[w] = (int32_t)lin3(g0, g1, g2, a.n2, a.n3);

        double tc[NCMAX];
#pragma unroll
        for (int k = 0; k < NCMAX; ++k) tc[k] = 0.0;

        // PGSE: running displacement sum and the lobe-edge events
        double p0 = 0.0, p1 = 0.0, p2 = 0.0;
        int evi = 0;
        int next_ev = (pgse && a.nevents > 0) ? a.ev_step[0] : -1;
        if (pgse)
            for (int k = 0; k < a.npairs * 3; ++k) a.vscr[(size_t)k * nthr + gtid] = 0.0;

        int next_rec = 0, rec = 0;   // the next recorded step and its record
        for (int i = 0; i < a.tn; ++i) {                            // main.cu:134
            if (active) {
                double fstep = 1.0;
                unsigned f0 = 0u, f1 = 0u;
                uint32_t ev = 0u;
                int nev = 0;
                // direction (main.cu:140-151)
                double vr = rng.next();
                const double cos_t = 1.0 - 2.0 * vr;
                const double sin_t = 2.0 * sqrt(vr * (1.0 - vr));
                vr = rng.next();
                double v0 = sin_t * cos(2.0 * kRefPi * vr);
                double v1 = sin_t * sin(2.0 * kRefPi * vr);
                double v2 = cos_t;

                for (int j = 0; (j < a.nite) && (fstep > 0); ++j) {  // main.cu:153
                    double tmin = 2.0;
                    int hit = -1;
                    face(0, v0, xt0, g0, tmin, hit);
                    face(1, v1, xt1, g1, tmin, hit);
                    face(2, v2, xt2, g2, tmin, hit);
                    if (tmin < 0.0) break;                          // main.cu:226-229

                    const double st = s_step[ai];                   // main.cu:231-244
                    if ((fstep * st) >= tmin) {
                        const double q = tmin / st;
                        fstep = fstep - q;
                        xt0 = xt0 + tmin * v0;
                        xt1 = xt1 + tmin * v1;
                        xt2 = xt2 + tmin * v2;
                        add_residence(tc, ai, q);
                    } else {
                        const double f = st * fstep;
                        xt0 = xt0 + f * v0;
                        xt1 = xt1 + f * v1;
                        xt2 = xt2 + f * v2;
                        add_residence(tc, ai, fstep);
                        fstep = 0.0;
                        break;
                    }
                    if (hit < 0) { atomicOr(a.err, kErrStep); break; }

                    // neighbour voxel; lattice wall (main.cu:246-265)
                    const double vh = hit == 0 ? v0 : (hit == 1 ? v1 : v2);
                    const int gh = hit == 0 ? g0 : (hit == 1 ? g1 : g2);
                    const int nh = hit == 0 ? a.n1 : (hit == 1 ? a.n2 : a.n3);
                    int gj = (vh >= 0.0) ? gh + 1 : gh - 1;
                    const int wall = (gj >= nh) ? 1 : ((gj < 0) ? -1 : 0);
                    if (wall != 0 && mirror) {
                        if (wall > 0) f1 |= 1u << hit; else f0 |= 1u << hit;
                        if (hit == 0) v0 = -v0; else if (hit == 1) v1 = -v1; else v2 = -v2;
                        ev |= ((1u << 2) | (uint32_t)hit) << (4 * nev++);
                        continue;
                    }
                    if (wall != 0) gj = (wall > 0) ? 0 : nh - 1;   // periodic neighbour

                    // membrane (main.cu:272-289)
                    const int j0 = hit == 0 ? gj : g0;
                    const int j1 = hit == 1 ? gj : g1;
                    const int j2 = hit == 2 ? gj : g2;
                    const int aj = (int)__ldg(a.labels + lin3(j0, j1, j2, a.n2, a.n3));
                    const double P = s_pij[ai * a.nc + aj];
                    bool cross;
                    if (P > 0.999999) {
                        cross = true;
                    } else if (P < 0.000001) {
                        cross = false;
                    } else {
                        cross = rng.next() < P;
                    }
                    if (cross) {
                        ai = aj;
                        g0 = j0; g1 = j1; g2 = j2;
                        if (wall != 0) {
                            const double shift = (wall > 0) ? -(double)nh : (double)nh;
                            if (hit == 0) { xt0 = xt0 + shift; xi0 = xi0 + shift; }
                            else if (hit == 1) { xt1 = xt1 + shift; xi1 = xi1 + shift; }
                            else { xt2 = xt2 + shift; xi2 = xi2 + shift; }
                            ev |= ((1u << 2) | (uint32_t)hit) << (4 * nev++);
                        } else {
                            ev |= ((3u << 2) | (uint32_t)hit) << (4 * nev++);
                        }
                    } else {
                        if (hit == 0) v0 = -v0; else if (hit == 1) v1 = -v1; else v2 = -v2;
                        ev |= ((2u << 2) | (uint32_t)hit) << (4 * nev++);
                    }
                }
                if (fstep > 0) ev |= 1u << 31;
                ev |= (uint32_t)nev << 28;

                // mirror the origin for each wall hit this step (main.cu:302-310)
                if (f0 & 1u) xi0 = -xi0;
                if (f1 & 1u) xi0 = 2.0 * (double)a.n1 - xi0;
                if (f0 & 2u) xi1 = -xi1;
                if (f1 & 2u) xi1 = 2.0 * (double)a.n2 - xi1;
                if (f0 & 4u) xi2 = -xi2;
                if (f1 & 4u) xi2 = 2.0 * (double)a.n3 - xi2;
                if (TRACE && w < a.trace_n) {
                    a.tr_vox[(size_t)w * a.tn + i] = (int32_t)lin3(g0, g1, g2, a.n2, a.n3);
                    a.tr_ev[(size_t)w * a.tn + i] = ev;
                    double* tp = a.tr_pos + ((size_t)w * a.tn + i) * 3;
                    tp[0] = xt0; tp[1] = xt1; tp[2] = xt2;
                }
            }

            if (pgse) {
                // displacement of this step's position (main_PGSE.cu:336-338)
                p0 = p0 + (xt0 - xi0) * a.res;
                p1 = p1 + (xt1 - xi1) * a.res;
                p2 = p2 + (xt2 - xi2) * a.res;
                if (i + 1 == next_ev) {
                    do {
                        const double cf = a.ev_coef[evi];
                        double* vv = a.vscr + (size_t)(a.ev_pair[evi] * 3) * nthr + gtid;
                        vv[0] = vv[0] + cf * p0;
                        vv[nthr] = vv[nthr] + cf * p1;
                        vv[2 * (size_t)nthr] = vv[2 * (size_t)nthr] + cf * p2;
                        ++evi;
                    } while (evi < a.nevents && a.ev_step[evi] == i + 1);
                    next_ev = (evi < a.nevents) ? a.ev_step[evi] : -1;
                }
                if (i == a.tn - 1) {
                    // final T2-weighted signal (main_PGSE.cu:348-357)
                    double s0 = 0.0;
#pragma unroll
                    for (int c = 0; c < NCMAX; ++c)
                        if (c < a.nc) s0 = s0 + tc[c] / s_t2[c];
                    s0 = active ? exp(-1.0 * s0) : 0.0;
                    for (int base = 0; base < a.ngrad; base += 32) {
                        double mine = 0.0;
                        const int cnt = min(32, a.ngrad - base);
                        for (int k = 0; k < cnt; ++k) {
                            const int jg = base + k;
                            const double* vv = a.vscr + (size_t)(a.gpair[jg] * 3) * nthr + gtid;
                            const double* g = a.grad + 6 * jg;
                            const double phase =
                                g[2] * (vv[0] * g[3] + vv[nthr] * g[4] + vv[2 * (size_t)nthr] * g[5]) * a.dt;
                            const double r = warp_sum(s0 * cos(phase));
                            if (lane == k) mine = r;
                        }
                        if (lane < cnt) sig_slot[base + lane] += mine;
                    }
                }
            }

            // record every tstep steps (main.cu:333-379; i % tstep == 0 as a countdown)
            if (i == next_rec) {
                const int tidx = rec++;
                next_rec += a.tstep;
                if (tidx < a.timepoints) {
                    double s0 = 0.0;
#pragma unroll
                    for (int c = 0; c < NCMAX; ++c)
                        if (c < a.nc) s0 = s0 + tc[c] / s_t2[c];
                    s0 = active ? exp(-1.0 * s0) : 0.0;
                    const double dx = (xt0 - xi0) * a.res;
                    const double dy = (xt1 - xi1) * a.res;
                    const double dz = (xt2 - xi2) * a.res;
                    double v[32];
                    v[0] = s0;
                    v[1] = s0 * dx * dx;  v[2] = s0 * dx * dy;  v[3] = s0 * dx * dz;
                    v[4] = s0 * dy * dy;  v[5] = s0 * dy * dz;  v[6] = s0 * dz * dz;
                    v[7] = s0 * dx * dx * dx * dx;   v[8] = s0 * dx * dx * dx * dy;
                    v[9] = s0 * dx * dx * dx * dz;   v[10] = s0 * dx * dx * dy * dy;
                    v[11] = s0 * dx * dx * dy * dz;  v[12] = s0 * dx * dx * dz * dz;
                    v[13] = s0 * dx * dy * dy * dy;  v[14] = s0 * dx * dy * dy * dz;
                    v[15] = s0 * dx * dy * dz * dz;  v[16] = s0 * dx * dz * dz * dz;
                    v[17] = s0 * dy * dy * dy * dy;  v[18] = s0 * dy * dy * dy * dz;
                    v[19] = s0 * dy * dy * dz * dz;  v[20] = s0 * dy * dz * dz * dz;
                    v[21] = s0 * dz * dz * dz * dz;
#pragma unroll
                    for (int c = 0; c < 10; ++c) v[kColCount + c] = (active && ai == c) ? 1.0 : 0.0;
                    const double r = warp_reduce_scatter32(v, lane);
                    double* row = slot + (size_t)tidx * a.nvals;
                    row[lane] += r;
                    if (!pgse) {
                        // narrow-pulse signal (main.cu:374-378)
                        for (int base = 0; base < a.nbvec; base += 32) {
                            double mine = 0.0;
                            const int cnt = min(32, a.nbvec - base);
                            for (int k = 0; k < cnt; ++k) {
                                const int jb = base + k;
                                const double qx = a.qtab[(size_t)tidx * a.nbvec + jb] *
                                                  (dx * a.bvec[jb * 3 + 0] + dy * a.bvec[jb * 3 + 1] +
                                                   dz * a.bvec[jb * 3 + 2]);
                                const double rr = warp_sum(s0 * cos(qx));
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

template <int NCMAX, bool TRACE>
int launch_t(const WalkArgs& a, int grid, int block, void* stream) {
    walk_compat_kernel<NCMAX, TRACE><<<grid, block, 0, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

}  // namespace

int launch_walk_compat(const WalkArgs& a, int grid, int block, bool trace, void* stream) {
    if (block != kBlock) return (int)cudaErrorInvalidValue;
    if (a.nc <= 4) return trace ? launch_t<4, true>(a, grid, block, stream)
                                : launch_t<4, false>(a, grid, block, stream);
    return trace ? launch_t<8, true>(a, grid, block, stream)
                 : launch_t<8, false>(a, grid, block, stream);
}

int walk_compat_blocks_per_sm(int nc, bool trace) {
    int n = 0;
    cudaError_t e;
    if (nc <= 4)
        e = trace ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, walk_compat_kernel<4, true>, kBlock, 0)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, walk_compat_kernel<4, false>, kBlock, 0);
    else
        e = trace ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, walk_compat_kernel<8, true>, kBlock, 0)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, walk_compat_kernel<8, false>, kBlock, 0);
    return e == cudaSuccess ? n : -1;
}

}  // namespace rms

// rms_adjoint.cu -- gradients of the waveform-mode signal by trajectory
// recomputation (rms_adjoint_run in include/rms.h).
//
// For the split walk in waveform mode (rms_walk_split.cu) with signals
// C_j = sum_w s0_w cos phi_jw, S_j = sum_w s0_w sin phi_jw and upstream weights
// (gC_j, gS_j), the loss is L = sum_w L_w, L_w = s0_w sum_j (gC_j cos phi_jw +
// gS_j sin phi_jw).  Each walker is walked twice from its counter-based random
// streams -- nothing of the trajectory is stored:
//
//  pass 1 accumulates phi_jw; the tangent dphi_jw/dl of the phase with respect
//    to the step length l with the event sequence frozen (the displacement's
//    tangent gains the step direction each step and flips its component at
//    every reflection, membrane or mirror wall; the origin image and periodic
//    wraps do not depend on l); the residence path per compartment (the T2
//    weight s0 = exp(-sum_c t_c / T2_c)); and the permeation score
//    E_w = sum over Bernoulli crossings of (1[crossed] - Pij), the derivative of
//    the log-probability of the crossing decisions with respect to log P for
//    Pij = P / (1 + P).  From these, a_jw = dL_w/dphi_jw, L_w E_w, E_w,
//    sum_j a_jw dphi_jw and L_w t_wc are summed over walkers;
//  pass 2 walks the walker again and adds a_jw X_wb (X_wb: the bin's
//    displacement sum, um) into dL/dwave[b][j] -- the phase is linear in the
//    waveform, so this gradient is exact pathwise.
//
// The host turns the sums into dL/dwave, dL/dT2_c (analytic), dL/dkappa
// (score function: dP/dkappa = P/kappa, with the walkers' mean loss as the
// baseline -- sum_w (L_w - mean L) E_w, unbiased since E[E_w] = 0, and far
// less noisy than sum_w L_w E_w) and dL/dD (pathwise via dl/dD = l/(2D), plus
// the score through dP/dD = -P/(2D)).  The walk itself is
// the split walk's step for step (same streams, same arithmetic), so the
// gradients belong to the function the forward run evaluates.
#include <cuda_runtime.h>
#include <math.h>

#include "philox.cuh"
#include "rms_internal.h"
#include "split_lattice.cuh"
#include "warp_reduce.cuh"

namespace rms {
namespace {

// Float reduce-scatter of 16 values: lanes l and l ^ 16 end with the
// warp-wide sum of v[l & 15].
__device__ __forceinline__ float warp_reduce_scatter16f(float (&v)[16], int lane) {
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] += __shfl_xor_sync(kFullMask, v[k], 16);
#pragma unroll
    for (int half = 8; half > 0; half >>= 1) {
        const bool upper = (lane & half) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const float send = upper ? v[k] : v[k + half];
            const float keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(kFullMask, send, half);
        }
    }
    return v[0];
}

__global__ void __launch_bounds__(kAdjBlock) adjoint_kernel(const __grid_constant__ AdjArgs a) {
    constexpr int NC = kAdjNc, BITS = 4, NW = kAdjWaves;
    constexpr int kTab = 2 * NC + 2 * NC * NC;
    __shared__ float s_tab[kTab];
    for (int i = threadIdx.x; i < kTab; i += blockDim.x)
        s_tab[i] = i < NC ? a.step[i]
                          : (i < 2 * NC ? a.kexp[i - NC]
                                        : (i < 2 * NC + NC * NC ? a.pij[i - 2 * NC] : a.ratio[i - 2 * NC - NC * NC]));
    __syncthreads();
    const float* t_step = s_tab;
    const float* t_k = s_tab + NC;
    const float* t_pij = s_tab + 2 * NC;
    const float* t_ratio = s_tab + 2 * NC + NC * NC;

    const int lane = threadIdx.x & 31;
    const int warp_global = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const bool mirror = (a.boundary == 0);
    constexpr int kWall = wall_code<BITS>();
    const uint32_t key0 = (uint32_t)a.seed, key1 = (uint32_t)(a.seed >> 32);
    const uint8_t* lat = a.lat;
    const int s0 = a.s0, s1 = a.s1;

    for (int64_t tile = warp_global; tile < a.ntiles; tile += nwarps) {
        const int64_t w = a.walker_begin + tile * 32 + lane;
        const bool live = w < a.walker_end;
        const uint32_t wlo = (uint32_t)w, whi = (uint32_t)((uint64_t)w >> 32);
        float phi[NW], dphi[NW], aj[NW], tc[NC];
#pragma unroll
        for (int j = 0; j < NW; ++j) phi[j] = dphi[j] = aj[j] = 0.0f;
#pragma unroll
        for (int c = 0; c < NC; ++c) tc[c] = 0.0f;
        float E = 0.0f;
        double w64 = 0.0;

        for (int pass = 0; pass < 2; ++pass) {
            // start position: uniform in the labelled voxels (the split walk's draws)
            bool active = live;
            float f0 = 0.5f, f1 = 0.5f, f2 = 0.5f;
            unsigned lin = 0;
            if (active) {
                DomainStream init;
                init.init(a.seed, (uint64_t)w, kDomInit);
                long long tries = 0;
                for (;;) {
                    const float x0 = init.next() * (float)a.n1;
                    const float x1 = init.next() * (float)a.n2;
                    const float x2 = init.next() * (float)a.n3;
                    const int g0 = min((int)x0, a.n1 - 1), g1 = min((int)x1, a.n2 - 1), g2 = min((int)x2, a.n3 - 1);
                    f0 = x0 - (float)g0; f1 = x1 - (float)g1; f2 = x2 - (float)g2;
                    lin = (unsigned)(g0 + 1) * (unsigned)s0 + (unsigned)(g1 + 1) * (unsigned)s1 + (unsigned)(g2 + 1);
                    if (label_at<BITS>(lat, lin) != 0) break;
                    if (++tries >= kInitTryCap) { atomicOr(a.err, kErrInitCap); active = false; break; }
                }
            }
            int ai = active ? label_at<BITS>(lat, lin) : 0;
            float cur_step = t_step[ai], cur_k = t_k[ai];
            int D0 = 0, D1 = 0, D2 = 0;
            float Fm0 = f0, Fm1 = f1, Fm2 = f2;
            float d0 = f0, d1 = f1, d2 = f2;
            unsigned up = 0u;
            DomainStream perm;
            perm.init(a.seed, (uint64_t)w, kDomPerm);
            w64 = 0.0;
            float w32 = 0.0f;
            double P0 = 0.0, P1 = 0.0, P2 = 0.0;     // bin displacement sums (voxels), folded
            float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
            float T0 = 0.0f, T1 = 0.0f, T2 = 0.0f;  // d(displacement)/dl (voxels per voxel of step)
            float B0 = 0.0f, B1 = 0.0f, B2 = 0.0f;  // bin sums of the tangent
            int bin = 0, next_bin = a.bin_steps;
            uint32_t spare_u1 = 0u, spare_u2 = 0u;
            const bool p1st = (pass == 0);

            for (int i = 0; i < a.tn; ++i) {
                uint32_t r1, r2;
                if ((i & 1) == 0) {
                    const U4 b = dir_block((uint32_t)(i >> 1), key0, key1, wlo, whi);
                    r1 = b.x; r2 = b.y; spare_u1 = b.z; spare_u2 = b.w;
                } else {
                    r1 = spare_u1; r2 = spare_u2;
                }
                if (active) {
                    const float u1 = u32_to_float(r1), u2 = u32_to_float(r2);
                    const float cz = 1.0f - 2.0f * u1;
                    const float s2 = u1 * (1.0f - u1);
                    const float sz = 2.0f * s2 * rsqrtf(s2);
                    float sp, cp;
                    __sincosf(6.283185307179586f * (u2 - 0.5f), &sp, &cp);
                    const float v0 = sz * cp, v1 = sz * sp, v2 = cz;
                    if (p1st) { T0 += v0; T1 += v1; T2 += v2; }
                    const unsigned nu = (v0 > 0.0f ? 1u : 0u) | (v1 > 0.0f ? 2u : 0u) | (v2 > 0.0f ? 4u : 0u);
                    if (a.flight && (cell_at<BITS>(lat, lin) & flight_bit<BITS>())) {
                        const float x0 = fmaf(cur_step, v0, (up & 1u) ? 1.0f - d0 : d0);
                        const float x1 = fmaf(cur_step, v1, (up & 2u) ? 1.0f - d1 : d1);
                        const float x2 = fmaf(cur_step, v2, (up & 4u) ? 1.0f - d2 : d2);
                        const float k0 = floorf(x0), k1 = floorf(x1), k2 = floorf(x2);
                        const int ik0 = (int)k0, ik1 = (int)k1, ik2 = (int)k2;
                        const float o0n = x0 - k0, o1n = x1 - k1, o2n = x2 - k2;
                        lin += (unsigned)(ik0 * s0 + ik1 * s1 + ik2);
                        D0 += ik0; D1 += ik1; D2 += ik2;
                        w32 = fmaf(cur_step, cur_k, w32);
                        if (p1st) {
#pragma unroll
                            for (int c = 0; c < NC; ++c) tc[c] += (ai == c) ? cur_step : 0.0f;
                        }
                        d0 = (nu & 1u) ? 1.0f - o0n : o0n;
                        d1 = (nu & 2u) ? 1.0f - o1n : o1n;
                        d2 = (nu & 4u) ? 1.0f - o2n : o2n;
                        up = nu;
                    } else {
                        const unsigned turn = nu ^ up;
                        if (turn & 1u) d0 = 1.0f - d0;
                        if (turn & 2u) d1 = 1.0f - d1;
                        if (turn & 4u) d2 = 1.0f - d2;
                        up = nu;
                        const float av0 = fabsf(v0), av1 = fabsf(v1), av2 = fabsf(v2);
                        const float iv0 = __fdividef(1.0f, av0), iv1 = __fdividef(1.0f, av1), iv2 = __fdividef(1.0f, av2);
                        int dl0 = (up & 1u) ? s0 : -s0;
                        int dl1 = (up & 2u) ? s1 : -s1;
                        int dl2 = (up & 4u) ? 1 : -1;
                        float rem = cur_step;
                        for (int j = 0; j < a.nite; ++j) {
                            const float t0 = d0 * iv0, t1 = d1 * iv1, t2 = d2 * iv2;
                            const float tm = fminf(t0, fminf(t1, t2));
                            if (rem < tm) {
                                d0 = fmaf(-rem, av0, d0); d1 = fmaf(-rem, av1, d1); d2 = fmaf(-rem, av2, d2);
                                w32 = fmaf(rem, cur_k, w32);
                                if (p1st) {
#pragma unroll
                                    for (int c = 0; c < NC; ++c) tc[c] += (ai == c) ? rem : 0.0f;
                                }
                                rem = 0.0f;
                                break;
                            }
                            const int hit = (t0 == tm) ? 0 : ((t1 == tm) ? 1 : 2);
                            const float tcs = fmaxf(tm, 0.0f);
                            d0 = fmaf(-tcs, av0, d0); d1 = fmaf(-tcs, av1, d1); d2 = fmaf(-tcs, av2, d2);
                            w32 = fmaf(tcs, cur_k, w32);
                            if (p1st) {
#pragma unroll
                                for (int c = 0; c < NC; ++c) tc[c] += (ai == c) ? tcs : 0.0f;
                            }
                            rem -= tcs;
                            const int dl = hit == 0 ? dl0 : (hit == 1 ? dl1 : dl2);
                            unsigned lj = lin + (unsigned)dl;
                            int aj2 = label_at<BITS>(lat, lj);
                            bool cross;
                            if (aj2 == ai && a.same_cross) {
                                cross = true;
                            } else {
                                if (aj2 == kWall) {
                                    const bool hi = (up >> hit) & 1u;
                                    const int nh = hit == 0 ? a.n1 : (hit == 1 ? a.n2 : a.n3);
                                    if (mirror) {
                                        const int g = hi ? nh - 1 : 0;
                                        if (hit == 0) { int I = g - D0; mirror_origin(I, Fm0, hi, nh); D0 = g - I; }
                                        else if (hit == 1) { int I = g - D1; mirror_origin(I, Fm1, hi, nh); D1 = g - I; }
                                        else { int I = g - D2; mirror_origin(I, Fm2, hi, nh); D2 = g - I; }
                                        aj2 = -1;
                                    } else {
                                        const int sh = hit == 0 ? s0 : (hit == 1 ? s1 : 1);
                                        lj = hi ? lin - (unsigned)(nh - 1) * (unsigned)sh
                                                : lin + (unsigned)(nh - 1) * (unsigned)sh;
                                        aj2 = label_at<BITS>(lat, lj);
                                    }
                                }
                                if (aj2 < 0) {
                                    cross = false;
                                } else {
                                    const float P = t_pij[ai * NC + aj2];
                                    if (P > 0.999999f) {
                                        cross = true;
                                    } else if (P >= 0.000001f) {
                                        cross = perm.next() < P;
                                        if (p1st) E += (cross ? 1.0f : 0.0f) - P;   // d log p / d log P
                                    } else {
                                        cross = false;
                                    }
                                }
                            }
                            if (cross) {
                                if (aj2 != ai) {
                                    rem *= t_ratio[ai * NC + aj2];
                                    cur_step = t_step[aj2];
                                    cur_k = t_k[aj2];
                                    ai = aj2;
                                }
                                lin = lj;
                                const int du = ((up >> hit) & 1u) ? 1 : -1;
                                if (hit == 0) D0 += du; else if (hit == 1) D1 += du; else D2 += du;
                            } else {
                                up ^= 1u << hit;
                                if (hit == 0) dl0 = -dl0; else if (hit == 1) dl1 = -dl1; else dl2 = -dl2;
                                if (p1st) {   // a reflection flips the tangent's component
                                    if (hit == 0) T0 = -T0; else if (hit == 1) T1 = -T1; else T2 = -T2;
                                }
                            }
                            if (hit == 0) d0 = 1.0f; else if (hit == 1) d1 = 1.0f; else d2 = 1.0f;
                            if (!(rem > 0.0f)) break;
                        }
                    }
                }
                const float o0 = (up & 1u) ? 1.0f - d0 : d0;
                const float o1 = (up & 2u) ? 1.0f - d1 : d1;
                const float o2 = (up & 4u) ? 1.0f - d2 : d2;
                p0 += (float)D0 + (o0 - Fm0);
                p1 += (float)D1 + (o1 - Fm1);
                p2 += (float)D2 + (o2 - Fm2);
                if (p1st) { B0 += T0; B1 += T1; B2 += T2; }
                const bool event = (i + 1 == next_bin);
                if (event || (i & 31) == 31) {
                    P0 += (double)p0; P1 += (double)p1; P2 += (double)p2;
                    p0 = p1 = p2 = 0.0f;
                    w64 += (double)w32;
                    w32 = 0.0f;
                }
                if (event) {
                    const double x0 = P0 * (double)a.res, x1 = P1 * (double)a.res, x2 = P2 * (double)a.res;
                    const double* wv = a.wave + (size_t)bin * a.nwave * 3;
                    if (p1st) {
#pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            if (j < a.nwave) {
                                const double g0 = __ldg(wv + 3 * j), g1 = __ldg(wv + 3 * j + 1), g2 = __ldg(wv + 3 * j + 2);
                                phi[j] += (float)(g0 * x0 + g1 * x1 + g2 * x2);
                                dphi[j] += (float)((g0 * B0 + g1 * B1 + g2 * B2) * (double)a.res);
                            }
                        }
                        B0 = B1 = B2 = 0.0f;
                    } else {
                        // dL/dwave[bin][j] += a_jw X_wb, summed over the warp's walkers
                        const float xs[3] = {(float)x0, (float)x1, (float)x2};
#pragma unroll
                        for (int ax = 0; ax < 3; ++ax) {
                            float v[NW];
#pragma unroll
                            for (int j = 0; j < NW; ++j) v[j] = aj[j] * xs[ax];
                            const float r = warp_reduce_scatter16f(v, lane);
                            if (lane < a.nwave) atomicAdd(a.dwave + ((size_t)bin * a.nwave + lane) * 3 + ax, r);
                        }
                    }
                    P0 = P1 = P2 = 0.0;
                    ++bin;
                    next_bin += a.bin_steps;
                }
            }
            w64 += (double)w32;

            if (p1st) {
                // this walker's loss, its derivatives, and the forward signal
                const float s0w = active ? (float)exp(-w64) : 0.0f;
                float Lw = 0.0f, G = 0.0f;
#pragma unroll
                for (int j = 0; j < NW; ++j) {
                    float sn = 0.0f, cs = 0.0f, gc = 0.0f, gs = 0.0f;
                    if (j < a.nwave) {
                        sincosf(phi[j], &sn, &cs);
                        gc = __ldg(a.gup + 2 * j);
                        gs = __ldg(a.gup + 2 * j + 1);
                    }
                    Lw += s0w * (gc * cs + gs * sn);
                    aj[j] = s0w * (gs * cs - gc * sn);
                    G += aj[j] * dphi[j];
                    const double C = warp_sum((double)(s0w * cs)), S = warp_sum((double)(s0w * sn));
                    if (lane == 0 && j < a.nwave) {
                        atomicAdd(a.sums + kAdjSumSig + 2 * j, C);
                        atomicAdd(a.sums + kAdjSumSig + 2 * j + 1, S);
                    }
                }
                const double L = warp_sum((double)Lw), LE = warp_sum((double)Lw * (double)E),
                             GP = warp_sum((double)G), ES = warp_sum(active ? (double)E : 0.0);
                if (lane == 0) {
                    atomicAdd(a.sums + kAdjSumL, L);
                    atomicAdd(a.sums + kAdjSumLE, LE);
                    atomicAdd(a.sums + kAdjSumPath, GP);
                    atomicAdd(a.sums + kAdjSumE, ES);
                }
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    // residence time in steps: path in compartment c / its step length
                    const float st = t_step[c];
                    const double LT = warp_sum(st > 0.0f ? (double)Lw * (double)(tc[c] / st) : 0.0);
                    if (lane == 0) atomicAdd(a.sums + kAdjSumLT + c, LT);
                }
            }
        }
    }
}

}  // namespace

int launch_adjoint(const AdjArgs& a, int grid, void* stream) {
    adjoint_kernel<<<grid, kAdjBlock, 0, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

int adjoint_blocks_per_sm() {
    int n = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjoint_kernel, kAdjBlock, 0);
    return e == cudaSuccess ? n : -1;
}

}  // namespace rms

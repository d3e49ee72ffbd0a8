// rms_adjoint.cu -- gradients of the waveform-mode signal by trajectory
// recomputation (rms_adjoint_run in include/rms.h).
//
// For the split walk in waveform mode (rms_walk_split.cu) with signals
// C_j = sum_w s0_w cos phi_jw, S_j = sum_w s0_w sin phi_jw and upstream weights
// (gC_j, gS_j), the loss is L = sum_w L_w, L_w = s0_w sum_j (gC_j cos phi_jw +
// gS_j sin phi_jw).  The estimators, as three walks of each walker from its
// counter-based random streams (FORM 0, nothing of the trajectory stored):
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
//    waveform, so this gradient is exact pathwise;
//  pass 3 (with permeable membranes) walks every walker that made nb_w > 0
//    permeation draws once more, with one of those draws, chosen uniformly
//    (its own counter domain), forced the other way and the rest of the walk
//    on the same streams, and sums nb_w Pij (1 - Pij) (L_w[crossed] -
//    L_w[reflected]): the weak derivative of the Bernoulli draws, an unbiased
//    estimate of dL/dlog P that measures what a crossing changes instead of
//    correlating the loss with rare crossings as the score function does.
//  By default (FORMs 1 and 2 below) pass 1 also records what pass 2 reads
//    (X_wb; the time-rescaling sums, linear in a_jw) so pass 2 is not walked,
//    and the walker's state at checkpoints: a forced walk repeats its
//    unforced walk up to the forced draw, so it is walked from the last
//    checkpoint before that draw, in a second launch over walkers grouped by
//    resume step.
//
// The host turns the sums into dL/dwave, dL/dT2_c (analytic), dL/dkappa
// (dP/dkappa = P/kappa: the forced-draw sum / kappa; the score function
// sum_w (L_w - mean L) E_w / kappa -- unbiased since E[E_w] = 0 -- is kept for
// comparison) and dL/dD.  dL/dD comes from time rescaling:
// a walk with diffusivity D(1 + eps) (and permeability kappa(1 + eps)) over
// [0, T] is, in law, the D-walk over [0, T(1 + eps)], so with x(t) the
// displacement, g_j the piecewise-constant waveform and W the T2 exponent
//   dphi_j/deps = -phi_j + sum_b t_b+1 (g_j,b - g_j,b+1) . x(t_b+1)  (g_j,nbins = 0)
//   dW/deps     = -W + T / T2(c_T)
// and D dL/dD = sum_w dL_w/deps - kappa dL/dkappa.  It sees the jumps of the
// walk at voxel corners, mirror walls and changed permeation draws, which the
// pathwise derivative through the step length (events frozen, also summed)
// does not; it is exact for the continuum process and carries the walk's
// time-discretisation error.  All passes walk the split walk's step
// (split_step.cuh: same streams, same arithmetic), so the gradients belong to
// the function the forward run evaluates.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "philox.cuh"
#include "rms_internal.h"
#include "split_lattice.cuh"
#include "split_step.cuh"
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

// What pass 1 records during a step (split_step's hooks): the path per
// compartment, the displacement's tangent with respect to the step length
// (flipped at every reflection) and the permeation score.
template <int NC>
struct AdjHooks {
    bool rec;             // pass 1 records; the others only walk
    bool force;           // pass 3: draw number force_at goes the other way
    float tc[NC];         // path per compartment (voxels)
    float T0, T1, T2;     // d(displacement)/dl, voxels per voxel of step
    float E;              // sum over Bernoulli draws of 1[crossed] - Pij
    int nb;               // Bernoulli draws so far
    int force_at;         // pass 3: the draw to flip
    float Pf;             // pass 3: its Pij
    bool xf;              // pass 3: its outcome before the flip
    __device__ __forceinline__ void path(int c, float len) {
        if (rec) {
#pragma unroll
            for (int k = 0; k < NC; ++k) tc[k] += (c == k) ? len : 0.0f;
        }
    }
    __device__ __forceinline__ void reflect(int axis) {
        if (rec) {
            if (axis == 0) T0 = -T0; else if (axis == 1) T1 = -T1; else T2 = -T2;
        }
    }
    __device__ __forceinline__ bool bernoulli(bool cross, float P) {
        if (rec) E += (cross ? 1.0f : 0.0f) - P;   // d log p / d log P
        if (force && nb == force_at) {
            Pf = P;
            xf = cross;
            cross = !cross;
        }
        ++nb;
        return cross;
    }
};

// JAC: instead of one weighted loss, the derivatives of every waveform's two
// signal sums C_j, S_j with respect to D, kappa and T2 (Jacobian columns; the
// sums at a.sums + kAdjSums, layout kJac* in rms_internal.h); dL/dwave is not
// formed.  The R_j of the time rescaling go to dphi[] in pass 2 (FORM 1: to
// their own array in pass 1) and the forced walk's phases to dphi[] in pass 3,
// so phi[] keeps pass 1's phases.
// One float per waveform for the calling lane, in shared memory: column
// threadIdx.x of a [NW][kAdjBlock] block (consecutive lanes, consecutive
// banks).  The walker's phases, tangents and a_jw are read and written only at
// bin ends and pass ends, so they need not hold registers through the step loop.
struct LaneArr {
    float* p;
    __device__ __forceinline__ float& operator[](int j) const { return p[j * kAdjBlock]; }
};

// Resident blocks per SM: at least 5 for the weighted-loss form (96 registers,
// no spills); the Jacobian form takes the compiler's choice (123 registers, 4
// blocks) except FORMs 1 and 2, held to 4 blocks (unbounded they took 248 and
// 134 registers).  FORM 1 of the weighted form also runs at 4 blocks: at 5
// (96 registers, 116 bytes spilled) the job below took 175 ms, at 4 (128
// registers, 48 bytes) 155 ms.
// Measured on a 64x64x512 axon, 1e6 walkers x 5000 steps, 16 waveforms, all
// passes in one launch: weighted 428 ms (518 ms at 4 blocks), Jacobian 390 ms
// (416 ms when held to 4 blocks at 115 registers); with the per-lane arrays
// in registers (3 blocks) 541 / 474 ms.  FORM 1, the dL/dwave reduction and
// FORM 2 (11 resume steps 480 steps apart): 155 / 149 ms (forward walk 154 ms;
// with pass 2 still walked and the forced walks grouped, 310 / 308 ms).
//
// FORM 0 walks all passes in this launch.  FORM 1 walks pass 1 only and
// leaves in memory what passes 2 and 3 need: the bin displacement sums X_wb
// and a_jw (weighted form; adjoint_dwave_kernel forms dL/dwave from them),
// the time-rescaling sums R_j summed in pass 1 from the displacement at each
// bin end (a_jw multiplies them only at the end), and the walker's state at
// every checkpoint step (a multiple of 3, 32 and the bin length, where no
// partial sum is in flight).  At the end it picks the forced draw and the last
// checkpoint before it and lists the walker under that resume step.  FORM 2
// walks the forced walks of those lists, 32 walkers of one resume step per
// warp, each from its checkpoint -- so a warp no longer walks from step 0
// because one lane's draw came early.  The sums are the single launch's up to
// the order of the float and FP64 sums.
constexpr int adj_min_blocks(bool jac, int form) { return form == 1 ? 4 : (jac ? (form == 2 ? 4 : 1) : 5); }

template <bool JAC, int FORM>
__global__ void __launch_bounds__(kAdjBlock, adj_min_blocks(JAC, FORM)) adjoint_kernel(const __grid_constant__ AdjArgs a) {
    constexpr int NC = kAdjNc, BITS = 4, NW = kAdjWaves;
    constexpr int kTab = 2 * NC + 2 * NC * NC;
    __shared__ float s_tab[kTab];
    // per lane: phi, dphi, aj (LaneArr); FORM 1: + the time-rescaling sums R_j
    __shared__ float s_lane[FORM == 1 ? 4 : 3][NW][kAdjBlock];
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
    const uint32_t key0 = (uint32_t)a.seed, key1 = (uint32_t)(a.seed >> 32);
    const uint8_t* lat = a.lat;
    const int s0 = a.s0, s1 = a.s1;

    for (int64_t tile = warp_global; tile < a.ntiles; tile += nwarps) {
        int64_t w;
        bool live;
        int gb = 0;   // FORM 2: the resume bucket of this tile
        int64_t wr = 0;   // the walker's index within the launch
        if (FORM == 2) {
            // tile -> (bucket, first entry): the buckets' tiles in order
            int64_t t = tile;
            int cnt = 0;
            for (gb = 0; gb < a.nbk; ++gb) {
                cnt = __ldg(a.bcount + gb);
                const int64_t nt = (cnt + 31) / 32;
                if (t < nt) break;
                t -= nt;
            }
            if (gb >= a.nbk) break;   // past the last listed walker (tiles only grow)
            const int64_t e = t * 32 + lane;
            live = e < cnt;
            wr = live ? (int64_t)__ldg(a.blist + (size_t)gb * a.nwalk + e) : 0;
        } else {
            wr = tile * 32 + lane;
            live = a.walker_begin + wr < a.walker_end;
        }
        w = a.walker_begin + wr;
        const uint32_t wlo = (uint32_t)w, whi = (uint32_t)((uint64_t)w >> 32);
        const LaneArr phi{&s_lane[0][0][threadIdx.x]}, dphi{&s_lane[1][0][threadIdx.x]}, aj{&s_lane[2][0][threadIdx.x]};
        const LaneArr rr{&s_lane[FORM == 1 ? 3 : 0][0][threadIdx.x]};   // FORM 1 only
#pragma unroll
        for (int j = 0; j < NW; ++j) phi[j] = dphi[j] = aj[j] = 0.0f;
        if (FORM == 1) {
#pragma unroll
            for (int j = 0; j < NW; ++j) rr[j] = 0.0f;
        }
        AdjHooks<NC> h;
#pragma unroll
        for (int c = 0; c < NC; ++c) h.tc[c] = 0.0f;
        h.E = 0.0f;
        h.force_at = -1;
        h.Pf = 0.0f;
        h.xf = false;
        double w64 = 0.0;
        float tr = 0.0f;   // this walker's time-rescaling derivative dL_w/d(eps)
        float Lkeep = 0.0f;   // this walker's loss (pass 1)
        int nb_w = 0;         // its Bernoulli draws (pass 1)
        float s0keep = 0.0f;  // JAC: its T2 weight s0 (pass 1)
        float wkeep = 0.0f;   // JAC: W - T / T2(c_T), the T2 weight's time-rescaling term (pass 1)
        int nb_at[kAdjCkMax];  // FORM 1: draws before checkpoint c (step c * ck_every)
        if (FORM == 2 && live) {
            // what pass 1 left for this walker (FORM 1's summary)
            const size_t nw = (size_t)a.nwalk;
            Lkeep = __uint_as_float(a.ws[0 * nw + wr]);
            nb_w = (int)a.ws[1 * nw + wr];
            s0keep = __uint_as_float(a.ws[2 * nw + wr]);
            if (JAC) {
#pragma unroll
                for (int j = 0; j < NW; ++j) phi[j] = __uint_as_float(a.ws[(3 + j) * nw + wr]);
            }
        }

        for (int pass = (FORM == 2 ? 2 : 0); pass < (FORM == 0 ? (a.force ? 3 : 2) : (FORM == 1 ? 1 : 3)); ++pass) {
            // pass 3 walks only the walkers that made a draw, and a warp with
            // none of them skips it
            if (FORM == 0 && pass == 2 && !__any_sync(kFullMask, live && nb_w > 0)) break;
            // start position: uniform in the labelled voxels (the split walk's draws)
            bool active = live && (pass < 2 || nb_w > 0);
            const bool resume = FORM == 2 && gb > 0;   // from a saved state, not from the start
            float f0 = 0.5f, f1 = 0.5f, f2 = 0.5f;
            unsigned lin = 0;
            if (active && !resume) {
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
            const int ai0 = (active && !resume) ? label_at<BITS>(lat, lin) : 0;
            SplitWalker wk{lin, (active && !resume) ? cell_at<BITS>(lat, lin) : 0u, f0, f1, f2, 0, 0, 0, f0, f1, f2,
                        ai0, t_step[ai0], t_k[ai0], 0.0f};
            const SplitGeom geo{lat, s0, s1, a.nite, (bool)a.flight, (bool)a.same_cross, mirror};
            auto nsize = [&](int axis) { return axis == 0 ? a.n1 : (axis == 1 ? a.n2 : a.n3); };
            DomainStream perm;
            perm.init(a.seed, (uint64_t)w, kDomPerm);
            w64 = 0.0;
            double P0 = 0.0, P1 = 0.0, P2 = 0.0;     // bin displacement sums (voxels), folded
            float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
            h.T0 = h.T1 = h.T2 = 0.0f;
            h.rec = (pass == 0);
            h.force = (pass == 2);
            h.nb = 0;
            if (pass == 2) {
                // the draw to flip, uniform over this walker's nb_w draws
                DomainStream fs;
                fs.init(a.seed, (uint64_t)w, kDomForce);
                h.force_at = min((int)(fs.next() * (float)nb_w), nb_w - 1);
            }
            if (pass > 0) {
#pragma unroll
                for (int j = 0; j < NW; ++j) {
                    if (JAC) dphi[j] = 0.0f;            // pass 2: R_j; pass 3: the forced phases
                    else if (pass == 2) phi[j] = 0.0f;  // pass 3: the forced phases
                }
            }
            int i_start = 0;
            if (resume) {
                // the state pass 1 saved at step gb * ck_every (layout: FORM 1's save below)
                i_start = gb * a.ck_every;
                if (active) {
                    const size_t nw = (size_t)a.nwalk;
                    const uint32_t* c = a.ck + (size_t)(gb - 1) * kAdjCkWords * nw + wr;
                    wk.lin = c[0 * nw]; wk.cell = c[1 * nw];
                    wk.o0 = __uint_as_float(c[2 * nw]); wk.o1 = __uint_as_float(c[3 * nw]);
                    wk.o2 = __uint_as_float(c[4 * nw]);
                    wk.D0 = (int)c[5 * nw]; wk.D1 = (int)c[6 * nw]; wk.D2 = (int)c[7 * nw];
                    wk.Fm0 = __uint_as_float(c[8 * nw]); wk.Fm1 = __uint_as_float(c[9 * nw]);
                    wk.Fm2 = __uint_as_float(c[10 * nw]);
                    wk.ai = (int)c[11 * nw];
                    wk.cur_step = __uint_as_float(c[12 * nw]); wk.cur_k = __uint_as_float(c[13 * nw]);
                    wk.w32 = __uint_as_float(c[14 * nw]);
                    perm.block = c[15 * nw]; perm.q1 = c[16 * nw]; perm.q2 = c[17 * nw]; perm.q3 = c[18 * nw];
                    perm.left = (int)c[19 * nw];
                    w64 = __hiloint2double((int)c[21 * nw], (int)c[20 * nw]);
                    h.nb = (int)c[22 * nw];
#pragma unroll
                    for (int j = 0; j < NW; ++j) {
                        const float v = __uint_as_float(c[(23 + j) * nw]);
                        if (JAC) dphi[j] = v;
                        else phi[j] = v;
                    }
                }
            }
            float B0 = 0.0f, B1 = 0.0f, B2 = 0.0f;  // bin sums of the tangent
            int bin = i_start / a.bin_steps, next_bin = (i_start / a.bin_steps + 1) * a.bin_steps;
            float q0 = 0.0f, q1 = 0.0f, q2 = 0.0f, q3 = 0.0f;   // the split walk's direction stream
            int phase = 0;
            uint32_t dblk = (uint32_t)(i_start / 3);
            const bool p1st = (pass == 0);
            int next_ck = (FORM == 1) ? 0 : -1;   // FORM 1: the next checkpoint step
            int ck_n = 0;

            for (int i = i_start; i < a.tn; ++i) {
                if (FORM == 1 && i == next_ck) {
                    // a checkpoint step: no partial sum is in flight here; the
                    // state at checkpoint c >= 1 goes to slot c - 1
                    if (ck_n < kAdjCkMax) nb_at[ck_n] = h.nb;
                    if (a.force && ck_n > 0 && ck_n < kAdjCkMax && live) {
                        const size_t nw = (size_t)a.nwalk;
                        uint32_t* c = a.ck + (size_t)(ck_n - 1) * kAdjCkWords * nw + wr;
                        c[0 * nw] = wk.lin; c[1 * nw] = wk.cell;
                        c[2 * nw] = __float_as_uint(wk.o0); c[3 * nw] = __float_as_uint(wk.o1);
                        c[4 * nw] = __float_as_uint(wk.o2);
                        c[5 * nw] = (uint32_t)wk.D0; c[6 * nw] = (uint32_t)wk.D1; c[7 * nw] = (uint32_t)wk.D2;
                        c[8 * nw] = __float_as_uint(wk.Fm0); c[9 * nw] = __float_as_uint(wk.Fm1);
                        c[10 * nw] = __float_as_uint(wk.Fm2);
                        c[11 * nw] = (uint32_t)wk.ai;
                        c[12 * nw] = __float_as_uint(wk.cur_step); c[13 * nw] = __float_as_uint(wk.cur_k);
                        c[14 * nw] = __float_as_uint(wk.w32);
                        c[15 * nw] = perm.block; c[16 * nw] = perm.q1; c[17 * nw] = perm.q2; c[18 * nw] = perm.q3;
                        c[19 * nw] = (uint32_t)perm.left;
                        c[20 * nw] = (uint32_t)__double2loint(w64); c[21 * nw] = (uint32_t)__double2hiint(w64);
                        c[22 * nw] = (uint32_t)h.nb;
#pragma unroll
                        for (int j = 0; j < NW; ++j) c[(23 + j) * nw] = __float_as_uint(phi[j]);
                    }
                    ++ck_n;
                    next_ck += a.ck_every;
                }
                float u1, u2;
                if (phase == 0) {
                    float u[6];
                    dir_fields(dir_block(dblk++, key0, key1, wlo, whi), u);
                    u1 = u[0]; u2 = u[1]; q0 = u[2]; q1 = u[3]; q2 = u[4]; q3 = u[5];
                    phase = 1;
                } else if (phase == 1) {
                    u1 = q0; u2 = q1; phase = 2;
                } else {
                    u1 = q2; u2 = q3; phase = 0;
                }
                if (active) {
                    float v0, v1, v2;
                    split_direction(u1, u2, v0, v1, v2);
                    if (p1st) { h.T0 += v0; h.T1 += v1; h.T2 += v2; }
                    split_step<NC, BITS, 0>(wk, v0, v1, v2, geo, t_step, t_k, t_pij, t_ratio, perm, nsize, h);
                }
                const float o0 = wk.o0, o1 = wk.o1, o2 = wk.o2;
                const int D0 = wk.D0, D1 = wk.D1, D2 = wk.D2;
                const float Fm0 = wk.Fm0, Fm1 = wk.Fm1, Fm2 = wk.Fm2;
                p0 += (float)D0 + (o0 - Fm0);
                p1 += (float)D1 + (o1 - Fm1);
                p2 += (float)D2 + (o2 - Fm2);
                if (p1st) { B0 += h.T0; B1 += h.T1; B2 += h.T2; }
                const bool event = (i + 1 == next_bin);
                if (event || (i & 31) == 31) {
                    P0 += (double)p0; P1 += (double)p1; P2 += (double)p2;
                    p0 = p1 = p2 = 0.0f;
                    w64 += (double)wk.w32;
                    wk.w32 = 0.0f;
                }
                if (event) {
                    const double x0 = P0 * (double)a.res, x1 = P1 * (double)a.res, x2 = P2 * (double)a.res;
                    const double* wv = a.wave + (size_t)bin * a.nwave * 3;
                    const float4* wq = a.wq + (size_t)bin * a.nwave * 2;   // [j]: g_j,b - g_j,b+1; g_j,b res
                    if (pass != 1) {
                        // the phases (pass 1: and their tangents; pass 3: of the forced walk)
#pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            if (j < a.nwave) {
                                const double g0 = __ldg(wv + 3 * j), g1 = __ldg(wv + 3 * j + 1), g2 = __ldg(wv + 3 * j + 2);
                                const float inc = (float)(g0 * x0 + g1 * x1 + g2 * x2);
                                if (JAC && pass == 2) dphi[j] += inc;
                                else phi[j] += inc;
                                if (p1st) {
                                    const float4 gr = __ldg(wq + 2 * j + 1);
                                    dphi[j] += fmaf(gr.z, B2, fmaf(gr.y, B1, gr.x * B0));
                                }
                            }
                        }
                        B0 = B1 = B2 = 0.0f;
                        if (FORM == 1) {
                            // X_wb for dL/dwave, and R_j += t (g_j,b - g_j,b+1) . x(t) as pass 2 sums it
                            if (!JAC && live) {
                                const size_t nw = (size_t)a.nwalk;
                                float* xb = a.xbin + (size_t)bin * 3 * nw + wr;
                                xb[0] = (float)x0;
                                xb[nw] = (float)x1;
                                xb[2 * nw] = (float)x2;
                            }
                            const float xe0 = ((float)D0 + (o0 - Fm0)) * a.res,
                                        xe1 = ((float)D1 + (o1 - Fm1)) * a.res,
                                        xe2 = ((float)D2 + (o2 - Fm2)) * a.res;
                            const float tb = (float)(i + 1);
#pragma unroll
                            for (int j = 0; j < NW; ++j) {
                                if (j < a.nwave) {
                                    const float4 q = __ldg(wq + 2 * j);
                                    rr[j] = fmaf(tb, q.x * xe0 + q.y * xe1 + q.z * xe2, rr[j]);
                                }
                            }
                        }
                    } else {
                        // time rescaling: at the end of bin b (time t = (b + 1) bin_steps dt)
                        // sum_j a_jw t (g_j,b - g_j,b+1) . x(t), g_j,nbins = 0
                        const float xe0 = ((float)D0 + (o0 - Fm0)) * a.res, xe1 = ((float)D1 + (o1 - Fm1)) * a.res,
                                    xe2 = ((float)D2 + (o2 - Fm2)) * a.res;
                        const float tb = (float)(i + 1);   // steps (the waveform table carries dt)
#pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            if (j < a.nwave) {
                                const float4 q = __ldg(wq + 2 * j);
                                if (JAC) dphi[j] = fmaf(tb, q.x * xe0 + q.y * xe1 + q.z * xe2, dphi[j]);   // R_j
                                else tr = fmaf(aj[j] * tb, q.x * xe0 + q.y * xe1 + q.z * xe2, tr);
                            }
                        }
                        if (!JAC) {
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
                    }
                    P0 = P1 = P2 = 0.0;
                    ++bin;
                    next_bin += a.bin_steps;
                }
            }
            w64 += (double)wk.w32;
            wk.w32 = 0.0f;

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
                    tr -= aj[j] * phi[j];
                    if (FORM == 1 && !JAC && j < a.nwave) {
                        tr = fmaf(aj[j], rr[j], tr);   // pass 2's time-rescaling sum
                        if (live) a.ajw[(size_t)j * a.nwalk + wr] = aj[j];
                    }
                    const double C = warp_sum((double)(s0w * cs)), S = warp_sum((double)(s0w * sn));
                    if (lane == 0 && j < a.nwave) {
                        atomicAdd(a.sums + kAdjSumSig + 2 * j, C);
                        atomicAdd(a.sums + kAdjSumSig + 2 * j + 1, S);
                    }
                    if (JAC && j < a.nwave) {
                        // score and residence sums of C_j and S_j
                        const double Ew = active ? (double)h.E : 0.0;
                        const double CE = warp_sum((double)(s0w * cs) * Ew), SE = warp_sum((double)(s0w * sn) * Ew);
                        double* js = a.sums + kAdjSums;
                        if (lane == 0) {
                            atomicAdd(js + kJacE + 2 * j, CE);
                            atomicAdd(js + kJacE + 2 * j + 1, SE);
                        }
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            const float st = t_step[c];
                            const double tcs = st > 0.0f ? (double)(h.tc[c] / st) : 0.0;
                            const double CT = warp_sum((double)(s0w * cs) * tcs), ST = warp_sum((double)(s0w * sn) * tcs);
                            if (lane == 0) {
                                atomicAdd(js + kJacLT + (2 * j) * NC + c, CT);
                                atomicAdd(js + kJacLT + (2 * j + 1) * NC + c, ST);
                            }
                        }
                    }
                }
                // the T2 weight under time rescaling: dW/d(eps) = -W + T / T2(c_T)
                wkeep = (float)(w64 - (double)a.tn * (double)(t_step[wk.ai] * t_k[wk.ai]));
                tr += Lw * wkeep;
                Lkeep = Lw;
                s0keep = s0w;
                nb_w = active ? h.nb : 0;
                if (FORM == 1) {
                    // pass 2's sums from what pass 1 kept
                    const double TR = warp_sum((double)tr);
                    if (lane == 0) atomicAdd(a.sums + kAdjSumTR, TR);
                    if (JAC) {
#pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            if (j < a.nwave) {
                                float sn = 0.0f, cs = 0.0f;
                                sincosf(phi[j], &sn, &cs);
                                const float Cw = active ? s0keep * cs : 0.0f, Sw = active ? s0keep * sn : 0.0f;
                                const float de = rr[j] - phi[j];
                                const double TC = warp_sum((double)(-Sw * de + Cw * wkeep));
                                const double TS = warp_sum((double)(Cw * de + Sw * wkeep));
                                if (lane == 0) {
                                    atomicAdd(a.sums + kAdjSums + kJacTR + 2 * j, TC);
                                    atomicAdd(a.sums + kAdjSums + kJacTR + 2 * j + 1, TS);
                                }
                            }
                        }
                    }
                    if (a.force && live && nb_w > 0) {
                        // the forced draw (as pass 3 picks it), the last checkpoint
                        // before it, and this walker listed under that resume step
                        DomainStream fs;
                        fs.init(a.seed, (uint64_t)w, kDomForce);
                        const int kf = min((int)(fs.next() * (float)nb_w), nb_w - 1);
                        const int nck = min(ck_n, kAdjCkMax);
                        int ck_r = 0;
                        for (int c = 1; c < nck; ++c)
                            if (nb_at[c] <= kf) ck_r = c;
                        const size_t nw = (size_t)a.nwalk;
                        a.ws[0 * nw + wr] = __float_as_uint(Lkeep);
                        a.ws[1 * nw + wr] = (uint32_t)nb_w;
                        a.ws[2 * nw + wr] = __float_as_uint(s0w);
                        if (JAC) {
#pragma unroll
                            for (int j = 0; j < NW; ++j) a.ws[(3 + j) * nw + wr] = __float_as_uint(phi[j]);
                        }
                        const int e = atomicAdd(a.bcount + ck_r, 1);
                        a.blist[(size_t)ck_r * a.nwalk + e] = (int)wr;
                    }
                }
                const double L = warp_sum((double)Lw), LE = warp_sum((double)Lw * (double)h.E),
                             GP = warp_sum((double)G), ES = warp_sum(active ? (double)h.E : 0.0);
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
                    const double LT = warp_sum(st > 0.0f ? (double)Lw * (double)(h.tc[c] / st) : 0.0);
                    if (lane == 0) atomicAdd(a.sums + kAdjSumLT + c, LT);
                }
            } else if (pass == 1) {
                const double TR = warp_sum((double)tr);
                if (lane == 0) atomicAdd(a.sums + kAdjSumTR, TR);
                if (JAC) {
                    // dC_j/deps = -S_j dphi_j/deps - C_j dW/deps, dS_j/deps = C_j dphi_j/deps - S_j dW/deps,
                    // dphi_j/deps = R_j - phi_j, -dW/deps = W - T / T2(c_T)
#pragma unroll
                    for (int j = 0; j < NW; ++j) {
                        if (j < a.nwave) {
                            float sn = 0.0f, cs = 0.0f;
                            sincosf(phi[j], &sn, &cs);
                            const float Cw = active ? s0keep * cs : 0.0f, Sw = active ? s0keep * sn : 0.0f;
                            const float de = dphi[j] - phi[j];
                            const double TC = warp_sum((double)(-Sw * de + Cw * wkeep));
                            const double TS = warp_sum((double)(Cw * de + Sw * wkeep));
                            if (lane == 0) {
                                atomicAdd(a.sums + kAdjSums + kJacTR + 2 * j, TC);
                                atomicAdd(a.sums + kAdjSums + kJacTR + 2 * j + 1, TS);
                            }
                        }
                    }
                }
            } else {
                // nb_w Pij (1 - Pij) (L[crossed] - L[reflected]) of the forced walk
                const float s0f = active ? (float)exp(-w64) : 0.0f;
                float Lf = 0.0f;
#pragma unroll
                for (int j = 0; j < NW; ++j) {
                    if (j < a.nwave) {
                        float sn, cs;
                        sincosf(phi[j], &sn, &cs);
                        Lf += s0f * (__ldg(a.gup + 2 * j) * cs + __ldg(a.gup + 2 * j + 1) * sn);
                    }
                }
                const float dL = h.xf ? Lkeep - Lf : Lf - Lkeep;
                const double wf = active ? (double)nb_w * (double)h.Pf * (1.0 - (double)h.Pf) : 0.0;
                const double F = warp_sum(wf * (double)dL);
                if (lane == 0) atomicAdd(a.sums + kAdjSumForce, F);
                if (JAC) {
                    // per waveform: C_j, S_j of the forced walk (phases in dphi[]) against pass 1's
#pragma unroll
                    for (int j = 0; j < NW; ++j) {
                        if (j < a.nwave) {
                            float sn, cs, snf, csf;
                            sincosf(phi[j], &sn, &cs);
                            sincosf(dphi[j], &snf, &csf);
                            const float dC = s0f * csf - s0keep * cs, dS = s0f * snf - s0keep * sn;
                            const double FC = warp_sum(wf * (double)(h.xf ? -dC : dC));
                            const double FS = warp_sum(wf * (double)(h.xf ? -dS : dS));
                            if (lane == 0) {
                                atomicAdd(a.sums + kAdjSums + kJacF + 2 * j, FC);
                                atomicAdd(a.sums + kAdjSums + kJacF + 2 * j + 1, FS);
                            }
                        }
                    }
                }
            }
        }
    }
}

// dL/dwave from pass 1's records: dwave[b][j][ax] += sum_w a_jw X_wb,ax over
// the launch's walkers (xbin [bin][axis][walker], ajw [waveform][walker]).
// Each block takes kDwSlab walkers (kDwPer per thread, their a_jw in
// registers) and rows [r0, r1) of the bin x axis table, kDwRows rows per
// step; per row a warp reduce-scatter, and per step one barrier and a sum over
// the block's warps leave one float atomic per row and waveform.  The next
// step's rows are loaded while this step's are summed (two register sets), so
// the X table streams from HBM instead of waiting out one load latency per
// row; it is read once (12 bytes per walker per bin).
constexpr int kDwBlock = 256, kDwPer = 4, kDwRows = 4, kDwSlab = kDwBlock * kDwPer;

__device__ __forceinline__ void dw_load(float (&xv)[kDwRows][kDwPer], const float* __restrict__ xbin, int64_t nwalk,
                                        int64_t w0, int rg, int r1) {
#pragma unroll
    for (int g = 0; g < kDwRows; ++g) {
        const int r = rg + g;
#pragma unroll
        for (int k = 0; k < kDwPer; ++k) {
            const int64_t w = w0 + (int64_t)k * kDwBlock;
            xv[g][k] = (r < r1 && w < nwalk) ? __ldcs(xbin + (size_t)r * nwalk + w) : 0.0f;
        }
    }
}

__device__ __forceinline__ void dw_rows(const float (&xv)[kDwRows][kDwPer], const float (&av)[kDwPer][kAdjWaves],
                                        float (&red)[kDwRows][kDwBlock / 32][kAdjWaves], int rg, int r1, int nwave,
                                        float* __restrict__ dwave) {
    constexpr int NW = kAdjWaves;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int g = 0; g < kDwRows; ++g) {
        float acc[NW];
#pragma unroll
        for (int j = 0; j < NW; ++j) acc[j] = 0.0f;
#pragma unroll
        for (int k = 0; k < kDwPer; ++k) {
#pragma unroll
            for (int j = 0; j < NW; ++j) acc[j] = fmaf(av[k][j], xv[g][k], acc[j]);
        }
        const float v = warp_reduce_scatter16f(acc, lane);   // lanes l, l ^ 16: waveform l & 15
        if (lane < 16) red[g][warp][lane] = v;
    }
    __syncthreads();
    if (threadIdx.x < kDwRows * 16) {
        const int g = threadIdx.x >> 4, j = threadIdx.x & 15, r = rg + g;
        if (j < nwave && r < r1) {
            float t = 0.0f;
#pragma unroll
            for (int q = 0; q < kDwBlock / 32; ++q) t += red[g][q][j];
            const int b = r / 3, ax = r - 3 * b;
            atomicAdd(dwave + ((size_t)b * nwave + j) * 3 + ax, t);
        }
    }
}

__global__ void __launch_bounds__(kDwBlock, 2) adjoint_dwave_kernel(const float* __restrict__ xbin,
                                                                   const float* __restrict__ ajw, int64_t nwalk,
                                                                   int nwave, int nrows, int rows_per_block,
                                                                   float* __restrict__ dwave) {
    constexpr int NW = kAdjWaves;
    // red[s]: the warps' row sums of every other step (one barrier per step:
    // a buffer is written again only after the next step's barrier, which its
    // readers pass after reading it)
    __shared__ float red[2][kDwRows][kDwBlock / 32][NW];
    const int64_t w0 = (int64_t)blockIdx.x * kDwSlab + threadIdx.x;
    float av[kDwPer][NW];
#pragma unroll
    for (int k = 0; k < kDwPer; ++k) {
        const int64_t w = w0 + (int64_t)k * kDwBlock;
#pragma unroll
        for (int j = 0; j < NW; ++j) av[k][j] = (w < nwalk && j < nwave) ? __ldg(ajw + (size_t)j * nwalk + w) : 0.0f;
    }
    const int r0 = blockIdx.y * rows_per_block, r1 = min(nrows, r0 + rows_per_block);
    float xa[kDwRows][kDwPer], xb[kDwRows][kDwPer];
    dw_load(xa, xbin, nwalk, w0, r0, r1);
    for (int rg = r0; rg < r1; rg += 2 * kDwRows) {
        dw_load(xb, xbin, nwalk, w0, rg + kDwRows, r1);
        dw_rows(xa, av, red[0], rg, r1, nwave, dwave);
        dw_load(xa, xbin, nwalk, w0, rg + 2 * kDwRows, r1);
        dw_rows(xb, av, red[1], rg + kDwRows, r1, nwave, dwave);
    }
}

}  // namespace

int launch_adjoint_dwave(const AdjArgs& a, int sms, void* stream) {
    const int nrows = a.nbins * 3;
    const int slabs = (int)((a.nwalk + kDwSlab - 1) / kDwSlab);
    // two waves of the 2 resident blocks per SM at least: split the rows when the walkers are few
    const int want = 4 * sms;
    const int groups = std::max(1, std::min(nrows, (want + slabs - 1) / slabs));
    const int per = (nrows + groups - 1) / groups;
    const dim3 grid((unsigned)slabs, (unsigned)((nrows + per - 1) / per));
    adjoint_dwave_kernel<<<grid, kDwBlock, 0, (cudaStream_t)stream>>>(a.xbin, a.ajw, a.nwalk, a.nwave, nrows, per,
                                                                     a.dwave);
    return (int)cudaGetLastError();
}

template <bool JAC>
static int launch_form(const AdjArgs& a, int form, int grid, cudaStream_t st) {
    if (form == 0) adjoint_kernel<JAC, 0><<<grid, kAdjBlock, 0, st>>>(a);
    else if (form == 1) adjoint_kernel<JAC, 1><<<grid, kAdjBlock, 0, st>>>(a);
    else adjoint_kernel<JAC, 2><<<grid, kAdjBlock, 0, st>>>(a);
    return (int)cudaGetLastError();
}

template <bool JAC>
static int blocks_form(int form) {
    int n = 0;
    const cudaError_t e =
        form == 0   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjoint_kernel<JAC, 0>, kAdjBlock, 0)
        : form == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjoint_kernel<JAC, 1>, kAdjBlock, 0)
                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjoint_kernel<JAC, 2>, kAdjBlock, 0);
    return e == cudaSuccess ? n : -1;
}

int launch_adjoint(const AdjArgs& a, bool jac, int form, int grid, void* stream) {
    return jac ? launch_form<true>(a, form, grid, (cudaStream_t)stream)
               : launch_form<false>(a, form, grid, (cudaStream_t)stream);
}

int adjoint_blocks_per_sm(bool jac, int form) { return jac ? blocks_form<true>(form) : blocks_form<false>(form); }

}  // namespace rms

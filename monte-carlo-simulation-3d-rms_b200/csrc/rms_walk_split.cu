// rms_walk_split.cu -- the split-precision walk (RMS_PREC_SPLIT).
//
// The same walk as the reference kernel `propagate` (hpc_code/lib/main.cu:
// 63-384, main_PGSE.cu:65-410) -- fixed-length isotropic steps, at most nite
// sub-segments, voxel-face reflection or Bernoulli(Pij) permeation, mirror
// walls, T2 weighting, moments and signal at the same records -- in the
// arithmetic a B200 issues fastest:
//
//  - position = voxel + FP32 offset inside it per axis (0..1, split_step.cuh).
//    A straight move is one FMA and a floor per axis.  The face loop works on
//    d_a, the distance to the next face in the direction of travel: the time
//    to a face is one multiply, and after any face event -- a cross into the
//    neighbour or a reflection -- the walker sits on that face with a whole
//    voxel ahead, d = 1 exactly, so no drift accumulates;
//  - the voxel is one linear index into a lattice padded with a one-voxel
//    border that holds a wall code: a face step is `lin += stride`, and
//    reaching a wall is a label like any other (rare branch); the integer
//    part of the displacement, D = voxel - origin image, is carried per axis;
//  - free flight: a voxel whose 26 neighbours all carry its label (and none
//    is a wall) has a flag bit in the lattice; a step that starts there is
//    shorter than a voxel, so it cannot meet a membrane or a wall and moves in
//    one straight line -- a floor per axis instead of the face loop.  It is
//    the face loop's own outcome (every face on the way is a same-label face,
//    always crossed) with at most three crossings, within the nite = 4 cap;
//  - labels packed 4 bits per voxel (3-bit label, wall = 7, plus the flag;
//    a padded 256x256x2048 lattice is 68 MB and stays in the 126 MB L2), or
//    one byte for Nc = 8;
//  - FP32 uniforms (21-bit), one Philox4x32-10 block per three steps;
//    hardware sine/cosine and reciprocal for the direction and face times;
//  - per-walker sums that grow over the walk (T2 exponent, PGSE displacement
//    sums) are carried in FP32 for at most 32 steps and folded into FP64;
//  - cross-walker sums: FP32 products per walker, staged in shared memory and
//    summed per column over the warp in FP64, per-warp FP64 rows, added into
//    each axon's totals with FP64 atomics (the no-allocation walk: an ordered
//    FP64 reduction, rms_reduce.cu).
//
// Mirror walls: the reference mirrors the origin image at the end of a step
// for each wall the step touched (main.cu:302-310).  A step shorter than a
// voxel touches a wall at most once per axis and nothing else moves the
// origin during the step, so the mirror is applied at the wall event itself.
//
// Random streams (philox.cuh): per walker, direction uniforms of steps 3k,
// 3k+1 and 3k+2 come from one Philox4x32-10 block indexed by k, so all lanes of
// a warp generate in lock step; start positions and partial-permeation draws
// read their own sequential counter domains.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>

#include "philox.cuh"
#include "rms_internal.h"
#include "split_lattice.cuh"
#include "split_step.cuh"
#include "warp_reduce.cuh"

namespace rms {
namespace {

// Launch variants (block size, minimum resident blocks per SM): the second
// number caps registers per thread at 65536 / (block * minb), trading spills
// in the rare record path for more resident warps to hide gather latency.
struct SplitVariant { int block, minb; };
constexpr int kLeapCap = 64;   // equal-step-length leap: tries per step before staying put
constexpr SplitVariant kVariants[] = {{256, 4}, {256, 3}, {256, 2}, {128, 8}, {512, 2}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Add a warp's accumulator rows (and PGSE signal row) into axon `axon`'s
// totals and clear them (multi-axon launches; other warps add concurrently).
__device__ __noinline__ void flush_rows(double* slot, double* sig_slot, double* out, double* os, size_t n,
                                        int ngrad, int lane) {
    for (size_t i = lane; i < n; i += 32) {
        const double x = slot[i];
        if (x != 0.0) {
            atomicAdd(out + i, x);
            slot[i] = 0.0;
        }
    }
    if (os) {
        for (int i = lane; i < ngrad; i += 32) {
            const double x = sig_slot[i];
            if (x != 0.0) {
                atomicAdd(os + i, x);
                sig_slot[i] = 0.0;
            }
        }
    }
}

// General waveforms, at the end of bin `bin`: X (voxels) is the bin's
// displacement sum; every waveform's phase gets wave_b . X res, and the bin's
// mean displacement (um) goes to the trajectory output when one is given.
__device__ __noinline__ void wave_bin(const double* __restrict__ wave, int nwave, int bin, double X0, double X1,
                                      double X2, double res, double* ph, int nthr, float* traj, int64_t tw,
                                      int nbins, int bin_steps, int split, int64_t traj_n) {
    const double x0 = X0 * res, x1 = X1 * res, x2 = X2 * res;
    const double* wv = wave + (size_t)bin * nwave * 3;
    for (int j = 0; j < nwave; ++j) ph[(size_t)j * nthr] += wv[3 * j] * x0 + wv[3 * j + 1] * x1 + wv[3 * j + 2] * x2;
    if (traj && tw >= 0) {
        const double inv = 1.0 / (double)bin_steps;
        const float m[3] = {(float)(x0 * inv), (float)(x1 * inv), (float)(x2 * inv)};
        const size_t at = ((size_t)tw * nbins + bin) * 3;
        if (split) {
            // BF16 pairs, hi = bf16(x), lo = bf16(x - hi): the operands of the
            // tensor-core contraction, split once here
            __nv_bfloat16* hi = reinterpret_cast<__nv_bfloat16*>(traj);
            __nv_bfloat16* lo = hi + (size_t)traj_n * nbins * 3;
            for (int k = 0; k < 3; ++k) {
                const __nv_bfloat16 h = __float2bfloat16_rn(m[k]);
                hi[at + k] = h;
                lo[at + k] = __float2bfloat16_rn(m[k] - __bfloat162float(h));
            }
        } else {
            traj[at] = m[0]; traj[at + 1] = m[1]; traj[at + 2] = m[2];
        }
    }
}

// General waveforms, after the last step: the warp's sums of s0 cos(phase) and
// s0 sin(phase) per waveform, (cos, sin) pairs into the signal row.
__device__ __noinline__ void wave_final(const double* ph, int nthr, int nwave, double s0, double* sig_slot,
                                        int lane) {
    for (int base = 0; base < 2 * nwave; base += 32) {
        double mine = 0.0;
        const int cnt = min(32, 2 * nwave - base);
        for (int k = 0; k < cnt; k += 2) {
            const int j = (base + k) >> 1;
            double sn, cs;
            sincos(ph[(size_t)j * nthr], &sn, &cs);
            const double rc = warp_sum(s0 * cs);
            const double rs = warp_sum(s0 * sn);
            if (lane == k) mine = rc;
            if (lane == k + 1) mine = rs;
        }
        if (lane < cnt) sig_slot[base + lane] += mine;
    }
}

// A record of the warp's 32 walkers added into the warp's row (row layout of
// rms_internal.h): each lane stages its 22 moments [sig0, dx2 x6, dx4 x15]
// (FP32 products) in shared memory, and lane c < 22 adds column c over the 32
// walkers in FP64, in lane order (four interleaved partials, combined in a
// fixed order); lanes 22.. take the compartment counts (integer warp sums).
// KC columns per pass.  Not inlined: the step loop keeps its registers (the
// inlined form cost the batch walk ~3 % more time).
template <int KC>
__device__ __noinline__ void record_row(double* row, float s0, float dx, float dy, float dz, int ai, bool active,
                                        int lane, float (*stage)[KC + 1]) {
    const float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    const float sxx = s0 * xx, syy = s0 * yy, szz = s0 * zz;
    const float mv[22] = {s0,      sxx,          s0 * dx * dy, s0 * dx * dz, syy,
                          s0 * dy * dz, szz,     sxx * xx,     sxx * dx * dy, sxx * dx * dz,
                          sxx * yy, sxx * dy * dz, sxx * zz,   syy * dx * dy, syy * dx * dz,
                          szz * dx * dy, szz * dx * dz, syy * yy, syy * dy * dz, syy * zz,
                          szz * dy * dz, szz * zz};
    double r = 0.0;
#pragma unroll
    for (int pass = 0; pass < 22 / KC; ++pass) {
        __syncwarp();
#pragma unroll
        for (int c = 0; c < KC; ++c) stage[lane][c] = mv[pass * KC + c];
        __syncwarp();
        const int col = lane - pass * KC;
        if (col >= 0 && col < KC) {
            double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
#pragma unroll
            for (int l = 0; l < 32; l += 4) {
                q0 += (double)stage[l][col];
                q1 += (double)stage[l + 1][col];
                q2 += (double)stage[l + 2][col];
                q3 += (double)stage[l + 3][col];
            }
            r = (q0 + q1) + (q2 + q3);
        }
    }
    unsigned cnt = 0u;
#pragma unroll
    for (int c = 0; c < 10; ++c) {
        const unsigned n = __reduce_add_sync(0xffffffffu, (active && ai == c) ? 1u : 0u);
        if (lane == kColCount + c) cnt = n;
    }
    if (lane >= kColCount) r = (double)cnt;
    row[lane] += r;
}

// ONE: the no-allocation walk's form -- one axon, whose scalars are read from
// the kernel parameters (a.axon0); every other launch reads the axon table.
template <int NCMAX, int BITS, int BLOCK, int MINB, bool ONE, int RULE = 0, int MODE = 0>
__global__ void __launch_bounds__(BLOCK, MINB) walk_split_kernel(const WalkArgs a) {
    // per warp, the current axon's tables: step (voxels), T2 exponent per voxel
    // of path, Pij and the step-length ratio that rescales the rest of a step
    constexpr int kTab = 2 * NCMAX + 2 * NCMAX * NCMAX;
    __shared__ float s_tab[BLOCK / 32][kTab];
    // per warp, a record's 22 moments of its 32 walkers, staged for the column
    // sums (all 22 at once up to 256 threads a block, else in two halves: the
    // static shared memory stays under 48 KB a block)
    constexpr int kCols = BLOCK <= 256 ? 22 : 11;
    __shared__ float s_stage[BLOCK / 32][32][kCols + 1];

    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    const int warp_global = gtid >> 5;
    const int nwarps = nthr >> 5;
    float* tab = s_tab[threadIdx.x >> 5];
    // the signal mode is compiled in: a walk carries no code of the others
    constexpr bool pgse = (MODE == 1);
    constexpr bool wave = (MODE == 2);
    constexpr bool sums = pgse || wave;   // displacement sums over the walk
    const bool mirror = (a.boundary == 0);

    // A warp keeps its rows for its current axon and, in the table form, adds
    // them into that axon's totals (FP64 atomics) when it moves on to another
    // axon or finishes.  ONE (the no-allocation walk) keeps one row set per
    // warp, summed in order afterwards.
    int ax = 0;          // current axon
    int held = -1;       // axon whose records the warp's rows hold
    int64_t next_tb = ONE ? INT64_MAX : ((a.naxons > 1) ? a.axons[1].tile_begin : INT64_MAX);
    // a field of the current axon: kernel parameters for ONE, else the axon
    // table (read where used, so it holds no registers)
#define AXF(f) (ONE ? a.axon0.f : a.axons[ax].f)
    double* slot = a.slots + (size_t)warp_global * a.timepoints * a.nvals;
    double* sig_slot = sums ? a.sig_slots + (size_t)warp_global * a.ngrad_pad : nullptr;

    // The table form (every SPLIT launch but the no-allocation walk, one axon
    // or many): a queue (one counter per launch) hands out tiles in order, so
    // the tiles in flight stay one narrow window of the list -- one or two
    // axons, whose lattices then share the L2 -- however far warps drift
    // apart.  ONE: tiles in strided order (warp w: w, w + nwarps, ...), so each
    // warp's rows, reduced in a fixed order, are the same every run.
    auto claim = [&]() -> int64_t {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(a.tile_ctr, 1ull);
        return (int64_t)__shfl_sync(0xffffffffu, t, 0);
    };
    for (int64_t tile = ONE ? warp_global : claim(); tile < a.ntiles; tile = ONE ? tile + nwarps : claim()) {
        if (!ONE) {
            while (tile >= next_tb) {
                ++ax;
                next_tb = (ax + 1 < a.naxons) ? a.axons[ax + 1].tile_begin : INT64_MAX;
            }
        }
        if (held != ax) {
            if (!ONE && held >= 0)
                flush_rows(slot, sig_slot, a.out_rows + (size_t)held * a.timepoints * a.nvals,
                           sums ? a.out_sig + (size_t)held * a.ngrad_pad : nullptr,
                           (size_t)a.timepoints * a.nvals, a.ngrad, lane);   // previous axon's records to its totals
            held = ax;
            // this axon's tables into the warp's shared memory
            __syncwarp();
            for (int i = lane; i < kTab; i += 32) {
                float v;
                if (i < NCMAX) v = AXF(step[i]);
                else if (i < 2 * NCMAX) v = AXF(k[i - NCMAX]);
                else if (i < 2 * NCMAX + NCMAX * NCMAX) {
                    const int r = (i - 2 * NCMAX) / NCMAX, c = (i - 2 * NCMAX) % NCMAX;
                    v = AXF(pij[r * kNcMax + c]);
                } else {
                    const int r = (i - 2 * NCMAX - NCMAX * NCMAX) / NCMAX, c = (i - 2 * NCMAX - NCMAX * NCMAX) % NCMAX;
                    v = AXF(ratio[r * kNcMax + c]);
                }
                tab[i] = v;
            }
            __syncwarp();
        }
        const uint8_t* lat = AXF(lat);
        const int s0 = AXF(s0), s1 = AXF(s1);
        const uint64_t seed = AXF(seed);   // a graph captures the table form, whose seed a replay rewrites
        const bool flight = AXF(flight);
        const bool same_certain = AXF(same_cross);
        const float* t_step = tab;
        const float* t_k = tab + NCMAX;
        const float* t_pij = tab + 2 * NCMAX;
        const float* t_ratio = tab + 2 * NCMAX + NCMAX * NCMAX;
        const uint32_t key0 = (uint32_t)seed, key1 = (uint32_t)(seed >> 32);

        const int64_t w = AXF(walker_begin) + (tile - (ONE ? 0 : AXF(tile_begin))) * 32 + lane;
        bool active = w < AXF(walker_end);
        const uint32_t wlo = (uint32_t)w, whi = (uint32_t)((uint64_t)w >> 32);

        // initial position: uniform in the labelled voxels (rejection sampling)
        float f0 = 0.5f, f1 = 0.5f, f2 = 0.5f;
        unsigned lin = 0;
        if (active) {
            DomainStream init;
            init.init(seed, (uint64_t)w, kDomInit);
            long long tries = 0;
            for (;;) {
                const int n1 = AXF(n1), n2 = AXF(n2), n3 = AXF(n3);
                const float x0 = init.next() * (float)n1;
                const float x1 = init.next() * (float)n2;
                const float x2 = init.next() * (float)n3;
                const int g0 = min((int)x0, n1 - 1), g1 = min((int)x1, n2 - 1), g2 = min((int)x2, n3 - 1);
                f0 = x0 - (float)g0; f1 = x1 - (float)g1; f2 = x2 - (float)g2;
                lin = (unsigned)(g0 + 1) * (unsigned)s0 + (unsigned)(g1 + 1) * (unsigned)s1 + (unsigned)(g2 + 1);
                if (label_at<BITS>(lat, lin) != 0) break;
                if (++tries >= kInitTryCap) { atomicOr(a.err, kErrInitCap); active = false; break; }
            }
        }
        const int ai0 = active ? label_at<BITS>(lat, lin) : 0;
        // displacement = D + (offset - Fm) per axis
        SplitWalker wk{lin, active ? cell_at<BITS>(lat, lin) : 0u, f0, f1, f2, 0, 0, 0, f0, f1, f2, ai0,
                        t_step[ai0], t_k[ai0], 0.0f};
        const SplitGeom geo{lat, s0, s1, a.nite, flight, same_certain, mirror};
        auto nsize = [&](int axis) { return axis == 0 ? AXF(n1) : (axis == 1 ? AXF(n2) : AXF(n3)); };
        NoHooks hooks;
        DomainStream perm;
        perm.init(seed, (uint64_t)w, kDomPerm);

        double w64 = 0.0;          // T2 exponent, folded
        double P0 = 0.0, P1 = 0.0, P2 = 0.0;   // displacement sums (voxels), folded
        float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
        int next_rec = 0, rec = 0;   // the next recorded step (0, tstep, 2 tstep, ...) and its record
        int evi = 0;   // next PGSE event, or current waveform bin
        int next_ev = pgse ? (a.nevents > 0 ? a.ev_step[0] : -1) : (wave ? a.bin_steps : -1);
        if (sums)
            for (int k = 0; k < (pgse ? a.npairs * 3 : a.nwave); ++k) a.vscr[(size_t)k * nthr + gtid] = 0.0;
        // direction uniforms: one Philox block per three steps, in lock step;
        // the next two steps' pairs wait in q0..q3
        float q0 = 0.0f, q1 = 0.0f, q2 = 0.0f, q3 = 0.0f;
        int phase = 0;
        uint32_t dblk = 0u;

        for (int i = 0; i < a.tn; ++i) {
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
                // RULE != 0: the step's start, restored when a membrane turns the step back
                const SplitWalker start = wk;
                for (int attempt = 0;; ++attempt) {
                    float v0, v1, v2;
                    split_direction(u1, u2, v0, v1, v2);
                    const bool back = split_step<NCMAX, BITS, RULE>(wk, v0, v1, v2, geo, t_step, t_k, t_pij, t_ratio,
                                                                    perm, nsize, hooks);
                    if (RULE == 0 || !back) break;
                    // the step is taken back (interaction.m:256-345): rejection
                    // sampling stays put for the step; the equal-step-length leap
                    // redraws the direction (partial-permeation stream) and walks
                    // the step again, up to kLeapCap tries, then stays
                    wk = start;
                    if (RULE == 1 || attempt + 1 >= kLeapCap) {
                        wk.w32 = fmaf(wk.cur_step, wk.cur_k, wk.w32);   // the step's time passes in place
                        break;
                    }
                    u1 = perm.next();
                    u2 = perm.next();
                }
            }
            // in-voxel offsets of the current position
            const float o0 = wk.o0, o1 = wk.o1, o2 = wk.o2;
            const int D0 = wk.D0, D1 = wk.D1, D2 = wk.D2;
            const float Fm0 = wk.Fm0, Fm1 = wk.Fm1, Fm2 = wk.Fm2;

            if (sums) {
                // displacement sums (voxels): PGSE, prefix sums read at the
                // lobe edges; waveforms, one sum per time bin
                p0 += (float)D0 + (o0 - Fm0);
                p1 += (float)D1 + (o1 - Fm1);
                p2 += (float)D2 + (o2 - Fm2);
                const bool event = (i + 1 == next_ev);
                if (event || (i & 31) == 31) {
                    P0 += (double)p0; P1 += (double)p1; P2 += (double)p2;
                    p0 = p1 = p2 = 0.0f;
                }
                if (event && wave) {
                    wave_bin(a.wave, a.nwave, evi, P0, P1, P2, (double)AXF(res), a.vscr + gtid, nthr, a.traj,
                             active ? w - AXF(walker_begin) : -1, a.nbins, a.bin_steps, a.traj_split, a.traj_n);
                    P0 = P1 = P2 = 0.0;
                    ++evi;
                    next_ev += a.bin_steps;
                } else if (event) {
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
                if (i == a.tn - 1 && wave) {
                    wave_final(a.vscr + gtid, nthr, a.nwave, active ? exp(-(w64 + (double)wk.w32)) : 0.0, sig_slot, lane);
                } else if (i == a.tn - 1) {
                    // final T2-weighted signal: phase_j = |g| (g_hat . V) res dt
                    const double s0 = active ? exp(-(w64 + (double)wk.w32)) : 0.0;
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

            if (i == next_rec) {
                const int tidx = rec++;
                next_rec += a.tstep;
                if (tidx < a.timepoints) {
                    w64 += (double)wk.w32;
                    wk.w32 = 0.0f;
                    const float s0 = active ? expf(-(float)w64) : 0.0f;
                    const float res = AXF(res);
                    const float dx = ((float)D0 + (o0 - Fm0)) * res;
                    const float dy = ((float)D1 + (o1 - Fm1)) * res;
                    const float dz = ((float)D2 + (o2 - Fm2)) * res;
                    double* row = slot + (size_t)tidx * a.nvals;
                    record_row<kCols>(row, s0, dx, dy, dz, wk.ai, active, lane, s_stage[threadIdx.x >> 5]);
                    if (!sums) {
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
    if (!ONE && held >= 0)
        flush_rows(slot, sig_slot, a.out_rows + (size_t)held * a.timepoints * a.nvals,
                   sums ? a.out_sig + (size_t)held * a.ngrad_pad : nullptr, (size_t)a.timepoints * a.nvals, a.ngrad,
                   lane);
}

#undef AXF

// Padded lattice: (n1+2) x (n2+2) x (n3+2), interior = the labels, border =
// the wall code.  An interior voxel also gets the free-flight flag when its 26
// neighbours carry its label -- with mirror walls counting only the neighbours
// inside the lattice (a straight line out through a wall is reflected in the
// walk), with periodic walls only for voxels off the lattice's faces.
template <int BITS>
__global__ void pad_pack_kernel(const uint8_t* __restrict__ labels, int n1, int n2, int n3, int mirror,
                                uint8_t* __restrict__ out, size_t nbytes) {
    const size_t P3 = (size_t)n3 + 2, P2 = (size_t)n2 + 2;
    const size_t nvox = ((size_t)n1 + 2) * P2 * P3;
    constexpr int per = 8 / BITS;
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbytes; b += (size_t)gridDim.x * blockDim.x) {
        unsigned v = 0;
#pragma unroll
        for (int k = 0; k < per; ++k) {
            const size_t p = b * per + k;
            const size_t pk = p % P3, pj = (p / P3) % P2, pi = p / (P3 * P2);
            unsigned cell;
            if (p >= nvox || pi == 0 || pi > (size_t)n1 || pj == 0 || pj > (size_t)n2 || pk == 0 || pk > (size_t)n3) {
                cell = (unsigned)wall_code<BITS>();
            } else {
                const long i = (long)pi - 1, j = (long)pj - 1, kk = (long)pk - 1;
                const unsigned lab = labels[((size_t)i * n2 + j) * (size_t)n3 + kk];
                cell = lab & label_mask<BITS>();
                const bool inner = i >= 1 && i + 1 < n1 && j >= 1 && j + 1 < n2 && kk >= 1 && kk + 1 < n3;
                if (mirror || inner) {
                    bool same = true;
                    for (int di = -1; di <= 1 && same; ++di)
                        for (int dj = -1; dj <= 1 && same; ++dj)
                            for (int dk = -1; dk <= 1; ++dk) {
                                const long qi = i + di, qj = j + dj, qk = kk + dk;
                                if (qi < 0 || qi >= n1 || qj < 0 || qj >= n2 || qk < 0 || qk >= n3) continue;
                                if (labels[((size_t)qi * n2 + qj) * (size_t)n3 + qk] != lab) {
                                    same = false;
                                    break;
                                }
                            }
                    if (same) cell |= flight_bit<BITS>();
                }
            }
            v |= cell << (BITS * k);
        }
        out[b] = (uint8_t)v;
    }
}

template <int NCMAX, int BITS, int B, int M, int MODE, int RULE>
int launch_k(const WalkArgs& a, int grid, void* stream) {
    if (a.naxons == 1 && !a.table_form)
        walk_split_kernel<NCMAX, BITS, B, M, true, RULE, MODE><<<grid, B, 0, (cudaStream_t)stream>>>(a);
    else
        walk_split_kernel<NCMAX, BITS, B, M, false, RULE, MODE><<<grid, B, 0, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

// Launch variants 2.. walk narrow-pulse and PGSE jobs with reflecting
// membranes; the first variant also walks waveforms and the alternative
// membrane rules (rejection sampling, equal-step-length leap).
template <int NCMAX, int BITS, int B, int M>
int launch_modes(const WalkArgs& a, int grid, void* stream) {
    if (a.rule != 0) return (int)cudaErrorInvalidValue;
    if (a.mode == 0) return launch_k<NCMAX, BITS, B, M, 0, 0>(a, grid, stream);
    if (a.mode == 1) return launch_k<NCMAX, BITS, B, M, 1, 0>(a, grid, stream);
    return (int)cudaErrorInvalidValue;
}

template <int NCMAX, int BITS>
int launch_first(const WalkArgs& a, int grid, void* stream) {
    constexpr int B = kVariants[0].block, M = kVariants[0].minb;
    switch (a.mode * 3 + a.rule) {
        case 0: return launch_k<NCMAX, BITS, B, M, 0, 0>(a, grid, stream);
        case 1: return launch_k<NCMAX, BITS, B, M, 0, 1>(a, grid, stream);
        case 2: return launch_k<NCMAX, BITS, B, M, 0, 2>(a, grid, stream);
        case 3: return launch_k<NCMAX, BITS, B, M, 1, 0>(a, grid, stream);
        case 4: return launch_k<NCMAX, BITS, B, M, 1, 1>(a, grid, stream);
        case 5: return launch_k<NCMAX, BITS, B, M, 1, 2>(a, grid, stream);
        case 6: return launch_k<NCMAX, BITS, B, M, 2, 0>(a, grid, stream);
        case 7: return launch_k<NCMAX, BITS, B, M, 2, 1>(a, grid, stream);
        case 8: return launch_k<NCMAX, BITS, B, M, 2, 2>(a, grid, stream);
        default: return (int)cudaErrorInvalidValue;
    }
}

template <int BLOCK, int MINB>
const void* kernel_ptr(int bits) {
    if (bits == 4) return (const void*)walk_split_kernel<8, 4, BLOCK, MINB, false>;
    return (const void*)walk_split_kernel<8, 8, BLOCK, MINB, false>;
}

template <int BLOCK, int MINB>
int launch_v(const WalkArgs& a, int bits, int grid, void* stream) {
    if (bits == 4) return a.nc <= 7 ? launch_modes<8, 4, BLOCK, MINB>(a, grid, stream) : (int)cudaErrorInvalidValue;
    if (bits == 8) return launch_modes<8, 8, BLOCK, MINB>(a, grid, stream);
    return (int)cudaErrorInvalidValue;
}

// Dispatch over the variant table (index v, 0-based).
template <class F>
auto by_variant(int v, F&& f) {
    switch (v) {
        case 0: return f.template operator()<256, 4>();
        case 1: return f.template operator()<256, 3>();
        case 2: return f.template operator()<256, 2>();
        case 3: return f.template operator()<128, 8>();
        default: return f.template operator()<512, 2>();
    }
}

}  // namespace

int split_lattice_bits(int nc) { return nc <= 7 ? 4 : 8; }

size_t padded_lattice_bytes(int n1, int n2, int n3, int bits) {
    const size_t nv = ((size_t)n1 + 2) * ((size_t)n2 + 2) * ((size_t)n3 + 2);
    return (nv * (size_t)bits + 7) / 8;
}

int pack_lattice_padded(const uint8_t* labels, int n1, int n2, int n3, int bits, int mirror, uint8_t* out,
                        void* stream) {
    const size_t nbytes = padded_lattice_bytes(n1, n2, n3, bits);
    size_t grid = (nbytes + 255) / 256;
    if (grid > 16384) grid = 16384;
    if (bits == 4)
        pad_pack_kernel<4><<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(labels, n1, n2, n3, mirror, out, nbytes);
    else
        pad_pack_kernel<8><<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(labels, n1, n2, n3, mirror, out, nbytes);
    return (int)cudaGetLastError();
}

int split_variant_count() { return kNumVariants; }
int split_variant_block(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].block : -1; }
int split_variant_minb(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].minb : -1; }

int launch_walk_split(const WalkArgs& a, int lattice_bits, int variant, int grid, void* stream) {
    if (variant < 0 || variant >= kNumVariants) return (int)cudaErrorInvalidValue;
    if (a.mode < 0 || a.mode > 2 || a.rule < 0 || a.rule > 2) return (int)cudaErrorInvalidValue;
    if (variant == 0) {
        if (lattice_bits == 4) return a.nc <= 7 ? launch_first<8, 4>(a, grid, stream) : (int)cudaErrorInvalidValue;
        if (lattice_bits == 8) return launch_first<8, 8>(a, grid, stream);
        return (int)cudaErrorInvalidValue;
    }
    return by_variant(variant, [&]<int B, int M>() { return launch_v<B, M>(a, lattice_bits, grid, stream); });
}

bool split_variant_walks(int variant, int mode, int rule) { return variant == 0 || (mode != 2 && rule == 0); }

int walk_split_blocks_per_sm(int nc, int lattice_bits, int variant) {
    if (variant < 0 || variant >= kNumVariants) return -1;
    const void* k = by_variant(variant, [&]<int B, int M>() { return kernel_ptr<B, M>(lattice_bits); });
    int n = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kVariants[variant].block, 0);
    return e == cudaSuccess ? n : -1;
}

}  // namespace rms

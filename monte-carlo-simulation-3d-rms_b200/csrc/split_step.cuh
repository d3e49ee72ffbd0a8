// split_step.cuh -- one step of the split-precision walk.  The walk
// (rms_walk_split.cu) and its adjoint (rms_adjoint.cu) both call split_step,
// so the adjoint's trajectories are the forward walk's by construction; the
// adjoint adds its bookkeeping through the Hooks argument.
//
// The step is the reference's (hpc_code/lib/main.cu:140-300): a fixed-length
// step in an isotropic direction, split at voxel faces into at most nite
// segments, each face crossed or reflected -- always crossed between voxels of
// one label, reflected at compartment 0 and at mirror walls, Bernoulli(Pij)
// otherwise -- in the split representation (see rms_walk_split.cu): between
// steps a walker is its voxel and its FP32 in-voxel offsets; the face loop
// works on the distances to the next faces along the direction of travel and
// converts back when it ends.
#pragma once
#include <cstdint>

#include "philox.cuh"
#include "split_lattice.cuh"

namespace rms {

// A walker between steps.
struct SplitWalker {
    unsigned lin;            // voxel: linear index into the padded lattice
    unsigned cell;           // its lattice cell (label + free-flight flag)
    float o0, o1, o2;        // in-voxel offset along each axis, 0..1 (1: on the upper face)
    int D0, D1, D2;          // integer part of the displacement: voxel - origin image
    float Fm0, Fm1, Fm2;     // fractional part of the origin image (mirrored at walls)
    int ai;                  // compartment (label)
    float cur_step, cur_k;   // step length (voxels), T2 exponent per voxel of path
    float w32;               // T2 exponent since the last fold
};

// What one step reads besides the walker: the padded lattice and its strides,
// the sub-segment cap and the per-axon switches.
struct SplitGeom {
    const uint8_t* lat;
    int s0, s1;              // padded strides of axes 0 and 1 (axis 2: 1)
    int nite;
    bool flight;             // straight moves allowed (same-label faces always crossed, nite >= 4)
    bool same_certain;       // same-label faces are crossed without a draw
    bool mirror;             // mirror walls (else periodic)
};

// The forward walk's hooks: nothing.  The adjoint's record the path per
// compartment, flip the displacement tangent at reflections, score the
// Bernoulli draws and, in its forced pass, flip one draw's outcome (bernoulli
// returns the outcome the step takes).
struct NoHooks {
    __device__ __forceinline__ void path(int, float) {}
    __device__ __forceinline__ void reflect(int) {}
    __device__ __forceinline__ bool bernoulli(bool cross, float) { return cross; }
};

// One step of walker s in direction v (unit vector); s.cell is the cell of
// the walker's voxel, and the step leaves the new voxel's cell there.
// Tables: t_step[c], t_k[c], t_pij[a * NCMAX + b], t_ratio[a * NCMAX + b]
// (step[b] / step[a]).
// nsize(axis) gives the lattice size along an axis (read where needed so it
// holds no registers).  Returns true when RULE != 0 and a membrane turned the
// step back (the caller's rule decides); the walker is then mid-step.
template <int NCMAX, int BITS, int RULE, class NSize, class Hooks>
__device__ __forceinline__ bool split_step(SplitWalker& s, float v0, float v1, float v2, const SplitGeom& g,
                                           const float* t_step, const float* t_k, const float* t_pij,
                                           const float* t_ratio, DomainStream& perm, NSize nsize, Hooks& h) {
    constexpr int kWall = wall_code<BITS>();
    const uint8_t* __restrict__ lat = g.lat;
    const int s0 = g.s0, s1 = g.s1;
    const unsigned nu = (v0 > 0.0f ? 1u : 0u) | (v1 > 0.0f ? 2u : 0u) | (v2 > 0.0f ? 4u : 0u);
    // Free flight: a voxel whose 26 neighbours all carry its label has a flag
    // bit; a step from there (shorter than a voxel) moves as one straight line
    // -- the face loop's own outcome, since every face on the way is a
    // same-label face, always crossed, with at most three crossings (within
    // nite = 4).  With mirror walls, voxels at the lattice's faces are flagged
    // when their neighbours inside the lattice carry their label: a line that
    // leaves through a wall is reflected there (the origin image mirrored), as
    // the face loop reflects it.  The new voxel's cell, which the next step
    // needs anyway, tells: it is a wall only if the line left the lattice.
    // Other voxels take the face loop.  (Checking the neighbours a step from an
    // unflagged voxel actually passes settles more steps without the face loop,
    // but measured on the 64-axon batch it costs every warp with such a lane
    // more than the face loops it saves.)
    if (g.flight && (s.cell & flight_bit<BITS>())) {
        float x0 = fmaf(s.cur_step, v0, s.o0);
        float x1 = fmaf(s.cur_step, v1, s.o1);
        float x2 = fmaf(s.cur_step, v2, s.o2);
        float k0 = floorf(x0), k1 = floorf(x1), k2 = floorf(x2);
        int ik0 = (int)k0, ik1 = (int)k1, ik2 = (int)k2;
        unsigned lj = s.lin + (unsigned)(ik0 * s0 + ik1 * s1 + ik2);
        unsigned cj = cell_at<BITS>(lat, lj);
        if ((cj & label_mask<BITS>()) == (unsigned)kWall) {
            // out through one or more mirror walls: reflect on each axis whose
            // face neighbour is a wall (x -> -x below the voxel, 2 - x above)
            if (ik0 != 0 && label_at<BITS>(lat, s.lin + (unsigned)(ik0 * s0)) == kWall) {
                const bool hi = ik0 > 0;
                const int nh = nsize(0), gw = hi ? nh - 1 : 0;
                int I = gw - s.D0; mirror_origin(I, s.Fm0, hi, nh); s.D0 = gw - I;
                x0 = hi ? 2.0f - x0 : -x0; k0 = 0.0f; ik0 = 0;
                h.reflect(0);
            }
            if (ik1 != 0 && label_at<BITS>(lat, s.lin + (unsigned)(ik1 * s1)) == kWall) {
                const bool hi = ik1 > 0;
                const int nh = nsize(1), gw = hi ? nh - 1 : 0;
                int I = gw - s.D1; mirror_origin(I, s.Fm1, hi, nh); s.D1 = gw - I;
                x1 = hi ? 2.0f - x1 : -x1; k1 = 0.0f; ik1 = 0;
                h.reflect(1);
            }
            if (ik2 != 0 && label_at<BITS>(lat, s.lin + (unsigned)ik2) == kWall) {
                const bool hi = ik2 > 0;
                const int nh = nsize(2), gw = hi ? nh - 1 : 0;
                int I = gw - s.D2; mirror_origin(I, s.Fm2, hi, nh); s.D2 = gw - I;
                x2 = hi ? 2.0f - x2 : -x2; k2 = 0.0f; ik2 = 0;
                h.reflect(2);
            }
            lj = s.lin + (unsigned)(ik0 * s0 + ik1 * s1 + ik2);
            cj = cell_at<BITS>(lat, lj);
        }
        s.lin = lj;
        s.cell = cj;
        s.D0 += ik0; s.D1 += ik1; s.D2 += ik2;
        s.w32 = fmaf(s.cur_step, s.cur_k, s.w32);
        h.path(s.ai, s.cur_step);
        s.o0 = x0 - k0; s.o1 = x1 - k1; s.o2 = x2 - k2;
        return false;
    }
    // the face loop: up to nite segments, one face event each, on the distances
    // to the next faces along the direction of travel (a face event leaves the
    // walker on the face with a whole voxel ahead: d = 1 exactly)
    unsigned up = nu;
    float d0 = (nu & 1u) ? 1.0f - s.o0 : s.o0;
    float d1 = (nu & 2u) ? 1.0f - s.o1 : s.o1;
    float d2 = (nu & 4u) ? 1.0f - s.o2 : s.o2;
    const float av0 = fabsf(v0), av1 = fabsf(v1), av2 = fabsf(v2);
    const float iv0 = __fdividef(1.0f, av0), iv1 = __fdividef(1.0f, av1), iv2 = __fdividef(1.0f, av2);
    // signed lattice step along each axis in the direction of travel
    int dl0 = (up & 1u) ? s0 : -s0;
    int dl1 = (up & 2u) ? s1 : -s1;
    int dl2 = (up & 4u) ? 1 : -1;
    float rem = s.cur_step;        // path left in this step, voxels
    for (int j = 0; j < g.nite; ++j) {
        const float t0 = d0 * iv0, t1 = d1 * iv1, t2 = d2 * iv2;
        const float tm = fminf(t0, fminf(t1, t2));
        if (rem < tm) {
            // the step ends inside the voxel
            d0 = fmaf(-rem, av0, d0); d1 = fmaf(-rem, av1, d1); d2 = fmaf(-rem, av2, d2);
            s.w32 = fmaf(rem, s.cur_k, s.w32);
            h.path(s.ai, rem);
            rem = 0.0f;
            break;
        }
        // onto the nearest face (lowest axis on ties, like the reference's scan)
        const int hit = (t0 == tm) ? 0 : ((t1 == tm) ? 1 : 2);
        const float tc = fmaxf(tm, 0.0f);
        d0 = fmaf(-tc, av0, d0); d1 = fmaf(-tc, av1, d1); d2 = fmaf(-tc, av2, d2);
        s.w32 = fmaf(tc, s.cur_k, s.w32);
        h.path(s.ai, tc);
        rem -= tc;
        const int dl = hit == 0 ? dl0 : (hit == 1 ? dl1 : dl2);
        unsigned lj = s.lin + (unsigned)dl;
        int aj = label_at<BITS>(lat, lj);
        bool cross;
        if (aj == s.ai && g.same_certain) {
            cross = true;
        } else {
            if (aj == kWall) {
                const bool hi = (up >> hit) & 1u;
                const int nh = nsize(hit);
                if (g.mirror) {
                    // mirror wall: reflect, and mirror the origin image
                    const int gw = hi ? nh - 1 : 0;
                    if (hit == 0) { int I = gw - s.D0; mirror_origin(I, s.Fm0, hi, nh); s.D0 = gw - I; }
                    else if (hit == 1) { int I = gw - s.D1; mirror_origin(I, s.Fm1, hi, nh); s.D1 = gw - I; }
                    else { int I = gw - s.D2; mirror_origin(I, s.Fm2, hi, nh); s.D2 = gw - I; }
                    aj = -1;   // reflect below
                } else {
                    // periodic: the neighbour is on the far side; the
                    // unfolded displacement just continues
                    const int sh = hit == 0 ? s0 : (hit == 1 ? s1 : 1);
                    lj = hi ? s.lin - (unsigned)(nh - 1) * (unsigned)sh : s.lin + (unsigned)(nh - 1) * (unsigned)sh;
                    aj = label_at<BITS>(lat, lj);
                }
            }
            if (aj < 0) {
                cross = false;
            } else {
                const float P = t_pij[s.ai * NCMAX + aj];
                if (P > 0.999999f) {
                    cross = true;
                } else if (P >= 0.000001f) {
                    cross = h.bernoulli(perm.next() < P, P);
                } else {
                    cross = false;
                }
                if (RULE != 0 && !cross) return true;   // a membrane sends the walker back: the rule decides
            }
        }
        if (cross) {
            if (aj != s.ai) {
                rem *= t_ratio[s.ai * NCMAX + aj];
                s.cur_step = t_step[aj];
                s.cur_k = t_k[aj];
                s.ai = aj;
            }
            s.lin = lj;
            const int du = ((up >> hit) & 1u) ? 1 : -1;
            if (hit == 0) s.D0 += du; else if (hit == 1) s.D1 += du; else s.D2 += du;
        } else {
            up ^= 1u << hit;
            if (hit == 0) dl0 = -dl0; else if (hit == 1) dl1 = -dl1; else dl2 = -dl2;
            h.reflect(hit);
        }
        // on the face, a whole voxel ahead
        if (hit == 0) d0 = 1.0f; else if (hit == 1) d1 = 1.0f; else d2 = 1.0f;
        if (!(rem > 0.0f)) break;
    }
    s.o0 = (up & 1u) ? 1.0f - d0 : d0;
    s.o1 = (up & 2u) ? 1.0f - d1 : d1;
    s.o2 = (up & 4u) ? 1.0f - d2 : d2;
    s.cell = cell_at<BITS>(lat, s.lin);
    return false;
}

// The isotropic direction of a step from two uniforms (u1: cos of the polar
// angle, u2: azimuth), in the split walk's FP32 arithmetic.
__device__ __forceinline__ void split_direction(float u1, float u2, float& v0, float& v1, float& v2) {
    const float cz = 1.0f - 2.0f * u1;
    const float s2 = u1 * (1.0f - u1);
    const float sz = 2.0f * s2 * rsqrtf(s2);
    float sp, cp;
    // azimuth 2 pi (u2 - 1/2): uniform on [-pi, pi), within the hardware
    // sine/cosine's accurate range
    __sincosf(6.283185307179586f * (u2 - 0.5f), &sp, &cp);
    v0 = sz * cp; v1 = sz * sp; v2 = cz;
}

}  // namespace rms

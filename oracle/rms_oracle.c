/*
 * oracle/rms_oracle.c -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * Plain-C restatement of the reference simulator's per-walker loop.  Every
 * block cites the reference line it follows; expressions keep the reference's
 * operand order and types so that, compiled without FMA contraction
 * (oracle/Makefile), a job run here equals the host build of the reference
 * (oracle/_ref) bit for bit.  See rms_oracle.h for the interface.
 */
#include "rms_oracle.h"
#include "philox_stream.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define OR_PI 3.14159265 /* main.cu:34 (the reference's truncated pi) */
#define OR_NC_MAX 16

static inline int64_t lin(const or_params* p, int i, int j, int k) {
    /* main.cu:124, 132, 272: NPix2*NPix3*i + NPix3*j + k */
    return (int64_t)p->n2 * p->n3 * i + (int64_t)p->n3 * j + k;
}

static int check(const or_params* p) {
    if (p->nc < 1 || p->nc > OR_NC_MAX) return -1;
    if (p->timepoints < 1 || p->tn < p->timepoints) return -2;
    if (p->nite < 1 || p->nite > 7) return -3;
    if (p->n1 < 1 || p->n2 < 1 || p->n3 < 1) return -4;
    if (p->mode == OR_MODE_PGSE && p->ngrad < 0) return -5;
    if (p->mode == OR_MODE_NARROW && p->nbvec < 0) return -5;
    if (p->mode == OR_MODE_WAVEFORM && (p->nwave < 1 || p->nbins < 1 || p->tn % p->nbins)) return -6;
    return 0;
}

static void walk_one(const or_params* p, int64_t w, or_outputs* out, double* phase,
                     int32_t* tr_init, int32_t* tr_vox, uint32_t* tr_ev, double* tr_pos) {
    const int Nc = p->nc;
    const int Tstep = p->tn / p->timepoints;               /* main.cu:68 */
    const int NPix[3] = {p->n1, p->n2, p->n3};             /* main.cu:86 */
    const uint8_t* APix = p->labels;
    const double* step = p->step;
    const double* Pij = p->pij;
    or_stream st;
    or_stream_init(&st, p->seed, (uint64_t)w);             /* main.cu:58-61, 66 */

    double xi[3] = {0}, xt[3] = {0}, vt[3] = {0};
    int xParGi[3] = {0}, xParGj[3] = {0};
    int flip0[3] = {0}, flip1[3] = {0};
    double t[OR_NC_MAX] = {0};
    int ai = 0, aj = 0, ii_hit = 0;

    /* initial position: rejection sampling in the box (main.cu:117-125) */
    for (;;) {
        xi[0] = or_stream_double(&st) * (double)p->n1;
        xi[1] = or_stream_double(&st) * (double)p->n2;
        xi[2] = or_stream_double(&st) * (double)p->n3;
        xParGi[0] = (int)floor(xi[0]);
        xParGi[1] = (int)floor(xi[1]);
        xParGi[2] = (int)floor(xi[2]);
        if (APix[lin(p, xParGi[0], xParGi[1], xParGi[2])] != 0) break;
    }
    /* main.cu:129-132 */
    xt[0] = xi[0]; xt[1] = xi[1]; xt[2] = xi[2];
    xParGi[0] = (int)floor(xt[0]); xParGi[1] = (int)floor(xt[1]); xParGi[2] = (int)floor(xt[2]);
    ai = APix[lin(p, xParGi[0], xParGi[1], xParGi[2])];
    if (tr_init) *tr_init = (int32_t)lin(p, xParGi[0], xParGi[1], xParGi[2]);

    for (int i = 0; i < p->tn; i++) {                      /* main.cu:134 */
        double fstep = 1.0;
        uint32_t ev = 0;
        int nev = 0;
        for (int jj = 0; jj < 3; jj++) { flip0[jj] = 0; flip1[jj] = 0; }
        /* direction (main.cu:140-151) */
        double vRand = or_stream_double(&st);
        double cos_theta = 1.0 - 2.0 * vRand;
        double sin_theta = 2.0 * sqrt(vRand * (1.0 - vRand));
        vRand = or_stream_double(&st);
        vt[0] = sin_theta * cos(2.0 * OR_PI * vRand);
        vt[1] = sin_theta * sin(2.0 * OR_PI * vRand);
        vt[2] = cos_theta;

        int j;
        for (j = 0; (j < p->nite) && (fstep > 0); j++) {   /* main.cu:153 */
            /* nearest voxel face along the ray (main.cu:199-219) */
            double tmin = 2.0, tmp, tt;
            ii_hit = -1;
            for (int ii = 0; ii < 3; ii++) {
                if (vt[ii] > 0.0) {
                    tmp = (double)xParGi[ii] + 1.0 - xt[ii];
                } else if (vt[ii] < 0.0) {
                    tmp = (double)xParGi[ii] - xt[ii];
                } else {
                    tmp = 2.0;
                }
                if (fabs(tmp) > fabs(vt[ii])) {
                    tt = 2.0;
                } else {
                    double q = tmp / vt[ii];
                    tt = (0.0 < q) ? q : 0.0;             /* std::max(0.0, q) */
                }
                if (tt < tmin) { tmin = tt; ii_hit = ii; }
            }
            if (tmin < 0.0) break;                         /* main.cu:226-229 */

            /* advance to the face or finish the step (main.cu:231-244) */
            if ((fstep * step[ai]) >= tmin) {
                fstep = fstep - tmin / step[ai];
                xt[0] = xt[0] + tmin * vt[0];
                xt[1] = xt[1] + tmin * vt[1];
                xt[2] = xt[2] + tmin * vt[2];
                t[ai] = t[ai] + tmin / step[ai];
            } else {
                xt[0] = xt[0] + step[ai] * fstep * vt[0];
                xt[1] = xt[1] + step[ai] * fstep * vt[1];
                xt[2] = xt[2] + step[ai] * fstep * vt[2];
                t[ai] = t[ai] + fstep;
                fstep = 0.0;   /* the reference breaks here (main.cu:243) */
                break;
            }

            /* neighbour voxel; domain wall (main.cu:246-265) */
            xParGj[0] = xParGi[0]; xParGj[1] = xParGi[1]; xParGj[2] = xParGi[2];
            int wall = 0;
            if (vt[ii_hit] >= 0.0) {
                xParGj[ii_hit] = xParGj[ii_hit] + 1;
                if (xParGj[ii_hit] >= NPix[ii_hit]) wall = 1;
            } else {
                xParGj[ii_hit] = xParGj[ii_hit] - 1;
                if (xParGj[ii_hit] < 0) wall = -1;
            }
            if (wall != 0 && p->boundary == OR_BOUNDARY_MIRROR) {
                if (wall > 0) flip1[ii_hit] = 1; else flip0[ii_hit] = 1;
                vt[ii_hit] = -vt[ii_hit];
                ev |= (OR_EV_MIRROR << 2 | (uint32_t)ii_hit) << (4 * nev++);
                continue;
            }
            if (wall != 0) {
                /* periodic extension: the neighbour is on the far side */
                xParGj[ii_hit] = (wall > 0) ? 0 : NPix[ii_hit] - 1;
            }

            /* membrane: cross, reflect or Bernoulli(Pij) (main.cu:272-289) */
            aj = APix[lin(p, xParGj[0], xParGj[1], xParGj[2])];
            int cross;
            if (Pij[ai * Nc + aj] > 0.999999) {
                cross = 1;
            } else if (Pij[ai * Nc + aj] < 0.000001) {
                cross = 0;
            } else {
                vRand = or_stream_double(&st);
                cross = (vRand < Pij[ai * Nc + aj]);
            }
            if (cross) {
                ai = aj;
                xParGi[ii_hit] = xParGj[ii_hit];
                if (wall != 0) {
                    double shift = (wall > 0) ? -(double)NPix[ii_hit] : (double)NPix[ii_hit];
                    xt[ii_hit] = xt[ii_hit] + shift;
                    xi[ii_hit] = xi[ii_hit] + shift;
                    ev |= (OR_EV_WRAP << 2 | (uint32_t)ii_hit) << (4 * nev++);
                } else {
                    ev |= (OR_EV_CROSS << 2 | (uint32_t)ii_hit) << (4 * nev++);
                }
            } else {
                vt[ii_hit] = -vt[ii_hit];
                ev |= (OR_EV_REFLECT << 2 | (uint32_t)ii_hit) << (4 * nev++);
            }
        }
        if (fstep > 0) ev |= 1u << 31;   /* sub-segment cap hit: remainder dropped */
        ev |= (uint32_t)nev << 28;

        /* mirror the origin for every wall hit this step (main.cu:302-310) */
        for (int jj = 0; jj < 3; jj++) {
            if (flip0[jj]) xi[jj] = -xi[jj];
            if (flip1[jj]) xi[jj] = 2.0 * (double)NPix[jj] - xi[jj];
            flip0[jj] = 0; flip1[jj] = 0;
        }
        if (tr_vox) {
            tr_vox[i] = (int32_t)lin(p, xParGi[0], xParGi[1], xParGi[2]);
            tr_ev[i] = ev;
        }
        if (tr_pos) {
            tr_pos[3 * i + 0] = xt[0];
            tr_pos[3 * i + 1] = xt[1];
            tr_pos[3 * i + 2] = xt[2];
        }

        double dx = 0, dy = 0, dz = 0, s0;
        if (p->mode == OR_MODE_PGSE) {
            /* PGSE phase per gradient (main_PGSE.cu:336-346) */
            dx = (xt[0] - xi[0]) * p->res;
            dy = (xt[1] - xi[1]) * p->res;
            dz = (xt[2] - xi[2]) * p->res;
            const double* g = p->grad;
            const double ti = (double)(i + 1) * p->dt;
            for (int jg = 0; jg < p->ngrad; jg++) {
                if (ti < g[jg * 6 + 1]) {
                    phase[jg] += g[jg * 6 + 2] * (dx * g[jg * 6 + 3] + dy * g[jg * 6 + 4] + dz * g[jg * 6 + 5]) * p->dt;
                } else if ((ti >= g[jg * 6]) & (ti < (g[jg * 6] + g[jg * 6 + 1]))) {
                    phase[jg] -= g[jg * 6 + 2] * (dx * g[jg * 6 + 3] + dy * g[jg * 6 + 4] + dz * g[jg * 6 + 5]) * p->dt;
                }
            }
            /* final T2-weighted signal (main_PGSE.cu:348-357) */
            if (i == (p->tn - 1)) {
                s0 = 0.0;
                for (int c = 0; c < Nc; c++) s0 = s0 + (t[c] / p->t2[c]);
                s0 = exp(-1.0 * s0);
                for (int jg = 0; jg < p->ngrad; jg++) out->sig[jg] += s0 * cos(phase[jg]);
            }
        }

        /* record moments every Tstep steps (main.cu:333-379) */
        if ((i % Tstep) == 0) {
            int tidx = i / Tstep;
            if (tidx >= p->timepoints) continue;   /* the reference writes past its arrays here */
            s0 = 0.0;
            for (int c = 0; c < Nc; c++) s0 = s0 + (t[c] / p->t2[c]);
            s0 = exp(-1.0 * s0);
            int nidx = Nc * tidx + ai;
            out->sig0[tidx] += s0;
            out->npar_count[nidx] += 1;
            dx = (xt[0] - xi[0]) * p->res;
            dy = (xt[1] - xi[1]) * p->res;
            dz = (xt[2] - xi[2]) * p->res;
            double* d2 = out->dx2 + 6 * tidx;
            d2[0] += s0 * dx * dx;
            d2[1] += s0 * dx * dy;
            d2[2] += s0 * dx * dz;
            d2[3] += s0 * dy * dy;
            d2[4] += s0 * dy * dz;
            d2[5] += s0 * dz * dz;
            double* d4 = out->dx4 + 15 * tidx;
            d4[0] += s0 * dx * dx * dx * dx;
            d4[1] += s0 * dx * dx * dx * dy;
            d4[2] += s0 * dx * dx * dx * dz;
            d4[3] += s0 * dx * dx * dy * dy;
            d4[4] += s0 * dx * dx * dy * dz;
            d4[5] += s0 * dx * dx * dz * dz;
            d4[6] += s0 * dx * dy * dy * dy;
            d4[7] += s0 * dx * dy * dy * dz;
            d4[8] += s0 * dx * dy * dz * dz;
            d4[9] += s0 * dx * dz * dz * dz;
            d4[10] += s0 * dy * dy * dy * dy;
            d4[11] += s0 * dy * dy * dy * dz;
            d4[12] += s0 * dy * dy * dz * dz;
            d4[13] += s0 * dy * dz * dz * dz;
            d4[14] += s0 * dz * dz * dz * dz;
            if (p->mode == OR_MODE_NARROW) {
                /* narrow-pulse signal (main.cu:374-378) */
                for (int jb = 0; jb < p->nbvec; jb++) {
                    double qx = sqrt(p->bval[jb] / p->td[tidx]) *
                                (dx * p->bvec[jb * 3 + 0] + dy * p->bvec[jb * 3 + 1] + dz * p->bvec[jb * 3 + 2]);
                    out->sigre[p->nbvec * tidx + jb] += s0 * cos(qx);
                }
            }
        }
    }
}

/* ---------------- FP64 replay of the split-precision walk ---------------- */

static void split_mirror_origin(double* xi, int hi, int n) {
    /* origin image x -> -x (lo wall) or 2N - x (hi wall), main.cu:302-310 */
    *xi = hi ? 2.0 * (double)n - *xi : -*xi;
}

/* Free flight of the split walk: the voxel's 26 neighbours all lie inside the
 * lattice and carry its label. */
static int homogeneous(const or_params* p, const int g[3]) {
    if (g[0] < 1 || g[0] + 1 >= p->n1 || g[1] < 1 || g[1] + 1 >= p->n2 || g[2] < 1 || g[2] + 1 >= p->n3) return 0;
    const uint8_t lab = p->labels[lin(p, g[0], g[1], g[2])];
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++)
                if (p->labels[lin(p, g[0] + a, g[1] + b, g[2] + c)] != lab) return 0;
    return 1;
}

/* Free flight with mirror walls: the voxel's neighbours inside the lattice
 * all carry its label (monte-carlo-simulation-3d-rms_b200/csrc/split_step.cuh:
 * a straight line out through a mirror wall is reflected there, the face
 * loop's own outcome). */
static int homogeneous_walls(const or_params* p, const int g[3]) {
    const uint8_t lab = p->labels[lin(p, g[0], g[1], g[2])];
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++) {
                const int q0 = g[0] + a, q1 = g[1] + b, q2 = g[2] + c;
                if (q0 < 0 || q0 >= p->n1 || q1 < 0 || q1 >= p->n2 || q2 < 0 || q2 >= p->n3) continue;
                if (p->labels[lin(p, q0, q1, q2)] != lab) return 0;
            }
    return 1;
}

/* Adjoint bookkeeping of one walker (or_adjoint_split; the GPU kernel's
 * pass-1 quantities, restated in FP64): the tangent of the displacement with
 * respect to the step length l with the event sequence frozen (gains the step
 * direction each step, flips its component at every reflection, membrane or
 * mirror wall), its bin sums folded into dphi, the permeation score
 * E = sum over Bernoulli crossings of (1[crossed] - Pij), the path per
 * compartment (voxels), the final T2 exponent and each bin's displacement sum. */
typedef struct {
    double T[3], B[3], E, tc[8], wexp;
    double* dphi;   /* [nwave] */
    double* xbin;   /* [nbins*3], um */
    double* rs;     /* [nwave]: sum over bin ends t (g_j,b - g_j,b+1) . x(t) (time rescaling) */
    int ai_end;     /* compartment after the last step */
    int nb;         /* permeation decisions drawn (0 < Pij < 1), counted */
    int force_at;   /* the decision whose outcome is flipped (-1: none) */
    double Pf;      /* its Pij */
    int xf;         /* its outcome before the flip */
} or_adj;

static void walk_split_core(const or_params* p, int64_t w, or_outputs* out, double* phase,
                            int32_t* tr_init, int32_t* tr_vox, uint32_t* tr_ev, double* tr_pos,
                            double* tr_bin, or_adj* adj) {
    const int Nc = p->nc;
    /* free flight applies when same-label faces are always crossed, no walker
     * can enter compartment 0, and three crossings fit the sub-segment cap */
    int flight = p->nite >= 4 && !p->no_flight;
    for (int c = 1; c < Nc; c++)
        if (!(p->pij[c * Nc + c] > 0.999999) || !(p->pij[c * Nc] < 0.000001)) flight = 0;
    const int Tstep = p->tn / p->timepoints;
    const int NPix[3] = {p->n1, p->n2, p->n3};
    const uint8_t* APix = p->labels;
    or_dstream init, perm;
    or_dstream_init(&init, p->seed, (uint64_t)w, OR_DOM_INIT);
    or_dstream_init(&perm, p->seed, (uint64_t)w, OR_DOM_PERM);
    int g[3];
    double f[3], xi[3];
    /* start position, formed in FP32 like the GPU */
    for (;;) {
        float x[3];
        for (int a = 0; a < 3; a++) {
            x[a] = or_dstream_float(&init) * (float)NPix[a];
            g[a] = (int)x[a];
            if (g[a] > NPix[a] - 1) g[a] = NPix[a] - 1;
            f[a] = (double)(x[a] - (float)g[a]);
        }
        if (APix[lin(p, g[0], g[1], g[2])] != 0) break;
    }
    for (int a = 0; a < 3; a++) xi[a] = (double)g[a] + f[a];
    int ai = APix[lin(p, g[0], g[1], g[2])];
    if (tr_init) *tr_init = (int32_t)lin(p, g[0], g[1], g[2]);
    double wexp = 0.0;   /* T2 exponent */
    double X[3] = {0.0, 0.0, 0.0};   /* waveform mode: the current bin's displacement sum (um) */
    const int bin_steps = p->mode == OR_MODE_WAVEFORM ? p->tn / p->nbins : 0;
    for (int i = 0; i < p->tn; i++) {
        float u1f, u2f;
        or_dir_uniforms(p->seed, (uint64_t)w, (uint32_t)i, &u1f, &u2f);
        double u1 = u1f, u2 = u2f;
        /* rule != reflect: the step's start, restored when a membrane turns it back */
        const int sg[3] = {g[0], g[1], g[2]}, sai = ai;
        const double sf[3] = {f[0], f[1], f[2]}, sxi[3] = {xi[0], xi[1], xi[2]}, swexp = wexp;
        double rem;
        int flo, fhi, nev;
        uint32_t ev;
        for (int attempt = 0;; attempt++) {
        int turned = 0;
        const double cz = 1.0 - 2.0 * u1;
        const double sz = 2.0 * sqrt(u1 * (1.0 - u1));
        const double phi = 6.283185307179586 * (u2 - 0.5);
        double v[3] = {sz * cos(phi), sz * sin(phi), cz};
        if (adj) for (int a = 0; a < 3; a++) adj->T[a] += v[a];
        rem = p->step[ai];
        flo = 0; fhi = 0; nev = 0;
        ev = 0;
        if (flight && (p->boundary == OR_BOUNDARY_MIRROR ? homogeneous_walls(p, g) : homogeneous(p, g))) {
            /* a straight line within the homogeneous neighbourhood, reflected at
             * mirror walls (the origin image mirrored at the end of the step) */
            for (int a = 0; a < 3; a++) {
                double x = f[a] + rem * v[a];
                double k = floor(x);
                if (g[a] + (int)k < 0) {
                    x = -x; k = 0.0; flo |= 1 << a;
                    if (adj) adj->T[a] = -adj->T[a];
                } else if (g[a] + (int)k >= NPix[a]) {
                    x = 2.0 - x; k = 0.0; fhi |= 1 << a;
                    if (adj) adj->T[a] = -adj->T[a];
                }
                g[a] += (int)k;
                f[a] = x - k;
            }
            wexp += rem / p->step[ai] / p->t2[ai];
            if (adj) adj->tc[ai] += rem;
            rem = 0.0;
        }
        for (int j = 0; j < p->nite && rem > 0.0; j++) {
            double t[3], tmin;
            for (int a = 0; a < 3; a++) {
                double d = (v[a] > 0.0) ? 1.0 - f[a] : f[a];
                if (d < 0.0) d = 0.0;
                t[a] = (v[a] == 0.0) ? INFINITY : d / fabs(v[a]);
            }
            tmin = fmin(t[0], fmin(t[1], t[2]));
            if (rem < tmin) {
                for (int a = 0; a < 3; a++) f[a] += rem * v[a];
                wexp += rem / p->step[ai] / p->t2[ai];
                if (adj) adj->tc[ai] += rem;
                rem = 0.0;
                break;
            }
            const int hit = (t[0] == tmin) ? 0 : ((t[1] == tmin) ? 1 : 2);
            for (int a = 0; a < 3; a++) f[a] += tmin * v[a];
            wexp += tmin / p->step[ai] / p->t2[ai];
            if (adj) adj->tc[ai] += tmin;
            rem -= tmin;
            const int up = v[hit] > 0.0;
            f[hit] = up ? 1.0 : 0.0;
            int gj = up ? g[hit] + 1 : g[hit] - 1;
            const int wall = (gj < 0 || gj >= NPix[hit]);
            if (wall && p->boundary == OR_BOUNDARY_MIRROR) {
                if (up) fhi |= 1 << hit; else flo |= 1 << hit;
                v[hit] = -v[hit];
                if (adj) adj->T[hit] = -adj->T[hit];
                ev |= (OR_EV_MIRROR << 2 | (uint32_t)hit) << (4 * nev++);
                if (!(rem > 0.0)) break;
                continue;
            }
            if (wall) gj = up ? 0 : NPix[hit] - 1;
            int gn[3] = {g[0], g[1], g[2]};
            gn[hit] = gj;
            const int aj = APix[lin(p, gn[0], gn[1], gn[2])];
            const double P = p->pij[ai * Nc + aj];
            int cross = (P > 0.999999) || (P >= 0.000001 && (double)or_dstream_float(&perm) < P);
            if (adj && !(P > 0.999999) && P >= 0.000001) {
                adj->E += (cross ? 1.0 : 0.0) - P;
                if (adj->nb == adj->force_at) {
                    adj->Pf = P;
                    adj->xf = cross;
                    cross = !cross;
                }
                adj->nb++;
            }
            if (p->rule != OR_RULE_REFLECT && !cross) {
                turned = 1;   /* the rule decides, after the loop */
                break;
            }
            if (cross) {
                if (aj != ai) {
                    rem *= p->step[aj] / p->step[ai];
                    ai = aj;
                }
                g[hit] = gj;
                f[hit] = up ? 0.0 : 1.0;
                if (wall) {
                    xi[hit] += up ? -(double)NPix[hit] : (double)NPix[hit];
                    ev |= (OR_EV_WRAP << 2 | (uint32_t)hit) << (4 * nev++);
                } else {
                    ev |= (OR_EV_CROSS << 2 | (uint32_t)hit) << (4 * nev++);
                }
            } else {
                v[hit] = -v[hit];
                if (adj) adj->T[hit] = -adj->T[hit];
                ev |= (OR_EV_REFLECT << 2 | (uint32_t)hit) << (4 * nev++);
            }
            if (!(rem > 0.0)) break;
        }
        if (p->rule == OR_RULE_REFLECT || !turned) break;
        /* taken back: rejection stays put for the step; the equal-step-length
         * leap redraws the direction from the permeation stream and walks the
         * step again, at most 64 tries (analysis/interaction.m:256-345) */
        for (int a = 0; a < 3; a++) { g[a] = sg[a]; f[a] = sf[a]; xi[a] = sxi[a]; }
        ai = sai;
        wexp = swexp;
        if (p->rule == OR_RULE_REJECT || attempt + 1 >= 64) {
            wexp += 1.0 / p->t2[ai];
            rem = 0.0;
            flo = fhi = nev = 0;
            ev = 0;
            break;
        }
        u1 = (double)or_dstream_float(&perm);
        u2 = (double)or_dstream_float(&perm);
        }
        if (rem > 0.0) ev |= 1u << 31;
        ev |= (uint32_t)nev << 28;
        for (int a = 0; a < 3; a++) {
            if (flo & (1 << a)) split_mirror_origin(&xi[a], 0, NPix[a]);
            if (fhi & (1 << a)) split_mirror_origin(&xi[a], 1, NPix[a]);
        }
        if (tr_vox) {
            tr_vox[i] = (int32_t)lin(p, g[0], g[1], g[2]);
            tr_ev[i] = ev;
        }
        if (tr_pos) for (int a = 0; a < 3; a++) tr_pos[3 * i + a] = (double)g[a] + f[a];
        const double dx = ((double)g[0] + f[0] - xi[0]) * p->res;
        const double dy = ((double)g[1] + f[1] - xi[1]) * p->res;
        const double dz = ((double)g[2] + f[2] - xi[2]) * p->res;
        if (p->mode == OR_MODE_PGSE) {
            const double* gr = p->grad;
            const double ti = (double)(i + 1) * p->dt;
            for (int jg = 0; jg < p->ngrad; jg++) {
                const double q = gr[jg * 6 + 2] * (dx * gr[jg * 6 + 3] + dy * gr[jg * 6 + 4] + dz * gr[jg * 6 + 5]) * p->dt;
                if (ti < gr[jg * 6 + 1]) phase[jg] += q;
                else if ((ti >= gr[jg * 6]) && (ti < (gr[jg * 6] + gr[jg * 6 + 1]))) phase[jg] -= q;
            }
            if (i == p->tn - 1) {
                const double s0 = exp(-wexp);
                for (int jg = 0; jg < p->ngrad; jg++) out->sig[jg] += s0 * cos(phase[jg]);
            }
        }
        if (p->mode == OR_MODE_WAVEFORM) {
            X[0] += dx; X[1] += dy; X[2] += dz;
            if (adj) for (int a = 0; a < 3; a++) adj->B[a] += adj->T[a];
            if ((i + 1) % bin_steps == 0) {
                const int b = (i + 1) / bin_steps - 1;
                for (int j = 0; j < p->nwave; j++) {
                    const double* wv = p->wave + ((size_t)j * p->nbins + b) * 3;
                    phase[j] += p->dt * (wv[0] * X[0] + wv[1] * X[1] + wv[2] * X[2]);
                    if (adj)
                        adj->dphi[j] += p->dt * (wv[0] * adj->B[0] + wv[1] * adj->B[1] + wv[2] * adj->B[2]) * p->res;
                }
                if (adj) {
                    for (int a = 0; a < 3; a++) adj->xbin[3 * b + a] = X[a];
                    adj->B[0] = adj->B[1] = adj->B[2] = 0.0;
                    /* time rescaling: the waveform's step at this bin end, t = (b + 1) bin_steps dt */
                    const double tb = (double)(i + 1) * p->dt;
                    for (int j = 0; j < p->nwave; j++) {
                        const double* wv = p->wave + ((size_t)j * p->nbins + b) * 3;
                        const double* wn = b + 1 < p->nbins ? wv + 3 : NULL;
                        adj->rs[j] += tb * ((wv[0] - (wn ? wn[0] : 0.0)) * dx + (wv[1] - (wn ? wn[1] : 0.0)) * dy +
                                            (wv[2] - (wn ? wn[2] : 0.0)) * dz);
                    }
                }
                if (tr_bin)
                    for (int a = 0; a < 3; a++) tr_bin[3 * b + a] = X[a] / (double)bin_steps;
                X[0] = X[1] = X[2] = 0.0;
            }
            if (i == p->tn - 1) {
                const double s0 = exp(-wexp);
                for (int j = 0; j < p->nwave; j++) {
                    out->sigw[2 * j] += s0 * cos(phase[j]);
                    out->sigw[2 * j + 1] += s0 * sin(phase[j]);
                }
            }
        }
        if ((i % Tstep) == 0) {
            const int tidx = i / Tstep;
            if (tidx >= p->timepoints) continue;
            const double s0 = exp(-wexp);
            out->sig0[tidx] += s0;
            out->npar_count[Nc * tidx + ai] += 1;
            const double d[3] = {dx, dy, dz};
            double* d2 = out->dx2 + 6 * tidx;
            double* d4 = out->dx4 + 15 * tidx;
            int k2 = 0, k4 = 0;
            for (int a = 0; a < 3; a++)
                for (int b = a; b < 3; b++) d2[k2++] += s0 * d[a] * d[b];
            for (int a = 0; a < 3; a++)
                for (int b = a; b < 3; b++)
                    for (int c = b; c < 3; c++)
                        for (int e = c; e < 3; e++) d4[k4++] += s0 * d[a] * d[b] * d[c] * d[e];
            if (p->mode == OR_MODE_NARROW) {
                for (int jb = 0; jb < p->nbvec; jb++) {
                    const double qx = sqrt(p->bval[jb] / p->td[tidx]) *
                                      (dx * p->bvec[jb * 3] + dy * p->bvec[jb * 3 + 1] + dz * p->bvec[jb * 3 + 2]);
                    out->sigre[p->nbvec * tidx + jb] += s0 * cos(qx);
                }
            }
        }
    }
    if (adj) {
        adj->wexp = wexp;
        adj->ai_end = ai;
    }
}

static void walk_one_split(const or_params* p, int64_t w, or_outputs* out, double* phase,
                           int32_t* tr_init, int32_t* tr_vox, uint32_t* tr_ev, double* tr_pos,
                           double* tr_bin) {
    walk_split_core(p, w, out, phase, tr_init, tr_vox, tr_ev, tr_pos, tr_bin, NULL);
}

typedef void (*walk_fn)(const or_params*, int64_t, or_outputs*, double*, int32_t*, int32_t*,
                        uint32_t*, double*, double*);

static int run_range(const or_params* p, int64_t w_begin, int64_t w_end, or_outputs* out,
                     or_trace* tr, walk_fn fn);

int or_run_split(const or_params* p, int64_t w_begin, int64_t w_end, or_outputs* out,
                 or_trace* tr) {
    int rc = check(p);
    if (rc) return rc;
    return run_range(p, w_begin, w_end, out, tr, walk_one_split);
}

int or_adjoint_split(const or_params* p, const double* gup, int64_t w_begin, int64_t w_end, double* sums,
                     double* dwave) {
    int rc = check(p);
    if (rc) return rc;
    if (p->mode != OR_MODE_WAVEFORM || p->rule != OR_RULE_REFLECT || p->nc > 8) return -6;
    const int nw = p->nwave, nb = p->nbins, nc = p->nc;
    double* phase = (double*)calloc((size_t)nw, sizeof(double));
    double* dphi = (double*)calloc((size_t)nw, sizeof(double));
    double* xbin = (double*)calloc((size_t)nb * 3, sizeof(double));
    double* rs = (double*)calloc((size_t)nw + 1, sizeof(double));
    or_outputs scratch;
    double* sbuf = (double*)calloc((size_t)p->timepoints * (1 + 6 + 15 + nc) + 2 * (size_t)nw + 1, sizeof(double));
    if (!phase || !dphi || !xbin || !sbuf || !rs) {
        free(phase); free(dphi); free(xbin); free(sbuf); free(rs);
        return -10;
    }
    scratch.sig0 = sbuf;
    scratch.dx2 = scratch.sig0 + p->timepoints;
    scratch.dx4 = scratch.dx2 + 6 * p->timepoints;
    scratch.npar_count = scratch.dx4 + 15 * p->timepoints;
    scratch.sigw = scratch.npar_count + (size_t)nc * p->timepoints;
    scratch.sigre = NULL;
    scratch.sig = NULL;
    for (int64_t w = w_begin; w < w_end; ++w) {
        or_adj adj;
        memset(&adj, 0, sizeof adj);
        memset(phase, 0, sizeof(double) * (size_t)nw);
        memset(dphi, 0, sizeof(double) * (size_t)nw);
        memset(rs, 0, sizeof(double) * (size_t)nw);
        adj.dphi = dphi;
        adj.xbin = xbin;
        adj.rs = rs;
        adj.force_at = -1;
        walk_split_core(p, w, &scratch, phase, NULL, NULL, NULL, NULL, NULL, &adj);
        /* this walker's loss L_w = s0 sum_j (gC_j cos phi_j + gS_j sin phi_j)
         * and a_j = dL_w / dphi_j */
        const double s0 = exp(-adj.wexp);
        double Lw = 0.0, G = 0.0, TR = 0.0;
        for (int j = 0; j < nw; j++) {
            const double c = cos(phase[j]), sn = sin(phase[j]);
            const double a = s0 * (gup[2 * j + 1] * c - gup[2 * j] * sn);
            Lw += s0 * (gup[2 * j] * c + gup[2 * j + 1] * sn);
            G += a * dphi[j];
            TR += a * (rs[j] - phase[j]);   /* dphi_j / deps of the time rescaling */
            sums[4 + nc + 2 * j] += s0 * c;
            sums[4 + nc + 2 * j + 1] += s0 * sn;
            for (int b = 0; b < nb; b++)
                for (int k = 0; k < 3; k++) dwave[((size_t)b * nw + j) * 3 + k] += a * xbin[3 * b + k];
        }
        /* the T2 exponent under time rescaling: dW/deps = -W + T / T2(c_T) */
        TR += Lw * (adj.wexp - (double)p->tn / p->t2[adj.ai_end]);
        sums[4 + nc + 2 * nw] += TR;
        sums[0] += Lw;
        sums[1] += Lw * adj.E;
        sums[2] += G;
        sums[3] += adj.E;
        for (int c = 0; c < nc; c++)
            if (p->step[c] > 0.0) sums[4 + c] += Lw * adj.tc[c] / p->step[c];
        /* forced decision: one of the walker's nb permeation decisions, chosen
         * uniformly (domain 3), is flipped and the walk repeated with the same
         * streams; nb Pij (1 - Pij) (L[crossed] - L[reflected]) estimates
         * d L_w / d log P (the weak derivative of the Bernoulli draws) */
        if (adj.nb > 0) {
            or_dstream fs;
            or_dstream_init(&fs, p->seed, (uint64_t)w, OR_DOM_FORCE);
            const float u = or_dstream_float(&fs);
            int K = (int)(u * (float)adj.nb);
            if (K > adj.nb - 1) K = adj.nb - 1;
            or_adj fa;
            memset(&fa, 0, sizeof fa);
            memset(phase, 0, sizeof(double) * (size_t)nw);
            fa.dphi = dphi;
            fa.xbin = xbin;
            fa.rs = rs;
            fa.force_at = K;
            walk_split_core(p, w, &scratch, phase, NULL, NULL, NULL, NULL, NULL, &fa);
            const double s0f = exp(-fa.wexp);
            double Lf = 0.0;
            for (int j = 0; j < nw; j++)
                Lf += s0f * (gup[2 * j] * cos(phase[j]) + gup[2 * j + 1] * sin(phase[j]));
            const double dL = fa.xf ? Lw - Lf : Lf - Lw;
            sums[5 + nc + 2 * nw] += (double)adj.nb * fa.Pf * (1.0 - fa.Pf) * dL;
        }
    }
    free(phase); free(dphi); free(xbin); free(sbuf); free(rs);
    return 0;
}

static void walk_one_ref(const or_params* p, int64_t w, or_outputs* out, double* phase, int32_t* ti,
                         int32_t* tv, uint32_t* te, double* tp, double* tb) {
    (void)tb;
    walk_one(p, w, out, phase, ti, tv, te, tp);
}

int or_run(const or_params* p, int64_t w_begin, int64_t w_end, or_outputs* out,
           or_trace* tr) {
    int rc = check(p);
    if (rc) return rc;
    if (p->mode == OR_MODE_WAVEFORM) return -6;   /* the reference's order has no waveform mode */
    if (p->rule != OR_RULE_REFLECT) return -7;    /* nor other membrane rules */
    return run_range(p, w_begin, w_end, out, tr, walk_one_ref);
}

static int run_range(const or_params* p, int64_t w_begin, int64_t w_end, or_outputs* out,
                     or_trace* tr, walk_fn fn) {
    double* phase = NULL;
    const int nph = p->mode == OR_MODE_PGSE ? p->ngrad : (p->mode == OR_MODE_WAVEFORM ? p->nwave : 0);
    if (nph > 0) {
        phase = (double*)malloc(sizeof(double) * (size_t)nph);
        if (!phase) return -10;
    }
    for (int64_t w = w_begin; w < w_end; ++w) {
        if (phase) memset(phase, 0, sizeof(double) * (size_t)nph);
        int32_t* ti = NULL; int32_t* tv = NULL; uint32_t* te = NULL; double* tp = NULL; double* tb = NULL;
        if (tr && w >= tr->w0 && w < tr->w0 + tr->nw) {
            int64_t r = w - tr->w0;
            ti = tr->init_voxel + r;
            tv = tr->voxel + r * p->tn;
            te = tr->events + r * p->tn;
            if (tr->pos) tp = tr->pos + r * p->tn * 3;
            if (tr->binmean && p->mode == OR_MODE_WAVEFORM) tb = tr->binmean + r * p->nbins * 3;
        }
        fn(p, w, out, phase, ti, tv, te, tp, tb);
    }
    free(phase);
    return 0;
}

static void zero_outputs(const or_params* p, or_outputs* o) {
    memset(o->sig0, 0, sizeof(double) * p->timepoints);
    memset(o->dx2, 0, sizeof(double) * p->timepoints * 6);
    memset(o->dx4, 0, sizeof(double) * p->timepoints * 15);
    memset(o->npar_count, 0, sizeof(double) * p->timepoints * p->nc);
    if (p->mode == OR_MODE_NARROW && p->nbvec > 0)
        memset(o->sigre, 0, sizeof(double) * p->timepoints * p->nbvec);
    if (p->mode == OR_MODE_PGSE && p->ngrad > 0) memset(o->sig, 0, sizeof(double) * p->ngrad);
    if (p->mode == OR_MODE_WAVEFORM) memset(o->sigw, 0, sizeof(double) * 2 * p->nwave);
}

static void add_outputs(const or_params* p, or_outputs* dst, const or_outputs* src) {
    for (int i = 0; i < p->timepoints; i++) dst->sig0[i] += src->sig0[i];
    for (int i = 0; i < p->timepoints * 6; i++) dst->dx2[i] += src->dx2[i];
    for (int i = 0; i < p->timepoints * 15; i++) dst->dx4[i] += src->dx4[i];
    for (int i = 0; i < p->timepoints * p->nc; i++) dst->npar_count[i] += src->npar_count[i];
    if (p->mode == OR_MODE_NARROW)
        for (int i = 0; i < p->timepoints * p->nbvec; i++) dst->sigre[i] += src->sigre[i];
    if (p->mode == OR_MODE_PGSE)
        for (int i = 0; i < p->ngrad; i++) dst->sig[i] += src->sig[i];
    if (p->mode == OR_MODE_WAVEFORM)
        for (int i = 0; i < 2 * p->nwave; i++) dst->sigw[i] += src->sigw[i];
}

static int run_parallel(const or_params* p, int64_t w_begin, int64_t w_end, int nthreads,
                        or_outputs* out, int split);

int or_run_parallel(const or_params* p, int64_t w_begin, int64_t w_end, int nthreads,
                    or_outputs* out) {
    return run_parallel(p, w_begin, w_end, nthreads, out, 0);
}

int or_run_split_parallel(const or_params* p, int64_t w_begin, int64_t w_end, int nthreads,
                          or_outputs* out) {
    return run_parallel(p, w_begin, w_end, nthreads, out, 1);
}

static int run_parallel(const or_params* p, int64_t w_begin, int64_t w_end, int nthreads,
                        or_outputs* out, int split) {
    int rc = check(p);
    if (rc) return rc;
    if (nthreads < 1) nthreads = 1;
    size_t per = (size_t)p->timepoints * (1 + 6 + 15 + p->nc) +
                 (size_t)p->timepoints * (p->mode == OR_MODE_NARROW ? p->nbvec : 0) +
                 (size_t)(p->mode == OR_MODE_PGSE ? p->ngrad : 0) +
                 (size_t)(p->mode == OR_MODE_WAVEFORM ? 2 * p->nwave : 0);
    double* buf = (double*)calloc(per * (size_t)nthreads, sizeof(double));
    or_outputs* priv = (or_outputs*)calloc((size_t)nthreads, sizeof(or_outputs));
    if (!buf || !priv) { free(buf); free(priv); return -10; }
    for (int t = 0; t < nthreads; t++) {
        double* b = buf + per * (size_t)t;
        priv[t].sig0 = b; b += p->timepoints;
        priv[t].dx2 = b; b += p->timepoints * 6;
        priv[t].dx4 = b; b += p->timepoints * 15;
        priv[t].npar_count = b; b += p->timepoints * p->nc;
        priv[t].sigre = b; if (p->mode == OR_MODE_NARROW) b += p->timepoints * p->nbvec;
        priv[t].sig = b; if (p->mode == OR_MODE_PGSE) b += p->ngrad;
        priv[t].sigw = b;
    }
    int64_t n = w_end - w_begin;
    int err = 0;
#pragma omp parallel num_threads(nthreads)
    {
        int t = omp_get_thread_num(), nt = omp_get_num_threads();
        int64_t lo = w_begin + n * t / nt, hi = w_begin + n * (t + 1) / nt;
        if ((split ? or_run_split(p, lo, hi, &priv[t], NULL) : or_run(p, lo, hi, &priv[t], NULL)) != 0) {
#pragma omp atomic write
            err = 1;
        }
    }
    if (!err) {
        zero_outputs(p, out);
        for (int t = 0; t < nthreads; t++) add_outputs(p, out, &priv[t]);
    }
    free(buf);
    free(priv);
    return err ? -11 : 0;
}

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    or_philox4x32(ctr, key, 10, out);
}

void or_stream_doubles(uint64_t seed, uint64_t walker, int n, double* out) {
    or_stream s;
    or_stream_init(&s, seed, walker);
    for (int i = 0; i < n; i++) out[i] = or_stream_double(&s);
}

void or_split_dir_uniforms(uint64_t seed, uint64_t walker, int nsteps, float* out) {
    for (int i = 0; i < nsteps; i++) or_dir_uniforms(seed, walker, (uint32_t)i, &out[2 * i], &out[2 * i + 1]);
}

void or_split_domain_floats(uint64_t seed, uint64_t walker, uint32_t dom, int n, float* out) {
    or_dstream s;
    or_dstream_init(&s, seed, walker, dom);
    for (int i = 0; i < n; i++) out[i] = or_dstream_float(&s);
}

void or_stream_floats(uint64_t seed, uint64_t walker, int n, float* out) {
    or_stream s;
    or_stream_init(&s, seed, walker);
    for (int i = 0; i < n; i++) out[i] = or_stream_float(&s);
}

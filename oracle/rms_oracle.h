/*
 * oracle/rms_oracle.h -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * A CPU restatement, in plain C, of the reference random-walk simulator's
 * per-walker algorithm (hpc_code/lib/main.cu:63-384 narrow-pulse,
 * hpc_code/lib/main_PGSE.cu:65-410 PGSE), plus the engine's documented
 * extensions (periodic boundary, explicit permeation table, configurable
 * timepoints and sub-segment cap) so the GPU kernels' extension paths have a
 * checker too.  With the reference settings it reproduces the host build of
 * the reference itself (oracle/_ref) bit for bit; tests pin that.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.
 */
#ifndef RMS_ORACLE_H
#define RMS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MODE_NARROW 0
#define OR_MODE_PGSE 1
#define OR_MODE_WAVEFORM 2   /* engine extension: general gradient waveforms */
#define OR_BOUNDARY_MIRROR 0
#define OR_BOUNDARY_PERIODIC 1

/* event codes, 4 bits per sub-segment event, oldest in the low bits */
#define OR_EV_MIRROR 1u   /* domain wall: direction flipped, origin mirrored */
#define OR_EV_REFLECT 2u  /* membrane: reflected */
#define OR_EV_CROSS 3u    /* membrane or same label: crossed */
#define OR_EV_WRAP 1u     /* periodic wall (shares the code of MIRROR) */

typedef struct or_params {
    int mode;            /* OR_MODE_NARROW / OR_MODE_PGSE */
    int64_t npar;        /* walkers in the job */
    int tn;              /* steps */
    int timepoints;      /* records; reference: 1000 (main.cu:35) */
    int nite;            /* sub-segment cap; reference: 4 (main.cu:36) */
    int nc;              /* compartments */
    int n1, n2, n3;      /* lattice, k (n3) fastest */
    int boundary;        /* OR_BOUNDARY_* ; reference: mirror */
    double res;          /* voxel size, um */
    double dt;           /* ms */
    uint64_t seed;
    const double* step;  /* [nc] step length in voxels: sqrt(6 dt D)/res */
    const double* t2;    /* [nc] T2 in steps (T2/dt) */
    const double* pij;   /* [nc*nc] permeation probability a->b */
    const uint8_t* labels; /* [n1*n2*n3] */
    /* narrow pulse */
    int nbvec;
    const double* bval;  /* [nbvec] */
    const double* bvec;  /* [nbvec*3] */
    const double* td;    /* [timepoints] */
    /* PGSE */
    int ngrad;
    const double* grad;  /* [ngrad*6] Delta, delta, |g|, gx, gy, gz */
    /* general waveforms (split replay only): phase_j = dt sum_b wave[j][b] . X_b,
     * X_b = sum over bin b's steps of the displacement (um) after each step */
    int nwave, nbins;
    const double* wave;  /* [nwave*nbins*3] */
    /* membrane rule of the split replay: reflect (the reference), reject
     * (stay for the step) or leap (redraw the direction), interaction.m */
    int rule;
    int no_flight;       /* 1: every split-replay step through the face loop (a
                            check that the straight moves are its outcome) */
} or_params;

#define OR_RULE_REFLECT 0
#define OR_RULE_REJECT 1
#define OR_RULE_LEAP 2

typedef struct or_outputs {
    double* sig0;        /* [timepoints] */
    double* dx2;         /* [timepoints*6] */
    double* dx4;         /* [timepoints*15] */
    double* sigre;       /* [timepoints*nbvec] narrow */
    double* sig;         /* [ngrad] PGSE */
    double* npar_count;  /* [timepoints*nc] */
    double* sigw;        /* [nwave*2] waveform mode: sums of s0 cos(phase), s0 sin(phase) */
} or_outputs;

typedef struct or_trace {
    int64_t w0;          /* first traced walker */
    int64_t nw;          /* number of traced walkers */
    int32_t* init_voxel; /* [nw] voxel of the initial position */
    int32_t* voxel;      /* [nw*tn] voxel after each step */
    uint32_t* events;    /* [nw*tn] event code of each step */
    double* pos;         /* [nw*tn*3] position (voxel units) after each step, or NULL */
    double* binmean;     /* [nw*nbins*3] waveform mode: bin mean displacement (um), or NULL */
} or_trace;

/* Walk walkers [w_begin, w_end) in order, adding into *out (which the caller
 * zeroes).  Returns 0, or a negative code for invalid parameters. */
int or_run(const or_params* p, int64_t w_begin, int64_t w_end, or_outputs* out,
           or_trace* trace);

/* Same job on nthreads OpenMP threads: contiguous walker ranges, private
 * accumulators summed in thread order. */
int or_run_parallel(const or_params* p, int64_t w_begin, int64_t w_end, int nthreads,
                    or_outputs* out);

/* FP64 replay of the engine's split-precision walk (RMS_PREC_SPLIT): the same
 * algorithm and the same random streams (philox_stream.h, split domains),
 * every quantity after the start position in FP64.  The start position is
 * formed in FP32 exactly as the GPU forms it, so both runs start from the same
 * point and differ only by the precision of the dynamics.  PGSE phases are
 * accumulated per step as in the reference (main_PGSE.cu:340-346). */
int or_run_split(const or_params* p, int64_t w_begin, int64_t w_end, or_outputs* out,
                 or_trace* trace);
int or_run_split_parallel(const or_params* p, int64_t w_begin, int64_t w_end, int nthreads,
                          or_outputs* out);

/* The project's stream, exposed for known-answer tests. */
/* The adjoint of the split walk in waveform mode (reflecting membranes), FP64:
 * per walker the tangent of the displacement with respect to the step length
 * with the event sequence frozen, the permeation score, the path per
 * compartment and the bin displacement sums, folded with the upstream weights
 * gup[2*nwave] (gC_j, gS_j) into walker sums:
 *   sums[0] = sum L_w, sums[1] = sum L_w E_w, sums[2] = sum_w sum_j a_jw dphi_jw,
 *   sums[3] = sum E_w, sums[4+c] = sum L_w t_wc / step_c (c < nc),
 *   sums[4+nc+2j], [4+nc+2j+1] = sum s0 cos phi_j, sum s0 sin phi_j;
 *   sums[4+nc+2nwave] = sum of the time-rescaling derivatives dL_w/deps;
 *   sums[5+nc+2nwave] = sum nb_w Pij (1 - Pij) (L_w[crossed] - L_w[reflected])
 *     over walkers with nb_w > 0 permeation draws, one of them (chosen from
 *     domain 3) flipped and the walk repeated on the same streams;
 *   dwave[(b*nwave + j)*3 + k] += sum a_jw X_wbk (um).
 * The same sums as the GPU adjoint kernel (csrc/rms_adjoint.cu); the caller
 * zeroes them.  Returns -6 for other modes or rules. */
int or_adjoint_split(const or_params* p, const double* gup, int64_t w_begin, int64_t w_end, double* sums,
                     double* dwave);

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void or_stream_doubles(uint64_t seed, uint64_t walker, int n, double* out);
void or_stream_floats(uint64_t seed, uint64_t walker, int n, float* out);
void or_split_dir_uniforms(uint64_t seed, uint64_t walker, int nsteps, float* out);  /* [nsteps*2] */
void or_split_domain_floats(uint64_t seed, uint64_t walker, uint32_t dom, int n, float* out);

#ifdef __cplusplus
}
#endif
#endif

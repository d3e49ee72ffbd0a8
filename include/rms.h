/*
 * rms.h -- C ABI of librms, the B200-native random-walk diffusion engine.
 *
 * The reference simulator (NYU-DiffusionMRI/monte-carlo-simulation-3D-RMS,
 * hpc_code/lib/main.cu and main_PGSE.cu) has no library interface: its
 * boundary is a process run with no arguments in a directory of text files
 * (part1_demo3_simulation.m:86-90).  This header is the library form of that
 * boundary; `rms_main` (the drop-in executable) is a thin client of it.
 *
 * Conventions
 *  - Every call returns an int status: RMS_OK (0) or a negative RMS_ERR_*.
 *    rms_last_error() gives a thread-local message for the last failure.
 *    No C++ exception and no exit() crosses this boundary.
 *  - The library owns rms_sim objects.  Caller buffers are borrowed for the
 *    duration of the call only (inputs are copied, outputs are written).
 *  - One rms_sim is not thread-safe; distinct rms_sim objects are independent.
 *  - Units follow the reference: ms, um, um^2/ms, |g| in rad/(um ms).
 */
#ifndef RMS_H
#define RMS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RMS_OK 0
#define RMS_ERR_ARG (-1)      /* invalid argument or configuration */
#define RMS_ERR_IO (-2)       /* file missing or unreadable / unwritable */
#define RMS_ERR_FORMAT (-3)   /* file content malformed or too short */
#define RMS_ERR_RANGE (-4)    /* value outside the supported range */
#define RMS_ERR_CUDA (-5)     /* CUDA runtime failure */
#define RMS_ERR_NOMEM (-6)    /* host or device allocation failed */
#define RMS_ERR_STATE (-7)    /* call out of order (e.g. get before run) */
#define RMS_ERR_TIMEOUT (-8)  /* a bounded device wait gave up */

/* Signal form: narrow-pulse b-table (main.cu) or rectangular PGSE (main_PGSE.cu). */
#define RMS_MODE_NARROW 0
#define RMS_MODE_PGSE 1
#define RMS_MODE_WAVEFORM 2   /* general gradient waveforms on time bins (SPLIT walk only) */
#define RMS_MODE_AUTO (-1)    /* rms_sim_load_dir: PGSE iff gradient_time.txt exists */

/* Lattice walls: mirror (the reference, main.cu:249-265, 302-310) or periodic. */
#define RMS_BOUNDARY_MIRROR 0
#define RMS_BOUNDARY_PERIODIC 1

/* Membrane permeation probability Pij between compartments a -> b.
 *  REFERENCE: 0 if a or b is 0, 1 if a == b, else min(1, sqrt(D_b/D_a))
 *             (main.cu:444-458).
 *  KAPPA:     0 if a or b is 0, 1 if a == b, else, from the permeability
 *             kappa (um/ms) and the step length ds_a = sqrt(6 D_a dt) (um),
 *             P = (2/3) kappa ds_a / D_a, then Pij = P / (1 + P).
 *  TABLE:     the caller's nc*nc table, used as given. */
#define RMS_PERM_REFERENCE 0
#define RMS_PERM_KAPPA 1
#define RMS_PERM_TABLE 2

/* Arithmetic of the walk.
 *  COMPAT: FP64 positions, FP64 uniforms, the reference's operation order;
 *          per-walker voxel/event sequences equal the CPU oracle's.
 *  SPLIT:  int32 voxel index + FP32 in-voxel offset, FP32 uniforms, FP64
 *          cross-walker sums; statistically equal to COMPAT.
 *  Repeatability: COMPAT sums each record's per-warp rows in a fixed order,
 *  so a rerun with the same seed is identical bit for bit; SPLIT adds the
 *  warps' rows into the totals with FP64 atomics, so a rerun has the same
 *  walkers and compartment counts and equal sums up to their order (about
 *  1e-15 relative). */
#define RMS_PREC_COMPAT 0
#define RMS_PREC_SPLIT 1

typedef struct rms_config {
    int mode;                  /* RMS_MODE_NARROW or RMS_MODE_PGSE */
    double dt;                 /* time step, ms */
    int tn;                    /* number of steps */
    int64_t npar;              /* number of walkers */
    int nc;                    /* number of compartments (labels 0..nc-1) */
    double res;                /* voxel size, um */
    int n1, n2, n3;            /* lattice size, n3 fastest */
    const double* diffusivity; /* [nc] um^2/ms; compartment 0 is the null one */
    const double* t2;          /* [nc] ms, > 0 */
    /* narrow pulse (main.cu:469-482) */
    int nbvec;
    const double* bval;        /* [nbvec] ms/um^2 */
    const double* bvec;        /* [nbvec*3] */
    /* PGSE (main_PGSE.cu:495-506) */
    int ngrad;
    const double* grad;        /* [ngrad*6]: Delta, delta, |g|, gx, gy, gz */
    /* general waveforms (RMS_MODE_WAVEFORM; no reference counterpart): nwave
     * waveforms, each piecewise constant on nbins equal time bins (TN must be
     * a multiple of nbins); wave[(j*nbins + b)*3 + axis] = gamma*g in
     * rad/(um ms).  Phase of walker and waveform j:
     *   phi_j = dt * sum_b wave_j,b . X_b,  X_b = sum over the bin's steps of
     *   the displacement (um) at the end of each step (the PGSE convention of
     *   main_PGSE.cu:340-346). */
    int nwave;
    int nbins;
    const double* wave;
    /* extensions; 0 selects the reference's value */
    int timepoints;            /* records; 0 -> 1000 (main.cu:35) */
    int nite;                  /* sub-segment cap per step; 0 -> 4 (main.cu:36) */
    int boundary;              /* RMS_BOUNDARY_* */
    int permeation;            /* RMS_PERM_* */
    double kappa;              /* um/ms, RMS_PERM_KAPPA */
    const double* pij;         /* [nc*nc], RMS_PERM_TABLE */
    int membrane_rule;         /* RMS_RULE_*: what a membrane does to a walker it
                                  turns back (SPLIT walk; COMPAT reflects) */
} rms_config;

/* Membrane rules.  REFLECT: elastic reflection at the membrane (the
 * reference simulator, main.cu:274-300).  REJECT: the whole step is
 * cancelled and the walker stays where it was for that step ("rejection
 * sampling", analysis/interaction.m:302-345).  LEAP: the step is cancelled and
 * taken again in a new direction (drawn from the partial-permeation stream)
 * until it stays clear, at most 64 tries, then the walker stays ("equal-step-
 * length random leap", interaction.m:256-300).  Mirror domain walls reflect
 * under every rule. */
#define RMS_RULE_REFLECT 0
#define RMS_RULE_REJECT 1
#define RMS_RULE_LEAP 2

typedef struct rms_run_opts {
    uint64_t seed;             /* RNG seed (the reference reads /dev/random) */
    int precision;             /* RMS_PREC_* */
    int device;                /* CUDA device ordinal */
    void* stream;              /* cudaStream_t to run on; NULL = library stream */
    int trace_walkers;         /* > 0: keep per-step voxel/event traces of
                                  walkers [0, trace_walkers) (COMPAT only) */
    int variant;               /* SPLIT walk launch variant: 0 = tuned default,
                                  k >= 1 = entry k of rms_split_variant() */
    int64_t walker_begin;      /* walk walkers [walker_begin, walker_end) of */
    int64_t walker_end;        /* the job; 0, 0 = all.  Lets ranks shard a job. */
    float* traj_out;           /* RMS_MODE_WAVEFORM, SPLIT: optional DEVICE buffer
                                  [walker - walker_begin][nbins][3] of each
                                  bin's mean displacement X_b / steps (um) */
    int traj_split;            /* nonzero: traj_out receives the means split into
                                  BF16 pairs, x = hi + lo: n*nbins*3 hi parts
                                  ([walker][nbins][3], n = walker_end -
                                  walker_begin), then n*nbins*3 lo parts -- the
                                  same bytes as the FP32 form; the input of
                                  RMS_CONTRACT_BF16X3_PRESPLIT */
    int shard_index;           /* shard_count > 1: every simulation of the call */
    int shard_count;           /* walks only its walkers [npar*shard_index/shard_count,
                                  npar*(shard_index+1)/shard_count): one rank's part
                                  of a job or of a batch.  Walker ids, and so the
                                  random streams, are the whole job's, so the
                                  shards' sums add up to the unsharded result.  A
                                  shard may be empty (npar < shard_count): its
                                  results are zero.  0 or 1 = all walkers; not
                                  combined with walker_begin/walker_end. */
} rms_run_opts;

typedef struct rms_sim rms_sim;

/* Output fields (rms_sim_get).  Layouts follow the reference's files
 * (main.cu:550-615, main_PGSE.cu:596-669): row-major [timepoints][cols]. */
#define RMS_FIELD_SIG0 0        /* [T]            sig0.txt */
#define RMS_FIELD_DX2 1         /* [T*6]          dx2.txt  xx xy xz yy yz zz */
#define RMS_FIELD_DX4 2         /* [T*15]         dx4.txt  (readRMS.m:16-18 order) */
#define RMS_FIELD_SIGRE 3       /* [T*nbvec]      sigRe.txt (narrow) */
#define RMS_FIELD_SIG 4         /* [ngrad]        sig.txt   (PGSE) */
#define RMS_FIELD_NPAR_COUNT 5  /* [T*nc]         NPar_count.txt */
#define RMS_FIELD_TD 6          /* [T]            diff_time.txt */
/* Derived tables, available without a run (main.cu:421-458): */
#define RMS_FIELD_DIFFUSIVITY 7 /* [nc]           um^2/ms */
#define RMS_FIELD_STEP 8        /* [nc]           step length in voxels */
#define RMS_FIELD_PIJ 9         /* [nc*nc]        permeation probability a -> b */
#define RMS_FIELD_SIGW 10       /* [nwave*2]      waveform signal: sum s0 cos phi, sum s0 sin phi */
/* Gradient tables as configured, available without a run: */
#define RMS_FIELD_BVAL 11       /* [nbvec]        bval.txt, ms/um^2 (narrow pulses; main.cu:469-474) */
#define RMS_FIELD_BVEC 12       /* [nbvec*3]      bvec.txt rows (narrow pulses; main.cu:477-482) */
#define RMS_FIELD_GRAD 13       /* [ngrad*6]      gradient_time.txt rows: Delta delta |g| gx gy gz
                                                   (PGSE; main_PGSE.cu:501-506) */
#define RMS_FIELD_SIM_PARA 14   /* [4]            sim_para.txt: dt (ms), TN, NPar, voxel size (um)
                                                   (main.cu:606-609), available without a run */

/* Build a simulation from a configuration (what main.cu:414-487 derives from
 * the text inputs).  Replaces: the input parsing + table set-up of
 * hpc_code/lib/main.cu:388-487 and main_PGSE.cu:414-527. */
int rms_sim_create(const rms_config* cfg, rms_sim** out);

/* Build a simulation from a run directory of reference inputs
 * (simParamInput.txt, diffusivity.txt, T2.txt, fiber.txt, and bval/bvec.txt
 * or gradient_Ngrad/gradient_time.txt).  mode: RMS_MODE_* or RMS_MODE_AUTO.
 * Replaces: the ifstream readers of main.cu:414-482, main_PGSE.cu:440-506. */
int rms_sim_load_dir(const char* dir, int mode, rms_sim** out);

/* Set (copy in) the label lattice, n3 fastest.  Labels must be < nc, and at
 * least 1e-7 of the voxels labelled (RMS_ERR_RANGE otherwise; a refused
 * lattice leaves the simulation's own in place).  Once the simulation has run
 * (it holds its device), the lattice is uploaded straight from `labels` (a
 * DMA when the buffer is pinned) and checked on the GPU; otherwise it is
 * checked and copied on the host.  Returns when `labels` is no longer read.
 * Replaces: fiber.txt -> APix (main.cu:461-466, :532). */
int rms_sim_set_lattice(rms_sim* sim, const uint8_t* labels, int n1, int n2, int n3);

/* Run the walk on the GPU; results stay in the sim until rms_sim_get.
 * Replaces: setup_kernel + propagate launch + copy-back
 * (main.cu:498-547, main_PGSE.cu:536-592). */
int rms_sim_run(rms_sim* sim, const rms_run_opts* opts);

/* Number of doubles in an output field. */
int rms_sim_field_size(const rms_sim* sim, int field, size_t* n);

/* Copy an output field into a caller buffer of n doubles (n must equal the
 * field size).  Replaces: thrust::copy back (main.cu:542-547). */
int rms_sim_get(const rms_sim* sim, int field, double* out, size_t n);

/* Per-step traces of the first trace_walkers walkers of the last COMPAT run:
 * init_voxel[w], voxel[w*tn+i] (linear index after step i), events[w*tn+i]
 * (4 bits per sub-segment event: axis | type<<2, type 1 wall, 2 reflect,
 * 3 cross; bits 28-30 event count; bit 31 remainder dropped).  No
 * reference counterpart: the test hook for step-by-step parity. */
int rms_sim_get_trace(const rms_sim* sim, int32_t* init_voxel, int32_t* voxel,
                      uint32_t* events, size_t nwalkers, size_t tn);

/* Position (voxel units, [w][i][xyz]) after each step of the traced walkers
 * of the last COMPAT run.  No reference counterpart: a parity test hook. */
int rms_sim_get_trace_positions(const rms_sim* sim, double* pos, size_t nwalkers, size_t tn);

/* Write the reference's output files into dir.  Replaces: the ofstream
 * writers of main.cu:550-615 and main_PGSE.cu:596-669. */
int rms_sim_write_dir(const rms_sim* sim, const char* dir);

/* Device time of the last run's walk kernel and of the whole run (ms), from
 * CUDA events on the run's stream; after rms_adjoint_run or
 * rms_adjoint_jacobian, both hold the reverse pass's time.  Replaces the
 * clock() print of main.cu:536-540. */
int rms_sim_last_timing(const rms_sim* sim, double* walk_ms, double* run_ms);

/* Run several simulations (e.g. one per axon) on one device.  Simulation k
 * walks with seed + k * 0x9E3779B97F4A7C15, so it reproduces rms_sim_run of
 * that simulation with that seed.  RMS_PREC_SPLIT walks all of them in ONE
 * persistent launch (uneven lattices and walker counts share the grid); they
 * must share TN, dt, timepoints, nite, walls and the b-table or gradient
 * table (lattice, Nc, D, T2, permeation, res and NPar may differ).
 * RMS_PREC_COMPAT runs them one after another.  opts->walker_begin/end are
 * ignored (every simulation walks all its walkers).
 * Replaces: the serial per-axon loop of part1_demo3_simulation.m:83-92. */
int rms_batch_run(rms_sim* const* sims, int n, const rms_run_opts* opts);

/* Thread-local message of the last failed call ("" if none). */
const char* rms_last_error(void);

void rms_sim_destroy(rms_sim* sim);

/* The engine's random stream on the host: n uniforms of walker `walker`
 * (Philox4x32-10; doubles take two words, floats one).  Replaces the draws of
 * curand_uniform_double (main.cu:118-120, 140, 144, 282); a test hook. */
int rms_rng_doubles(uint64_t seed, uint64_t walker, int n, double* out);
int rms_rng_floats(uint64_t seed, uint64_t walker, int n, float* out);
int rms_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The SPLIT walk's streams on the host: domain 0 gives the direction
 * uniforms of steps 0, 1, ... (two per step, n values), domain 1 the start
 * position draws, domain 2 the partial-permeation draws.  A test hook. */
int rms_rng_split(uint64_t seed, uint64_t walker, int domain, int n, float* out);

/* Lattice of one tube along z built on the GPU: voxel (i, j, k) gets
 * `inside` when ((i+0.5) res - cx[k])^2 + ((j+0.5) res - cy[k])^2 < r2[k],
 * else `outside` (per-slice radius^2 and centre, um, n3 values each: the
 * caliber variation and undulation of an axon, analysis/visualizeaxon.m:28-67).
 * Every operation is rounded on its own, so the lattice equals one built on
 * the host in FP64 from the same tables.  Replaces the sim's lattice (a host
 * copy is kept). */
int rms_sim_set_tube_lattice(rms_sim* sim, const double* r2, const double* cx, const double* cy, int inside,
                             int outside, int device);

/* Cumulants of a finished run, the formulas analysis/readRMS.m applies to the
 * output files (:44-45 normalisation by sig0 with the tensor multiplicities,
 * :96-103 D = <x^2>/(2t), K = <x^4>/<x^2>^2 - 3) along ndir unit directions
 * dirs[ndir*3] (NULL: x, y, z): D[t*ndir + q], K[t*ndir + q] for the
 * timepoints t.  rms_combine_cumulants combines per-axon D, K ([axon][t][dir])
 * with volume fractions f[axon] as part1_demo4_analysis.m:88-90 does:
 * D = sum f D_i, K = 3 (sum f D_i^2 - D^2) / D^2 + sum f D_i^2 K_i / D^2. */
int rms_sim_cumulants(const rms_sim* sim, const double* dirs, int ndir, double* D, double* K);
int rms_combine_cumulants(int naxons, int T, int ndir, const double* f, const double* D_axons,
                          const double* K_axons, double* D, double* K);

/* DKI fits of a signal table (host functions; no simulation needed).
 * sig[T*m]: signal per timepoint and measurement, normalised as the readers do
 * (narrow pulses: |sigRe| / sig0, readRMS.m:47-48; PGSE: |sig|,
 * readRMS_pgse.m:56); bvec[m*3] gradient directions, bval[m] b-values.
 *
 * rms_dki_shell (readRMS.m:51-78; readRMS_pgse.m:60-89 with intercept = 1):
 * per unique direction (exact row equality) the least-squares fit of
 * log(S + eps) against [1] -b, b^2/6, ..., b^nb/6 (nb = number of distinct
 * b-values), D = first slope, K = second / D^2; then <x^2> = 2 D td[t] and
 * <x^4> = (K + 3) <x^2>^2 per direction, fitted over the directions by the 6
 * second-order and 15 fourth-order tensor elements: dt[t*21 + 0..5], [6..20].
 * rms_dki_lls (readRMS.m:80-91): log(S + eps) fitted by the 21 DKI terms
 * -b D_cnt g_i g_j and b^2/6 W_cnt g_i g_j g_k g_l (unit directions):
 * dt[t*21 + 0..20] (the reference returns the transpose, [21][T]).
 * Each least-squares solve is MATLAB's backslash: QR with column pivoting,
 * and for a rank-deficient system (the intercept form always is: a direction
 * has one more column than distinct b-values; fewer than 15 directions; one
 * b-shell) its basic solution, where MATLAB also prints a warning.  Fewer
 * than two distinct b-values is RMS_ERR_ARG (the reference indexes past X).
 *
 * rms_akc_shell (readRMS.m:105-112): D and K along ndir directions from a
 * shell fit: x2 = dt[0..5].n2, x4 = dt[6..20].n4, D = x2/(2 td), K = x4/x2^2 - 3.
 * rms_akc_lls (readRMS.m:114-117, whose DKI.akc is an external MATLAB class
 * the reference does not ship): the DKI signal model
 * ln S = -b D(n) + b^2 D(n)^2 K(n)/6 read off the LLS coefficients,
 * D(n) = sum D_cnt dt_ij n_i n_j, K(n) = sum W_cnt dt_ijkl n_i n_j n_k n_l / D(n)^2.
 * Outputs D[t*ndir + q], K[t*ndir + q]. */
int rms_dki_shell(int T, int m, const double* sig, const double* bvec, const double* bval, const double* td,
                  int intercept, double* dt);
int rms_dki_lls(int T, int m, const double* sig, const double* bvec, const double* bval, double* dt);
int rms_akc_shell(int T, const double* dt, int ndir, const double* dirs, const double* td, double* D, double* K);
int rms_akc_lls(int T, const double* dt, int ndir, const double* dirs, double* D, double* K);

/* A batch launch captured once as a CUDA graph and replayed with new seeds.
 * rms_batch_graph_create plans the SPLIT launch of rms_batch_run(sims, n,
 * opts) (uploads the tables, sizes the buffers) and captures its device work
 * -- axon table from pinned memory, accumulators cleared, the persistent walk,
 * the reduction, results to pinned memory -- on opts->stream (or the first
 * simulation's own stream); rms_graph_run(g, seed) replays it with member k's
 * seed = seed + k * 0x9E3779B97F4A7C15 (as rms_batch_run), waits, and unpacks
 * the results into the simulations (rms_sim_get as usual).  The graph refers
 * to the simulations' device buffers: it stays valid while the simulations
 * exist and no other call gives them a new lattice or larger buffers;
 * rms_graph_run checks both and returns RMS_ERR_STATE otherwise.  Destroy the
 * graph before its simulations.  No reference counterpart. */
typedef struct rms_graph rms_graph;
int rms_batch_graph_create(rms_sim* const* sims, int n, const rms_run_opts* opts, rms_graph** graph);
int rms_graph_run(rms_graph* graph, uint64_t seed);
void rms_graph_destroy(rms_graph* graph);

/* Autotuner of the SPLIT walk's launch variant for a batch (n >= 1 sims, as
 * rms_batch_run would walk them with opts): every variant walks the same
 * subset of each simulation's walkers (about four waves of the GPU), the
 * fastest walk kernel wins; *variant receives its number (pass it as
 * rms_run_opts.variant), variant_ms (optional, one per variant) the times.
 * Results are cached per device, lattice encoding, Nc, axon count and size
 * class, so later calls return at once.  The simulations' results are
 * overwritten by the tuning runs.  No reference counterpart (the reference
 * launches one fixed shape, hpc_code/lib/main.cu:499-504). */
int rms_autotune(rms_sim* const* sims, int n, const rms_run_opts* opts, int* variant, double* variant_ms);

/* Launch variants of the SPLIT walk (block size x minimum resident blocks per
 * SM).  rms_split_variant(k, ...) describes entry k >= 1; returns RMS_ERR_ARG
 * past the end.  No reference counterpart (the reference launches one fixed
 * shape, hpc_code/lib/main.cu:499-504). */
int rms_split_variant(int k, int* block, int* min_blocks_per_sm);

/* ---- Walk without allocating device memory --------------------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * call cudaMalloc: applications whose device memory is all owned by their own
 * allocator (a framework pool, a fixed pre-reserved budget), and code that
 * must not hit cudaMalloc/cudaFree because they synchronise the whole device.
 * Runs the SPLIT walk of `sim` (its configuration and tables; the sim itself is
 * not changed) on device buffers the caller owns:
 *   d_labels  [n1*n2*n3] uint8 lattice, n3 fastest, labels < nc (nc <= 7);
 *             checked on the device before the walk, as rms_sim_set_lattice
 *             checks a host lattice (RMS_ERR_RANGE: a label >= nc, or fewer
 *             than 1e-7 of the voxels labelled)
 *   d_rows    [timepoints * W] doubles, W = 32 (PGSE) or 32 + 32*ceil(nbvec/32)
 *             (narrow); row t holds sig0 at column 0, dx2 at 1-6, dx4 at 7-21,
 *             compartment counts at 22.., sigRe at 32..
 *   d_sig     [32*ceil(max(ngrad,1)/32)] doubles (PGSE; NULL for narrow)
 * on opts->stream (NULL = the default stream), and returns after the walk
 * finished.  All scratch lives in one fixed device array of
 * RMS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit; a job needing more scratch than that is refused with RMS_ERR_RANGE,
 * and large jobs run on fewer warps than rms_sim_run uses.  The first call on
 * each device looks up the array's device address: make it before any stream
 * capture.  Calls share the array, so calls that overlap on the GPU race:
 * serialise them.  No memory is allocated, host or device. */
#define RMS_NOALLOC_SCRATCH_BYTES ((size_t)128 << 20)
int rms_sim_run_noalloc(const rms_sim* sim, const rms_run_opts* opts, const uint8_t* d_labels,
                        double* d_rows, double* d_sig);

/* ---- Adjoint of the waveform-mode signal ----------------------------------
 * No counterpart in the reference.  For a RMS_MODE_WAVEFORM simulation (at
 * most 16 waveforms, Nc <= 4, one diffusivity D shared by every labelled
 * compartment) and upstream weights g_sigw[2j] = dL/dC_j, g_sigw[2j+1] =
 * dL/dS_j of the signal sums C_j = sum_w s0 cos(phase_j), S_j = sum_w s0
 * sin(phase_j) (RMS_FIELD_SIGW), computes the gradients of
 * L = sum_j g_sigw[2j] C_j + g_sigw[2j+1] S_j for the same walkers and seed
 * as rms_sim_run with opts (SPLIT precision):
 *   d_wave[nwave*nbins*3]  dL/dwave, the layout of rms_config.wave; exact
 *                          pathwise (the phase is linear in the waveform)
 *   d_t2[c]                dL/dT2_c (ms), analytic through s0
 *   d_kappa                dL/dkappa (RMS_PERM_KAPPA with kappa > 0, else
 *                          0) by forced draws: per walker with nb > 0
 *                          permeation draws, one of them (chosen uniformly)
 *                          is walked the other way with the rest of the walk
 *                          on the same streams, and nb Pij (1 - Pij)
 *                          (L[crossed] - L[reflected]) / kappa is summed (the
 *                          weak derivative of the Bernoulli draws; unbiased)
 *   d_kappa_score          the same derivative by the score function of the
 *                          draws, sum_w (L_w - mean L) sum (1[crossed] - Pij)
 *                          / kappa (unbiased, noisier where crossings are rare)
 *   d_diffusivity          dL/dD by time rescaling: a walk with D(1 + eps)
 *                          and kappa(1 + eps) over [0, T] is, in law, the
 *                          D-walk over [0, T(1 + eps)], so D dL/dD is the
 *                          derivative of the walk stretched in time (phases
 *                          through the waveform's bin edges, the T2 weight
 *                          through the final compartment) minus kappa dL/dkappa.
 *                          It includes the jumps of the walk's output at
 *                          voxel corners, mirror walls and changed permeation
 *                          draws; it is exact for the continuum process and
 *                          carries the walk's time-discretisation error
 *   d_diffusivity_pathwise dL/dD through the step length with the event
 *                          sequence fixed (plus the forced-draw term through
 *                          the kappa-mode permeation probability): low variance,
 *                          exact where the walk is continuous in the step
 *                          length (flat membranes, periodic walls), blind to
 *                          the jumps above; the T2 weight's dependence on D
 *                          through residence times is not included
 * Each walker is walked once, recording its bin displacement sums (12 bytes
 * per bin) and its state every ck steps (at most 16 checkpoints; ck a multiple
 * of 96 and of the bin length); with permeation draws each walker that made a
 * draw is walked once more from the last checkpoint before its forced draw.
 * The records go in device scratch held by the simulation (walkers in chunks
 * of at most half the free memory and 16 GiB, or RMS_ADJOINT_SCRATCH_MB
 * mebibytes when that is set and smaller); where even 65536 walkers'
 * records do not fit, or with RMS_ADJOINT_GROUPED=0 in the environment, each
 * walker is walked two or three times from its random streams instead, with
 * nothing stored (the same gradients up to the order of float sums).  d_wave
 * (caller-allocated host array) and sigw (optional, [nwave*2], the run's own
 * signal sums) may be NULL. */
typedef struct rms_adjoint_grads {
    double* d_wave;
    double d_diffusivity;
    double d_kappa;
    double d_t2[8];
    double loss;
    double* sigw;
    double d_diffusivity_pathwise;
    double d_kappa_score;
} rms_adjoint_grads;
int rms_adjoint_run(rms_sim* sim, const rms_run_opts* opts, const double* g_sigw, rms_adjoint_grads* out);

/* Jacobian of every waveform's signal sums with respect to the scalar
 * parameters, in one adjoint run (the walks of rms_adjoint_run).  No counterpart in the reference.  For waveform j and
 * signal sum s (0: C_j, 1: S_j), row q = 2j + s of jac[2*nwave*RMS_JAC_COLS]
 * holds d(sum)/d(parameter) in the columns below: the estimators of
 * rms_adjoint_run with the loss L = that sum (D by time rescaling, kappa by
 * forced draws and by the score function, T2 analytic; unused columns 0).
 * sigw (optional, [nwave*2]) receives the run's signal sums. */
#define RMS_JAC_D 0
#define RMS_JAC_KAPPA 1
#define RMS_JAC_KAPPA_SCORE 2
#define RMS_JAC_T2 3             /* + compartment c, c < Nc */
#define RMS_JAC_COLS 11
int rms_adjoint_jacobian(rms_sim* sim, const rms_run_opts* opts, double* jac, double* sigw);

/* ---- Multi-waveform phase contraction -------------------------------------
 * No counterpart in the reference (its only gradient form is the PGSE pair,
 * hpc_code/lib/main_PGSE.cu:336-346, summed per step per gradient).  For
 * walker positions sampled on time bins and many gradient waveforms:
 *   d_pos   [nwalk][nbins][3] float, um (e.g. the trajectory output of a
 *           RMS_MODE_WAVEFORM run: bin mean displacements)
 *   d_wave  [nwave][nbins][3] float, phase per um of a bin's position
 *           (gamma g times the bin's duration)
 *   d_out   [nwave][2] double: sum over walkers of cos(phi), sin(phi),
 *           phi[w][j] = sum_{b,axis} pos[w][b][axis] wave[j][b][axis]
 * All three are device buffers on the current device; the call runs on
 * `stream` and returns when the contraction has finished.  Methods:
 * RMS_CONTRACT_FP32 (FP32 products and sums on the CUDA cores) and
 * RMS_CONTRACT_BF16X3 (both operands split into BF16 hi + lo parts, three
 * tensor-core products hi.hi + hi.lo + lo.hi summed in FP32; needs
 * nbins % 4 == 0 and a 16-byte aligned d_pos).  Phases are reduced mod 2 pi in
 * FP32 before the sine and cosine; the per-waveform sums are FP64.
 * kernel_ms (optional, may be NULL) receives the kernel's device time. */
#define RMS_CONTRACT_FP32 0
#define RMS_CONTRACT_BF16X3 1
/* d_pos holds the BF16 pairs a waveform walk wrote with traj_split (hi parts
 * then lo parts); the tensor cores read them as they lie (TMA), no FP32 ->
 * BF16 conversion in the contraction.  Needs nbins % 8 == 0. */
#define RMS_CONTRACT_BF16X3_PRESPLIT 2
int rms_contract_phases(const float* d_pos, int64_t nwalk, int nbins, const float* d_wave, int nwave, int method,
                        double* d_out, void* stream, float* kernel_ms);

/* Library version string. */
const char* rms_version(void);

#ifdef __cplusplus
}
#endif
#endif

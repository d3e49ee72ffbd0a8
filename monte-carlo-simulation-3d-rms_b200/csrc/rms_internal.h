// rms_internal.h -- engine internals shared by the host library (C++) and the
// kernels (CUDA).  Not part of the C ABI (include/rms.h).
#pragma once
#include <cstddef>
#include <cstdint>

namespace rms {

constexpr int kWarp = 32;
constexpr int kNcMax = 8;          // compartments supported by the kernels
constexpr int kRowHead = 32;       // record row: [sig0, dx2 x6, dx4 x15, count x nc, pad] then signals
constexpr int kColSig0 = 0;
constexpr int kColDx2 = 1;
constexpr int kColDx4 = 7;
constexpr int kColCount = 22;      // + compartment
constexpr int kMaxTimepoints = 1 << 20;
constexpr long long kInitTryCap = 1ll << 26;   // rejection-sampling attempts per walker
constexpr int kErrInitCap = 1;                  // a walker found no labelled voxel in kInitTryCap tries
constexpr int kErrStep = 2;                     // a segment found no face (step >= 1 voxel)
constexpr int kErrTimeout = 4;                  // a bounded wait of a pipelined kernel ran out

// One simulation ("axon") of a split-precision launch.  A launch walks the
// tiles (32 walkers) of all its axons; axon k owns global tiles
// [tile_begin, tile_begin + ceil((walker_end - walker_begin) / 32)).
struct AxonDesc {
    const uint8_t* lat;         // padded, packed lattice of this axon
    int n1, n2, n3, nc;
    int s0, s1;                 // padded lattice strides: (n2+2)(n3+2), n3+2
    int64_t walker_begin, walker_end;   // walker ids (random streams) within the axon's job
    int64_t tile_begin;
    uint64_t seed;
    float res;
    int same_cross;             // same-label faces always crossed, compartment 0 never entered
    int flight;                 // free flight allowed (same_cross and nite >= 4)
    float step[kNcMax];         // step length, voxels
    float k[kNcMax];            // T2 exponent per voxel of path
    float pij[kNcMax * kNcMax]; // [a * kNcMax + b]
    float ratio[kNcMax * kNcMax];   // step[b] / step[a]
};

// Arguments of the walk kernels (passed by value; pointers are device memory).
struct WalkArgs {
    const uint8_t* labels;      // [n1*n2*n3], n3 fastest
    int n1, n2, n3;
    int64_t walker_begin, walker_end;
    int tn, tstep, timepoints, nite, nc, boundary, mode;
    double res, dt;
    uint64_t seed;
    const double* step;         // [nc] voxels
    const double* t2;           // [nc] steps
    const double* pij;          // [nc*nc]
    int nvals;                  // doubles per record row, multiple of 32
    double* slots;              // [nslots][timepoints][nvals]
    // narrow pulse
    int nbvec;
    const double* qtab;         // [timepoints][nbvec] = sqrt(bval/TD)
    const double* bvec;         // [nbvec*3]
    // PGSE
    int ngrad, ngrad_pad, npairs, nevents;
    const int* ev_step;         // [nevents], ascending: P(ev_step) enters pair ev_pair
    const int* ev_pair;
    const double* ev_coef;      // +1 or -1
    const double* grad;         // [ngrad*6]
    const int* gpair;           // [ngrad] timing pair of each gradient
    double* vscr;               // [npairs*3][nthreads] per-thread window sums
    double* sig_slots;          // [nslots][ngrad_pad]
    // split precision (FP32 arithmetic): per-compartment FP32 tables
    const float* stepf;         // [nc]
    const float* t2invf;        // [nc] 1 / (T2 in steps)
    const float* pijf;          // [nc*nc]
    int* err;                   // device error word (kErr* bits), zeroed per run
    unsigned long long* tile_ctr;   // table-form launches: next tile to hand out, zeroed per run
    int table_form;             // walk even one axon from the axon table (what a graph replay rewrites)
    // split launches: the axons and their tiles; with several axons each warp
    // adds its rows into out_rows[axon][timepoints][nvals] / out_sig[axon][ngrad_pad]
    const AxonDesc* axons;
    int naxons;
    int64_t ntiles;
    double* out_rows;
    double* out_sig;
    // general waveforms: phase per um of a bin's displacement sum (waveform x
    // dt), [bin][waveform][axis]; optional per-walker bin means out,
    // [walker - walker_begin][bin][axis] in um
    int nwave, nbins, bin_steps;
    int rule;                   // membrane rule: 0 reflect, 1 reject (stay), 2 leap (redraw)
    const double* wave;
    float* traj;
    int traj_split;             // traj holds BF16 hi parts, then lo parts (per walker, bin, axis)
    int64_t traj_n;             // walkers in the trajectory buffer
    AxonDesc axon0;             // the first axon, by value (read from kernel parameters)
    // traces (COMPAT)
    int64_t trace_n;
    int32_t* tr_init;
    int32_t* tr_vox;
    uint32_t* tr_ev;
    double* tr_pos;             // [trace_n*tn*3] position after each step (voxels)
};

// Launchers (rms_walk_*.cu, rms_reduce.cu).  All asynchronous on `stream`;
// they return a cudaError_t value (0 = success).
int launch_walk_compat(const WalkArgs& a, int grid, int block, bool trace, void* stream);
// Split walk over a.naxons axons (a.axons, a.ntiles, per-warp a.slots, and
// a.out_rows/out_sig for several axons); lattice_bits: packed lattice format.
int launch_walk_split(const WalkArgs& a, int lattice_bits, int variant, int grid, void* stream);
int split_variant_count();
bool split_variant_walks(int variant, int mode, int rule);   // variants past the first: narrow/PGSE, reflecting
int split_variant_block(int variant);   // threads per block of a launch variant
int split_variant_minb(int variant);    // its minimum resident blocks per SM
// The split walk's lattice: (n1+2) x (n2+2) x (n3+2) with a wall-code border;
// 4 bits per voxel (3-bit label + free-flight flag) when Nc <= 7 (every split
// walk, the no-allocation one included), else one byte.
int split_lattice_bits(int nc);
size_t padded_lattice_bytes(int n1, int n2, int n3, int bits);
// mirror: flag voxels at the lattice's faces too (mirror walls; see pad_pack_kernel)
int pack_lattice_padded(const uint8_t* labels, int n1, int n2, int n3, int bits, int mirror, uint8_t* out,
                        void* stream);
int launch_reduce_slots(const double* slots, int nslots, size_t row, double* out, void* stream);
// Resident blocks per SM of the walk kernels (occupancy API); -1 on error.
int walk_compat_blocks_per_sm(int nc, bool trace);
int walk_split_blocks_per_sm(int nc, int lattice_bits, int variant);
const char* cuda_error_string(int code);

// A tube lattice on the device (rms_geometry.cu).
int build_tube_lattice(uint8_t* d_out, int n1, int n2, int n3, double res, const double* d_r2, const double* d_cx,
                       const double* d_cy, uint8_t inside, uint8_t outside, void* stream);
// A lattice in device memory checked on the GPU: d_counts[0] += voxels with a
// label >= nc, d_counts[1] += labelled voxels (the caller zeroes d_counts).
int check_labels(const uint8_t* d_labels, size_t n, unsigned nc, unsigned long long* d_counts, int sms,
                 void* stream);

// Adjoint of the waveform-mode split walk (rms_adjoint.cu): one axon, labels
// below kAdjNc, at most kAdjWaves waveforms.
constexpr int kAdjWaves = 16;
constexpr int kAdjNc = 4;
// sums[]: sum_w L_w, sum_w L_w E_w, sum_w sum_j a_jw dphi_jw, sum_w L_w t_wc
// (steps, per compartment), sum_w E_w, the signal sums (cos, sin) per
// waveform, then sum_w dL_w/deps of the time rescaling (rms_adjoint.cu)
constexpr int kAdjSumL = 0, kAdjSumLE = 1, kAdjSumPath = 2, kAdjSumLT = 3, kAdjSumE = 3 + kAdjNc,
              kAdjSumSig = 4 + kAdjNc, kAdjSumTR = kAdjSumSig + 2 * kAdjWaves, kAdjSumForce = kAdjSumTR + 1;
constexpr int kAdjSums = kAdjSumForce + 1;
// Jacobian sums (rms_adjoint_jacobian), after the kAdjSums: for waveform j and
// signal sum s (0: C_j = sum s0 cos phi_j, 1: S_j = sum s0 sin phi_j), q = 2j + s:
//   kJacE + q           sum_w X_qw E_w (score of the permeation draws)
//   kJacTR + q          sum_w dX_qw/deps (time rescaling)
//   kJacF + q           sum_w nb_w Pij (1 - Pij) (X_qw[crossed] - X_qw[reflected]) (forced draws)
//   kJacLT + q*NC + c   sum_w X_qw t_wc / step_c (residence in compartment c, steps)
constexpr int kJacE = 0, kJacTR = 2 * kAdjWaves, kJacF = 4 * kAdjWaves, kJacLT = 6 * kAdjWaves;
constexpr int kJacSums = kJacLT + 2 * kAdjWaves * kAdjNc;
struct AdjArgs {
    const uint8_t* lat;          // padded 4-bit lattice with free-flight flags
    int n1, n2, n3, s0, s1;
    int64_t walker_begin, walker_end, ntiles;
    uint64_t seed;
    int tn, nbins, bin_steps, nwave, nite, boundary;
    float res;
    int flight, same_cross;
    int force;                   // a third pass: one permeation decision per walker forced the other way
    float step[kAdjNc], kexp[kAdjNc], pij[kAdjNc * kAdjNc], ratio[kAdjNc * kAdjNc];
    const double* wave;          // [bin][waveform][axis], x dt
    const float4* wq;            // [bin][waveform][2]: (g_b - g_b+1, 0), (g_b res, 0) as floats (g_nbins = 0)
    const float* gup;            // [waveform][2]: dL/d(sum cos), dL/d(sum sin)
    double* sums;                // [kAdjSums]
    // pass 1 alone, then the forced walks grouped (adjoint_kernel FORM 1 and
    // 2): checkpoint every ck_every steps (nbk resume steps b * ck_every); per
    // walker of the launch (nwalk): its states at checkpoints 1..nbk-1,
    // ck[checkpoint - 1][word][walker]; its summary ws[word][walker]; bucket
    // lists blist[b][nwalk] with counts bcount[b]; weighted form: the bin
    // displacement sums xbin[bin][axis][walker] (um) and a_jw, ajw[j][walker]
    int ck_every, nbk;
    int64_t nwalk;
    uint32_t* ck;
    uint32_t* ws;
    int* blist;
    int* bcount;
    float* xbin;
    float* ajw;
    float* dwave;                // [bin][waveform][axis]: sum_w a_jw X_wb (um)
    int* err;
};
// form 0: all passes in one launch; 1: pass 1 with checkpoints, X_wb, a_jw
// and the buckets of the forced walks; 2: the forced walks, grouped by resume
// step.  launch_adjoint_dwave: dL/dwave from form 1's X_wb and a_jw.
constexpr int kAdjCkWords = 23 + kAdjWaves, kAdjWsWords = 3 + kAdjWaves, kAdjCkMax = 16;
int launch_adjoint(const AdjArgs& a, bool jac, int form, int grid, void* stream);
int launch_adjoint_dwave(const AdjArgs& a, int sms, void* stream);
int adjoint_blocks_per_sm(bool jac, int form);
constexpr int kAdjBlock = 128;

// Multi-waveform phase contraction (rms_contract.cu): out[j] = (sum_w cos phi,
// sum_w sin phi), phi[w][j] = sum_k pos[w][k] wave[j][k], K = 3 nbins.
// method RMS_CONTRACT_FP32 or RMS_CONTRACT_BF16X3.  Returns an RMS_* status;
// msg gets a reason on failure.
int contract_phases(const float* d_pos, int64_t nwalk, int nbins, const float* d_wave, int nwave, int method,
                    double* d_out, void* stream, const char** msg, float* kernel_ms);

}  // namespace rms

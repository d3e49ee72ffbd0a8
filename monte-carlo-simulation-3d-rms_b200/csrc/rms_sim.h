// rms_sim.h -- the library's simulation object (host side, C++).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rms.h"

struct rms_device_state;  // rms_api.cpp

struct rms_sim {
    // configuration, owned copies (what hpc_code/lib/main.cu:414-482 reads)
    int mode = RMS_MODE_NARROW;
    double dt = 0.0;
    int tn = 0;
    int64_t npar = 0;
    int nc = 0;
    double res = 0.0;
    int n1 = 0, n2 = 0, n3 = 0;
    std::vector<double> diffusivity, t2, bval, bvec, grad, pij_in, wave;
    int nwave = 0, nbins = 0;
    int timepoints = 1000, nite = 4, boundary = RMS_BOUNDARY_MIRROR,
        permeation = RMS_PERM_REFERENCE;
    double kappa = 0.0;
    int rule = 0;              // RMS_RULE_*

    // derived tables (main.cu:433-458, 484-487)
    int tstep = 1;
    std::vector<double> step;       // [nc] voxels
    std::vector<double> t2_steps;   // [nc] T2 / dt
    std::vector<double> pij;        // [nc*nc]
    std::vector<double> td;         // [timepoints]
    std::vector<double> qtab;       // [timepoints*nbvec] sqrt(bval/TD)

    // PGSE lobe schedule: per gradient its timing pair; per pair the steps at
    // which the running displacement sum enters the pair's window sum
    int npairs = 0;
    std::vector<int> gpair;          // [ngrad]
    std::vector<int> ev_step, ev_pair;
    std::vector<double> ev_coef;

    // lattice
    std::vector<uint8_t> labels;
    bool have_lattice = false;
    bool lattice_dirty = true;
    bool host_stale = false;   // the device holds a newer lattice than `labels`

    // device resources (lazily created)
    rms_device_state* dev = nullptr;

    // results of the last run
    bool have_results = false;
    bool have_timing = false;   // walk_ms / run_ms hold a run's or an adjoint's times
    std::vector<double> sig0, dx2, dx4, sigre, sig, sigw, npar_count;
    int64_t trace_n = 0;
    std::vector<int32_t> tr_init, tr_vox;
    std::vector<uint32_t> tr_ev;
    std::vector<double> tr_pos;
    double walk_ms = 0.0, run_ms = 0.0;
    int last_grid = 0, last_block = 0;

    int nbvec() const { return (int)bval.size(); }
    int ngrad() const { return (int)(grad.size() / 6); }
};

namespace rms {
struct AxonDesc;
// describe one simulation as an axon of a split launch (rms_internal.h)
void fill_axon_desc(AxonDesc& x, const rms_sim* s, int64_t w0, int64_t w1, int64_t tile_begin, uint64_t seed,
                    const uint8_t* lat);
// walkers [w0, w1) a call asks of s: its walker range, its shard, or all
// (only a shard can be empty); batch_range ignores the walker range
int walker_range(const rms_sim* s, const rms_run_opts* o, int64_t& w0, int64_t& w1);
int batch_range(const rms_sim* s, const rms_run_opts* o, int64_t& w0, int64_t& w1);
// zero results of a simulation that walked no walkers (an empty shard)
void zero_results(rms_sim* s);
// error reporting (thread-local message behind rms_last_error)
int set_error(int code, const std::string& msg);
// derive tables and validate a filled-in configuration
int finalize_config(rms_sim* s);
// text formats of the reference (rms_io.cpp)
int load_run_dir(const char* dir, int mode, rms_sim* s);
int write_run_dir(const rms_sim* s, const char* dir);
int parse_lattice_text(const std::string& path, size_t n, std::vector<uint8_t>& out, int nc);
}  // namespace rms

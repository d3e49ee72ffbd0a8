// rms_api.cpp -- the C ABI of include/rms.h: configuration, derived tables,
// device resources, launch and result unpacking.
//
// Host-side counterpart of the reference's main() (hpc_code/lib/main.cu:388-621,
// main_PGSE.cu:414-675): it derives the same tables, then runs the walk
// kernels (rms_walk_*.cu) and the ordered reduction (rms_reduce.cu) instead of
// `propagate` with FP64 CAS atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <tuple>

#include "philox.cuh"
#include "rms_internal.h"
#include "rms_sim.h"

namespace {
thread_local std::string g_last_error;

constexpr int kCompatBlock = 128;
constexpr int kSplitVariantDefault = 0;   // 256 threads, >= 4 blocks per SM (64 registers): fastest measured
constexpr int kMaxGrad = 1 << 16;
constexpr uint64_t kBatchSeedStep = 0x9E3779B97F4A7C15ull;   // seed of batch member k: seed + k * this

// One device allocation that only grows.
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

struct HostPinned {
    void* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMallocHost(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};
}  // namespace

struct rms_device_state {
    int device = -1;
    cudaStream_t own = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    DevBuf labels, packed, axons, wavef, tables, tablesf, slots, sig_slots, vscr, qtab, bvec, grad, gpair, ev_step,
        ev_pair, ev_coef, out, out_sig, err, tr_init, tr_vox, tr_ev, tr_pos, adj_g, adj_sums, adj_dwave, adj_ck, adj_ws, adj_blist, adj_bcount, adj_xbin, adj_ajw, adj_wq,
        stage, counts;
    HostPinned h_out, h_axons;
    size_t labels_bytes = 0;
    bool packed_valid = false;
    int packed_bits = 0;       // cell width of the packed lattice (4 or 8)

    ~rms_device_state() {
        if (device >= 0) cudaSetDevice(device);
        for (DevBuf* b : {&labels, &packed, &axons, &wavef, &tables, &tablesf, &slots, &sig_slots, &vscr, &qtab, &bvec, &grad,
                          &gpair, &ev_step, &ev_pair, &ev_coef, &out, &out_sig, &err, &tr_init,
                          &tr_vox, &tr_ev, &tr_pos, &adj_g, &adj_sums, &adj_dwave, &adj_ck, &adj_ws, &adj_blist,
                          &adj_bcount, &adj_xbin, &adj_ajw, &adj_wq, &stage, &counts})
            b->release();
        h_out.release();
        h_axons.release();
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (e2) cudaEventDestroy(e2);
        if (own) cudaStreamDestroy(own);
    }
};

namespace rms {

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

namespace {

int cuda_fail(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return set_error(RMS_ERR_CUDA, m);
}

#define RMS_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Number of steps i in [0, tn) whose end time (i+1)*dt lies below x; the same
// double comparison as main_PGSE.cu:341-343, found by bisection (monotone in i).
int count_below(double x, int tn, double dt) {
    int lo = 0, hi = tn;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (static_cast<double>(mid + 1) * dt < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// PGSE lobes as step windows (main_PGSE.cu:340-346): lobe 1 is the steps with
// t < delta; lobe 2 the remaining steps with Delta <= t < Delta + delta.
// With P(n) = sum of the first n displacements, a gradient's phase is
// |g| dt g_hat . (P(n1) + P(a) - P(b)), lobe 2 = [a, b).  Gradients sharing
// (n1, a, b) share one window sum ("timing pair").
void build_pgse_schedule(rms_sim* s) {
    std::map<std::tuple<int, int, int>, int> pairs;
    s->gpair.assign(s->ngrad(), 0);
    std::vector<std::tuple<int, int, int>> keys;
    for (int j = 0; j < s->ngrad(); ++j) {
        const double Del = s->grad[6 * j + 0], del = s->grad[6 * j + 1];
        const int n1 = count_below(del, s->tn, s->dt);
        const int n2 = count_below(Del, s->tn, s->dt);
        const int n3 = count_below(Del + del, s->tn, s->dt);
        const int a = std::max(n1, n2);
        const int b = std::max(a, n3);
        auto key = std::make_tuple(n1, a, b);
        auto it = pairs.find(key);
        if (it == pairs.end()) {
            it = pairs.emplace(key, (int)keys.size()).first;
            keys.push_back(key);
        }
        s->gpair[j] = it->second;
    }
    s->npairs = (int)keys.size();
    struct Ev { int step, pair; double coef; };
    std::vector<Ev> evs;
    for (int p = 0; p < s->npairs; ++p) {
        const int n1 = std::get<0>(keys[p]), a = std::get<1>(keys[p]), b = std::get<2>(keys[p]);
        if (n1 > 0) evs.push_back({n1, p, 1.0});
        if (a != b) {
            if (a > 0) evs.push_back({a, p, 1.0});
            evs.push_back({b, p, -1.0});
        }
    }
    std::stable_sort(evs.begin(), evs.end(), [](const Ev& x, const Ev& y) { return x.step < y.step; });
    s->ev_step.clear(); s->ev_pair.clear(); s->ev_coef.clear();
    for (const Ev& e : evs) {
        s->ev_step.push_back(e.step);
        s->ev_pair.push_back(e.pair);
        s->ev_coef.push_back(e.coef);
    }
}

}  // namespace

// Walkers [w0, w1) of simulation s that a call asks for: an explicit range
// (walker_begin/walker_end), shard shard_index of shard_count, or all of them.
// Only a shard may be empty (a job with fewer walkers than shards).
int walker_range(const rms_sim* s, const rms_run_opts* o, int64_t& w0, int64_t& w1) {
    w0 = o ? o->walker_begin : 0;
    w1 = o ? o->walker_end : 0;
    const int nsh = o ? o->shard_count : 0;
    if (nsh > 1) {
        if (w0 != 0 || w1 != 0) return set_error(RMS_ERR_ARG, "give a walker range or a shard, not both");
        const int r = o->shard_index;
        if (r < 0 || r >= nsh) return set_error(RMS_ERR_ARG, "shard_index outside [0, shard_count)");
        w0 = (int64_t)((__int128)s->npar * r / nsh);
        w1 = (int64_t)((__int128)s->npar * (r + 1) / nsh);
        return RMS_OK;
    }
    if (nsh < 0 || (o && (o->shard_index < 0 || (nsh <= 1 && o->shard_index > 0))))
        return set_error(RMS_ERR_ARG, "shard_index outside [0, shard_count)");
    if (w0 == 0 && w1 == 0) w1 = s->npar;
    if (w0 < 0 || w1 > s->npar || w0 >= w1) return set_error(RMS_ERR_ARG, "walker range outside [0, NPar)");
    return RMS_OK;
}

// Results of a simulation that walked no walkers (an empty shard): zeros in
// the shapes a run leaves.
void zero_results(rms_sim* s) {
    const int T = s->timepoints, nb = s->nbvec();
    s->sig0.assign(T, 0.0);
    s->dx2.assign((size_t)T * 6, 0.0);
    s->dx4.assign((size_t)T * 15, 0.0);
    s->npar_count.assign((size_t)T * s->nc, 0.0);
    s->sigre.assign((size_t)T * nb, 0.0);
    s->sig.assign(s->mode == RMS_MODE_PGSE ? s->ngrad() : 0, 0.0);
    s->sigw.assign(s->mode == RMS_MODE_WAVEFORM ? 2 * s->nwave : 0, 0.0);
    s->trace_n = 0;
    s->walk_ms = s->run_ms = 0.0;
    s->have_results = true;
    s->have_timing = true;
}

// The walkers a batch call walks in simulation s: all of them, or the call's
// shard (a batch ignores walker_begin/walker_end).
int batch_range(const rms_sim* s, const rms_run_opts* o, int64_t& w0, int64_t& w1) {
    rms_run_opts x = o ? *o : rms_run_opts{};
    x.walker_begin = x.walker_end = 0;
    return walker_range(s, &x, w0, w1);
}

void fill_axon_desc(AxonDesc& x, const rms_sim* s, int64_t w0, int64_t w1, int64_t tile_begin, uint64_t seed,
                    const uint8_t* lat) {
    std::memset(&x, 0, sizeof x);
    x.lat = lat;
    x.n1 = s->n1; x.n2 = s->n2; x.n3 = s->n3; x.nc = s->nc;
    x.s1 = s->n3 + 2;
    x.s0 = (s->n2 + 2) * (s->n3 + 2);
    x.walker_begin = w0; x.walker_end = w1;
    x.tile_begin = tile_begin;
    x.seed = seed;
    x.res = (float)s->res;
    bool same = true;
    for (int c = 0; c < s->nc; ++c) {
        x.step[c] = (float)s->step[c];
        x.k[c] = s->step[c] > 0.0 ? (float)(1.0 / (s->step[c] * s->t2_steps[c])) : 0.0f;
        for (int e = 0; e < s->nc; ++e) {
            x.pij[c * kNcMax + e] = (float)s->pij[(size_t)c * s->nc + e];
            x.ratio[c * kNcMax + e] = s->step[c] > 0.0 ? (float)(s->step[e] / s->step[c]) : 0.0f;
        }
        if (c >= 1) same = same && s->pij[(size_t)c * s->nc + c] > 0.999999 && s->pij[(size_t)c * s->nc] < 0.000001;
    }
    x.same_cross = same ? 1 : 0;
    x.flight = (same && s->nite >= 4) ? 1 : 0;
}

int finalize_config(rms_sim* s) {
    std::ostringstream m;
    if (s->mode != RMS_MODE_NARROW && s->mode != RMS_MODE_PGSE && s->mode != RMS_MODE_WAVEFORM)
        return set_error(RMS_ERR_ARG, "mode");
    if (s->rule < RMS_RULE_REFLECT || s->rule > RMS_RULE_LEAP) return set_error(RMS_ERR_ARG, "membrane rule");
    if (!(s->dt > 0.0) || !std::isfinite(s->dt)) return set_error(RMS_ERR_RANGE, "dt must be > 0");
    if (s->tn < 1) return set_error(RMS_ERR_RANGE, "TN must be >= 1");
    if (s->npar < 1 || s->npar > (int64_t)1 << 40) return set_error(RMS_ERR_RANGE, "NPar out of range");
    if (s->nc < 1 || s->nc > kNcMax) {
        m << "Nc = " << s->nc << " outside [1, " << kNcMax << "]";
        return set_error(RMS_ERR_RANGE, m.str());
    }
    if (!(s->res > 0.0)) return set_error(RMS_ERR_RANGE, "voxel size must be > 0");
    if (s->n1 < 1 || s->n2 < 1 || s->n3 < 1) return set_error(RMS_ERR_RANGE, "lattice size must be >= 1");
    if ((double)s->n1 * s->n2 * s->n3 >= 2147483648.0 ||
        ((double)s->n1 + 2) * ((double)s->n2 + 2) * ((double)s->n3 + 2) >= 4294967296.0)
        return set_error(RMS_ERR_RANGE, "lattice larger than 2^31 voxels");
    if ((int)s->diffusivity.size() != s->nc || (int)s->t2.size() != s->nc)
        return set_error(RMS_ERR_ARG, "diffusivity and T2 need Nc values");
    if (s->timepoints == 0) s->timepoints = 1000;
    if (s->nite == 0) s->nite = 4;
    if (s->timepoints < 1 || s->timepoints > kMaxTimepoints)
        return set_error(RMS_ERR_RANGE, "timepoints out of range");
    if (s->tn < s->timepoints) {
        m << "TN = " << s->tn << " is below the " << s->timepoints
          << " recorded timepoints (the reference divides by TN/timepoints)";
        return set_error(RMS_ERR_RANGE, m.str());
    }
    if (s->nite < 1 || s->nite > 7) return set_error(RMS_ERR_RANGE, "nite must be in [1, 7]");
    if (s->boundary != RMS_BOUNDARY_MIRROR && s->boundary != RMS_BOUNDARY_PERIODIC)
        return set_error(RMS_ERR_ARG, "boundary");
    if (s->permeation < RMS_PERM_REFERENCE || s->permeation > RMS_PERM_TABLE)
        return set_error(RMS_ERR_ARG, "permeation");
    if ((int)s->bvec.size() != 3 * s->nbvec()) return set_error(RMS_ERR_ARG, "bvec needs 3 values per b-value");
    if (s->mode == RMS_MODE_PGSE && s->ngrad() > kMaxGrad) return set_error(RMS_ERR_RANGE, "Ngrad too large");
    if (s->grad.size() % 6) return set_error(RMS_ERR_ARG, "grad needs 6 values per gradient");
    if (s->mode == RMS_MODE_WAVEFORM) {
        if (s->nbins < 1 || s->tn % s->nbins) return set_error(RMS_ERR_RANGE, "waveforms need TN to be a multiple of nbins >= 1");
        if (s->nwave < 1 || s->nwave > kMaxGrad) return set_error(RMS_ERR_RANGE, "nwave out of range");
        if (s->wave.size() != (size_t)s->nwave * s->nbins * 3) return set_error(RMS_ERR_ARG, "wave needs nwave*nbins*3 values");
        for (double x : s->wave)
            if (!std::isfinite(x)) return set_error(RMS_ERR_RANGE, "waveform values must be finite");
    }

    const int nc = s->nc;
    s->tstep = s->tn / s->timepoints;                       // main.cu:68
    s->step.assign(nc, 0.0);
    s->t2_steps.assign(nc, 0.0);
    for (int i = 0; i < nc; i++) {
        const double D = s->diffusivity[i];
        if (!(D >= 0.0) || !std::isfinite(D)) return set_error(RMS_ERR_RANGE, "diffusivity must be >= 0");
        if (!(s->t2[i] > 0.0)) return set_error(RMS_ERR_RANGE, "T2 must be > 0 (T2 = 0 gives 0/0)");
        s->t2_steps[i] = s->t2[i] / s->dt;                   // main.cu:433
        s->step[i] = std::sqrt(6.0 * s->dt * D) / s->res;    // main.cu:440
        if (i > 0 && !(s->step[i] < 1.0)) {
            m << "step length of compartment " << i << " is " << s->step[i]
              << " voxels; it must be below one voxel (cf. analysis/setupRMS.m:65-68)";
            return set_error(RMS_ERR_RANGE, m.str());
        }
    }
    s->pij.assign((size_t)nc * nc, 0.0);
    for (int i = 0; i < nc; i++) {
        for (int j = 0; j < nc; j++) {
            double p;
            if (s->permeation == RMS_PERM_TABLE) {
                if ((int)s->pij_in.size() != nc * nc) return set_error(RMS_ERR_ARG, "pij table needs Nc*Nc values");
                p = s->pij_in[(size_t)i * nc + j];
                if (!(p >= 0.0 && p <= 1.0)) return set_error(RMS_ERR_RANGE, "pij values must be in [0, 1]");
            } else if (i == 0 || j == 0) {                   // main.cu:448-454
                p = 0.0;
            } else if (i == j) {
                p = 1.0;
            } else if (s->permeation == RMS_PERM_REFERENCE) {
                p = std::fmin(1.0, std::sqrt(s->diffusivity[j] / s->diffusivity[i]));
            } else {
                // analysis/interaction.m:437-439 (3-D): P = 2/3 kappa ds / D0, P/(1+P)
                if (!(s->kappa >= 0.0)) return set_error(RMS_ERR_RANGE, "kappa must be >= 0");
                const double D = s->diffusivity[i];
                const double ds = std::sqrt(6.0 * D * s->dt);
                double P = D > 0.0 ? 2.0 / 3.0 * s->kappa * ds / D : 0.0;
                p = P / (1.0 + P);
            }
            s->pij[(size_t)i * nc + j] = p;
        }
    }
    const int T = s->timepoints;
    s->td.resize(T);
    for (int i = 0; i < T; i++) s->td[i] = (i * s->tstep + 1) * s->dt;   // main.cu:485-487
    const int nb = s->nbvec();
    s->qtab.assign((size_t)T * nb, 0.0);
    for (int t = 0; t < T; ++t)
        for (int j = 0; j < nb; ++j) s->qtab[(size_t)t * nb + j] = std::sqrt(s->bval[j] / s->td[t]);  // main.cu:375
    if (s->mode == RMS_MODE_PGSE) build_pgse_schedule(s);
    else { s->npairs = 0; s->gpair.clear(); s->ev_step.clear(); s->ev_pair.clear(); s->ev_coef.clear(); }
    return RMS_OK;
}

namespace {

// Run fn(begin, end) over [0, n) split across host threads: one range below
// 32 MB, at most 8 ranges (the lattice scans and copies are memory-bound).
template <class F>
void host_parallel(size_t n, F fn) {
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::min<size_t>({8, hw, std::max<size_t>(1, n >> 25)});
    if (parts <= 1) {
        fn(size_t(0), n, 0);
        return;
    }
    std::vector<std::thread> pool;
    const size_t chunk = (n + parts - 1) / parts;
    for (size_t p = 1; p < parts; ++p)
        pool.emplace_back(fn, std::min(n, p * chunk), std::min(n, (p + 1) * chunk), (int)p);
    fn(size_t(0), std::min(n, chunk), 0);
    for (std::thread& t : pool) t.join();
}

// Check a lattice: every label below Nc, enough labelled voxels.  The scan is
// branch-free per voxel (largest label and labelled count in 255-voxel blocks
// of 8-bit counters), so it vectorises and runs at memory speed on lattices
// of gigabytes; only on an error is the lattice scanned again, for the first
// offending voxel.
int validate_lattice(const uint8_t* labels, size_t n, int nc) {
    size_t part_nonzero[8] = {0};
    uint8_t part_top[8] = {0};
    host_parallel(n, [&](size_t lo, size_t hi, int part) {
        size_t nonzero = 0;
        uint8_t top = 0;
        for (size_t b = lo; b < hi; b += 255) {
            const size_t e = std::min(hi, b + 255);
            uint8_t mx = 0, cnt = 0;
            for (size_t i = b; i < e; ++i) {
                const uint8_t v = labels[i];
                mx = v > mx ? v : mx;
                cnt += (uint8_t)(v != 0);
            }
            top = mx > top ? mx : top;
            nonzero += cnt;
        }
        part_nonzero[part] = nonzero;
        part_top[part] = top;
    });
    size_t nonzero = 0;
    uint8_t top = 0;
    for (int k = 0; k < 8; ++k) {
        nonzero += part_nonzero[k];
        top = std::max(top, part_top[k]);
    }
    if (top >= nc) {
        size_t i = 0;
        while (labels[i] < nc) ++i;
        std::ostringstream m;
        m << "label " << (int)labels[i] << " at voxel " << i << " is not below Nc = " << nc;
        return set_error(RMS_ERR_RANGE, m.str());
    }
    if (nonzero == 0) return set_error(RMS_ERR_RANGE, "lattice has no voxel with a non-zero label");
    if ((double)nonzero / (double)n < 1e-7)
        return set_error(RMS_ERR_RANGE, "labelled voxels are below 1e-7 of the lattice; "
                                        "rejection-sampled initial positions would not finish");
    return RMS_OK;
}

// The device holds the simulation's current lattice and the host copy is
// older (rms_sim_set_lattice checked and kept a lattice on the device only):
// copy it back, for a path that walks from the host copy.
int sync_host_labels(rms_sim* s) {
    if (!s->host_stale) return RMS_OK;
    rms_device_state* d = s->dev;
    const size_t n = (size_t)s->n1 * s->n2 * s->n3;
    s->labels.resize(n);
    RMS_CUDA(cudaSetDevice(d->device));
    RMS_CUDA(cudaMemcpyAsync(s->labels.data(), d->labels.p, n, cudaMemcpyDeviceToHost, d->own));
    RMS_CUDA(cudaStreamSynchronize(d->own));
    s->host_stale = false;
    return RMS_OK;
}

int ensure_device(rms_sim* s, int device) {
    if (s->dev && s->dev->device == device) return RMS_OK;
    int rc = sync_host_labels(s);
    if (rc) return rc;
    delete s->dev;
    s->dev = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return set_error(RMS_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= count) return set_error(RMS_ERR_ARG, "device ordinal out of range");
    RMS_CUDA(cudaSetDevice(device));
    auto* d = new rms_device_state();
    d->device = device;
    e = cudaStreamCreateWithFlags(&d->own, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&d->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&d->e1);
    if (e == cudaSuccess) e = cudaEventCreate(&d->e2);
    if (e != cudaSuccess) { delete d; return cuda_fail(e, "stream/event creation"); }
    s->dev = d;
    s->lattice_dirty = true;
    return RMS_OK;
}

template <class T>
cudaError_t upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
    const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
    cudaError_t e = b.ensure(bytes);
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

// One simulation of a launch: its walker range and seed.
struct LaunchJob {
    rms_sim* s;
    int64_t w0, w1;
    uint64_t seed;
};

// Upload a simulation's lattice (when changed) and, for the split walk, its
// padded packed copy; both live in the simulation's own device state.
int prepare_lattice(rms_sim* s, cudaStream_t st, bool split, int bits) {
    rms_device_state* d = s->dev;
    if (s->lattice_dirty || d->labels_bytes != s->labels.size()) {
        if (s->host_stale) return set_error(RMS_ERR_STATE, "the simulation's lattice is on a device it no longer holds");
        RMS_CUDA(d->labels.ensure(s->labels.size()));
        RMS_CUDA(cudaMemcpyAsync(d->labels.p, s->labels.data(), s->labels.size(), cudaMemcpyHostToDevice, st));
        d->labels_bytes = s->labels.size();
        d->packed_valid = false;
        s->lattice_dirty = false;
    }
    // packed again when the launch needs another cell width (a batch's widest
    // Nc decides it for all its members)
    if (split && (!d->packed_valid || d->packed_bits != bits)) {
        RMS_CUDA(d->packed.ensure(padded_lattice_bytes(s->n1, s->n2, s->n3, bits)));
        int pe = pack_lattice_padded(d->labels.as<uint8_t>(), s->n1, s->n2, s->n3, bits,
                                     s->boundary == RMS_BOUNDARY_MIRROR ? 1 : 0, d->packed.as<uint8_t>(), st);
        if (pe) return cuda_fail((cudaError_t)pe, "label packing");
        d->packed_valid = true;
        d->packed_bits = bits;
    }
    return RMS_OK;
}

// Settings every simulation of one split launch must share (the signal
// tables and the record schedule are the launch's).
bool same_schedule(const rms_sim* a, const rms_sim* b) {
    return a->mode == b->mode && a->tn == b->tn && a->dt == b->dt && a->timepoints == b->timepoints &&
           a->tstep == b->tstep && a->nite == b->nite && a->boundary == b->boundary && a->bval == b->bval &&
           a->bvec == b->bvec && a->grad == b->grad && a->nbins == b->nbins && a->wave == b->wave &&
           a->rule == b->rule;
}

// One launch, in three parts: plan (validate, shape, allocate, upload the
// tables), enqueue (device work only: accumulators cleared, axon table, walk,
// reduction, results to pinned host memory -- what a CUDA graph captures),
// finish (wait, check the error word, unpack into the simulations).
struct LaunchPlan {
    WalkArgs a{};
    rms_device_state* d = nullptr;
    cudaStream_t st = nullptr;
    int prec = 0, grid = 0, block = 0, variant = 0, bits = 8, naxons = 0, T = 0, nb = 0, ngrad = 0,
        ngrad_pad = 0, nvals = 0, nseg = 0;
    size_t row = 0, nrow = 0, nsig = 0;
    bool multi = false, has_sig = false, wavemode = false;
    int64_t trace_n = 0;
    std::vector<AxonDesc> axons;
};

// Run one launch: COMPAT (one simulation) or SPLIT (one or more simulations,
// "axons", walked by one persistent grid).  The first job's simulation owns
// the launch's accumulators.
int plan_launch(std::vector<LaunchJob>& jobs, const rms_run_opts* o, LaunchPlan& p) {
    rms_sim* s = jobs[0].s;
    const int prec = o ? o->precision : RMS_PREC_COMPAT;
    if (prec != RMS_PREC_COMPAT && prec != RMS_PREC_SPLIT) return set_error(RMS_ERR_ARG, "precision");
    if (prec == RMS_PREC_COMPAT && jobs.size() != 1) return set_error(RMS_ERR_ARG, "a COMPAT launch walks one simulation");
    if (prec == RMS_PREC_COMPAT && s->mode == RMS_MODE_WAVEFORM)
        return set_error(RMS_ERR_ARG, "general waveforms are walked by the SPLIT walk");
    if (prec == RMS_PREC_COMPAT && s->rule != RMS_RULE_REFLECT)
        return set_error(RMS_ERR_ARG, "the COMPAT walk reflects at membranes (the reference's rule); other rules walk SPLIT");
    float* traj = o ? o->traj_out : nullptr;
    if (traj && (s->mode != RMS_MODE_WAVEFORM || prec != RMS_PREC_SPLIT || jobs.size() != 1))
        return set_error(RMS_ERR_ARG, "trajectory output needs a one-simulation SPLIT run in waveform mode");
    const int device = o ? o->device : 0;
    for (LaunchJob& j : jobs) {
        if (!j.s->have_lattice) return set_error(RMS_ERR_STATE, "no lattice: call rms_sim_set_lattice or load a run directory");
        if (!same_schedule(s, j.s)) return set_error(RMS_ERR_ARG, "simulations of one launch need the same steps, records, walls and signal tables");
        int rc = ensure_device(j.s, device);
        if (rc) return rc;
    }
    rms_device_state* d = s->dev;
    RMS_CUDA(cudaSetDevice(device));
    cudaStream_t st = (o && o->stream) ? (cudaStream_t)o->stream : d->own;
    const int naxons = (int)jobs.size();

    int64_t trace_n = (o && o->trace_walkers > 0) ? o->trace_walkers : 0;
    if (trace_n && prec != RMS_PREC_COMPAT) return set_error(RMS_ERR_ARG, "traces are recorded by the COMPAT walk only");
    if (trace_n && jobs[0].w0 != 0) return set_error(RMS_ERR_ARG, "traces need walker_begin = 0");
    trace_n = std::min<int64_t>(trace_n, jobs[0].w1);

    // launch shape: persistent grid
    int dev_sms = 0;
    RMS_CUDA(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device));
    int block = kCompatBlock, per_sm, variant = 0, lattice_bits = 8;
    int nc_max = 0;
    for (LaunchJob& j : jobs) nc_max = std::max(nc_max, j.s->nc);
    if (prec == RMS_PREC_COMPAT) {
        per_sm = walk_compat_blocks_per_sm(s->nc, trace_n > 0);
    } else {
        lattice_bits = split_lattice_bits(nc_max);
        variant = (o && o->variant > 0) ? o->variant - 1 : kSplitVariantDefault;
        if (!split_variant_walks(variant, s->mode, s->rule)) variant = 0;   // waveforms and rules: first variant
        if (variant >= split_variant_count()) return set_error(RMS_ERR_ARG, "variant out of range");
        block = split_variant_block(variant);
        per_sm = walk_split_blocks_per_sm(nc_max, lattice_bits, variant);
    }
    if (per_sm <= 0) return set_error(RMS_ERR_CUDA, "occupancy query failed (kernel image missing for this GPU?)");
    std::vector<int64_t> tile_begin(naxons + 1, 0);
    for (int k = 0; k < naxons; ++k) tile_begin[k + 1] = tile_begin[k] + (jobs[k].w1 - jobs[k].w0 + 31) / 32;
    const int64_t ntiles = tile_begin[naxons];
    const int64_t warps_per_block = block / 32;
    const int64_t grid64 = std::min<int64_t>((int64_t)dev_sms * per_sm, (ntiles + warps_per_block - 1) / warps_per_block);
    const int grid = (int)std::max<int64_t>(grid64, 1);
    const int nthr = grid * block;
    const int nwarps = nthr / 32;
    const int T = s->timepoints;
    const int nb = s->nbvec();
    const int nvals = (s->mode == RMS_MODE_NARROW) ? kRowHead + ((nb + 31) / 32) * 32 : kRowHead;
    const bool wavemode = s->mode == RMS_MODE_WAVEFORM;
    const bool has_sig = s->mode != RMS_MODE_NARROW;
    // signal row: PGSE, one value per gradient; waveforms, (cos, sin) per waveform
    const int ngrad = wavemode ? 2 * s->nwave : s->ngrad();
    const int ngrad_pad = std::max(32, ((ngrad + 31) / 32) * 32);
    const size_t row = (size_t)T * nvals;

    const int nseg = nwarps;   // one accumulator row set per warp
    // The SPLIT walk runs in the table form (axon fields and seeds from device
    // memory, tiles from a queue, each warp's rows added into the axon totals
    // with FP64 atomics): for one axon too, where it is 1.3x faster than the
    // form reading kernel parameters (fewer registers), at the price of sums
    // repeatable only up to their order.  COMPAT: per-warp rows, ordered sum.
    const bool multi = prec == RMS_PREC_SPLIT;

    // inputs
    for (LaunchJob& j : jobs) {
        int rc = prepare_lattice(j.s, st, prec == RMS_PREC_SPLIT, lattice_bits);
        if (rc) return rc;
    }
    std::vector<double> tables;
    tables.insert(tables.end(), s->step.begin(), s->step.end());
    tables.insert(tables.end(), s->t2_steps.begin(), s->t2_steps.end());
    tables.insert(tables.end(), s->pij.begin(), s->pij.end());
    RMS_CUDA(upload(d->tables, tables, st));
    RMS_CUDA(upload(d->qtab, s->qtab, st));
    RMS_CUDA(upload(d->bvec, s->bvec, st));
    RMS_CUDA(upload(d->grad, s->grad, st));
    RMS_CUDA(upload(d->gpair, s->gpair, st));
    RMS_CUDA(upload(d->ev_step, s->ev_step, st));
    RMS_CUDA(upload(d->ev_pair, s->ev_pair, st));
    RMS_CUDA(upload(d->ev_coef, s->ev_coef, st));
    if (wavemode) {
        // [bin][waveform][axis], scaled by dt: the phase per um of X_b
        std::vector<double> wf((size_t)s->nbins * s->nwave * 3);
        for (int j = 0; j < s->nwave; ++j)
            for (int b = 0; b < s->nbins; ++b)
                for (int x = 0; x < 3; ++x)
                    wf[((size_t)b * s->nwave + j) * 3 + x] = s->wave[((size_t)j * s->nbins + b) * 3 + x] * s->dt;
        RMS_CUDA(upload(d->wavef, wf, st));
    }
    if (prec == RMS_PREC_SPLIT) {
        p.axons.resize(naxons);
        for (int k = 0; k < naxons; ++k)
            fill_axon_desc(p.axons[k], jobs[k].s, jobs[k].w0, jobs[k].w1, tile_begin[k], jobs[k].seed,
                           jobs[k].s->dev->packed.as<uint8_t>());
        RMS_CUDA(d->axons.ensure(sizeof(AxonDesc) * naxons));
    }

    // accumulators
    RMS_CUDA(d->slots.ensure((size_t)nseg * row * sizeof(double)));
    RMS_CUDA(d->out.ensure((size_t)naxons * row * sizeof(double)));
    RMS_CUDA(d->err.ensure(16));   // error word, then the multi-axon tile counter at byte 8
    if (has_sig) {
        RMS_CUDA(d->sig_slots.ensure((size_t)nseg * ngrad_pad * sizeof(double)));
        RMS_CUDA(d->out_sig.ensure((size_t)naxons * ngrad_pad * sizeof(double)));
        const size_t per_thread = wavemode ? (size_t)s->nwave : (size_t)s->npairs * 3;
        RMS_CUDA(d->vscr.ensure(std::max<size_t>(per_thread * nthr * sizeof(double), 16)));
    }
    if (trace_n) {
        RMS_CUDA(d->tr_init.ensure((size_t)trace_n * sizeof(int32_t)));
        RMS_CUDA(d->tr_vox.ensure((size_t)trace_n * s->tn * sizeof(int32_t)));
        RMS_CUDA(d->tr_ev.ensure((size_t)trace_n * s->tn * sizeof(uint32_t)));
        RMS_CUDA(d->tr_pos.ensure((size_t)trace_n * s->tn * 3 * sizeof(double)));
    }
    const size_t nrow = (size_t)naxons * row, nsig = (size_t)naxons * ngrad_pad;
    RMS_CUDA(d->h_out.ensure((nrow + nsig + 1) * sizeof(double)));
    if (prec == RMS_PREC_SPLIT) RMS_CUDA(d->h_axons.ensure(sizeof(AxonDesc) * naxons));

    WalkArgs& a = p.a;
    a = WalkArgs{};
    a.labels = d->labels.as<uint8_t>();
    a.n1 = s->n1; a.n2 = s->n2; a.n3 = s->n3;
    a.walker_begin = jobs[0].w0; a.walker_end = jobs[0].w1;
    a.tn = s->tn; a.tstep = s->tstep; a.timepoints = T; a.nite = s->nite; a.nc = nc_max;
    a.boundary = s->boundary; a.mode = s->mode;
    a.res = s->res; a.dt = s->dt;
    a.seed = jobs[0].seed;
    a.rule = s->rule;
    a.table_form = multi ? 1 : 0;
    a.step = d->tables.as<double>();
    a.t2 = a.step + s->nc;
    a.pij = a.t2 + s->nc;
    a.nvals = nvals;
    a.slots = d->slots.as<double>();
    a.nbvec = nb;
    a.qtab = d->qtab.as<double>();
    a.bvec = d->bvec.as<double>();
    a.ngrad = ngrad; a.ngrad_pad = ngrad_pad; a.npairs = s->npairs; a.nevents = (int)s->ev_step.size();
    a.ev_step = d->ev_step.as<int>(); a.ev_pair = d->ev_pair.as<int>(); a.ev_coef = d->ev_coef.as<double>();
    a.grad = d->grad.as<double>(); a.gpair = d->gpair.as<int>();
    a.vscr = d->vscr.as<double>();
    a.sig_slots = d->sig_slots.as<double>();
    a.err = d->err.as<int>();
    a.tile_ctr = reinterpret_cast<unsigned long long*>(static_cast<char*>(d->err.p) + 8);
    a.axons = d->axons.as<AxonDesc>();
    a.naxons = naxons;
    a.ntiles = ntiles;
    a.nwave = wavemode ? s->nwave : 0;
    a.nbins = wavemode ? s->nbins : 0;
    a.bin_steps = wavemode ? s->tn / s->nbins : 0;
    a.wave = d->wavef.as<double>();
    a.traj = traj;
    a.traj_split = (o && o->traj_split) ? 1 : 0;
    a.traj_n = jobs[0].w1 - jobs[0].w0;
    a.out_rows = d->out.as<double>();
    a.out_sig = d->out_sig.as<double>();
    if (!p.axons.empty()) a.axon0 = p.axons[0];
    a.trace_n = trace_n;
    a.tr_init = d->tr_init.as<int32_t>(); a.tr_vox = d->tr_vox.as<int32_t>(); a.tr_ev = d->tr_ev.as<uint32_t>();
    a.tr_pos = d->tr_pos.as<double>();

    p.d = d; p.st = st; p.prec = prec; p.grid = grid; p.block = block; p.variant = variant; p.bits = lattice_bits;
    p.naxons = naxons; p.T = T; p.nb = nb; p.ngrad = ngrad; p.ngrad_pad = ngrad_pad; p.nvals = nvals; p.nseg = nseg;
    p.row = row; p.nrow = nrow; p.nsig = nsig; p.multi = multi; p.has_sig = has_sig; p.wavemode = wavemode;
    p.trace_n = trace_n;
    return RMS_OK;
}

// Device work of one launch, all asynchronous on p.st.  The axon table comes
// from the pinned host copy (which the caller fills); `events` brackets the
// walk and the reduction with the timing events (not inside a graph).
int enqueue_launch(LaunchPlan& p, rms_sim* s, bool events) {
    rms_device_state* d = p.d;
    cudaStream_t st = p.st;
    const WalkArgs& a = p.a;
    if (p.prec == RMS_PREC_SPLIT)
        RMS_CUDA(cudaMemcpyAsync(d->axons.p, d->h_axons.p, sizeof(AxonDesc) * p.naxons, cudaMemcpyHostToDevice, st));
    RMS_CUDA(cudaMemsetAsync(d->slots.p, 0, (size_t)p.nseg * p.row * sizeof(double), st));
    if (p.multi) RMS_CUDA(cudaMemsetAsync(d->out.p, 0, p.nrow * sizeof(double), st));
    RMS_CUDA(cudaMemsetAsync(d->err.p, 0, 16, st));
    if (p.has_sig) {
        RMS_CUDA(cudaMemsetAsync(d->sig_slots.p, 0, (size_t)p.nseg * p.ngrad_pad * sizeof(double), st));
        if (p.multi) RMS_CUDA(cudaMemsetAsync(d->out_sig.p, 0, p.nsig * sizeof(double), st));
    }
    if (events) RMS_CUDA(cudaEventRecord(d->e0, st));
    int e = (p.prec == RMS_PREC_COMPAT) ? launch_walk_compat(a, p.grid, p.block, p.trace_n > 0, st)
                                        : launch_walk_split(a, p.bits, p.variant, p.grid, st);
    if (e) return cuda_fail((cudaError_t)e, "walk kernel launch");
    if (events) RMS_CUDA(cudaEventRecord(d->e1, st));
    if (!p.multi) {
        // COMPAT: the warps' rows summed in a fixed order (repeatable)
        e = launch_reduce_slots(a.slots, p.nseg, p.row, d->out.as<double>(), st);
        if (!e && p.has_sig)
            e = launch_reduce_slots(a.sig_slots, p.nseg, (size_t)p.ngrad_pad, d->out_sig.as<double>(), st);
        if (e) return cuda_fail((cudaError_t)e, "reduce launch");
    }
    if (events) RMS_CUDA(cudaEventRecord(d->e2, st));

    // results back (one pinned staging buffer: rows, then signals, then the error word)
    double* h = static_cast<double*>(d->h_out.p);
    RMS_CUDA(cudaMemcpyAsync(h, d->out.p, p.nrow * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (p.has_sig)
        RMS_CUDA(cudaMemcpyAsync(h + p.nrow, d->out_sig.p, p.nsig * sizeof(double), cudaMemcpyDeviceToHost, st));
    int* herr = reinterpret_cast<int*>(h + p.nrow + p.nsig);
    RMS_CUDA(cudaMemcpyAsync(herr, d->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (p.trace_n) {
        const size_t tn = (size_t)s->tn, n = (size_t)p.trace_n;
        s->tr_init.resize(n);
        s->tr_vox.resize(n * tn);
        s->tr_ev.resize(n * tn);
        s->tr_pos.resize(n * tn * 3);
        RMS_CUDA(cudaMemcpyAsync(s->tr_init.data(), d->tr_init.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        RMS_CUDA(cudaMemcpyAsync(s->tr_vox.data(), d->tr_vox.p, s->tr_vox.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        RMS_CUDA(cudaMemcpyAsync(s->tr_ev.data(), d->tr_ev.p, s->tr_ev.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        RMS_CUDA(cudaMemcpyAsync(s->tr_pos.data(), d->tr_pos.p, s->tr_pos.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    return RMS_OK;
}

int finish_launch(std::vector<LaunchJob>& jobs, LaunchPlan& p, bool events) {
    rms_device_state* d = p.d;
    RMS_CUDA(cudaStreamSynchronize(p.st));
    const double* h = static_cast<const double*>(d->h_out.p);
    const int herr = *reinterpret_cast<const int*>(h + p.nrow + p.nsig);
    if (herr & kErrInitCap)
        return set_error(RMS_ERR_RANGE, "a walker found no labelled voxel within the rejection-sampling cap");
    if (herr & kErrStep) return set_error(RMS_ERR_RANGE, "a step segment found no voxel face (step >= 1 voxel)");

    float ms_walk = 0.f, ms_run = 0.f;
    if (events) {
        RMS_CUDA(cudaEventElapsedTime(&ms_walk, d->e0, d->e1));
        RMS_CUDA(cudaEventElapsedTime(&ms_run, d->e0, d->e2));
    } else {
        RMS_CUDA(cudaEventElapsedTime(&ms_walk, d->e0, d->e1));
        ms_run = ms_walk;
    }

    // unpack record rows into the reference's field layouts
    const int T = p.T, nb = p.nb, ngrad = p.ngrad;
    for (int k = 0; k < p.naxons; ++k) {
        rms_sim* sk = jobs[k].s;
        const double* hk = h + (size_t)k * p.row;
        const int nc = sk->nc;
        sk->sig0.assign(T, 0.0);
        sk->dx2.assign((size_t)T * 6, 0.0);
        sk->dx4.assign((size_t)T * 15, 0.0);
        sk->npar_count.assign((size_t)T * nc, 0.0);
        sk->sigre.assign((size_t)T * nb, 0.0);
        for (int t = 0; t < T; ++t) {
            const double* r = hk + (size_t)t * p.nvals;
            sk->sig0[t] = r[kColSig0];
            for (int q = 0; q < 6; ++q) sk->dx2[t * 6 + q] = r[kColDx2 + q];
            for (int q = 0; q < 15; ++q) sk->dx4[t * 15 + q] = r[kColDx4 + q];
            for (int c = 0; c < nc; ++c) sk->npar_count[t * nc + c] = r[kColCount + c];
            if (sk->mode == RMS_MODE_NARROW)
                for (int q = 0; q < nb; ++q) sk->sigre[(size_t)t * nb + q] = r[kRowHead + q];
        }
        sk->sig.assign(sk->mode == RMS_MODE_PGSE ? ngrad : 0, 0.0);
        for (int q = 0; q < (int)sk->sig.size(); ++q) sk->sig[q] = h[p.nrow + (size_t)k * p.ngrad_pad + q];
        sk->sigw.assign(p.wavemode ? ngrad : 0, 0.0);
        for (int q = 0; q < (int)sk->sigw.size(); ++q) sk->sigw[q] = h[p.nrow + (size_t)k * p.ngrad_pad + q];
        sk->trace_n = k == 0 ? p.trace_n : 0;
        sk->walk_ms = ms_walk;
        sk->run_ms = ms_run;
        sk->last_grid = p.grid;
        sk->last_block = p.block;
        sk->have_results = true;
        sk->have_timing = true;
    }
    return RMS_OK;
}

// RMS_TRACE set (and not "0"): every launch prints one line to stderr with its
// phases -- plan (validation, shape, uploads), enqueue, finish (wait, error
// word, unpack) on the host clock, and the walk / walk+reduce kernel times the
// launch's events measured.  Read once per process.
bool trace_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("RMS_TRACE");
        return v && *v && std::strcmp(v, "0") != 0;
    }();
    return on;
}

int run_launch(std::vector<LaunchJob>& jobs, const rms_run_opts* o) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    LaunchPlan p;
    int rc = plan_launch(jobs, o, p);
    if (rc) return rc;
    if (p.prec == RMS_PREC_SPLIT)
        std::memcpy(p.d->h_axons.p, p.axons.data(), sizeof(AxonDesc) * p.naxons);
    const auto t1 = clk::now();
    rc = enqueue_launch(p, jobs[0].s, true);
    if (rc) return rc;
    const auto t2 = clk::now();
    rc = finish_launch(jobs, p, true);
    if (rc == RMS_OK && trace_enabled()) {
        const auto t3 = clk::now();
        auto ms = [](clk::time_point a, clk::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        std::fprintf(stderr,
                     "rms trace: %s %d sim(s) %lld walker-steps: plan %.3f ms, enqueue %.3f ms, finish %.3f ms; "
                     "kernels: walk %.3f ms, walk+reduce %.3f ms; grid %d x %d\n",
                     p.prec == RMS_PREC_SPLIT ? "split" : "compat", p.naxons,
                     (long long)[&] {
                         long long n = 0;
                         for (const LaunchJob& j : jobs) n += (long long)(j.w1 - j.w0) * j.s->tn;
                         return n;
                     }(),
                     ms(t0, t1), ms(t1, t2), ms(t2, t3), jobs[0].s->walk_ms, jobs[0].s->run_ms, p.grid, p.block);
    }
    return rc;
}

}  // namespace
}  // namespace rms

// A captured batch launch (rms_batch_graph_create): the plan, the simulations
// it walks, and the device buffers the graph refers to.
struct rms_graph {
    std::vector<rms::LaunchJob> jobs;
    rms::LaunchPlan plan;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> buffers;
    int device = 0;
    ~rms_graph() {
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace rms {
namespace {

std::vector<const void*> graph_buffers(const rms_graph* g) {
    const rms_device_state* d = g->plan.d;
    std::vector<const void*> v{d->axons.p, d->slots.p, d->out.p, d->err.p, d->sig_slots.p, d->out_sig.p,
                               d->vscr.p, d->tables.p, d->qtab.p, d->bvec.p, d->grad.p, d->gpair.p,
                               d->ev_step.p, d->ev_pair.p, d->ev_coef.p, d->wavef.p, d->h_out.p, d->h_axons.p};
    for (const LaunchJob& j : g->jobs) v.push_back(j.s->dev ? j.s->dev->packed.p : nullptr);
    return v;
}

int graph_create(rms_sim* const* sims, int n, const rms_run_opts* o, rms_graph** out) {
    if (!o || o->precision != RMS_PREC_SPLIT) return set_error(RMS_ERR_ARG, "a graph captures the SPLIT walk");
    if (o->trace_walkers > 0 || o->traj_out) return set_error(RMS_ERR_ARG, "a graph records no traces or trajectories");
    std::unique_ptr<rms_graph> g(new rms_graph());
    g->device = o->device;
    for (int i = 0; i < n; ++i) {
        int64_t w0 = 0, w1 = 0;
        int rc = batch_range(sims[i], o, w0, w1);
        if (rc) return rc;
        g->jobs.push_back(LaunchJob{sims[i], w0, w1, o->seed + (uint64_t)i * kBatchSeedStep});
    }
    rms_run_opts oo = *o;
    int rc = plan_launch(g->jobs, &oo, g->plan);
    if (rc) return rc;
    LaunchPlan& p = g->plan;
    if (!o->stream) p.st = p.d->own;   // capture needs a stream other than the legacy default stream
    std::memcpy(p.d->h_axons.p, p.axons.data(), sizeof(AxonDesc) * p.naxons);
    RMS_CUDA(cudaStreamBeginCapture(p.st, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_launch(p, g->jobs[0].s, false);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(p.st, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "stream capture of the batch launch");
    g->graph = graph;
    RMS_CUDA(cudaGraphInstantiate(&g->exec, graph, 0));
    g->buffers = graph_buffers(g.get());
    *out = g.release();
    return RMS_OK;
}

int graph_run(rms_graph* g, uint64_t seed) {
    for (const LaunchJob& j : g->jobs)
        if (j.s->lattice_dirty || !j.s->dev || !j.s->dev->packed_valid || j.s->dev->packed_bits != g->plan.bits)
            return set_error(RMS_ERR_STATE, "a simulation of the graph has a new lattice: create the graph again");
    if (graph_buffers(g) != g->buffers)
        return set_error(RMS_ERR_STATE, "the graph's device buffers were reallocated by another run: create the graph again");
    LaunchPlan& p = g->plan;
    RMS_CUDA(cudaSetDevice(g->device));
    for (int k = 0; k < p.naxons; ++k) p.axons[k].seed = seed + (uint64_t)k * kBatchSeedStep;
    std::memcpy(p.d->h_axons.p, p.axons.data(), sizeof(AxonDesc) * p.naxons);
    RMS_CUDA(cudaEventRecord(p.d->e0, p.st));
    RMS_CUDA(cudaGraphLaunch(g->exec, p.st));
    RMS_CUDA(cudaEventRecord(p.d->e1, p.st));
    return finish_launch(g->jobs, p, false);
}

// Launch-variant autotuner: each variant walks the same subset of every
// simulation's walkers (the first fraction f of each, f chosen so the subset
// fills about four waves of the widest variant), one untimed launch first;
// the fastest walk kernel wins.  Results are cached per (device, lattice
// encoding, Nc, axon count, log2 of the lattice voxels, log2 of the steps).
struct TuneKey {
    int device, bits, nc, naxons, vox_log2, tn_log2, mode;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, bits, nc, naxons, vox_log2, tn_log2, mode) <
               std::tie(o.device, o.bits, o.nc, o.naxons, o.vox_log2, o.tn_log2, o.mode);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, std::vector<double>>> g_tune;

int autotune(rms_sim* const* sims, int n, const rms_run_opts* opts, int* variant, double* variant_ms) {
    const int device = opts ? opts->device : 0;
    int nc_max = 0;
    double vox = 0.0;
    int64_t total = 0;
    std::vector<int64_t> r0(n), r1(n);
    for (int i = 0; i < n; ++i) {
        int rc = batch_range(sims[i], opts, r0[i], r1[i]);
        if (rc) return rc;
        nc_max = std::max(nc_max, sims[i]->nc);
        vox += (double)sims[i]->n1 * sims[i]->n2 * sims[i]->n3;
        total += r1[i] - r0[i];
    }
    const TuneKey key{device, split_lattice_bits(nc_max), nc_max, n, (int)std::log2(std::max(vox, 1.0)),
                      (int)std::log2((double)std::max(sims[0]->tn, 1)), sims[0]->mode};
    const int nv = split_variant_count();
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            *variant = it->second.first;
            if (variant_ms)
                for (int v = 0; v < nv; ++v) variant_ms[v] = it->second.second[v];
            return RMS_OK;
        }
    }
    int sms = 0;
    RMS_CUDA(cudaSetDevice(device));
    RMS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const double want = 4.0 * sms * 4 * 256;     // four waves of 256 x 4 blocks per SM
    const double f = std::min(1.0, want / (double)std::max<int64_t>(total, 1));
    std::vector<LaunchJob> jobs;
    const uint64_t seed = opts ? opts->seed : 0;
    for (int i = 0; i < n; ++i) {
        const int64_t ni = r1[i] - r0[i];
        const int64_t m = std::max<int64_t>(std::min<int64_t>(32, ni), (int64_t)std::ceil(f * ni));
        jobs.push_back(LaunchJob{sims[i], r0[i], r0[i] + std::min<int64_t>(m, ni), seed + (uint64_t)i * kBatchSeedStep});
    }
    rms_run_opts o = opts ? *opts : rms_run_opts{};
    o.precision = RMS_PREC_SPLIT;
    o.trace_walkers = 0;
    o.traj_out = nullptr;
    std::vector<double> ms(nv, 0.0);
    int best = 0;
    for (int v = -1; v < nv; ++v) {
        if (v >= 0 && !split_variant_walks(v, sims[0]->mode, sims[0]->rule)) {
            ms[v] = INFINITY;                    // built for the first variant only
            continue;
        }
        o.variant = (v < 0 ? 0 : v) + 1;
        int rc = run_launch(jobs, &o);
        if (rc) return rc;
        if (v < 0) continue;                     // warm-up launch
        ms[v] = jobs[0].s->walk_ms;
        if (ms[v] < ms[best]) best = v;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = {best + 1, ms};
    }
    *variant = best + 1;
    if (variant_ms)
        for (int v = 0; v < nv; ++v) variant_ms[v] = ms[v];
    return RMS_OK;
}

int run_one(rms_sim* s, const rms_run_opts* o) {
    int64_t w0 = 0, w1 = 0;
    int rc = walker_range(s, o, w0, w1);
    if (rc) return rc;
    if (w0 == w1) {
        // an empty shard: nothing to walk, zero results
        zero_results(s);
        return RMS_OK;
    }
    std::vector<LaunchJob> jobs{LaunchJob{s, w0, w1, o ? o->seed : 0}};
    return run_launch(jobs, o);
}

// Gradients of L = sum_j g_cos[j] C_j + g_sin[j] S_j for a waveform-mode
// simulation, by the two-pass walk of rms_adjoint.cu.
int run_adjoint(rms_sim* s, const rms_run_opts* o, const double* g_sigw, rms_adjoint_grads* out, double* jac) {
    if (s->mode != RMS_MODE_WAVEFORM) return set_error(RMS_ERR_ARG, "the adjoint differentiates a waveform-mode simulation");
    if (s->rule != RMS_RULE_REFLECT) return set_error(RMS_ERR_ARG, "the adjoint walks with reflecting membranes");
    if (s->nwave > kAdjWaves) return set_error(RMS_ERR_RANGE, "the adjoint takes at most 16 waveforms per run");
    if (s->nc > kAdjNc) return set_error(RMS_ERR_RANGE, "the adjoint supports Nc <= 4");
    if (!s->have_lattice) return set_error(RMS_ERR_STATE, "no lattice: call rms_sim_set_lattice or load a run directory");
    double D = 0.0;
    for (int c = 1; c < s->nc; ++c) {
        if (D == 0.0) D = s->diffusivity[c];
        if (s->diffusivity[c] != D)
            return set_error(RMS_ERR_ARG, "the adjoint needs one diffusivity for all labelled compartments");
    }
    if (!(D > 0.0)) return set_error(RMS_ERR_ARG, "the adjoint needs a positive diffusivity");
    int64_t w0 = 0, w1 = 0;
    int rc0 = walker_range(s, o, w0, w1);
    if (rc0) return rc0;
    if (w0 == w1) return set_error(RMS_ERR_ARG, "the adjoint's shard holds no walkers");
    const int device = o ? o->device : 0;
    int rc = ensure_device(s, device);
    if (rc) return rc;
    rms_device_state* d = s->dev;
    RMS_CUDA(cudaSetDevice(device));
    cudaStream_t st = (o && o->stream) ? (cudaStream_t)o->stream : d->own;
    rc = prepare_lattice(s, st, true, 4);
    if (rc) return rc;

    AxonDesc x;
    fill_axon_desc(x, s, w0, w1, 0, o ? o->seed : 0, d->packed.as<uint8_t>());
    AdjArgs a{};
    a.lat = x.lat;
    a.n1 = x.n1; a.n2 = x.n2; a.n3 = x.n3; a.s0 = x.s0; a.s1 = x.s1;
    a.walker_begin = w0; a.walker_end = w1;
    a.ntiles = (w1 - w0 + 31) / 32;
    a.seed = x.seed;
    a.tn = s->tn; a.nbins = s->nbins; a.bin_steps = s->tn / s->nbins; a.nwave = s->nwave;
    a.nite = s->nite; a.boundary = s->boundary;
    a.res = x.res;
    a.flight = x.flight; a.same_cross = x.same_cross;
    // the forced-draw pass runs when some face is crossed by a draw
    a.force = 0;
    for (int c = 0; c < s->nc; ++c)
        for (int e = 0; e < s->nc; ++e) {
            const float P = x.pij[c * kNcMax + e];
            if (P >= 0.000001f && !(P > 0.999999f)) a.force = 1;
        }
    for (int c = 0; c < kAdjNc; ++c) {
        a.step[c] = c < s->nc ? x.step[c] : 0.0f;
        a.kexp[c] = c < s->nc ? x.k[c] : 0.0f;
        for (int e = 0; e < kAdjNc; ++e) {
            a.pij[c * kAdjNc + e] = (c < s->nc && e < s->nc) ? x.pij[c * kNcMax + e] : 0.0f;
            a.ratio[c * kAdjNc + e] = (c < s->nc && e < s->nc) ? x.ratio[c * kNcMax + e] : 0.0f;
        }
    }
    std::vector<double> wf((size_t)s->nbins * s->nwave * 3);
    for (int j = 0; j < s->nwave; ++j)
        for (int b = 0; b < s->nbins; ++b)
            for (int k = 0; k < 3; ++k)
                wf[((size_t)b * s->nwave + j) * 3 + k] = s->wave[((size_t)j * s->nbins + b) * 3 + k] * s->dt;
    RMS_CUDA(upload(d->wavef, wf, st));
    // the float terms of the time rescaling and of the step-length tangent:
    // (float)(g_b - g_b+1) with g_nbins = 0, and (float)(g_b res)
    std::vector<float> wq((size_t)s->nbins * s->nwave * 8, 0.0f);
    for (int b = 0; b < s->nbins; ++b)
        for (int j = 0; j < s->nwave; ++j)
            for (int k = 0; k < 3; ++k) {
                const double g = wf[((size_t)b * s->nwave + j) * 3 + k];
                const double gn = b + 1 < s->nbins ? wf[((size_t)(b + 1) * s->nwave + j) * 3 + k] : 0.0;
                float* e = wq.data() + ((size_t)b * s->nwave + j) * 8;
                e[k] = (float)(g - gn);
                e[4 + k] = (float)(g * (double)x.res);
            }
    RMS_CUDA(upload(d->adj_wq, wq, st));
    std::vector<float> gup((size_t)2 * s->nwave);
    for (int j = 0; j < 2 * s->nwave; ++j) gup[j] = (float)(g_sigw ? g_sigw[j] : 0.0);
    RMS_CUDA(upload(d->adj_g, gup, st));
    const size_t ndw = (size_t)s->nbins * s->nwave * 3;
    const int nsums = kAdjSums + (jac ? kJacSums : 0);
    RMS_CUDA(d->adj_sums.ensure(sizeof(double) * nsums));
    RMS_CUDA(cudaMemsetAsync(d->adj_sums.p, 0, sizeof(double) * nsums, st));
    RMS_CUDA(d->adj_dwave.ensure(sizeof(float) * ndw));
    RMS_CUDA(cudaMemsetAsync(d->adj_dwave.p, 0, sizeof(float) * ndw, st));
    RMS_CUDA(d->err.ensure(sizeof(int)));
    RMS_CUDA(cudaMemsetAsync(d->err.p, 0, sizeof(int), st));
    a.wave = d->wavef.as<double>();
    a.wq = d->adj_wq.as<float4>();
    a.gup = d->adj_g.as<float>();
    a.sums = d->adj_sums.as<double>();
    a.dwave = d->adj_dwave.as<float>();
    a.err = d->err.as<int>();

    int sms = 0;
    RMS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int64_t wpb = kAdjBlock / 32;
    auto grid_for = [&](int form, int64_t tiles, int& grid) -> int {
        const int per_sm = adjoint_blocks_per_sm(jac != nullptr, form);
        if (per_sm <= 0) return set_error(RMS_ERR_CUDA, "occupancy query failed (kernel image missing for this GPU?)");
        grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, (tiles + wpb - 1) / wpb));
        return RMS_OK;
    };
    // Pass 1 alone, then the forced walks grouped by resume step.  Checkpoints
    // every E steps, E a multiple of 3 (the direction blocks), 32 (the float
    // folds) and the bin length, at most kAdjCkMax of them; each forced walk
    // resumes from the last checkpoint before its forced draw.  Per walker:
    // the checkpoints, the summary, a bucket entry per resume step and
    // (weighted form) X_wb and a_jw; the walkers go in chunks that fit the
    // scratch budget (half the free memory, at most 16 GiB, or less with
    // RMS_ADJOINT_SCRATCH_MB).
    int64_t base = 96;   // lcm(3, 32)
    {
        int64_t x = base, y = a.bin_steps;
        while (y) { const int64_t t = x % y; x = y; y = t; }
        base = base / x * a.bin_steps;
    }
    const int64_t ck_every = base * std::max<int64_t>(1, (s->tn + base * kAdjCkMax - 1) / (base * kAdjCkMax));
    const int nbk = (int)((s->tn - 1) / ck_every + 1);
    const int64_t nwalk = w1 - w0;
    const size_t per_walker =
        (jac ? 0 : sizeof(float) * ((size_t)3 * s->nbins + s->nwave)) +
        (a.force ? sizeof(uint32_t) * ((size_t)kAdjCkWords * (nbk - 1) + kAdjWsWords + nbk) : 0);
    size_t mfree = 0, mtotal = 0;
    if (cudaMemGetInfo(&mfree, &mtotal) != cudaSuccess) {
        (void)cudaGetLastError();
        mfree = 0;
    }
    size_t budget = std::min<size_t>(mfree / 2, (size_t)16 << 30);
    if (const char* cap = std::getenv("RMS_ADJOINT_SCRATCH_MB")) {
        const long long mb = std::atoll(cap);
        if (mb > 0) budget = std::min<size_t>(budget, (size_t)mb << 20);
    }
    int64_t chunk = std::min<int64_t>(nwalk, (int64_t)(budget / std::max<size_t>(per_walker, 1)));
    if (chunk < nwalk) chunk = chunk / 32 * 32;
    const char* genv = std::getenv("RMS_ADJOINT_GROUPED");
    bool grouped = !(genv && genv[0] == '0') && chunk >= std::min<int64_t>(nwalk, 65536);
    if (grouped) {
        const size_t nwc = (size_t)chunk;
        bool ok = true;
        if (!jac) {
            ok = ok && d->adj_xbin.ensure(sizeof(float) * 3 * (size_t)s->nbins * nwc) == cudaSuccess;
            ok = ok && d->adj_ajw.ensure(sizeof(float) * (size_t)s->nwave * nwc) == cudaSuccess;
        }
        if (a.force) {
            ok = ok && d->adj_ck.ensure(sizeof(uint32_t) * kAdjCkWords * (size_t)(nbk - 1) * nwc) == cudaSuccess;
            ok = ok && d->adj_ws.ensure(sizeof(uint32_t) * kAdjWsWords * nwc) == cudaSuccess;
            ok = ok && d->adj_blist.ensure(sizeof(int) * (size_t)nbk * nwc) == cudaSuccess;
            ok = ok && d->adj_bcount.ensure(sizeof(int) * kAdjCkMax) == cudaSuccess;
        }
        if (!ok) {
            // without room for the records the single launch walks all passes
            (void)cudaGetLastError();   // a failed allocation is not sticky; clear it
            for (DevBuf* b : {&d->adj_xbin, &d->adj_ajw, &d->adj_ck, &d->adj_ws, &d->adj_blist}) b->release();
            grouped = false;
        }
    }
    RMS_CUDA(cudaEventRecord(d->e0, st));
    if (!grouped) {
        int grid = 0;
        rc = grid_for(0, a.ntiles, grid);
        if (rc) return rc;
        const int e = launch_adjoint(a, jac != nullptr, 0, grid, st);
        if (e) return cuda_fail((cudaError_t)e, "adjoint kernel launch");
    } else {
        a.ck_every = (int)ck_every;
        a.nbk = nbk;
        a.xbin = d->adj_xbin.as<float>();
        a.ajw = d->adj_ajw.as<float>();
        a.ck = d->adj_ck.as<uint32_t>();
        a.ws = d->adj_ws.as<uint32_t>();
        a.blist = d->adj_blist.as<int>();
        a.bcount = d->adj_bcount.as<int>();
        for (int64_t c0 = w0; c0 < w1; c0 += chunk) {
            a.walker_begin = c0;
            a.walker_end = std::min<int64_t>(w1, c0 + chunk);
            a.nwalk = a.walker_end - a.walker_begin;
            a.ntiles = (a.nwalk + 31) / 32;
            if (a.force) RMS_CUDA(cudaMemsetAsync(d->adj_bcount.p, 0, sizeof(int) * kAdjCkMax, st));
            int grid = 0;
            rc = grid_for(1, a.ntiles, grid);
            if (rc) return rc;
            int e = launch_adjoint(a, jac != nullptr, 1, grid, st);
            if (e) return cuda_fail((cudaError_t)e, "adjoint kernel launch (pass 1)");
            if (!jac) {
                e = launch_adjoint_dwave(a, sms, st);
                if (e) return cuda_fail((cudaError_t)e, "adjoint dL/dwave launch");
            }
            if (a.force) {
                // the buckets' tiles: at most one partial tile per bucket beyond nwalk / 32
                a.ntiles = a.nwalk / 32 + nbk;
                rc = grid_for(2, a.ntiles, grid);
                if (rc) return rc;
                e = launch_adjoint(a, jac != nullptr, 2, grid, st);
                if (e) return cuda_fail((cudaError_t)e, "adjoint kernel launch (forced walks)");
            }
        }
    }
    RMS_CUDA(cudaEventRecord(d->e1, st));
    std::vector<double> sums(nsums);
    std::vector<float> dw(ndw);
    int herr = 0;
    RMS_CUDA(cudaMemcpyAsync(sums.data(), d->adj_sums.p, sizeof(double) * nsums, cudaMemcpyDeviceToHost, st));
    RMS_CUDA(cudaMemcpyAsync(dw.data(), d->adj_dwave.p, sizeof(float) * ndw, cudaMemcpyDeviceToHost, st));
    RMS_CUDA(cudaMemcpyAsync(&herr, d->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    RMS_CUDA(cudaStreamSynchronize(st));
    if (herr & kErrInitCap)
        return set_error(RMS_ERR_RANGE, "a walker found no labelled voxel within the rejection-sampling cap");
    float ms = 0.f;
    RMS_CUDA(cudaEventElapsedTime(&ms, d->e0, d->e1));
    s->walk_ms = ms;
    s->run_ms = ms;
    s->have_timing = true;

    // dL/dwave: phase_j = dt sum_b wave_j,b . X_b
    if (out->d_wave)
        for (int j = 0; j < s->nwave; ++j)
            for (int b = 0; b < s->nbins; ++b)
                for (int k = 0; k < 3; ++k)
                    out->d_wave[((size_t)j * s->nbins + b) * 3 + k] =
                        s->dt * (double)dw[((size_t)b * s->nwave + j) * 3 + k];
    out->loss = sums[kAdjSumL];
    // dL/dlog P of the permeation draws (Pij = P / (1 + P)), two unbiased
    // estimates: the forced draws, sum_w nb_w Pij (1 - Pij) (L[crossed] -
    // L[reflected]); and the score with the mean loss as baseline,
    // sum_w (L_w - L/N) E_w (E[E_w] = 0 keeps it unbiased)
    const double forced = sums[kAdjSumForce];
    const double score = sums[kAdjSumLE] - sums[kAdjSumL] / (double)(w1 - w0) * sums[kAdjSumE];
    // time rescaling: D dL/dD = sum_w dL_w/deps - kappa dL/dkappa.  In kappa mode
    // kappa dL/dkappa = dL/dlog P; with a fixed permeation probability the
    // continuum permeability of the rescaled walk scales as (1 + eps)^(-1/2)
    // relative to kappa (1 + eps), so half of it comes off.
    const bool kap = s->permeation == RMS_PERM_KAPPA;
    out->d_diffusivity = (sums[kAdjSumTR] - (kap ? forced : 0.5 * forced)) / D;
    // pathwise, events frozen: l = sqrt(6 D dt) / res, dl/dD = l / (2 D); in
    // kappa mode P ~ kappa D^(-1/2)
    const double step = s->step[s->nc > 1 ? 1 : 0];
    out->d_diffusivity_pathwise = (sums[kAdjSumPath] * step / 2.0 - (kap ? forced / 2.0 : 0.0)) / D;
    out->d_kappa = (kap && s->kappa > 0.0) ? forced / s->kappa : 0.0;
    out->d_kappa_score = (kap && s->kappa > 0.0) ? score / s->kappa : 0.0;
    for (int c = 0; c < 8; ++c) out->d_t2[c] = 0.0;
    for (int c = 0; c < s->nc; ++c) {
        const double T2 = s->t2[c];
        out->d_t2[c] = sums[kAdjSumLT + c] * s->dt / (T2 * T2);   // s0 = exp(-sum_c t_c / T2_c), t_c in ms
    }
    if (out->sigw)
        for (int j = 0; j < 2 * s->nwave; ++j) out->sigw[j] = sums[kAdjSumSig + j];
    if (jac) {
        // each signal sum X_q (q = 2j + s) as the loss L = X_q: the formulas above with
        // the walker sums of X_q
        const double* js = sums.data() + kAdjSums;
        const double N = (double)(w1 - w0);
        for (int q = 0; q < 2 * s->nwave; ++q) {
            double* row = jac + (size_t)q * RMS_JAC_COLS;
            for (int k = 0; k < RMS_JAC_COLS; ++k) row[k] = 0.0;
            const double Xq = sums[kAdjSumSig + q];
            const double fq = js[kJacF + q];
            const double sq = js[kJacE + q] - Xq / N * sums[kAdjSumE];
            row[RMS_JAC_D] = (js[kJacTR + q] - (kap ? fq : 0.5 * fq)) / D;
            row[RMS_JAC_KAPPA] = (kap && s->kappa > 0.0) ? fq / s->kappa : 0.0;
            row[RMS_JAC_KAPPA_SCORE] = (kap && s->kappa > 0.0) ? sq / s->kappa : 0.0;
            for (int c = 0; c < s->nc; ++c) {
                const double T2 = s->t2[c];
                row[RMS_JAC_T2 + c] = js[kJacLT + q * kAdjNc + c] * s->dt / (T2 * T2);
            }
        }
    }
    return RMS_OK;
}

bool field_size(const rms_sim* s, int field, size_t& n) {
    const size_t T = s->timepoints;
    switch (field) {
        case RMS_FIELD_SIG0: n = T; return true;
        case RMS_FIELD_DX2: n = T * 6; return true;
        case RMS_FIELD_DX4: n = T * 15; return true;
        case RMS_FIELD_SIGRE: n = s->mode == RMS_MODE_NARROW ? T * s->nbvec() : 0; return true;
        case RMS_FIELD_SIG: n = s->mode == RMS_MODE_PGSE ? (size_t)s->ngrad() : 0; return true;
        case RMS_FIELD_NPAR_COUNT: n = T * s->nc; return true;
        case RMS_FIELD_TD: n = T; return true;
        case RMS_FIELD_DIFFUSIVITY: n = s->nc; return true;
        case RMS_FIELD_STEP: n = s->nc; return true;
        case RMS_FIELD_PIJ: n = (size_t)s->nc * s->nc; return true;
        case RMS_FIELD_SIGW: n = s->mode == RMS_MODE_WAVEFORM ? (size_t)2 * s->nwave : 0; return true;
        case RMS_FIELD_BVAL: n = s->mode == RMS_MODE_NARROW ? (size_t)s->nbvec() : 0; return true;
        case RMS_FIELD_BVEC: n = s->mode == RMS_MODE_NARROW ? (size_t)3 * s->nbvec() : 0; return true;
        case RMS_FIELD_GRAD: n = s->mode == RMS_MODE_PGSE ? (size_t)6 * s->ngrad() : 0; return true;
        case RMS_FIELD_SIM_PARA: n = 4; return true;
        default: return false;
    }
}

constexpr int kNoDevicePath = 1;   // set_lattice_on_device: take the host path instead

int set_lattice_on_device(rms_sim* s, const uint8_t* labels, size_t n) {
    rms_device_state* d = s->dev;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(d->device) != cudaSuccess) return kNoDevicePath;
    struct Restore {
        int dev;
        ~Restore() { if (dev >= 0) cudaSetDevice(dev); }
    } restore{prev};
    if (d->stage.ensure(n) != cudaSuccess || d->counts.ensure(2 * sizeof(unsigned long long)) != cudaSuccess) {
        d->stage.release();
        return kNoDevicePath;
    }
    int sms = 0;
    RMS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device));
    unsigned long long hcount[2] = {0, 0};
    RMS_CUDA(cudaMemsetAsync(d->counts.p, 0, sizeof(hcount), d->own));
    RMS_CUDA(cudaMemcpyAsync(d->stage.p, labels, n, cudaMemcpyHostToDevice, d->own));
    // from here the stream reads the caller's buffer: every return waits for it
    cudaError_t e = (cudaError_t)check_labels(d->stage.as<uint8_t>(), n, (unsigned)s->nc,
                                              d->counts.as<unsigned long long>(), sms, d->own);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hcount, d->counts.p, sizeof(hcount), cudaMemcpyDeviceToHost, d->own);
    const cudaError_t es = cudaStreamSynchronize(d->own);
    if (e != cudaSuccess) return cuda_fail(e, "lattice check");
    if (es != cudaSuccess) return cuda_fail(es, "lattice upload");
    if (hcount[0] || hcount[1] == 0 || (double)hcount[1] / (double)n < 1e-7) {
        // refused: the host scan names the first offending voxel
        const int rc = validate_lattice(labels, n, s->nc);
        return rc ? rc : set_error(RMS_ERR_RANGE, "lattice refused by the device check");
    }
    std::swap(d->labels, d->stage);
    d->labels_bytes = n;
    d->packed_valid = false;
    s->have_lattice = true;
    s->lattice_dirty = false;
    s->host_stale = true;
    return RMS_OK;
}

}  // namespace
}  // namespace rms

using namespace rms;

extern "C" {

const char* rms_last_error(void) { return g_last_error.c_str(); }

const char* rms_version(void) { return "rms_b200 0.1 (sm_100a)"; }

int rms_contract_phases(const float* d_pos, int64_t nwalk, int nbins, const float* d_wave, int nwave, int method,
                        double* d_out, void* stream, float* kernel_ms) {
    const char* msg = nullptr;
    const int rc = contract_phases(d_pos, nwalk, nbins, d_wave, nwave, method, d_out, stream, &msg, kernel_ms);
    if (rc != RMS_OK) {
        std::string m = std::string("contraction: ") + (msg ? msg : "failed");
        const cudaError_t ce = cudaGetLastError();
        if (rc == RMS_ERR_CUDA && ce != cudaSuccess) m += std::string(" (") + cudaGetErrorString(ce) + ")";
        return set_error(rc, m);
    }
    return RMS_OK;
}

int rms_split_variant(int k, int* block, int* min_blocks_per_sm) {
    if (k < 1 || k > split_variant_count()) return set_error(RMS_ERR_ARG, "no such variant");
    if (block) *block = split_variant_block(k - 1);
    if (min_blocks_per_sm) *min_blocks_per_sm = split_variant_minb(k - 1);
    return RMS_OK;
}

int rms_sim_create(const rms_config* cfg, rms_sim** out) {
    if (!cfg || !out) return set_error(RMS_ERR_ARG, "null argument");
    *out = nullptr;
    auto* s = new (std::nothrow) rms_sim();
    if (!s) return set_error(RMS_ERR_NOMEM, "out of host memory");
    s->mode = cfg->mode;
    s->dt = cfg->dt;
    s->tn = cfg->tn;
    s->npar = cfg->npar;
    s->nc = cfg->nc;
    s->res = cfg->res;
    s->n1 = cfg->n1; s->n2 = cfg->n2; s->n3 = cfg->n3;
    auto copy = [](const double* p, size_t n, std::vector<double>& v) -> bool {
        if (n && !p) return false;
        v.assign(p, p + n);
        return true;
    };
    const int nc = cfg->nc > 0 ? cfg->nc : 0;
    bool ok = copy(cfg->diffusivity, nc, s->diffusivity) && copy(cfg->t2, nc, s->t2);
    if (cfg->mode == RMS_MODE_NARROW) {
        ok = ok && cfg->nbvec >= 0 && copy(cfg->bval, cfg->nbvec, s->bval) &&
             copy(cfg->bvec, (size_t)cfg->nbvec * 3, s->bvec);
    } else if (cfg->mode == RMS_MODE_PGSE) {
        ok = ok && cfg->ngrad >= 0 && copy(cfg->grad, (size_t)cfg->ngrad * 6, s->grad);
    } else if (cfg->mode == RMS_MODE_WAVEFORM) {
        ok = ok && cfg->nwave >= 0 && cfg->nbins >= 0 &&
             copy(cfg->wave, (size_t)cfg->nwave * cfg->nbins * 3, s->wave);
        s->nwave = cfg->nwave;
        s->nbins = cfg->nbins;
    }
    if (cfg->permeation == RMS_PERM_TABLE) ok = ok && copy(cfg->pij, (size_t)nc * nc, s->pij_in);
    if (!ok) { delete s; return set_error(RMS_ERR_ARG, "missing array for a non-zero count"); }
    s->timepoints = cfg->timepoints;
    s->nite = cfg->nite;
    s->boundary = cfg->boundary;
    s->permeation = cfg->permeation;
    s->kappa = cfg->kappa;
    s->rule = cfg->membrane_rule;
    int rc = finalize_config(s);
    if (rc) { delete s; return rc; }
    *out = s;
    return RMS_OK;
}

int rms_sim_load_dir(const char* dir, int mode, rms_sim** out) {
    if (!dir || !out) return set_error(RMS_ERR_ARG, "null argument");
    *out = nullptr;
    auto* s = new (std::nothrow) rms_sim();
    if (!s) return set_error(RMS_ERR_NOMEM, "out of host memory");
    int rc = load_run_dir(dir, mode, s);
    if (rc == RMS_OK) rc = validate_lattice(s->labels.data(), s->labels.size(), s->nc);
    if (rc) { delete s; return rc; }
    *out = s;
    return RMS_OK;
}


int rms_sim_set_lattice(rms_sim* s, const uint8_t* labels, int n1, int n2, int n3) {
    if (!s || !labels) return set_error(RMS_ERR_ARG, "null argument");
    if (n1 != s->n1 || n2 != s->n2 || n3 != s->n3) {
        std::ostringstream m;
        m << "lattice " << n1 << "x" << n2 << "x" << n3 << " does not match the configured "
          << s->n1 << "x" << s->n2 << "x" << s->n3;
        return set_error(RMS_ERR_ARG, m.str());
    }
    const size_t n = (size_t)n1 * n2 * n3;
    // A simulation that has run has its device: the lattice goes up straight
    // from the caller's buffer (a DMA when it is pinned) into a staging buffer
    // and is checked there by one GPU pass; only a lattice that passes becomes
    // the simulation's device lattice, and the host copy is brought up to date
    // only if a later call needs it.  Without a device, the lattice is checked
    // and copied on the host.  Either way a rejected lattice leaves the
    // simulation's own as it was, and the call returns once the caller's
    // buffer is no longer read.
    if (s->dev) {
        int rc = set_lattice_on_device(s, labels, n);
        if (rc != kNoDevicePath) return rc;
    }
    int rc = validate_lattice(labels, n, s->nc);
    if (rc) return rc;
    s->labels.resize(n);
    uint8_t* dst = s->labels.data();
    host_parallel(n, [&](size_t lo, size_t hi, int) { std::memcpy(dst + lo, labels + lo, hi - lo); });
    s->have_lattice = true;
    s->lattice_dirty = true;
    s->host_stale = false;
    return RMS_OK;
}

int rms_adjoint_run(rms_sim* s, const rms_run_opts* opts, const double* g_sigw, rms_adjoint_grads* out) {
    if (!s || !out) return set_error(RMS_ERR_ARG, "null argument");
    if (opts && opts->precision != RMS_PREC_SPLIT) return set_error(RMS_ERR_ARG, "the adjoint walks the SPLIT walk");
    if (opts && opts->traj_out) return set_error(RMS_ERR_ARG, "the adjoint writes no trajectory");
    return run_adjoint(s, opts, g_sigw, out, nullptr);
}

int rms_adjoint_jacobian(rms_sim* s, const rms_run_opts* opts, double* jac, double* sigw) {
    if (!s || !jac) return set_error(RMS_ERR_ARG, "null argument");
    if (opts && opts->precision != RMS_PREC_SPLIT) return set_error(RMS_ERR_ARG, "the adjoint walks the SPLIT walk");
    if (opts && opts->traj_out) return set_error(RMS_ERR_ARG, "the adjoint writes no trajectory");
    rms_adjoint_grads g{};
    g.sigw = sigw;
    return run_adjoint(s, opts, nullptr, &g, jac);
}

int rms_sim_run(rms_sim* s, const rms_run_opts* opts) {
    if (!s) return set_error(RMS_ERR_ARG, "null sim");
    try {
        return run_one(s, opts);
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

int rms_sim_set_tube_lattice(rms_sim* s, const double* r2, const double* cx, const double* cy, int inside,
                             int outside, int device) {
    if (!s || !r2 || !cx || !cy) return set_error(RMS_ERR_ARG, "null argument");
    if (inside < 0 || inside >= s->nc || outside < 0 || outside >= s->nc)
        return set_error(RMS_ERR_RANGE, "labels must be below Nc");
    if (inside == 0 && outside == 0) return set_error(RMS_ERR_RANGE, "a lattice needs labelled voxels");
    try {
        int rc = ensure_device(s, device);
        if (rc) return rc;
        rms_device_state* d = s->dev;
        RMS_CUDA(cudaSetDevice(device));
        cudaStream_t st = d->own;
        const size_t nvox = (size_t)s->n1 * s->n2 * s->n3;
        std::vector<double> tab;
        tab.insert(tab.end(), r2, r2 + s->n3);
        tab.insert(tab.end(), cx, cx + s->n3);
        tab.insert(tab.end(), cy, cy + s->n3);
        RMS_CUDA(upload(d->tables, tab, st));
        RMS_CUDA(d->labels.ensure(nvox));
        const double* t = d->tables.as<double>();
        int e = build_tube_lattice(d->labels.as<uint8_t>(), s->n1, s->n2, s->n3, s->res, t, t + s->n3, t + 2 * s->n3,
                                   (uint8_t)inside, (uint8_t)outside, st);
        if (e) return cuda_fail((cudaError_t)e, "lattice kernel launch");
        s->labels.resize(nvox);
        RMS_CUDA(cudaMemcpyAsync(s->labels.data(), d->labels.p, nvox, cudaMemcpyDeviceToHost, st));
        RMS_CUDA(cudaStreamSynchronize(st));
        size_t nonzero = 0;
        for (size_t i = 0; i < nvox; ++i) nonzero += s->labels[i] != 0;
        if (nonzero == 0) return set_error(RMS_ERR_RANGE, "the lattice has no labelled voxel");
        // the device already holds these labels; the packed form is rebuilt at the next run
        s->have_lattice = true;
        s->lattice_dirty = false;
        s->host_stale = false;
        d->labels_bytes = nvox;
        d->packed_valid = false;
        return RMS_OK;
    } catch (const std::exception& ex) {
        return set_error(RMS_ERR_NOMEM, ex.what());
    }
}

int rms_sim_cumulants(const rms_sim* s, const double* dirs, int ndir, double* D, double* K) {
    if (!s || !D || !K) return set_error(RMS_ERR_ARG, "null argument");
    if (!s->have_results) return set_error(RMS_ERR_STATE, "no results: run the simulation first");
    static const double axes[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (!dirs) {
        dirs = axes;
        ndir = 3;
    }
    if (ndir < 1) return set_error(RMS_ERR_ARG, "ndir must be >= 1");
    // readRMS.m:13-18: tensor multiplicities and index lists of dx2 / dx4
    static const double dcnt[6] = {1, 2, 2, 1, 2, 1};
    static const double wcnt[15] = {1, 4, 4, 6, 12, 6, 4, 12, 12, 4, 1, 4, 6, 4, 1};
    static const int dind[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    static const int wind[15][4] = {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 0, 2}, {0, 0, 1, 1}, {0, 0, 1, 2},
                                    {0, 0, 2, 2}, {0, 1, 1, 1}, {0, 1, 1, 2}, {0, 1, 2, 2}, {0, 2, 2, 2},
                                    {1, 1, 1, 1}, {1, 1, 1, 2}, {1, 1, 2, 2}, {1, 2, 2, 2}, {2, 2, 2, 2}};
    const int T = s->timepoints;
    for (int q = 0; q < ndir; ++q) {
        const double* n = dirs + 3 * q;
        double n2[6], n4[15];
        for (int i = 0; i < 6; ++i) n2[i] = n[dind[i][0]] * n[dind[i][1]];
        for (int i = 0; i < 15; ++i) n4[i] = n[wind[i][0]] * n[wind[i][1]] * n[wind[i][2]] * n[wind[i][3]];
        for (int t = 0; t < T; ++t) {
            // readRMS.m:44-45 (normalise by sig0 with multiplicities), :96-103 (D, K)
            double x2 = 0.0, x4 = 0.0;
            for (int i = 0; i < 6; ++i) x2 += s->dx2[(size_t)t * 6 + i] * dcnt[i] / s->sig0[t] * n2[i];
            for (int i = 0; i < 15; ++i) x4 += s->dx4[(size_t)t * 15 + i] * wcnt[i] / s->sig0[t] * n4[i];
            D[(size_t)t * ndir + q] = x2 / 2.0 / s->td[t];
            K[(size_t)t * ndir + q] = x4 / (x2 * x2) - 3.0;
        }
    }
    return RMS_OK;
}

int rms_combine_cumulants(int naxons, int T, int ndir, const double* f, const double* Din, const double* Kin,
                          double* D, double* K) {
    if (naxons < 1 || T < 1 || ndir < 1 || !f || !Din || !Kin || !D || !K) return set_error(RMS_ERR_ARG, "bad argument");
    const size_t m = (size_t)T * ndir;
    for (size_t i = 0; i < m; ++i) {
        // part1_demo4_analysis.m:88-90
        double d = 0.0, d2 = 0.0, d2k = 0.0;
        for (int a = 0; a < naxons; ++a) {
            const double di = Din[(size_t)a * m + i];
            d += f[a] * di;
            d2 += f[a] * di * di;
            d2k += f[a] * di * di * Kin[(size_t)a * m + i];
        }
        D[i] = d;
        K[i] = 3.0 * (d2 - d * d) / (d * d) + d2k / (d * d);
    }
    return RMS_OK;
}

int rms_batch_graph_create(rms_sim* const* sims, int n, const rms_run_opts* opts, rms_graph** out) {
    if (!sims || n < 1 || !out) return set_error(RMS_ERR_ARG, "null argument");
    for (int i = 0; i < n; ++i)
        if (!sims[i]) return set_error(RMS_ERR_ARG, "null simulation in the batch");
    *out = nullptr;
    try {
        return graph_create(sims, n, opts, out);
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

int rms_graph_run(rms_graph* g, uint64_t seed) {
    if (!g) return set_error(RMS_ERR_ARG, "null graph");
    try {
        return graph_run(g, seed);
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

void rms_graph_destroy(rms_graph* g) { delete g; }

int rms_autotune(rms_sim* const* sims, int n, const rms_run_opts* opts, int* variant, double* variant_ms) {
    if (!sims || n < 1 || !variant) return set_error(RMS_ERR_ARG, "null argument");
    for (int i = 0; i < n; ++i)
        if (!sims[i]) return set_error(RMS_ERR_ARG, "null simulation in the batch");
    try {
        return autotune(sims, n, opts, variant, variant_ms);
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

int rms_batch_run(rms_sim* const* sims, int n, const rms_run_opts* opts) {
    if (!sims || n < 0) return set_error(RMS_ERR_ARG, "null argument");
    for (int i = 0; i < n; ++i)
        if (!sims[i]) return set_error(RMS_ERR_ARG, "null simulation in the batch");
    if (n == 0) return RMS_OK;
    const int prec = opts ? opts->precision : RMS_PREC_COMPAT;
    const uint64_t seed = opts ? opts->seed : 0;
    try {
        if (prec == RMS_PREC_SPLIT) {
            // one persistent launch over all simulations
            std::vector<LaunchJob> jobs;
            for (int i = 0; i < n; ++i) {
                int64_t w0 = 0, w1 = 0;
                int rc = batch_range(sims[i], opts, w0, w1);
                if (rc) return rc;
                jobs.push_back(LaunchJob{sims[i], w0, w1, seed + (uint64_t)i * kBatchSeedStep});
            }
            return run_launch(jobs, opts);
        }
        for (int i = 0; i < n; ++i) {
            rms_run_opts oi = opts ? *opts : rms_run_opts{};
            oi.seed = seed + (uint64_t)i * kBatchSeedStep;
            oi.walker_begin = oi.walker_end = 0;
            int rc = run_one(sims[i], &oi);
            if (rc) {
                std::ostringstream m;
                m << "simulation " << i << ": " << g_last_error;
                return set_error(rc, m.str());
            }
        }
        return RMS_OK;
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

int rms_sim_field_size(const rms_sim* s, int field, size_t* n) {
    if (!s || !n) return set_error(RMS_ERR_ARG, "null argument");
    if (!field_size(s, field, *n)) return set_error(RMS_ERR_ARG, "unknown field");
    return RMS_OK;
}

int rms_sim_get(const rms_sim* s, int field, double* out, size_t n) {
    if (!s || (!out && n)) return set_error(RMS_ERR_ARG, "null argument");
    size_t want = 0;
    if (!field_size(s, field, want)) return set_error(RMS_ERR_ARG, "unknown field");
    if (n != want) {
        std::ostringstream m;
        m << "field holds " << want << " values, buffer has " << n;
        return set_error(RMS_ERR_ARG, m.str());
    }
    const std::vector<double>* table = nullptr;
    if (field == RMS_FIELD_TD) table = &s->td;
    if (field == RMS_FIELD_DIFFUSIVITY) table = &s->diffusivity;
    if (field == RMS_FIELD_STEP) table = &s->step;
    if (field == RMS_FIELD_PIJ) table = &s->pij;
    if (field == RMS_FIELD_BVAL) table = &s->bval;
    if (field == RMS_FIELD_BVEC) table = &s->bvec;
    if (field == RMS_FIELD_GRAD) table = &s->grad;
    if (field == RMS_FIELD_SIM_PARA) {
        out[0] = s->dt;
        out[1] = (double)s->tn;
        out[2] = (double)s->npar;
        out[3] = s->res;
        return RMS_OK;
    }
    if (table) {
        std::copy(table->begin(), table->begin() + want, out);
        return RMS_OK;
    }
    if (!s->have_results) return set_error(RMS_ERR_STATE, "no results: run the simulation first");
    const std::vector<double>* v = nullptr;
    switch (field) {
        case RMS_FIELD_SIG0: v = &s->sig0; break;
        case RMS_FIELD_DX2: v = &s->dx2; break;
        case RMS_FIELD_DX4: v = &s->dx4; break;
        case RMS_FIELD_SIGRE: v = &s->sigre; break;
        case RMS_FIELD_SIG: v = &s->sig; break;
        case RMS_FIELD_NPAR_COUNT: v = &s->npar_count; break;
        case RMS_FIELD_SIGW: v = &s->sigw; break;
    }
    std::copy(v->begin(), v->end(), out);
    return RMS_OK;
}

int rms_sim_get_trace(const rms_sim* s, int32_t* init_voxel, int32_t* voxel, uint32_t* events,
                      size_t nwalkers, size_t tn) {
    if (!s || !init_voxel || !voxel || !events) return set_error(RMS_ERR_ARG, "null argument");
    if (!s->have_results || s->trace_n == 0) return set_error(RMS_ERR_STATE, "the last run kept no traces");
    if (nwalkers != (size_t)s->trace_n || tn != (size_t)s->tn)
        return set_error(RMS_ERR_ARG, "trace buffer shape differs from the last run");
    std::copy(s->tr_init.begin(), s->tr_init.end(), init_voxel);
    std::copy(s->tr_vox.begin(), s->tr_vox.end(), voxel);
    std::copy(s->tr_ev.begin(), s->tr_ev.end(), events);
    return RMS_OK;
}

int rms_sim_get_trace_positions(const rms_sim* s, double* pos, size_t nwalkers, size_t tn) {
    if (!s || !pos) return set_error(RMS_ERR_ARG, "null argument");
    if (!s->have_results || s->trace_n == 0) return set_error(RMS_ERR_STATE, "the last run kept no traces");
    if (nwalkers != (size_t)s->trace_n || tn != (size_t)s->tn)
        return set_error(RMS_ERR_ARG, "trace buffer shape differs from the last run");
    std::copy(s->tr_pos.begin(), s->tr_pos.end(), pos);
    return RMS_OK;
}

int rms_sim_write_dir(const rms_sim* s, const char* dir) {
    if (!s || !dir) return set_error(RMS_ERR_ARG, "null argument");
    return write_run_dir(s, dir);
}

int rms_sim_last_timing(const rms_sim* s, double* walk_ms, double* run_ms) {
    if (!s) return set_error(RMS_ERR_ARG, "null sim");
    if (!s->have_timing) return set_error(RMS_ERR_STATE, "no run yet");
    if (walk_ms) *walk_ms = s->walk_ms;
    if (run_ms) *run_ms = s->run_ms;
    return RMS_OK;
}

void rms_sim_destroy(rms_sim* s) {
    if (!s) return;
    delete s->dev;
    delete s;
}

int rms_rng_doubles(uint64_t seed, uint64_t walker, int n, double* out) {
    if (n < 0 || (n && !out)) return set_error(RMS_ERR_ARG, "bad buffer");
    DoubleStream r;
    r.init(seed, walker);
    for (int i = 0; i < n; ++i) out[i] = r.next();
    return RMS_OK;
}

int rms_rng_floats(uint64_t seed, uint64_t walker, int n, float* out) {
    if (n < 0 || (n && !out)) return set_error(RMS_ERR_ARG, "bad buffer");
    FloatStream r;
    r.init(seed, walker);
    for (int i = 0; i < n; ++i) out[i] = r.next();
    return RMS_OK;
}

int rms_rng_split(uint64_t seed, uint64_t walker, int domain, int n, float* out) {
    if (n < 0 || (n && !out)) return set_error(RMS_ERR_ARG, "bad buffer");
    if (domain < 0 || domain > 2) return set_error(RMS_ERR_ARG, "domain must be 0, 1 or 2");
    if (domain == (int)kDomDir) {
        // step i's pair: fields 2(i % 3), 2(i % 3) + 1 of block i / 3
        for (int i = 0; 2 * i < n; ++i) {
            float u[6];
            dir_fields(dir_block((uint32_t)(i / 3), (uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)walker,
                                 (uint32_t)(walker >> 32)), u);
            out[2 * i] = u[2 * (i % 3)];
            if (2 * i + 1 < n) out[2 * i + 1] = u[2 * (i % 3) + 1];
        }
        return RMS_OK;
    }
    DomainStream r;
    r.init(seed, walker, (uint32_t)domain);
    for (int i = 0; i < n; ++i) out[i] = r.next();
    return RMS_OK;
}

int rms_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    if (!ctr || !key || !out) return set_error(RMS_ERR_ARG, "null argument");
    const U4 r = philox4x32_10(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
    return RMS_OK;
}

}  // extern "C"

// rms_noalloc.cu -- the split-precision walk for callers that cannot allocate
// device memory.
//
// Who needs this: a host application whose device memory is entirely owned by
// its own allocator (a framework memory pool, a fixed pre-reserved budget), so
// a library may not take memory behind its back; and code that must never hit
// cudaMalloc/cudaFree, which synchronise the whole device and would stall
// work the caller keeps in flight on other streams.  rms_sim_run_noalloc asks
// nothing of the allocator: the caller hands in the lattice and the output
// buffers (device memory it already owns), and every scratch buffer the walk
// needs -- per-warp accumulator rows, PGSE window sums, tables, the error word
// -- is carved out of one file-scope device array of fixed size,
// RMS_NOALLOC_SCRATCH_BYTES, which each GPU that loads the library holds until
// the process exits.
//
// The kernels are the library's own split walk and ordered reduction
// (rms_walk_split.cu, rms_reduce.cu), launched on that scratch.  The grid is
// sized so the per-warp rows fit in the scratch; a job whose fixed tables or
// single block of rows do not fit is refused with RMS_ERR_RANGE.  The walk
// reads the same padded, packed lattice as rms_sim_run (4 bits per voxel with
// the free-flight flags, Nc <= 7), built in the scratch too: 68 MB for
// 256x256x2048.  Same lattice, same kernel, same walkers: the results equal
// rms_sim_run's up to the order of the final sums.  The caller's lattice is
// checked on the device first (labels below Nc, enough labelled voxels), as
// rms_sim_set_lattice checks a host lattice.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in).  The first call on each device, with that
// device current, looks the address up with cudaGetSymbolAddress and keeps it;
// make that first call before any stream capture begins.  All calls share the
// one array and it keeps the last call's contents: each call clears what must
// start at zero, and calls that overlap on the GPU (two streams, two host
// threads) race on it -- serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <sstream>

#include "philox.cuh"
#include "rms_internal.h"
#include "rms_sim.h"

namespace rms {
namespace {

constexpr size_t kScratchBytes = RMS_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr int kVariant = 0;   // 256 threads, >= 4 resident blocks per SM
constexpr int kNoallocNc = 7;  // compartments of the 4-bit packed lattice (label 7 is the wall code)
constexpr int kTabMax = 2 * kNoallocNc + kNoallocNc * kNoallocNc;   // step, T2, Pij

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (looked up once).
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return set_error(RMS_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(RMS_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                               cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return RMS_OK;
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Bump allocator over the scratch array (offsets only; nothing is allocated).
struct Carve {
    unsigned char* base;
    size_t used = 0;
    template <class T> T* take(size_t count) {
        T* p = reinterpret_cast<T*>(base + used);
        used += align256(std::max<size_t>(count, 1) * sizeof(T));
        return p;
    }
};

template <class T>
cudaError_t put(T* dst, const T* src, size_t count, cudaStream_t st) {
    if (!count) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, st);
}

}  // namespace
}  // namespace rms

using namespace rms;

extern "C" int rms_sim_run_noalloc(const rms_sim* s, const rms_run_opts* o, const uint8_t* d_labels,
                                   double* d_rows, double* d_sig) {
    if (!s || !o || !d_labels || !d_rows) return set_error(RMS_ERR_ARG, "null argument");
    if (s->mode == RMS_MODE_WAVEFORM) return set_error(RMS_ERR_ARG, "the no-allocation walk records narrow-pulse and PGSE runs");
    if (s->rule != RMS_RULE_REFLECT) return set_error(RMS_ERR_ARG, "the no-allocation walk reflects at membranes");
    if (o->traj_out) return set_error(RMS_ERR_ARG, "the no-allocation walk writes no trajectory");
    if (s->mode == RMS_MODE_PGSE && !d_sig) return set_error(RMS_ERR_ARG, "PGSE needs the sig buffer");
    if (s->nc > kNoallocNc) return set_error(RMS_ERR_RANGE, "the no-allocation walk supports Nc <= 7");
    cudaError_t e = cudaSetDevice(o->device);
    if (e != cudaSuccess) return set_error(RMS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    unsigned char* base = nullptr;
    int rc = scratch_address(o->device, &base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)o->stream;

    int64_t w0 = 0, w1 = 0;
    rc = walker_range(s, o, w0, w1);
    if (rc) return rc;
    if (w0 == w1) return set_error(RMS_ERR_ARG, "the call's shard holds no walkers");

    const int T = s->timepoints, nc = s->nc, nb = s->nbvec(), ngrad = s->ngrad();
    const int nvals = (s->mode == RMS_MODE_NARROW) ? kRowHead + ((nb + 31) / 32) * 32 : kRowHead;
    const int ngrad_pad = std::max(32, ((ngrad + 31) / 32) * 32);
    const size_t row = (size_t)T * nvals;
    const int block = split_variant_block(kVariant);
    const int warps_per_block = block / 32;

    // fixed part of the scratch
    const int bits = split_lattice_bits(nc);
    const size_t lat_bytes = padded_lattice_bytes(s->n1, s->n2, s->n3, bits);
    const size_t fixed = align256(lat_bytes) + align256(sizeof(AxonDesc)) + align256(sizeof(int)) + align256(sizeof(double) * (2 * nc + nc * nc)) +
                         align256(sizeof(float) * (2 * nc + nc * nc)) + align256(sizeof(double) * s->qtab.size()) +
                         align256(sizeof(double) * s->bvec.size()) + align256(sizeof(double) * s->grad.size()) +
                         align256(sizeof(int) * s->gpair.size()) + align256(sizeof(int) * s->ev_step.size()) +
                         align256(sizeof(int) * s->ev_pair.size()) + align256(sizeof(double) * s->ev_coef.size()) +
                         align256(2 * sizeof(unsigned long long)) + 256;
    // per block: its warps' rows, PGSE signal rows and per-thread window sums
    const size_t per_block = (size_t)warps_per_block * row * sizeof(double) +
                             (s->mode == RMS_MODE_PGSE ? (size_t)warps_per_block * ngrad_pad * sizeof(double) +
                                                             (size_t)s->npairs * 3 * block * sizeof(double)
                                                       : 0);
    if (fixed + per_block + 3 * 256 > kScratchBytes) {
        std::ostringstream m;
        m << "job needs " << (fixed + per_block) << " bytes of scratch for one block; the no-allocation walk has "
          << kScratchBytes << " (fewer timepoints, b-values or PGSE timing pairs fit)";
        return set_error(RMS_ERR_RANGE, m.str());
    }
    int dev_sms = 0;
    e = cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, o->device);
    if (e != cudaSuccess) return set_error(RMS_ERR_CUDA, cudaGetErrorString(e));
    const int per_sm = walk_split_blocks_per_sm(nc, bits, kVariant);
    if (per_sm <= 0) return set_error(RMS_ERR_CUDA, "occupancy query failed");
    const int64_t ntiles = (w1 - w0 + 31) / 32;
    int64_t grid64 = std::min<int64_t>((int64_t)dev_sms * per_sm, (ntiles + warps_per_block - 1) / warps_per_block);
    grid64 = std::min<int64_t>(grid64, (int64_t)((kScratchBytes - fixed - 3 * 256) / per_block));
    const int grid = (int)std::max<int64_t>(grid64, 1);
    const int nthr = grid * block, nslots = nthr / 32;

    Carve c{base};
    uint8_t* d_lat = c.take<uint8_t>(lat_bytes);
    AxonDesc* d_axon = c.take<AxonDesc>(1);
    int* d_err = c.take<int>(1);
    unsigned long long* d_counts = c.take<unsigned long long>(2);
    double* d_tab = c.take<double>(2 * nc + nc * nc);
    float* d_tabf = c.take<float>(2 * nc + nc * nc);
    double* d_qtab = c.take<double>(s->qtab.size());
    double* d_bvec = c.take<double>(s->bvec.size());
    double* d_grad = c.take<double>(s->grad.size());
    int* d_gpair = c.take<int>(s->gpair.size());
    int* d_evs = c.take<int>(s->ev_step.size());
    int* d_evp = c.take<int>(s->ev_pair.size());
    double* d_evc = c.take<double>(s->ev_coef.size());
    double* d_slots = c.take<double>((size_t)nslots * row);
    double* d_sigslots = c.take<double>(s->mode == RMS_MODE_PGSE ? (size_t)nslots * ngrad_pad : 1);
    double* d_vscr = c.take<double>(s->mode == RMS_MODE_PGSE ? (size_t)s->npairs * 3 * nthr : 1);
    if (c.used > kScratchBytes) return set_error(RMS_ERR_RANGE, "no-allocation scratch overflow");

    // tables (FP64 and FP32 copies built on the stack: Nc <= kNoallocNc)
    double tab[kTabMax];
    float tabf[kTabMax];
    for (int i = 0; i < nc; ++i) {
        tab[i] = s->step[i];
        tab[nc + i] = s->t2_steps[i];
        tabf[i] = (float)s->step[i];
        tabf[nc + i] = (float)(1.0 / s->t2_steps[i]);
    }
    for (int i = 0; i < nc * nc; ++i) {
        tab[2 * nc + i] = s->pij[i];
        tabf[2 * nc + i] = (float)s->pij[i];
    }
    if ((e = put(d_tab, tab, 2 * nc + nc * nc, st)) != cudaSuccess ||
        (e = put(d_tabf, tabf, 2 * nc + nc * nc, st)) != cudaSuccess ||
        (e = put(d_qtab, s->qtab.data(), s->qtab.size(), st)) != cudaSuccess ||
        (e = put(d_bvec, s->bvec.data(), s->bvec.size(), st)) != cudaSuccess ||
        (e = put(d_grad, s->grad.data(), s->grad.size(), st)) != cudaSuccess ||
        (e = put(d_gpair, s->gpair.data(), s->gpair.size(), st)) != cudaSuccess ||
        (e = put(d_evs, s->ev_step.data(), s->ev_step.size(), st)) != cudaSuccess ||
        (e = put(d_evp, s->ev_pair.data(), s->ev_pair.size(), st)) != cudaSuccess ||
        (e = put(d_evc, s->ev_coef.data(), s->ev_coef.size(), st)) != cudaSuccess)
        return set_error(RMS_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
    AxonDesc axon;
    fill_axon_desc(axon, s, w0, w1, 0, o->seed, d_lat);
    if ((e = put(d_axon, &axon, 1, st)) != cudaSuccess)
        return set_error(RMS_ERR_CUDA, std::string("axon upload: ") + cudaGetErrorString(e));
    // what must start at zero: error word and the accumulator rows
    if ((e = cudaMemsetAsync(d_err, 0, sizeof(int), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(d_slots, 0, (size_t)nslots * row * sizeof(double), st)) != cudaSuccess ||
        (s->mode == RMS_MODE_PGSE &&
         (e = cudaMemsetAsync(d_sigslots, 0, (size_t)nslots * ngrad_pad * sizeof(double), st)) != cudaSuccess))
        return set_error(RMS_ERR_CUDA, std::string("scratch clear: ") + cudaGetErrorString(e));

    // the lattice is the caller's device memory: check it before walking it (a
    // label >= Nc would index the compartment tables past their Nc entries)
    const size_t nvox = (size_t)s->n1 * s->n2 * s->n3;
    unsigned long long hcount[2] = {0, 0};
    if ((e = cudaMemsetAsync(d_counts, 0, sizeof(hcount), st)) != cudaSuccess)
        return set_error(RMS_ERR_CUDA, std::string("scratch clear: ") + cudaGetErrorString(e));
    if ((e = (cudaError_t)check_labels(d_labels, nvox, (unsigned)nc, d_counts, dev_sms, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hcount, d_counts, sizeof(hcount), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return set_error(RMS_ERR_CUDA, std::string("lattice check: ") + cudaGetErrorString(e));
    if (hcount[0]) {
        std::ostringstream m;
        m << hcount[0] << " voxel(s) of the device lattice carry a label that is not below Nc = " << nc;
        return set_error(RMS_ERR_RANGE, m.str());
    }
    if (hcount[1] == 0) return set_error(RMS_ERR_RANGE, "lattice has no voxel with a non-zero label");
    if ((double)hcount[1] / (double)nvox < 1e-7)
        return set_error(RMS_ERR_RANGE, "labelled voxels are below 1e-7 of the lattice; "
                                        "rejection-sampled initial positions would not finish");

    int pe = pack_lattice_padded(d_labels, s->n1, s->n2, s->n3, bits, s->boundary == RMS_BOUNDARY_MIRROR ? 1 : 0,
                                 d_lat, st);
    if (pe) return set_error(RMS_ERR_CUDA, std::string("lattice packing: ") + cudaGetErrorString((cudaError_t)pe));

    WalkArgs a{};
    a.labels = d_labels;
    a.n1 = s->n1; a.n2 = s->n2; a.n3 = s->n3;
    a.walker_begin = w0; a.walker_end = w1;
    a.tn = s->tn; a.tstep = s->tstep; a.timepoints = T; a.nite = s->nite; a.nc = nc;
    a.boundary = s->boundary; a.mode = s->mode;
    a.res = s->res; a.dt = s->dt;
    a.seed = o->seed;
    a.step = d_tab; a.t2 = d_tab + nc; a.pij = d_tab + 2 * nc;
    a.stepf = d_tabf; a.t2invf = d_tabf + nc; a.pijf = d_tabf + 2 * nc;
    a.nvals = nvals;
    a.slots = d_slots;
    a.nbvec = nb; a.qtab = d_qtab; a.bvec = d_bvec;
    a.ngrad = ngrad; a.ngrad_pad = ngrad_pad; a.npairs = s->npairs; a.nevents = (int)s->ev_step.size();
    a.ev_step = d_evs; a.ev_pair = d_evp; a.ev_coef = d_evc;
    a.grad = d_grad; a.gpair = d_gpair;
    a.vscr = d_vscr;
    a.sig_slots = d_sigslots;
    a.err = d_err;
    a.axons = d_axon;
    a.axon0 = axon;
    a.naxons = 1;
    a.ntiles = ntiles;

    int ke = launch_walk_split(a, bits, kVariant, grid, st);
    if (ke) return set_error(RMS_ERR_CUDA, std::string("walk launch: ") + cudaGetErrorString((cudaError_t)ke));
    ke = launch_reduce_slots(d_slots, nslots, row, d_rows, st);
    if (!ke && s->mode == RMS_MODE_PGSE) ke = launch_reduce_slots(d_sigslots, nslots, (size_t)ngrad_pad, d_sig, st);
    if (ke) return set_error(RMS_ERR_CUDA, std::string("reduce launch: ") + cudaGetErrorString((cudaError_t)ke));
    int herr = 0;
    if ((e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return set_error(RMS_ERR_CUDA, std::string("no-allocation walk: ") + cudaGetErrorString(e));
    if (herr & kErrInitCap)
        return set_error(RMS_ERR_RANGE, "a walker found no labelled voxel within the rejection-sampling cap");
    if (herr & kErrStep) return set_error(RMS_ERR_RANGE, "a step segment found no voxel face");
    return RMS_OK;
}

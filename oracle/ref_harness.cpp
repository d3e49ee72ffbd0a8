/*
 * oracle/ref_harness.cpp -- TEST INFRASTRUCTURE (the oracle).
 *
 * Drives the reference simulator's own kernels (hpc_code/lib/main.cu:63-384
 * `propagate`, hpc_code/lib/main_PGSE.cu:65-410 `propagate`), compiled for
 * the host through oracle/ref_shim/, in two ways:
 *
 *  - ref_narrow_main_dir / ref_pgse_main_dir: the reference's whole program
 *    (its main(): file parsing, tables, launch, output writing) run in a run
 *    directory, exactly as `./main_cuda` would be (part1_demo3_simulation.m:86-90).
 *  - ref_run_narrow / ref_run_pgse: the reference's `propagate` on walkers
 *    [0, nsample) of an NPar-walker job, spread over OpenMP threads.  Each
 *    thread owns a contiguous walker range and private accumulators; the
 *    private sums are added in thread order, so a run is repeatable.  This
 *    is the timed CPU baseline (one walker = one reference "thread",
 *    RNG subsequence = walker id, as main.cu:58-61 + 64-70 arrange it).
 *
 * Built by oracle/Makefile into oracle/_ref/.
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <unistd.h>
#include <omp.h>
#include "ref_shim/rms_ref_shim.hpp"

thread_local _shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

void ref_narrow_main(int argc, char* argv[]);
void ref_pgse_main(int argc, char* argv[]);

void ref_narrow_propagate(curandStatePhilox4_32_10_t* state, double* sig0, double* dx2,
                          double* dx4, double* sigRe, double* NPar_count, const double* TD,
                          const int TN, const int NPar, const int Nbvec, const int Nc,
                          const double res, const double* step, const int NPix1,
                          const int NPix2, const int NPix3, const double* T2,
                          const double* Pij, const double* bval, const double* bvec,
                          const int* APix);

void ref_pgse_propagate(curandStatePhilox4_32_10_t* state, double* sig0, double* dx2,
                        double* dx4, double* sig, double* NPar_count, const int TN,
                        const int NPar, const int Nc, const double res, const double dt,
                        const double* step, const int NPix1, const int NPix2,
                        const int NPix3, const int Ngrad, const double* grad,
                        const double* T2, const double* Pij, const int* APix);

namespace {
int run_main_in_dir(void (*fn)(int, char**), const char* dir) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return -1;
    if (chdir(dir) != 0) return -2;
    char name[] = "main_cuda";
    char* argv[] = {name, nullptr};
    fn(1, argv);
    if (chdir(cwd) != 0) return -3;
    return 0;
}

constexpr int kTimepoints = 1000;   // main.cu:35

struct Acc {
    std::vector<double> sig0, dx2, dx4, sig, npar;
    Acc(int nsig, int nc)
        : sig0(kTimepoints, 0.0), dx2(kTimepoints * 6, 0.0), dx4(kTimepoints * 15, 0.0),
          sig(nsig, 0.0), npar(kTimepoints * nc, 0.0) {}
};

void add_into(std::vector<double>& dst, const std::vector<double>& src) {
    for (size_t i = 0; i < dst.size(); ++i) dst[i] += src[i];
}

/* Run body(walker, acc) for walkers [0, nsample) on nthreads threads with
 * contiguous ranges, then sum the private accumulators in thread order. */
template <class Body>
void run_parallel(int64_t nsample, int nthreads, int nsig, int nc, Body body,
                  double* sig0, double* dx2, double* dx4, double* sig, double* npar) {
    if (nthreads < 1) nthreads = 1;
    std::vector<Acc> accs;
    accs.reserve(nthreads);
    for (int t = 0; t < nthreads; ++t) accs.emplace_back(nsig, nc);
#pragma omp parallel num_threads(nthreads)
    {
        int t = omp_get_thread_num();
        int nt = omp_get_num_threads();
        int64_t lo = nsample * t / nt, hi = nsample * (t + 1) / nt;
        for (int64_t w = lo; w < hi; ++w) body(w, accs[t]);
    }
    Acc total(nsig, nc);
    for (int t = 0; t < nthreads; ++t) {
        add_into(total.sig0, accs[t].sig0);
        add_into(total.dx2, accs[t].dx2);
        add_into(total.dx4, accs[t].dx4);
        add_into(total.sig, accs[t].sig);
        add_into(total.npar, accs[t].npar);
    }
    std::memcpy(sig0, total.sig0.data(), total.sig0.size() * sizeof(double));
    std::memcpy(dx2, total.dx2.data(), total.dx2.size() * sizeof(double));
    std::memcpy(dx4, total.dx4.data(), total.dx4.size() * sizeof(double));
    if (nsig) std::memcpy(sig, total.sig.data(), total.sig.size() * sizeof(double));
    std::memcpy(npar, total.npar.data(), total.npar.size() * sizeof(double));
}

/* One reference "thread" per walker: blockDim = 1, gridDim = NPar, so
 * idx = walker and the grid-stride loop of main.cu:70 visits that walker only. */
void set_thread(int64_t walker, int npar) {
    blockDim = _shim_dim3{1, 1, 1};
    gridDim = _shim_dim3{(unsigned)npar, 1, 1};
    blockIdx = _shim_dim3{(unsigned)walker, 0, 0};
    threadIdx = _shim_dim3{0, 0, 0};
}
}  // namespace

extern "C" {

int ref_narrow_main_dir(const char* dir) { return run_main_in_dir(ref_narrow_main, dir); }
int ref_pgse_main_dir(const char* dir) { return run_main_in_dir(ref_pgse_main, dir); }

/* Tables as the reference's main() derives them (main.cu:421-458, 484-487):
 * step in voxels, T2 already divided by dt, TD[1000]. */
int ref_run_narrow(unsigned long long seed, int TN, int NPar, int64_t nsample, int Nbvec,
                   int Nc, double res, const double* step, int NPix1, int NPix2, int NPix3,
                   const double* T2, const double* Pij, const double* bval,
                   const double* bvec, const int* APix, const double* TD, int nthreads,
                   double* sig0, double* dx2, double* dx4, double* sigRe, double* npar) {
    if (nsample > NPar) return -1;
    std::vector<curandStatePhilox4_32_10_t> states((size_t)nsample);
    auto body = [&](int64_t w, Acc& a) {
        set_thread(w, NPar);
        curand_init(seed, (unsigned long long)w, 0, &states[w]);
        curandStatePhilox4_32_10_t* base = states.data();
        ref_narrow_propagate(base, a.sig0.data(), a.dx2.data(), a.dx4.data(), a.sig.data(),
                             a.npar.data(), TD, TN, NPar, Nbvec, Nc, res, step, NPix1, NPix2,
                             NPix3, T2, Pij, bval, bvec, APix);
    };
    run_parallel(nsample, nthreads, kTimepoints * Nbvec, Nc, body, sig0, dx2, dx4, sigRe, npar);
    return 0;
}

int ref_run_pgse(unsigned long long seed, int TN, int NPar, int64_t nsample, int Nc,
                 double res, double dt, const double* step, int NPix1, int NPix2, int NPix3,
                 int Ngrad, const double* grad, const double* T2, const double* Pij,
                 const int* APix, int nthreads, double* sig0, double* dx2, double* dx4,
                 double* sig, double* npar) {
    if (nsample > NPar) return -1;
    std::vector<curandStatePhilox4_32_10_t> states((size_t)nsample);
    auto body = [&](int64_t w, Acc& a) {
        set_thread(w, NPar);
        curand_init(seed, (unsigned long long)w, 0, &states[w]);
        ref_pgse_propagate(states.data(), a.sig0.data(), a.dx2.data(), a.dx4.data(),
                           a.sig.data(), a.npar.data(), TN, NPar, Nc, res, dt, step, NPix1,
                           NPix2, NPix3, Ngrad, grad, T2, Pij, APix);
    };
    run_parallel(nsample, nthreads, Ngrad, Nc, body, sig0, dx2, dx4, sig, npar);
    return 0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

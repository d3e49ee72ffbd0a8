// rms_main.cpp -- drop-in for the reference's `./main_cuda`.
//
// Run with no arguments in a run directory, as part1_demo3_simulation.m:86-90
// runs the reference: reads the same text inputs, writes the same outputs
// (hpc_code/lib/main.cu:388-621 narrow pulse; main_PGSE.cu:414-675 PGSE) and
// prints the same stdout lines, ending with "Done! Elpased time N s" (the
// reference's spelling, which analysis/read_slurm_cuda.m:9-11 parses).
//
//   rms_main [--dir D] [--pgse|--narrow] [--seed S] [--precision compat|split]
//            [--device N] [--metrics]
// --metrics adds one JSON line on stderr after the run: walker-steps, the
// walk and run kernel times (CUDA events), the wall time of the run call and
// the walker-steps/s of each (stdout stays the reference's lines).
// The mode defaults to PGSE when gradient_time.txt exists.  The seed defaults
// to 8 bytes of /dev/urandom, like the reference's /dev/random read
// (main.cu:492-496).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/rms.h"

static int fail(const char* what) {
    std::fprintf(stderr, "rms_main: %s: %s\n", what, rms_last_error());
    return 1;
}

int main(int argc, char** argv) {
    std::string dir = ".";
    int mode = RMS_MODE_AUTO;
    bool have_seed = false;
    bool metrics = false;
    unsigned long long seed = 0;
    rms_run_opts opts{};
    opts.precision = RMS_PREC_COMPAT;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](const char* name) -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "rms_main: %s needs a value\n", name); std::exit(2); }
            return argv[++i];
        };
        if (a == "--dir") dir = next("--dir");
        else if (a == "--pgse") mode = RMS_MODE_PGSE;
        else if (a == "--narrow") mode = RMS_MODE_NARROW;
        else if (a == "--seed") { seed = std::strtoull(next("--seed"), nullptr, 0); have_seed = true; }
        else if (a == "--device") opts.device = std::atoi(next("--device"));
        else if (a == "--metrics") metrics = true;
        else if (a == "--precision") {
            std::string p = next("--precision");
            if (p == "compat") opts.precision = RMS_PREC_COMPAT;
            else if (p == "split") opts.precision = RMS_PREC_SPLIT;
            else { std::fprintf(stderr, "rms_main: unknown precision %s\n", p.c_str()); return 2; }
        } else {
            std::fprintf(stderr, "usage: rms_main [--dir D] [--pgse|--narrow] [--seed S] "
                                 "[--precision compat|split] [--device N] [--metrics]\n");
            return 2;
        }
    }
    if (!have_seed) {
        FILE* f = std::fopen("/dev/urandom", "rb");
        if (!f || std::fread(&seed, sizeof seed, 1, f) != 1) { std::fprintf(stderr, "rms_main: cannot read /dev/urandom\n"); return 1; }
        std::fclose(f);
    }
    opts.seed = seed;

    rms_sim* sim = nullptr;
    if (rms_sim_load_dir(dir.c_str(), mode, &sim) != RMS_OK) return fail("loading inputs");
    size_t nc = 0;
    rms_sim_field_size(sim, RMS_FIELD_DIFFUSIVITY, &nc);
    std::vector<double> D(nc), pij(nc * nc);
    rms_sim_get(sim, RMS_FIELD_DIFFUSIVITY, D.data(), nc);
    rms_sim_get(sim, RMS_FIELD_PIJ, pij.data(), nc * nc);
    for (double d : D) std::cout << "diffusivity=" << d << std::endl;          // main.cu:425
    for (double p : pij) std::cout << "permeation probability=" << p << std::endl;  // main.cu:455

    const auto t0 = std::chrono::steady_clock::now();
    if (rms_sim_run(sim, &opts) != RMS_OK) { rms_sim_destroy(sim); return fail("simulation"); }
    const auto t1 = std::chrono::steady_clock::now();
    double walk_ms = 0, run_ms = 0;
    rms_sim_last_timing(sim, &walk_ms, &run_ms);
    const long secs = (long)std::chrono::duration<double>(t1 - t0).count();
    std::cout << "Done! Elpased time " << double(secs) << " s" << std::endl;   // main.cu:540
    if (metrics) {
        double para[4] = {0, 0, 0, 0};      // dt, TN, NPar, res
        rms_sim_get(sim, RMS_FIELD_SIM_PARA, para, 4);
        const double steps = para[1] * para[2];
        const double wall_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        std::fprintf(stderr,
                     "{\"walker_steps\": %.0f, \"precision\": \"%s\", \"seed\": %llu, \"walk_ms\": %.3f, "
                     "\"run_ms\": %.3f, \"wall_ms\": %.3f, \"walker_steps_per_s_walk\": %.6g, "
                     "\"walker_steps_per_s_wall\": %.6g}\n",
                     steps, opts.precision == RMS_PREC_SPLIT ? "split" : "compat", seed, walk_ms, run_ms, wall_ms,
                     walk_ms > 0 ? steps / (walk_ms * 1e-3) : 0.0, wall_ms > 0 ? steps / (wall_ms * 1e-3) : 0.0);
    }
    if (rms_sim_write_dir(sim, dir.c_str()) != RMS_OK) { rms_sim_destroy(sim); return fail("writing outputs"); }
    rms_sim_destroy(sim);
    return 0;
}

// cutauleaping -- command-line drop-in for the reference binary.
//
//   cutauleaping input_folder threads blocks gpu offset output_folder prefix
//                fitness force_ssa verbose
//
// Same argument contract as the reference main() (kernel.cu:74-436,
// README.md:37): N = threads*blocks simulations read from rows
// [offset, offset+N) of MX_0 / c_matrix; fitness 0 = dynamics files,
// 1 = fitness to ./pref_allfit, 2 = fitness to stdout; verbose 1 = verbose,
// 2 = dynamics to stdout.  threads/blocks fix N (and the fitness grouping);
// the launch shape is chosen by the library and never changes results.
//
// Extras through the environment (the 10-argument contract is unchanged):
//   CTL_SEED       Philox seed (default: time(NULL), like kernel.cu:176)
//   CTL_FLAGS      quirk switches (ctl.h CTL_Q*_OFF), default 0
//   CTL_EPS, CTL_NC, CTL_MAX_STEPS, CTL_GROUP, CTL_THREADS, CTL_WARP_SIMS
//   CTL_SPEC       kernels compiled for the network at run time (ctl.h
//                  ctl_run_cfg.spec): 0 library choice, 1 always, -1 never
//   CTL_OUTPUT_EXISTING_OK=1  write into an existing output folder instead of
//                  falling back to "./" (the reference falls back on any
//                  mkdir failure, tau.cu:3133-3139)
//   CTL_BINARY_OUTPUT=1  one binary file <output_folder><prefix>.ctlbin
//                  (ctl_write_samples_binary) instead of a text file per
//                  simulation
//   CTL_REPORT=<path>  a JSON run report (ctl_write_run_report): rates,
//                  step counts, per-status counts, launch shape
#include <sys/stat.h>
#include <sys/types.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <new>
#include <string>
#include <vector>

#include "../../include/ctl.h"

static void usage_exit() {
    // check_args (tau.cu:57-75)
    printf("ERROR: please specify:\n");
    printf("                       the folder which contains the model\n");
    printf("                       the number of parallel threads\n");
    printf("                       the number of blocks\n");
    printf("                       the device's number\n");
    printf("                       the offset of data for this GPU\n");
    printf("                       the output folder\n");
    printf("                       the prefix for the output files\n");
    printf("                       the type of fitness (0 to disable)\n");
    printf("       for instance: cuTauLeaping ./input 128 4 1 0 output prefix 0\n");
    exit(-1);
}

static int exit_code(ctl_status st, const char* what) {
    std::string msg = ctl_last_error();
    fprintf(stderr, "ERROR (%s): %s%s%s\n", what, ctl_status_str(st), msg.empty() ? "" : ": ", msg.c_str());
    // The reference's exit codes (tau.cu:70,246,598,630,646,1139), from the
    // status and its detail code, never from the message text.
    switch (ctl_last_error_detail()) {
        case CTL_DETAIL_ROWS_SHORT: return -4;
        case CTL_DETAIL_MX0_ROW: return -5;
        case CTL_DETAIL_MX0_UNREADABLE: return -6;
        case CTL_DETAIL_TARGET_ASSIGN: return -10;
        default: break;
    }
    if (st == CTL_ERR_OOM) return -3;
    return -1;
}

static std::string output_folder(int argc, const char* arg, bool verbose) {
    // get_output_folder (tau.cu:3114-3148)
    std::string folder = "./";
    if (argc > 3 && arg) {
        folder = arg;
        if (folder.empty() || folder.back() != '/') folder += "/";
        mode_t mask = umask(0);
        if (mkdir(folder.c_str(), S_IRWXU | S_IRGRP | S_IXGRP) != 0) {
            const char* ok = getenv("CTL_OUTPUT_EXISTING_OK");
            struct stat sb;
            bool exists = stat(folder.c_str(), &sb) == 0 && S_ISDIR(sb.st_mode);
            if (!(ok && ok[0] == '1' && exists)) {
                if (verbose) {
                    printf("ERROR: unable to create results folder %s", folder.c_str());
                    perror("");
                }
                folder = "./";
            }
        }
        umask(mask);
    }
    return folder;
}

static double env_d(const char* k, double d) {
    const char* v = getenv(k);
    return v ? atof(v) : d;
}
static unsigned long long env_u(const char* k, unsigned long long d) {
    const char* v = getenv(k);
    return v ? strtoull(v, nullptr, 0) : d;
}

// threads / blocks / offset as the reference reads them (atoi), but a
// negative value is an error instead of a huge unsigned one.
static bool count_arg(const char* s, unsigned& v) {
    const long x = atol(s);
    if (x < 0 || x > 0xffffffffL) return false;
    v = (unsigned)x;
    return true;
}

// Rows of MX_0 (lines, as the library counts them), to reject a batch that
// cannot fit before allocating host buffers for it; -1 if unreadable.
static long long mx0_rows(const char* folder) {
    std::ifstream in((std::string(folder) + "/MX_0").c_str());
    if (!in.is_open()) return -1;
    long long rows = 0;
    for (std::string line; std::getline(in, line);) rows++;
    return rows;
}

static int run_cli(int argc, const char* argv[]) {
    if (argc < 6) usage_exit();
    const bool verbose = argc > 10 && std::string(argv[10]) == "1";
    const bool stdout_dyn = argc > 10 && std::string(argv[10]) == "2";
    const char* folder = argv[1];
    unsigned threads = 0, blocks = 0, offset = 0;
    const int gpu = atoi(argv[4]);
    if (!count_arg(argv[2], threads) || !count_arg(argv[3], blocks) || !count_arg(argv[5], offset) ||
        (unsigned long long)threads * blocks > 0xffffffffull) {
        fprintf(stderr, "ERROR: threads, blocks and offset must be non-negative and threads*blocks < 2^32\n");
        return -1;
    }
    const unsigned N = threads * blocks;
    if (verbose) {
        printf(" * Required %d threads per block using %d blocks", threads, blocks);
        printf(" * Launching simulations on GPU %d \n", gpu);
        printf(" * Data offset: %d to %d threads\n", offset, offset + N);
    }
    std::string out_dir = output_folder(argc, argc > 6 ? argv[6] : nullptr, verbose);
    std::string prefix = argc > 7 ? argv[7] : "";
    if (verbose) printf(" * Output path: %s%s.\n", out_dir.c_str(), prefix.c_str());
    bool just_fitness = true, text_fitness = true, force_ssa = false;
    if (argc > 8) {
        just_fitness = std::string(argv[8]) != "0";
        text_fitness = std::string(argv[8]) == "2";
    }
    if (argc > 9) {
        force_ssa = std::string(argv[9]) != "0";
        if (force_ssa) fprintf(stdout, " * tau-leaping disabled: cuTauLeaping will force SSA instead.\n");
    }
    if (N == 0) {
        fprintf(stderr, "ERROR: threads*blocks must be positive\n");
        return -1;
    }

    ctl_model* model = nullptr;
    ctl_status st = ctl_model_load(folder, &model);
    if (st != CTL_OK) return exit_code(st, "model");
    {
        std::ifstream probe((std::string(folder) + "/cs_vector").c_str());
        if (!probe.is_open())
            printf("WARNING: chemical species to sample vector not found, saving ALL species as default.\n");
    }
    ctl_model_dims dims;
    ctl_model_dims_get(model, &dims);
    const long long rows = mx0_rows(folder);
    if (rows >= 0 && (long long)offset + N > rows) {  // the library's message and exit code, before any allocation
        fprintf(stderr, "ERROR: input files rows (%lld) and requested threads (%u) do not fit\n", rows, N);
        return -4;
    }
    std::vector<int32_t> X0((size_t)N * dims.S);
    std::vector<float> c((size_t)N * dims.R);
    st = ctl_rows_load(folder, dims.S, dims.R, offset, N, X0.data(), c.data());
    if (st != CTL_OK) return exit_code(st, "rows");

    ctl_target* target = nullptr;
    if (just_fitness) {
        st = ctl_target_load(folder, model, threads, blocks, &target);
        if (st != CTL_OK) return exit_code(st, "fitness target");
        uint32_t rep = 0, prep = 0, tq = 0, ex = 0;
        ctl_target_dims(target, &rep, &prep, &tq, &ex);
        if (verbose) printf(" * Experiments: %d, repetitions: %d target quantities: %d\n", ex, rep, tq);
        for (uint32_t d = 0; d < ex; d++) printf("\n");  // the reference's normalizer dump (tau.cu:1232-1237)
    }

    ctl_run_cfg cfg;
    ctl_run_cfg_default(&cfg);
    cfg.seed = env_u("CTL_SEED", (unsigned long long)time(nullptr));
    cfg.flags = (uint32_t)env_u("CTL_FLAGS", 0) | (force_ssa ? CTL_FORCE_SSA : 0u);
    cfg.eps = (float)env_d("CTL_EPS", 0.03);
    cfg.nc = (uint32_t)env_u("CTL_NC", 10);
    cfg.max_steps = (uint32_t)env_u("CTL_MAX_STEPS", 0xFFFFFFFFull);
    cfg.group = (int32_t)env_u("CTL_GROUP", 0);
    cfg.threads = (int32_t)env_u("CTL_THREADS", 0);
    cfg.warp_sims = (int32_t)env_u("CTL_WARP_SIMS", 0);
    cfg.spec = (int32_t)env_u("CTL_SPEC", 0);
    cfg.device = gpu;
    cfg.sim_base = offset;
    if (verbose) {
        printf(" * Seed: %llu\n", (unsigned long long)cfg.seed);
        fprintf(stdout, " * 3P-tau-leaping starting on GPU%d\n", gpu);
    }

    std::vector<ctl_sim_info> info(N);
    std::vector<uint32_t> samples;
    std::vector<double> fit;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    if (just_fitness) {
        // fitness mode: samples are summed per parameter set on the device
        fit.assign(N, 0.0);
        st = ctl_fitness_run(model, target, &cfg, X0.data(), c.data(), fit.data(), info.data());
    } else {
        samples.resize((size_t)N * dims.ns * dims.s_out);
        st = ctl_run(model, &cfg, N, X0.data(), c.data(), samples.data(), info.data());
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (st != CTL_OK && st != CTL_ERR_STEP_LIMIT) return exit_code(st, just_fitness ? "fitness" : "run");
    if (st == CTL_ERR_STEP_LIMIT) fprintf(stderr, "WARNING: %s\n", ctl_last_error());
    const double run_s = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
    if (verbose) printf(" * RUNNING TIME: %f seconds.\n", run_s);
    if (const char* rep = getenv("CTL_REPORT")) {
        ctl_launch_info li;
        const bool have = ctl_launch_query(model, &cfg, N, &li) == CTL_OK;
        if (ctl_write_run_report(model, rep, N, info.data(), run_s > 0.0 ? run_s : 1e-9, have ? &li : nullptr) !=
            CTL_OK)
            fprintf(stderr, "WARNING: %s\n", ctl_last_error());
    }

    std::string dumpfile = out_dir + prefix;
    if (!just_fitness) {
        if (!stdout_dyn && env_u("CTL_BINARY_OUTPUT", 0) == 1) {
            const std::string bin = dumpfile + ".ctlbin";
            printf(" * Writing dynamics to file %s\n", bin.c_str());
            fflush(stdout);
            st = ctl_write_samples_binary(model, bin.c_str(), N, samples.data(), 0);
        } else if (!stdout_dyn) {
            printf(" * Writing dynamics to file %s\n", dumpfile.c_str());
            fflush(stdout);
            st = ctl_write_dynamics(model, dumpfile.c_str(), N, samples.data(), 0, 0);
        } else {
            fflush(stdout);
            st = ctl_print_dynamics(model, N, samples.data());
        }
        if (st != CTL_OK) return exit_code(st, "output");
    } else {
        if (verbose) printf(" * Calculating fitnesses.\n");
        uint32_t prep = 1;
        ctl_target_dims(target, nullptr, &prep, nullptr, nullptr);
        fflush(stdout);
        if (text_fitness) {
            for (unsigned sw = 0; sw < blocks / prep; sw++) {
                for (unsigned part = 0; part < threads; part++) std::cout << fit[(size_t)sw * threads + part] << "\t";
                std::cout << "\t";
            }
            std::cout.flush();
        } else {
            printf(" * Dumping fitness to file.\n");
            std::ofstream dump("./pref_allfit");
            dump << std::fixed << std::showpoint << std::setprecision(20);
            for (unsigned sw = 0; sw < blocks; sw++) {
                for (unsigned part = 0; part < threads; part++) dump << fit[(size_t)sw * threads + part] << "\t";
                dump << "\n";
            }
        }
        ctl_target_free(target);
    }
    ctl_model_free(model);
    return 0;
}

int main(int argc, const char* argv[]) {
    try {
        return run_cli(argc, argv);
    } catch (const std::bad_alloc&) {
        fprintf(stderr, "ERROR: out of host memory\n");
        return -3;
    }
}

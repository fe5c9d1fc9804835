// Internal declarations shared by the host library (ctl_host.cpp) and the
// CUDA sweep (ctl_sweep.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ctl.h"

namespace ctl {

// Packed table entries: index in the high 24 bits, coefficient in the low 8
// (unsigned stoichiometry for reactants, two's-complement for net changes).
inline uint32_t pack(uint32_t idx, int coef) { return (idx << 8) | (uint32_t)(uint8_t)(int8_t)coef; }

// Flattened model tables; every list keeps the reference's flattening order
// (2phase_n-tau-leaping.cu:212-225 reactants r-major, 314-326 RAV
// species-major, 330-342 feed-masked F r-major).
struct HostTables {
    int S = 0, R = 0, P = 2, logP = 1, ns = 0, s_out = 0;
    std::vector<uint32_t> reac_off, reac_ent;  // reactants (left > 0), r-major: s<<8|st
    std::vector<uint32_t> reac_desc;           // [2R]: up to two reactant entries (s<<8|st, 0 = none);
                                               // 0xffffffff in slot 0 = use the general list
    std::vector<uint32_t> vs_off, vs_ent;      // V = right-left, species-major: r<<8|v
    std::vector<uint32_t> fs_off, fs_ent;      // F (feed-masked V), species-major: r<<8|f
    std::vector<uint32_t> fr_off, fr_ent;      // F, reaction-major: s<<8|f
    std::vector<uint32_t> dep_off, dep_ent;    // reactions whose propensity a firing changes
    std::vector<uint8_t> hor, hort;            // Cao HOR / HORtype (tau.cu:402-432)
    std::vector<double> tvec;                  // sample instants
    std::vector<uint32_t> cs;                  // sampled species
    double tmax = 0.0;
};

struct DeviceCopy {
    int device = -1;
    void* buf = nullptr;         // all tables, one allocation
    size_t bytes = 0;
    uint32_t* ctrl = nullptr;    // [0] = work-queue ticket, [1..] spare
    size_t off_reac_off = 0, off_reac_ent = 0, off_vs_off = 0, off_vs_ent = 0;
    size_t off_fs_off = 0, off_fs_ent = 0, off_fr_off = 0, off_fr_ent = 0;
    size_t off_dep_off = 0, off_dep_ent = 0, off_hor = 0, off_hort = 0, off_tvec = 0, off_cs = 0;
    size_t off_reac_desc = 0;
};

// Shifts of the stored levels of the propensity sum tree over P = 2^logP
// leaves: 3, 6, 9, ... below logP, then logP (the root).  Stored level li
// holds the nodes that cover 2^shift leaves.
inline int stored_level_shifts(int logP, int (&shift)[10]) {
    int n = 0;
    for (int l = 3; l < logP; l += 3) shift[n++] = l;
    shift[n++] = logP;
    return n;
}

void set_error(const std::string& msg);
ctl_status build_tables(int S, int R, const int32_t* left, const int32_t* right,
                        const int32_t* feed, int ns, const double* tvec, int s_out,
                        const int32_t* cs, HostTables& t);

}  // namespace ctl

struct ctl_model {
    ctl::HostTables t;
    std::mutex mu;
    ctl::DeviceCopy dev[16];
    // autotune cache: (device, log2 of the batch size, rate mode, flags) -> launch shape
    struct Tuned { int device; uint32_t nbucket, uniform, flags; int group, threads, ssa_budget, dec_budget, min_blocks, sched, warp_sims; };
    std::vector<Tuned> tuned;
};

struct ctl_target {
    uint32_t repetitions = 0, p_rep = 0, target_quantities = 0, experiments = 0;
    uint32_t threads = 0, blocks = 0, ns = 0, s_out = 0;
    std::vector<uint8_t> thread2experiment;  // [threads*blocks]
    std::vector<uint32_t> series;            // [ns][experiments][repetitions][target_quantities]
};

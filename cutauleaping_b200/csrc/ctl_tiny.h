// Register-resident sweep for tiny networks: limits, the kernel's parameter
// block and the host-side helpers (ctl_tiny.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <string>

#include "ctl_internal.h"

namespace ctl {
namespace tiny {

constexpr int MAX_R = 16;    // reactions (tree leaves up to 16)
constexpr int MAX_S = 8;     // species, and sampled species
constexpr int NET_MAX_E = 3; // reactant entries per reaction (the kernel body's MAX_E)

// The model as a kernel parameter (constant bank; every value is the same
// for all threads).  Species-major tables hold entries in ascending reaction
// order, the reference's flattening order (tau.cu:314-342).
struct Net {
    int32_t S, R, ns, s_out;
    double tmax;
    const double* tvec;         // device copy of the sample instants
    uint8_t ne[MAX_R];          // reactant entries of reaction r
    uint8_t es[MAX_R][NET_MAX_E];  // their species, ascending
    uint8_t ec[MAX_R][NET_MAX_E];  // their coefficients
    int8_t V[MAX_S][MAX_R];     // tau1 table: V species-major (F when quirk Q5 is off)
    uint8_t vnz[MAX_S];         // species s has an entry in V
    int8_t Fm[MAX_S][MAX_R];    // feed-masked net change F, species-major (leap test)
    uint8_t hor[MAX_S], hort[MAX_S];
    uint8_t cs[MAX_S];          // sampled species
    uint32_t frow[MAX_R][2];    // F reaction-major: 8 signed bytes per reaction (SSA update)
};

}  // namespace tiny

// Networks the register-resident sweep runs: R <= 16, S <= 8, at most 8
// sampled species, at most 3 reactant entries per reaction.
bool tiny_eligible(const HostTables& t);
// Species bound of the kernel variant (4 or 8).
int tiny_species_bound(const HostTables& t);
// Parameter block for a run with `flags` (quirk Q5 picks the tau1 table).
void tiny_net(const HostTables& t, uint32_t flags, const double* d_tvec, tiny::Net& n);
// Kernel for P tree leaves (2, 4, 8, 16) and species bound SM (4, 8).
const void* tiny_kernel_ptr(int P, int SM);

// Parameter block of a model-specialised kernel: everything else is
// compiled in.
struct SpecNet {
    const double* tvec;
    double tmax;
};
// The kernel compiled for this network and tau1 table (quirk Q5 in flags)
// by NVRTC, for minb resident 256-thread blocks per SM (its register
// budget: 2, 3 or 4) and one schedule (1 block rounds, 2 warp lockstep), or
// nullptr when NVRTC is missing or the compilation failed (the reason in
// *why).  Compiled once per process, network, budget and schedule; takes a
// lock.
const void* tiny_spec_kernel(const HostTables& t, uint32_t flags, int minb, int sched, std::string* why);

// Compiles `src` for sm_100a with NVRTC (-fmad=false, the same arithmetic as
// the library's kernels; the device headers ctl_devmath.cuh,
// ctl_tiny_body.cuh and ctl_sweep_dev.cuh can be included), loads the CUBIN
// and returns the kernel `name`, or nullptr with the reason in `why` when
// NVRTC is missing or a step fails.  No caching and no lock: callers keep
// their own cache.
const void* nvrtc_kernel(const std::string& src, const char* name, std::string& why);

}  // namespace ctl

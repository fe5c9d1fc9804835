// Register-resident sweep for tiny networks (at most 16 reactions and 8
// species, e.g. the Schlogl model of schlogl.xml) on sm_100a.
//
// The shared-memory sweep (ctl_sweep_dev.cuh) keeps each simulation's state
// in shared memory and steps groups of lanes in block rounds; for a network
// of a handful of reactions its SSA step is a long chain of shared-memory
// round trips, table loads and barriers, and a batch of a few thousand
// bistable simulations is timed by its slowest simulation.  Here one thread
// owns one simulation and keeps everything in registers (ctl_tiny_body.cuh).
//
// Two kinds of kernel run that code:
//   * the library's own, one per (tree leaves P, species bound SM), reading
//     the model as a parameter block (Net, constant bank, warp-uniform);
//   * a kernel compiled at run time for one model by NVRTC, with the model's
//     tables as compile-time constants.  For a 4-reaction network the
//     generic kernel spends most of an SSA step on uniform branches and
//     table selects around four propensities; the specialised one computes
//     them as straight-line arithmetic.  It is compiled once per (network,
//     tau1 table) and process, loaded with cudaLibraryLoadData, and used
//     whenever NVRTC is present; the library's kernels are the fallback.
// Both give the same bits as the shared-memory sweep and the CPU oracle.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "ctl_tiny.h"
#include "ctl_tiny_body.cuh"

namespace ctl {
namespace tiny {

// The model read from the parameter block at run time.
struct NetRT {
    Net n;
    __device__ __forceinline__ int S() const { return n.S; }
    __device__ __forceinline__ int R() const { return n.R; }
    __device__ __forceinline__ int ns() const { return n.ns; }
    __device__ __forceinline__ int s_out() const { return n.s_out; }
    __device__ __forceinline__ double tmax() const { return n.tmax; }
    __device__ __forceinline__ const double* tvec() const { return n.tvec; }
    __device__ __forceinline__ int ne(int r) const { return n.ne[r]; }
    __device__ __forceinline__ uint32_t es(int r, int e) const { return n.es[r][e]; }
    __device__ __forceinline__ int ec(int r, int e) const { return n.ec[r][e]; }
    __device__ __forceinline__ int V(int q, int r) const { return n.V[q][r]; }
    __device__ __forceinline__ bool vnz(int q) const { return n.vnz[q] != 0; }
    __device__ __forceinline__ int Fm(int q, int r) const { return n.Fm[q][r]; }
    __device__ __forceinline__ uint32_t hor(int q) const { return n.hor[q]; }
    __device__ __forceinline__ uint32_t hort(int q) const { return n.hort[q]; }
    __device__ __forceinline__ uint32_t cs(int k) const { return n.cs[k]; }
    __device__ __forceinline__ uint32_t frow(int r, int w) const { return n.frow[r][w]; }
};

// One thread per simulation; see run_sweep().
template <int P, int SM>
__global__ void __launch_bounds__(256, 2) tiny_kernel(const __grid_constant__ NetRT net,
                                                      const __grid_constant__ dev::Run run, uint32_t lanes) {
    run_sweep<NetRT, P, SM>(net, run, lanes);
}

static_assert(NET_MAX_E == MAX_E, "parameter block and kernel body agree on reactant entries");

}  // namespace tiny

// Host side: which networks qualify, their parameter block, the kernels.

bool tiny_eligible(const HostTables& t) {
    if (t.R > tiny::MAX_R || t.S > tiny::MAX_S || t.s_out > tiny::MAX_S) return false;
    for (int r = 0; r < t.R; r++)
        if (t.reac_off[r + 1] - t.reac_off[r] > (uint32_t)tiny::NET_MAX_E) return false;
    return true;
}

int tiny_species_bound(const HostTables& t) { return t.S <= 4 ? 4 : 8; }

void tiny_net(const HostTables& t, uint32_t flags, const double* d_tvec, tiny::Net& n) {
    std::memset(&n, 0, sizeof(n));
    n.S = t.S;
    n.R = t.R;
    n.ns = t.ns;
    n.s_out = t.s_out;
    n.tmax = t.tmax;
    n.tvec = d_tvec;
    for (int r = 0; r < t.R; r++) {
        n.ne[r] = (uint8_t)(t.reac_off[r + 1] - t.reac_off[r]);
        for (uint32_t e = t.reac_off[r]; e < t.reac_off[r + 1]; e++) {
            n.es[r][e - t.reac_off[r]] = (uint8_t)(t.reac_ent[e] >> 8);
            n.ec[r][e - t.reac_off[r]] = (uint8_t)(t.reac_ent[e] & 0xffu);
        }
    }
    // tau1 table: V species-major, or the feed-masked F when Q5 is off
    const bool q5off = (flags & dev::F_Q5_OFF) != 0;
    const std::vector<uint32_t>& vo = q5off ? t.fs_off : t.vs_off;
    const std::vector<uint32_t>& ve = q5off ? t.fs_ent : t.vs_ent;
    for (int s = 0; s < t.S; s++) {
        n.vnz[s] = vo[s + 1] != vo[s] ? 1 : 0;
        for (uint32_t e = vo[s]; e < vo[s + 1]; e++) n.V[s][ve[e] >> 8] = (int8_t)(ve[e] & 0xffu);
        for (uint32_t e = t.fs_off[s]; e < t.fs_off[s + 1]; e++) n.Fm[s][t.fs_ent[e] >> 8] = (int8_t)(t.fs_ent[e] & 0xffu);
        n.hor[s] = t.hor[s];
        n.hort[s] = t.hort[s];
    }
    for (int k = 0; k < t.s_out; k++) n.cs[k] = (uint8_t)t.cs[k];
    for (int r = 0; r < t.R; r++)
        for (uint32_t e = t.fr_off[r]; e < t.fr_off[r + 1]; e++) {
            const uint32_t s = t.fr_ent[e] >> 8;
            n.frow[r][s >> 2] |= (t.fr_ent[e] & 0xffu) << (8 * (s & 3));
        }
}

const void* tiny_kernel_ptr(int P, int SM) {
    if (SM == 4) {
        switch (P) {
            case 2: return reinterpret_cast<const void*>(&tiny::tiny_kernel<2, 4>);
            case 4: return reinterpret_cast<const void*>(&tiny::tiny_kernel<4, 4>);
            case 8: return reinterpret_cast<const void*>(&tiny::tiny_kernel<8, 4>);
            case 16: return reinterpret_cast<const void*>(&tiny::tiny_kernel<16, 4>);
        }
    } else if (SM == 8) {
        switch (P) {
            case 2: return reinterpret_cast<const void*>(&tiny::tiny_kernel<2, 8>);
            case 4: return reinterpret_cast<const void*>(&tiny::tiny_kernel<4, 8>);
            case 8: return reinterpret_cast<const void*>(&tiny::tiny_kernel<8, 8>);
            case 16: return reinterpret_cast<const void*>(&tiny::tiny_kernel<16, 8>);
        }
    }
    return nullptr;
}

// ---------------------------------------------------------------------------
// Model-specialised kernels (NVRTC)
// ---------------------------------------------------------------------------

// The sources of ctl_devmath.cuh, ctl_tiny_body.cuh and ctl_sweep_dev.cuh,
// embedded by the build (cutauleaping_b200/build.py writes them into
// ctl_tiny_src.cpp).
extern const char* const ctl_src_devmath;
extern const char* const ctl_src_tiny_body;
extern const char* const ctl_src_sweep_dev;

namespace {

// NVRTC, opened at run time: the library has no link-time dependency on it
// and falls back to its own kernels when it is absent.
struct Nvrtc {
    bool ok = false;
    std::string why;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

Nvrtc open_nvrtc() {
    Nvrtc n;
    void* h = nullptr;
    for (const char* name : {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"})
        if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
        n.why = "NVRTC (libnvrtc.so.12) not found";
        return n;
    }
    n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    if (!n.ok) n.why = "NVRTC lacks a required entry point";
    return n;
}

std::mutex g_spec_mu;
struct SpecEntry {
    std::string source;
    const void* kernel;
    std::string why;
};
std::vector<SpecEntry> g_spec;

// A table accessor as a switch over its nonzero entries (folded away for
// the constant arguments the unrolled kernel passes).
template <class F>
void accessor(std::ostringstream& o, const char* decl, int rows, int cols, F&& value) {
    o << "    __device__ __forceinline__ " << decl << " const { switch (a * " << cols << " + b) {";
    for (int i = 0; i < rows; i++)
        for (int j = 0; j < cols; j++) {
            const long long v = value(i, j);
            if (v) o << " case " << i * cols + j << ": return " << v << ";";
        }
    o << " default: return 0; } }\n";
}

std::string spec_source(const HostTables& t, uint32_t flags, int minb, int sched) {
    tiny::Net n;
    tiny_net(t, flags, nullptr, n);
    const int P = t.P, SM = tiny_species_bound(t);
    std::ostringstream o;
    o << "#include \"ctl_tiny_body.cuh\"\n";
    o << "struct NetCT {\n    const double* tv;\n    double tm;\n";
    o << "    __device__ __forceinline__ int S() const { return " << n.S << "; }\n";
    o << "    __device__ __forceinline__ int R() const { return " << n.R << "; }\n";
    o << "    __device__ __forceinline__ int ns() const { return " << n.ns << "; }\n";
    o << "    __device__ __forceinline__ int s_out() const { return " << n.s_out << "; }\n";
    o << "    __device__ __forceinline__ double tmax() const { return tm; }\n";
    o << "    __device__ __forceinline__ const double* tvec() const { return tv; }\n";
    accessor(o, "int ne(int a, int b = 0)", tiny::MAX_R, 1, [&](int i, int) { return (long long)n.ne[i]; });
    accessor(o, "unsigned es(int a, int b)", tiny::MAX_R, tiny::NET_MAX_E, [&](int i, int j) { return (long long)n.es[i][j]; });
    accessor(o, "int ec(int a, int b)", tiny::MAX_R, tiny::NET_MAX_E, [&](int i, int j) { return (long long)n.ec[i][j]; });
    accessor(o, "int V(int a, int b)", tiny::MAX_S, tiny::MAX_R, [&](int i, int j) { return (long long)n.V[i][j]; });
    accessor(o, "int vnz(int a, int b = 0)", tiny::MAX_S, 1, [&](int i, int) { return (long long)n.vnz[i]; });
    accessor(o, "int Fm(int a, int b)", tiny::MAX_S, tiny::MAX_R, [&](int i, int j) { return (long long)n.Fm[i][j]; });
    accessor(o, "unsigned hor(int a, int b = 0)", tiny::MAX_S, 1, [&](int i, int) { return (long long)n.hor[i]; });
    accessor(o, "unsigned hort(int a, int b = 0)", tiny::MAX_S, 1, [&](int i, int) { return (long long)n.hort[i]; });
    accessor(o, "unsigned cs(int a, int b = 0)", tiny::MAX_S, 1, [&](int i, int) { return (long long)n.cs[i]; });
    accessor(o, "unsigned frow(int a, int b)", tiny::MAX_R, 2, [&](int i, int j) { return (long long)n.frow[i][j]; });
    o << "};\n";
    // one schedule per kernel: warp lockstep (2) or block rounds (1)
    o << "extern \"C\" __global__ void __launch_bounds__(256, " << minb << ") ctl_tiny_spec("
         "const __grid_constant__ NetCT net, const __grid_constant__ ctl::dev::Run run, unsigned lanes) {\n";
    if (sched == 2)
        o << "    ctl::tiny::sweep<NetCT, " << P << ", " << SM << ">(net, run, lanes);\n}\n";
    else
        o << "    extern __shared__ unsigned ctl_tiny_xs[];\n"
             "    ctl::tiny::sweep_rounds<NetCT, " << P << ", " << SM << ">(net, run, lanes, ctl_tiny_xs);\n}\n";
    return o.str();
}

}  // namespace

const void* nvrtc_kernel(const std::string& src, const char* name, std::string& why) {
    static Nvrtc nv = open_nvrtc();
    if (!nv.ok) {
        why = nv.why;
        return nullptr;
    }
    const char* headers[] = {ctl_src_devmath, ctl_src_tiny_body, ctl_src_sweep_dev};
    const char* names[] = {"ctl_devmath.cuh", "ctl_tiny_body.cuh", "ctl_sweep_dev.cuh"};
    nvrtcProgram prog;
    if (nv.create(&prog, src.c_str(), "ctl_spec.cu", 3, headers, names) != NVRTC_SUCCESS) {
        why = "nvrtcCreateProgram failed";
        return nullptr;
    }
    const char* opts[] = {"--gpu-architecture=sm_100a", "-fmad=false", "--std=c++17"};
    const nvrtcResult r = nv.compile(prog, 3, opts);
    std::vector<char> cubin;
    if (r == NVRTC_SUCCESS) {
        size_t n = 0;
        if (nv.cubin_size(prog, &n) == NVRTC_SUCCESS && n) {
            cubin.resize(n);
            if (nv.cubin(prog, cubin.data()) != NVRTC_SUCCESS) cubin.clear();
        }
    } else {
        size_t n = 0;
        nv.log_size(prog, &n);
        std::string log(n, '\0');
        if (n) nv.log(prog, &log[0]);
        why = "NVRTC compilation failed: " + log.substr(0, 2000);
    }
    nv.destroy(&prog);
    if (cubin.empty()) {
        if (why.empty()) why = "NVRTC produced no CUBIN";
        return nullptr;
    }
    cudaLibrary_t lib;
    cudaError_t e = cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) {
        why = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e);
        return nullptr;
    }
    cudaKernel_t k;
    e = cudaLibraryGetKernel(&k, lib, name);
    if (e != cudaSuccess) {
        why = std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(e);
        return nullptr;
    }
    return reinterpret_cast<const void*>(k);
}

const void* tiny_spec_kernel(const HostTables& t, uint32_t flags, int minb, int sched, std::string* why) {
    const std::string src = spec_source(t, flags & dev::F_Q5_OFF, minb, sched);
    std::lock_guard<std::mutex> lk(g_spec_mu);
    for (const auto& e : g_spec)
        if (e.source == src) {
            if (why) *why = e.why;
            return e.kernel;
        }
    std::string w;
    const void* k = nvrtc_kernel(src, "ctl_tiny_spec", w);
    g_spec.push_back({src, k, w});
    if (why) *why = w;
    return k;
}

}  // namespace ctl

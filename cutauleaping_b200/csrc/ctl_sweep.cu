// Persistent tau-leaping / SSA sweep for sm_100a.
//
// Replaces the reference's host loop (kernel.cu:242-345) and its kernels
// PreCalculations (2phase_n-tau-leaping.cu:1568-2093), EventualSSASteps
// (2099-2273), LightweightSSA (2280-2454), setup_random (2974-2988),
// PrepareVariables (1269-1297) and ParallelVoting (2990-3002) with ONE
// launch: every group of G lanes owns a shared-memory slot, pulls a
// simulation from a device work queue (atomic ticket), runs it to the end
// (leaps, SSA bursts, samples) and pulls the next one.  No host round trip
// per leap, no per-pass reload of state from global memory.
//
// Determinism contract (what makes any launch shape give identical bits):
//   * every random word comes from Philox4x32-10 with key = seed and counter
//     (block, tag, step, sim): a draw depends on which simulation, which step
//     and what it is for, never on which thread computes it;
//   * every FP64 sum over reactions (A0, the critical sum a0c) is the root of
//     a fixed binary tree over the reactions padded to P = 2^k leaves, and
//     the SSA / critical-reaction searches descend that same tree;
//   * per-species sums (mu, sigma^2, population updates) run over a fixed
//     entry order by one lane.
// The CPU oracle (oracle/ctl_oracle.c) implements the same contract.
//
// Built with -fmad=false: no implicit FMA contraction; fma() is called
// explicitly where it is meant.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <chrono>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "ctl_internal.h"

#include "ctl_sweep_dev.cuh"
#include "ctl_tiny.h"

namespace ctl {
namespace dev {

// calculateFitness (tau.cu:3324-3408): one thread per parameter set.
__global__ void fitness_kernel(const uint32_t* __restrict__ samples, const uint32_t* __restrict__ target,
                               const uint8_t* __restrict__ swarm, double* __restrict__ fitness,
                               uint32_t threads, uint32_t nsets, uint32_t p_rep, uint32_t ns,
                               uint32_t so, uint32_t E, uint32_t REP) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nsets) return;
    const uint32_t b = tid / threads, t = tid % threads;
    const uint32_t ex = swarm[tid];
    float sub = 0.0f;
    for (uint32_t c = 0; c < ns; c++) {
        for (uint32_t s = 0; s < so; s++) {
            double acc = 0.0;
            for (uint32_t par = 0; par < p_rep; par++) {
                const size_t gid = (size_t)(b * p_rep + par) * threads + t;
                acc = acc + (double)samples[(gid * ns + c) * so + s];
            }
            acc = acc / (double)p_rep;
            for (uint32_t e = 0; e < REP; e++) {
                const int tgt = (int)target[((size_t)(c * E + ex) * REP + e) * so + s];
                double dist = fabs((double)tgt - acc);
                if (tgt != 0) dist = dist / (double)tgt;
                sub = (float)((double)sub + dist);
            }
        }
    }
    fitness[tid] = ((1.0 / (double)ns) * (1.0 / (double)so)) * (double)sub;
}

// The same from per-set sample sums (fitness mode of the sweep): the
// reference's FP64 running sum of p_rep integer samples is exact, so it
// equals the integer sum converted once; the rest is calculateFitness.
__global__ void fitness_sums_kernel(const unsigned long long* __restrict__ sums, const uint32_t* __restrict__ target,
                                    const uint8_t* __restrict__ swarm, double* __restrict__ fitness,
                                    uint32_t nsets, uint32_t p_rep, uint32_t ns, uint32_t so, uint32_t E,
                                    uint32_t REP) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nsets) return;
    const uint32_t ex = swarm[tid];
    float sub = 0.0f;
    for (uint32_t c = 0; c < ns; c++) {
        for (uint32_t s = 0; s < so; s++) {
            const double acc = (double)sums[((size_t)tid * ns + c) * so + s] / (double)p_rep;
            for (uint32_t e = 0; e < REP; e++) {
                const int tgt = (int)target[((size_t)(c * E + ex) * REP + e) * so + s];
                double dist = fabs((double)tgt - acc);
                if (tgt != 0) dist = dist / (double)tgt;
                sub = (float)((double)sub + dist);
            }
        }
    }
    fitness[tid] = ((1.0 / (double)ns) * (1.0 / (double)so)) * (double)sub;
}

}  // namespace dev

// ---------------------------------------------------------------------------
// Host launch side
// ---------------------------------------------------------------------------

static ctl_status cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CTL_ERR_CUDA;
}
#define CTL_CUDA(call)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);         \
    } while (0)

static size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// The model tables in one device buffer: offsets of every array (`place`
// returns the next 16-byte aligned offset) and the copy of its contents
// (`put` returns false to stop); shared by the cached per-device copy and the
// allocation-free path.
template <class Place>
static void table_layout(const HostTables& t, DeviceCopy& d, Place&& place) {
    d.off_reac_off = place(t.reac_off.size() * 4);
    d.off_reac_ent = place(std::max<size_t>(1, t.reac_ent.size()) * 4);
    d.off_reac_desc = place(t.reac_desc.size() * 4);
    d.off_vs_off = place(t.vs_off.size() * 4);
    d.off_vs_ent = place(std::max<size_t>(1, t.vs_ent.size()) * 4);
    d.off_fs_off = place(t.fs_off.size() * 4);
    d.off_fs_ent = place(std::max<size_t>(1, t.fs_ent.size()) * 4);
    d.off_fr_off = place(t.fr_off.size() * 4);
    d.off_fr_ent = place(std::max<size_t>(1, t.fr_ent.size()) * 4);
    d.off_dep_off = place(t.dep_off.size() * 4);
    d.off_dep_ent = place(std::max<size_t>(1, t.dep_ent.size()) * 4);
    d.off_hor = place(t.hor.size());
    d.off_hort = place(t.hort.size());
    d.off_tvec = place(t.tvec.size() * 8);
    d.off_cs = place(t.cs.size() * 4);
}

template <class Put>
static void table_fill(const HostTables& t, const DeviceCopy& d, Put&& put) {
    put(d.off_reac_off, t.reac_off.data(), t.reac_off.size() * 4) &&
        put(d.off_reac_ent, t.reac_ent.data(), t.reac_ent.size() * 4) &&
        put(d.off_reac_desc, t.reac_desc.data(), t.reac_desc.size() * 4) &&
        put(d.off_vs_off, t.vs_off.data(), t.vs_off.size() * 4) &&
        put(d.off_vs_ent, t.vs_ent.data(), t.vs_ent.size() * 4) &&
        put(d.off_fs_off, t.fs_off.data(), t.fs_off.size() * 4) &&
        put(d.off_fs_ent, t.fs_ent.data(), t.fs_ent.size() * 4) &&
        put(d.off_fr_off, t.fr_off.data(), t.fr_off.size() * 4) &&
        put(d.off_fr_ent, t.fr_ent.data(), t.fr_ent.size() * 4) &&
        put(d.off_dep_off, t.dep_off.data(), t.dep_off.size() * 4) &&
        put(d.off_dep_ent, t.dep_ent.data(), t.dep_ent.size() * 4) &&
        put(d.off_hor, t.hor.data(), t.hor.size()) &&
        put(d.off_hort, t.hort.data(), t.hort.size()) &&
        put(d.off_tvec, t.tvec.data(), t.tvec.size() * 8) &&
        put(d.off_cs, t.cs.data(), t.cs.size() * 4);
}

// Upload the model tables to `device` once; later runs reuse them.
static ctl_status ensure_device(ctl_model* m, int device, DeviceCopy*& out) {
    if (device < 0 || device >= 16) {
        set_error("device ordinal out of range");
        return CTL_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(m->mu);
    DeviceCopy& d = m->dev[device];
    if (d.buf) {
        out = &d;
        return CTL_OK;
    }
    const HostTables& t = m->t;
    size_t off = 0;
    auto place = [&](size_t bytes) {
        size_t o = off;
        off = align16(off + bytes);
        return o;
    };
    table_layout(t, d, place);
    size_t ctrl_off = place(256);
    d.bytes = off;
    std::vector<unsigned char> h(d.bytes, 0);
    auto put = [&](size_t o, const void* p, size_t bytes) {
        if (bytes) std::memcpy(h.data() + o, p, bytes);
    };
    table_fill(t, d, [&](size_t o, const void* p, size_t bytes) {
        put(o, p, bytes);
        return true;
    });
    int prev = 0;
    CTL_CUDA(cudaGetDevice(&prev));
    CTL_CUDA(cudaSetDevice(device));
    void* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, d.bytes);
    if (e != cudaSuccess) {
        cudaSetDevice(prev);
        set_error(std::string("cudaMalloc(model tables): ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CTL_ERR_OOM : CTL_ERR_CUDA;
    }
    e = cudaMemcpy(buf, h.data(), d.bytes, cudaMemcpyHostToDevice);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaFree(buf);
        return cuda_fail(e, "cudaMemcpy(model tables)");
    }
    d.buf = buf;
    d.device = device;
    d.ctrl = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(buf) + ctrl_off);
    out = &d;
    return CTL_OK;
}

static void tree_levels(const HostTables& t, dev::Model& dm);

static dev::Model make_dev_model(const ctl_model* m, const DeviceCopy& d, uint32_t flags) {
    const HostTables& t = m->t;
    auto P = [&](size_t o) { return static_cast<const unsigned char*>(d.buf) + o; };
    dev::Model dm;
    dm.S = t.S; dm.R = t.R; dm.P = t.P; dm.logP = t.logP; dm.ns = t.ns; dm.s_out = t.s_out;
    dm.reac_off = reinterpret_cast<const uint32_t*>(P(d.off_reac_off));
    dm.reac_ent = reinterpret_cast<const uint32_t*>(P(d.off_reac_ent));
    dm.reac_desc = reinterpret_cast<const uint2*>(P(d.off_reac_desc));
    const bool q5off = (flags & dev::F_Q5_OFF) != 0;
    dm.v_off = reinterpret_cast<const uint32_t*>(P(q5off ? d.off_fs_off : d.off_vs_off));
    dm.v_ent = reinterpret_cast<const uint32_t*>(P(q5off ? d.off_fs_ent : d.off_vs_ent));
    dm.fs_off = reinterpret_cast<const uint32_t*>(P(d.off_fs_off));
    dm.fs_ent = reinterpret_cast<const uint32_t*>(P(d.off_fs_ent));
    dm.fr_off = reinterpret_cast<const uint32_t*>(P(d.off_fr_off));
    dm.fr_ent = reinterpret_cast<const uint32_t*>(P(d.off_fr_ent));
    dm.dep_off = reinterpret_cast<const uint32_t*>(P(d.off_dep_off));
    dm.dep_ent = reinterpret_cast<const uint32_t*>(P(d.off_dep_ent));
    dm.hor = P(d.off_hor);
    dm.hort = P(d.off_hort);
    dm.tvec = reinterpret_cast<const double*>(P(d.off_tvec));
    dm.cs = reinterpret_cast<const uint32_t*>(P(d.off_cs));
    dm.tmax = t.tmax;
    tree_levels(t, dm);
    return dm;
}

struct LaunchPlan {
    int G = 1, minb = 1, sched = 1, threads = 256, NS = 256, blocks = 1, blocks_per_sm = 1, sm_count = 1, regs = 0;
    int ssa_budget = 0, dec_budget = 0;
    size_t smem = 0;
    dev::Layout lay{};
    int warp_sims = 0;           // > 0: register-resident sweep, simulations per warp
    int tinyP = 0, tinySM = 0;   // its kernel variant: tree leaves, species bound
    const void* spec = nullptr;  // the kernel compiled for this network, if any
};

// Stored levels of the sum tree for P = 2^k leaves: 3, 6, ... below k, then
// k (the root).  Level li is the pairwise sum of 2^d nodes of level li-1.
static void tree_levels(const HostTables& t, dev::Model& dm) {
    int shift[10];
    const int nlev = stored_level_shifts(t.logP, shift);
    int prev = 0, base = 0;
    for (int li = 0; li < nlev; li++) {
        dm.lev_shift_v[li] = shift[li];
        dm.lev_d_v[li] = shift[li] - prev;
        dm.lev_base_v[li] = base;
        dm.lev_count_v[li] = t.P >> shift[li];
        base += t.P >> shift[li];
        prev = shift[li];
    }
    dm.nlev = nlev;
}

static int tree_words(const HostTables& t) {
    dev::Model dm;
    tree_levels(t, dm);
    return dm.lev_base_v[dm.nlev - 1] + 1;
}

// Shared-memory bytes of a block with NS slots of group size G.
static size_t slot_layout(const HostTables& t, int G, int NS, bool uniform_c, dev::Layout& lay, bool sums = false) {
    size_t off = 0;
    auto region = [&](size_t bytes) {
        size_t o = off;
        off = align16(off + bytes);
        return (uint32_t)o;
    };
    const int tw = tree_words(t);
    if (G == 1) {
        lay.len_S = (uint32_t)t.S;
        lay.len_P = (uint32_t)t.P;
        lay.len_C = (uint32_t)t.P;
        lay.len_T = (uint32_t)tw;
        lay.len_O = (uint32_t)t.s_out;
    } else {
        lay.len_S = (uint32_t)(t.S | 1);
        lay.len_P = (uint32_t)(t.P + 1);
        lay.len_C = (uint32_t)(((t.P + 3) & ~3) + 4);
        lay.len_T = (uint32_t)(tw | 1);
        lay.len_O = (uint32_t)(t.s_out | 1);
    }
    lay.off_tree = region((size_t)NS * lay.len_T * 8);
    lay.off_state = region((size_t)NS * (4 * 8 + 9 * 4));
    lay.off_X = region((size_t)NS * lay.len_S * 4);
    lay.off_X1 = region((size_t)NS * lay.len_S * 4);
    lay.off_a = region((size_t)NS * lay.len_P * 4);
    lay.off_K = region((size_t)NS * lay.len_P * 4);
    lay.off_c = region(uniform_c ? (size_t)t.P * 4 : (size_t)NS * lay.len_P * 4);
    lay.off_list = region((size_t)NS * 4);
    lay.off_crit = region((size_t)NS * lay.len_C);
    lay.off_grp = region((size_t)NS * (16 * (G > 32 ? G / 32 : 1) + 16));  // multi-warp group scratch
    lay.off_last = region(sums ? (size_t)NS * lay.len_O * 4 : 0);         // fitness mode only
    return off;
}

static const void* kernel_for(int G, int minb) {
    switch (G) {
        case 1: return sweep_kernel_g1(minb);
        case 2: return sweep_kernel_g2(minb);
        case 4: return sweep_kernel_g4(minb);
        case 8: return sweep_kernel_g8(minb);
        case 16: return sweep_kernel_g16(minb);
        case 32: return sweep_kernel_g32(minb);
        case 64: return sweep_kernel_g64(minb);
        case 128: return sweep_kernel_g128(minb);
        case 256: return sweep_kernel_g256(minb);
    }
    return nullptr;
}

// Lanes per simulation when the caller does not choose: about 16
// reactions per lane up to one warp (measured best for 64 x 128: G = 8;
// tiny networks: 1), about 8 per lane beyond (512 x 1024: G = 128, 1.8x
// the throughput of G = 32).
static int heuristic_group(const HostTables& t) {
    const int g = t.P >= 1024 ? t.P / 8 : t.P / 16;
    const int cap = t.P >= 1024 ? 256 : 32;
    int G = 1;
    while (G < g && G < cap) G <<= 1;
    return G;
}

// Launch shape for (model, cfg, n): group size, threads, slots and grid.
// Small batches use smaller blocks so that every SM gets work.
// Device attributes and kernel occupancy, cached: querying them costs far
// more than a small sweep launch.
struct DevAttr {
    int sm_count = 0, smem_optin = 0;
};
static std::mutex g_attr_mu;
static DevAttr g_attr[16];

static ctl_status device_attr(int dev, DevAttr& out) {
    if (dev < 0 || dev >= 16) return CTL_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (!g_attr[dev].sm_count) {
        DevAttr a;
        CTL_CUDA(cudaDeviceGetAttribute(&a.sm_count, cudaDevAttrMultiProcessorCount, dev));
        CTL_CUDA(cudaDeviceGetAttribute(&a.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        g_attr[dev] = a;
    }
    out = g_attr[dev];
    return CTL_OK;
}

// Per (device, G): the kernel's registers and the largest dynamic shared
// memory a launch may ask for (the opt-in maximum less the kernel's static
// shared memory).  The first query raises the kernel's dynamic-memory
// ceiling to that limit once, so every shape (cached or new) can launch.
struct KernAttr {
    int dev;
    const void* k;
    int regs;
    size_t dyn_max;
};
static std::vector<KernAttr> g_kattr;

static ctl_status kernel_attr(int dev, const void* k, KernAttr& out) {
    DevAttr da;
    if (device_attr(dev, da) != CTL_OK) return CTL_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const auto& a : g_kattr)
        if (a.dev == dev && a.k == k) {
            out = a;
            return CTL_OK;
        }
    cudaFuncAttributes fa;
    CTL_CUDA(cudaFuncGetAttributes(&fa, k));
    if ((size_t)da.smem_optin <= fa.sharedSizeBytes) {
        set_error("sweep kernel's static shared memory exceeds the device limit");
        return CTL_ERR_SHAPE;
    }
    KernAttr a{dev, k, fa.numRegs, (size_t)da.smem_optin - fa.sharedSizeBytes};
    CTL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.dyn_max));
    g_kattr.push_back(a);
    out = a;
    return CTL_OK;
}

struct OccKey {
    int dev;
    const void* k;
    int threads;
    size_t smem;
    int bps;
};
static std::vector<OccKey> g_occ;

static ctl_status occupancy(int dev, const void* k, int threads, size_t smem, int& bps, int& regs) {
    KernAttr ka;
    ctl_status st = kernel_attr(dev, k, ka);
    if (st != CTL_OK) return st;
    regs = ka.regs;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const auto& o : g_occ)
        if (o.dev == dev && o.k == k && o.threads == threads && o.smem == smem) {
            bps = o.bps;
            return CTL_OK;
        }
    CTL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, threads, smem));
    g_occ.push_back({dev, k, threads, smem, bps});
    return CTL_OK;
}

// ---------------------------------------------------------------------------
// Shared-memory sweep compiled for one network (NVRTC)
// ---------------------------------------------------------------------------
// The kernel body of ctl_sweep_dev.cuh instantiated with the network's
// geometry as compile-time constants: species, reactions, tree leaves, the
// stored tree levels (shift, fan-in, offset, count), sample instants and
// sampled species.  Loops over levels unroll and every level's offsets fold
// into the code; the tables stay in device memory (dev::Tables, the same
// kernel parameter as the first part of dev::Model).  On the 64 x 128
// network of the 65,536-simulation benchmark at 8 lanes per simulation this
// takes a sweep from 1,672 to 1,232 ms on one B200, with identical bits.
// Compiled once per process and (geometry, group size, register budget).

// Batches of at least this many simulations use the compiled kernel when
// the caller leaves the choice to the library (ctl_run_cfg.spec == 0); a
// compilation takes seconds, which a smaller batch would not recover.
static constexpr uint32_t SPEC_MIN_SIMS = 4096;

static std::string sweep_spec_source(const HostTables& t, int G, int minb) {
    dev::Model dm;
    tree_levels(t, dm);
    std::ostringstream o;
    o << "#define CTL_SPEC_GEOMETRY 1\n#include \"ctl_sweep_dev.cuh\"\n";
    o << "struct ModelCT : ctl::dev::Tables {\n";
    o << "    static constexpr int S = " << t.S << ", R = " << t.R << ", P = " << t.P << ", logP = " << t.logP
      << ", ns = " << t.ns << ", s_out = " << t.s_out << ", nlev = " << dm.nlev << ";\n";
    auto table = [&](const char* name, const int* v) {
        o << "    __host__ __device__ static constexpr int " << name << "(int li) { return ";
        for (int li = 0; li + 1 < dm.nlev; li++) o << "li == " << li << " ? " << v[li] << " : ";
        o << v[dm.nlev - 1] << "; }\n";
    };
    table("lev_shift", dm.lev_shift_v);
    table("lev_d", dm.lev_d_v);
    table("lev_base", dm.lev_base_v);
    table("lev_count", dm.lev_count_v);
    o << "};\n";
    o << "static_assert(sizeof(ModelCT) == sizeof(ctl::dev::Tables), \"kernel parameter layout\");\n";
    o << "extern \"C\" __global__ void __launch_bounds__(256, " << minb << ") ctl_sweep_spec("
         "const __grid_constant__ ModelCT m, const __grid_constant__ ctl::dev::Run run, "
         "const __grid_constant__ ctl::dev::Layout lay) {\n";
    o << "    ctl::dev::sweep_body<" << G << ">(m, run, lay);\n}\n";
    return o.str();
}

static std::mutex g_sspec_mu;
struct SweepSpec {
    std::string source;
    const void* kernel;
    std::string why;
};
static std::vector<SweepSpec> g_sspec;

// The compiled kernel for (network geometry, G, minb), or nullptr when NVRTC
// is missing or the compilation failed (the reason in *why).
static const void* sweep_spec_kernel(const HostTables& t, int G, int minb, std::string* why) {
    const std::string src = sweep_spec_source(t, G, minb);
    std::lock_guard<std::mutex> lk(g_sspec_mu);
    for (const auto& e : g_sspec)
        if (e.source == src) {
            if (why) *why = e.why;
            return e.kernel;
        }
    std::string w;
    const void* k = nvrtc_kernel(src, "ctl_sweep_spec", w);
    g_sspec.push_back({src, k, w});
    if (why) *why = w;
    return k;
}

// Host-buffer runs stage through stream-ordered allocations; keep the
// device's default pool from returning that memory to the driver at every
// synchronisation, so that repeated calls reuse it.
static void keep_pool_memory(int dev) {
    static bool done[16];
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (dev < 0 || dev >= 16 || done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[dev] = true;
}

static uint32_t n_bucket(uint32_t n) {
    uint32_t b = 0;
    while ((1u << b) < n && b < 31) b++;
    return b;
}

// Autotuned shape for (device, batch bucket, rate mode, flags), if any.
static bool find_tuned(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, ctl_model::Tuned& out) {
    std::lock_guard<std::mutex> lk(m->mu);
    for (const auto& e : m->tuned)
        if (e.device == cfg->device && e.nbucket == n_bucket(n) && e.uniform == (uint32_t)(cfg->uniform_rates != 0) &&
            e.flags == cfg->flags) {
            out = e;
            return true;
        }
    return false;
}

// SSA steps per round when neither the caller nor the tuner chose: 16, or 8
// when the whole batch fits in one wave of resident simulations -- the
// slowest simulation then sets the time, and its decisions wait less for the
// block's SSA bursts (Schlogl, 4,096 simulations on one B200: 87.7k against
// 80.2k sims/s).
static int default_ssa_budget(bool one_wave) { return one_wave ? 8 : 16; }
static int default_dec_budget(int G) { return G > 32 ? 2 : 1; }

// Launch shape of the register-resident sweep for tiny networks: one thread
// per simulation, `warp_sims` working lanes per warp.  Library choice of
// warp_sims: spread a small batch so that about 8 warps per SM work (each
// warp then runs the union of fewer simulations' paths), whole warps once the
// batch fills them; smaller blocks while the batch would not reach every SM.
struct TinyOcc {
    int dev;
    const void* kernel;
    int threads;
    size_t smem;
    int bps, regs;
};
static std::vector<TinyOcc> g_tiny_occ;

// Scheduling of the register-resident sweep when the caller does not choose.
static constexpr int TINY_DEFAULT_SCHED = 1;
// Block rounds: a block whose queue is closed finishes a lone simulation in
// warp lockstep (Schlogl's slowest simulation alone: 6.6 ms against 8.8 ms
// in rounds); with 2 or more the rounds keep their advantage (16,384
// simulations: 538k sims/s with 2, 551k with 1, 555k with none).
static constexpr uint32_t TINY_TAIL_SIMS = 1;

static ctl_status plan_tiny(const HostTables& t, const ctl_run_cfg* cfg, uint32_t n, LaunchPlan& pl) {
    DevAttr da;
    if (device_attr(cfg->device, da) != CTL_OK) return CTL_ERR_CUDA;
    pl.tinyP = t.P;
    pl.tinySM = tiny_species_bound(t);
    // register budget of the kernel compiled for the network (the library's
    // own is built for 2): 1 by default, which leaves the Schlogl kernels
    // unspilled (254 registers for block rounds, 187 for warp lockstep,
    // against 128 with spills at 2) -- 4,096 simulations on one B200: 330k
    // against 295k sims/s; 65,536: 722k against 650k
    const int minb = cfg->min_blocks > 0 ? cfg->min_blocks : 1;
    const int sched = cfg->sched > 0 ? cfg->sched : TINY_DEFAULT_SCHED;
    pl.spec = cfg->spec >= 0 ? tiny_spec_kernel(t, cfg->flags, minb, sched, nullptr) : nullptr;
    const void* k = pl.spec ? pl.spec : tiny_kernel_ptr(pl.tinyP, pl.tinySM);
    if (!k) {
        set_error("no register-resident kernel for this network");
        return CTL_ERR_SHAPE;
    }
    int threads = cfg->threads > 0 ? cfg->threads : (sched == 1 ? 64 : 256);
    if (threads % 32 || threads < 32 || threads > 256 || (sched == 1 && threads < 64)) {
        set_error("threads per block must be a multiple of 32, at most 256 (at least 64 for block rounds)");
        return CTL_ERR_ARG;
    }
    int ws = cfg->warp_sims;
    size_t smem = 0;
    uint64_t need = 0;
    if (sched == 1) {
        // Block rounds with regrouping: `ws` live simulations per warp of the
        // block on average, slots = ws * warps per block (at most 16 per warp
        // leaves a whole warp for the deciding ones in a 64-thread block);
        // a small batch is spread over every SM.
        const uint64_t wpb = (uint64_t)threads / 32;
        if (ws <= 0) {
            // 8 per warp (16 live simulations in a 64-thread block) measured
            // best for Schlogl, 4,096 simulations: 291k sims/s against 254k
            // with 14 (one block per SM) and 239k for warp lockstep
            const uint64_t per = ((uint64_t)n + (uint64_t)da.sm_count * wpb - 1) / ((uint64_t)da.sm_count * wpb);
            ws = (int)std::min<uint64_t>(8, std::max<uint64_t>(1, per));
        }
        const uint64_t slots = (uint64_t)ws * wpb;
        smem = (size_t)(2 * pl.tinySM + 20 + pl.tinyP) * (size_t)threads * 4;  // Packed<P, SM>::WORDS
        need = ((uint64_t)n + slots - 1) / slots;
    } else {
        if (ws <= 0) {
            const uint64_t target_warps = (uint64_t)da.sm_count * 8;
            ws = 1;
            while (ws < 32 && (uint64_t)n > target_warps * (uint64_t)ws) ws <<= 1;
        }
        const uint64_t warps = ((uint64_t)n + ws - 1) / ws;
        // a batch of about one wave: blocks of two warps spread it evenly over
        // the SMs (Schlogl, 4,096 simulations, 4 per warp: 230k against 212k
        // sims/s with 192-thread blocks, which leave some SMs one block and
        // others two)
        if (cfg->threads <= 0 && warps <= (uint64_t)da.sm_count * 8) threads = 64;
        need = (warps * 32 + threads - 1) / threads;
    }
    if (smem > (size_t)da.smem_optin) {
        set_error("register-resident sweep: the block-round exchange needs more shared memory than a block has");
        return CTL_ERR_SHAPE;
    }
    int bps = 0, regs = 0;
    {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        if (smem > 48 * 1024) {  // above the default dynamic limit: raise the kernel's ceiling once
            static std::vector<std::pair<int, const void*>> raised;
            bool done = false;
            for (const auto& r : raised) done = done || (r.first == cfg->device && r.second == k);
            if (!done) {
                cudaFuncAttributes fa;
                CTL_CUDA(cudaFuncGetAttributes(&fa, k));
                if (smem + fa.sharedSizeBytes > (size_t)da.smem_optin) {
                    set_error("register-resident sweep: the block-round exchange needs more shared memory than a "
                              "block has");
                    return CTL_ERR_SHAPE;
                }
                CTL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              da.smem_optin - (int)fa.sharedSizeBytes));
                raised.push_back({cfg->device, k});
            }
        }
        for (const auto& o : g_tiny_occ)
            if (o.dev == cfg->device && o.kernel == k && o.threads == threads && o.smem == smem) {
                bps = o.bps;
                regs = o.regs;
            }
        if (!bps) {
            cudaFuncAttributes fa;
            CTL_CUDA(cudaFuncGetAttributes(&fa, k));
            CTL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, threads, smem));
            regs = fa.numRegs;
            g_tiny_occ.push_back({cfg->device, k, threads, smem, bps, regs});
        }
    }
    if (bps < 1) {
        set_error("register-resident sweep cannot be resident with this shape");
        return CTL_ERR_SHAPE;
    }
    pl.G = 1;
    pl.threads = threads;
    pl.NS = sched == 1 ? ws * threads / 32 : threads / 32 * ws;
    pl.blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)bps * da.sm_count));
    pl.blocks_per_sm = bps;
    pl.sm_count = da.sm_count;
    pl.regs = regs;
    pl.smem = smem;
    pl.minb = pl.spec ? minb : 2;
    pl.sched = sched;
    // rounds of 16 SSA steps and 2 decisions for block rounds (a deciding warp
    // then takes about as long as a stepping one), 16 and 1 in warp lockstep
    pl.ssa_budget = cfg->ssa_budget > 0 ? cfg->ssa_budget : 16;
    pl.dec_budget = cfg->dec_budget > 0 ? cfg->dec_budget : (sched == 1 ? 2 : 1);
    pl.warp_sims = ws;
    return CTL_OK;
}

static ctl_status plan_launch(ctl_model* m, const ctl_run_cfg* cfg_in, uint32_t n, LaunchPlan& pl,
                              bool sums = false, bool use_tuned = true) {
    const HostTables& t = m->t;
    ctl_run_cfg tuned_cfg = *cfg_in;
    if (use_tuned && cfg_in->group <= 0 && cfg_in->threads <= 0) {
        ctl_model::Tuned e;
        if (find_tuned(m, cfg_in, n, e)) {
            tuned_cfg.group = e.group;
            tuned_cfg.threads = e.threads;
            if (tuned_cfg.ssa_budget <= 0) tuned_cfg.ssa_budget = e.ssa_budget;
            if (tuned_cfg.dec_budget <= 0) tuned_cfg.dec_budget = e.dec_budget;
            if (tuned_cfg.min_blocks <= 0) tuned_cfg.min_blocks = e.min_blocks;
            if (tuned_cfg.sched <= 0) tuned_cfg.sched = e.sched;
            if (tuned_cfg.warp_sims == 0) tuned_cfg.warp_sims = e.warp_sims;
        }
    }
    const ctl_run_cfg* cfg = &tuned_cfg;
    const bool tiny_ok = tiny_eligible(t);
    if (cfg->warp_sims > 0 && !tiny_ok) {
        set_error("warp_sims: the register-resident sweep takes at most 16 reactions, 8 species, 8 sampled "
                  "species and 3 reactant entries per reaction");
        return CTL_ERR_ARG;
    }
    if (tiny_ok && (cfg->warp_sims > 0 || (cfg->warp_sims == 0 && cfg->group <= 0)))
        return plan_tiny(t, cfg, n, pl);
    if (cfg->min_blocks == 1) {
        set_error("min_blocks 1 applies to the register-resident sweep only; the shared-memory sweep takes 2, 3 or 4");
        return CTL_ERR_ARG;
    }
    pl.ssa_budget = cfg->ssa_budget;
    pl.dec_budget = cfg->dec_budget;
    pl.sched = cfg->sched > 0 ? cfg->sched : 1;
    int G = cfg->group > 0 ? cfg->group : heuristic_group(t);
    if (cfg->group <= 0) {
        // small batches (fewer lanes than one 256-thread block per SM): more
        // lanes per simulation so that every SM gets warps
        DevAttr da0;
        if (device_attr(cfg->device, da0) != CTL_OK) return CTL_ERR_CUDA;
        const int gmax = std::min(t.P, 32);
        while (G < gmax && (uint64_t)n * G < (uint64_t)256 * da0.sm_count) G <<= 1;
    }
    if (G != 1 && G != 2 && G != 4 && G != 8 && G != 16 && G != 32 && G != 64 && G != 128 && G != 256) {
        set_error("group must be a power of two from 1 to 256");
        return CTL_ERR_ARG;
    }
    if (G > t.P) G = t.P;
    const int tstep = G > 32 ? G : 32;  // blocks hold whole groups and whole warps
    int threads = cfg->threads > 0 ? cfg->threads : 256;
    if (threads % tstep || threads < tstep || threads > 256) {
        set_error("threads per block must be a multiple of 32 and of the group size, at most 256");
        return CTL_ERR_ARG;
    }
    int dev_id = cfg->device;
    DevAttr da;
    if (device_attr(dev_id, da) != CTL_OK) return CTL_ERR_CUDA;
    KernAttr ka;
    const bool uni = cfg->uniform_rates != 0;
    // Register budget: for groups of 8 lanes or more, as many resident
    // blocks as the slot memory of a full 256-thread block allows (2 or 3);
    // smaller groups keep 2 (their spills cost more than the occupancy
    // gains: Schlogl at G = 1, 62k vs 56k sims/s); 4 only when chosen or tuned.
    int minb = cfg->min_blocks;
    if (minb <= 0) {
        const size_t full = slot_layout(t, G, 256 / G, uni, pl.lay, sums);
        minb = G >= 8 && 3 * (full + 1024) <= (size_t)da.smem_optin + 1024 ? 3 : 2;
    }
    // The kernel compiled for this network when asked (spec 1) or when the
    // batch is large enough to recover the compilation (spec 0), else, or
    // when NVRTC is unavailable, the library's own kernel.
    if (kernel_for(G, minb) == nullptr) {
        set_error("no sweep kernel for this group size and register budget");
        return CTL_ERR_ARG;
    }
    const bool want_spec = cfg->spec > 0 || (cfg->spec == 0 && n >= SPEC_MIN_SIMS);
    pl.spec = want_spec ? sweep_spec_kernel(t, G, minb, nullptr) : nullptr;
    const void* kern = pl.spec ? pl.spec : kernel_for(G, minb);
    if (ctl_status st = kernel_attr(dev_id, kern, ka); st != CTL_OK) return st;
    const size_t smem_max = ka.dyn_max;
    if (cfg->threads <= 0) {
        while (threads > tstep && (uint64_t)n * G < (uint64_t)threads * da.sm_count) threads -= tstep;
    }
    for (;;) {
        int NS = threads / G;
        size_t bytes = slot_layout(t, G, NS, uni, pl.lay, sums);
        if (bytes <= smem_max) {
            pl.smem = bytes;
            pl.NS = NS;
            break;
        }
        if (threads <= tstep) {
            set_error("network too large: one simulation slot needs " + std::to_string(bytes / NS) +
                      " bytes of shared memory");
            return CTL_ERR_SHAPE;
        }
        threads -= tstep;
    }
    pl.G = G;
    // Round budgets when neither the caller nor the tuner chose: 16 SSA steps
    // (8 for a batch of one wave, below) and one leap decision per round (one
    // B200, against 8 and 2: +7 % on the 64 x 128 network, +10 % on Schlogl,
    // +12 % on the uneven batch); groups of whole warps keep two decisions
    // (512 x 1024: 2.7 % better).
    if (pl.dec_budget <= 0) pl.dec_budget = default_dec_budget(G);
    pl.threads = threads;
    int bps = 0, regs = 0;
    if (ctl_status st = occupancy(dev_id, kern, threads, pl.smem, bps, regs); st != CTL_OK) return st;
    pl.minb = minb;
    if (bps < 1) {
        set_error("sweep kernel cannot be resident with this shape");
        return CTL_ERR_SHAPE;
    }
    pl.regs = regs;
    pl.blocks_per_sm = bps;
    pl.sm_count = da.sm_count;
    uint64_t need = (n + (uint64_t)pl.NS - 1) / pl.NS;
    uint64_t cap = (uint64_t)bps * da.sm_count;
    pl.blocks = (int)std::max<uint64_t>(1, std::min(need, cap));
    if (pl.ssa_budget <= 0) pl.ssa_budget = default_ssa_budget((uint64_t)n <= (uint64_t)pl.blocks * pl.NS);
    return CTL_OK;
}

static ctl_status enqueue_sweep(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* dX0,
                                const float* dc, uint32_t* dout, ctl_sim_info* dinfo,
                                cudaStream_t stream, const LaunchPlan& pl, const DeviceCopy& d,
                                unsigned long long* sums = nullptr, uint32_t sum_threads = 1,
                                uint32_t sum_prep = 1, uint32_t* done = nullptr, uint32_t done_shift = 0,
                                uint32_t* out_host = nullptr) {
    dev::Run run;
    run.seed = cfg->seed;
    run.eps = cfg->eps;
    run.nc = cfg->nc;
    run.ssa_factor = cfg->ssa_factor;
    run.ssa_steps = cfg->ssa_steps;
    run.flags = cfg->flags;
    run.max_steps = cfg->max_steps;
    run.sim_base = cfg->sim_base;
    run.n = n;
    run.uniform_c = cfg->uniform_rates != 0;
    run.ssa_budget = (uint32_t)pl.ssa_budget;
    run.dec_budget = (uint32_t)pl.dec_budget;
    run.warp_local = pl.sched == 2 ? 1u : 0u;
    run.tail_sims = TINY_TAIL_SIMS;
    run.X0 = dX0;
    run.c = dc;
    run.out = dout;
    run.sums = sums;
    run.sum_threads = sum_threads;
    run.sum_prep = sum_prep;
    run.done = done;
    run.done_shift = done_shift;
    run.out_host = out_host;
    run.info = dinfo;
    run.queue = d.ctrl;
    dev::Model dm = make_dev_model(m, d, cfg->flags);
    CTL_CUDA(cudaMemsetAsync(d.ctrl, 0, sizeof(uint32_t), stream));
    if (pl.warp_sims > 0) {
        // warp lockstep: simulations per warp; block rounds: live simulations per block
        uint32_t lanes = (uint32_t)(pl.sched == 1 ? pl.NS : pl.warp_sims);
        if (pl.spec) {
            SpecNet sn{dm.tvec, dm.tmax};
            void* sargs[] = {&sn, &run, &lanes};
            CTL_CUDA(cudaLaunchKernel(pl.spec, dim3((unsigned)pl.blocks), dim3((unsigned)pl.threads), sargs, pl.smem,
                                      stream));
        } else {
            tiny::Net net;
            tiny_net(m->t, cfg->flags, dm.tvec, net);
            void* targs[] = {&net, &run, &lanes};
            CTL_CUDA(cudaLaunchKernel(tiny_kernel_ptr(pl.tinyP, pl.tinySM), dim3((unsigned)pl.blocks),
                                      dim3((unsigned)pl.threads), targs, pl.smem, stream));
        }
        return CTL_OK;
    }
    // The compiled kernel's first parameter is the tables alone (the leading
    // part of dev::Model); the library's kernel takes the whole model.
    void* args[] = {pl.spec ? static_cast<void*>(static_cast<dev::Tables*>(&dm)) : static_cast<void*>(&dm), &run,
                    const_cast<dev::Layout*>(&pl.lay)};
    CTL_CUDA(cudaLaunchKernel(pl.spec ? pl.spec : kernel_for(pl.G, pl.minb), dim3((unsigned)pl.blocks),
                              dim3((unsigned)pl.threads), args, pl.smem, stream));
    return CTL_OK;
}

// Host rows given to ctl_run / ctl_fitness_run: counts >= 0 and rate
// constants finite and >= 0 (row 0 only when the caller declares every row
// equal).  A NaN or infinite rate makes the propensity sum non-finite, and
// simulated time then never reaches the next sample instant: the simulation
// would run to its step cap.
static ctl_status check_host_rows(const HostTables& t, uint32_t n, const int32_t* X0, const float* c,
                                  bool uniform) {
    const size_t nx = (size_t)n * (size_t)t.S;
    for (size_t i = 0; i < nx; i++)
        if (X0[i] < 0) {
            set_error("X0: negative count in row " + std::to_string(i / (size_t)t.S));
            return CTL_ERR_ARG;
        }
    const size_t nc = (uniform ? (size_t)1 : (size_t)n) * (size_t)t.R;
    for (size_t i = 0; i < nc; i++)
        if (!(c[i] >= 0.0f) || !std::isfinite(c[i])) {
            set_error("c: rate constant in row " + std::to_string(i / (size_t)t.R) + " is negative or not finite");
            return CTL_ERR_ARG;
        }
    return CTL_OK;
}

static ctl_status check_cfg(const ctl_run_cfg* cfg) {
    if (!cfg) {
        set_error("null run configuration");
        return CTL_ERR_ARG;
    }
    if (cfg->ssa_steps == 0) {
        set_error("ssa_steps must be positive");
        return CTL_ERR_ARG;
    }
    if (cfg->min_blocks != 0 && (cfg->min_blocks < 1 || cfg->min_blocks > 4)) {
        set_error("min_blocks must be 0 (library choice), 1 (register-resident sweep only), 2, 3 or 4");
        return CTL_ERR_ARG;
    }
    if (cfg->sched < 0 || cfg->sched > 2) {
        set_error("sched must be 0 (library choice), 1 (block regrouping) or 2 (warp-local)");
        return CTL_ERR_ARG;
    }
    if (cfg->warp_sims < -1 || cfg->warp_sims > 32) {
        set_error("warp_sims must be -1 (never), 0 (library choice) or 1..32");
        return CTL_ERR_ARG;
    }
    if (cfg->spec < -1 || cfg->spec > 1) {
        set_error("spec must be 0 (library choice), 1 (kernels compiled for the network whenever possible) or -1 "
                  "(never)");
        return CTL_ERR_ARG;
    }
    return CTL_OK;
}

struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;  // result of making the device current
    explicit DeviceGuard(int d) {
        cudaGetDevice(&prev);
        err = cudaSetDevice(d);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace ctl

using namespace ctl;

struct ctl_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
};

extern "C" void ctl_model_free(ctl_model* m) {
    if (!m) return;
    for (auto& d : m->dev) {
        if (d.buf) {
            int prev = 0;
            cudaGetDevice(&prev);
            cudaSetDevice(d.device);
            cudaFree(d.buf);
            cudaSetDevice(prev);
            d.buf = nullptr;
        }
    }
    delete m;
}

extern "C" ctl_status ctl_launch_query(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                                       ctl_launch_info* li) {
    if (!m || !li) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    DeviceGuard dg(cfg->device);
    LaunchPlan pl;
    st = plan_launch(m, cfg, n, pl);
    if (st != CTL_OK) return st;
    li->group = pl.G;
    li->threads = pl.threads;
    li->blocks = pl.blocks;
    li->slots_per_block = pl.NS;
    li->smem_bytes = (int32_t)pl.smem;
    li->regs_per_thread = pl.regs;
    li->blocks_per_sm = pl.blocks_per_sm;
    li->sm_count = pl.sm_count;
    li->min_blocks = pl.minb;
    li->sched = pl.sched;
    li->ssa_budget = pl.ssa_budget;
    li->dec_budget = pl.dec_budget;
    li->warp_sims = pl.warp_sims;
    li->specialized = pl.spec != nullptr ? 1 : 0;
    return CTL_OK;
}

extern "C" ctl_status ctl_run_device(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                                     const int32_t* d_X0, const float* d_c, uint32_t* d_samples,
                                     ctl_sim_info* d_info, void* stream) {
    if (!m) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    if (n == 0) return CTL_OK;
    if (!d_X0 || !d_c || !d_samples || !d_info) {
        set_error("null device buffer");
        return CTL_ERR_ARG;
    }
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    LaunchPlan pl;
    if ((st = plan_launch(m, cfg, n, pl)) != CTL_OK) return st;
    return enqueue_sweep(m, cfg, n, d_X0, d_c, d_samples, d_info, static_cast<cudaStream_t>(stream), pl, *d);
}

extern "C" ctl_status ctl_run(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* X0,
                              const float* c, uint32_t* samples, ctl_sim_info* info) {
    if (!m) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    if (n == 0) return CTL_OK;
    if (!X0 || !c || !samples || !info) {
        set_error("null host buffer");
        return CTL_ERR_ARG;
    }
    const HostTables& t = m->t;
    if ((st = check_host_rows(t, n, X0, c, cfg->uniform_rates != 0)) != CTL_OK) return st;
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    ctl_run_cfg rc = *cfg;
    if (!rc.uniform_rates) {  // one shared copy of c when every row equals row 0
        bool same = true;
        for (uint32_t i = 1; i < n && same; i++)
            same = std::memcmp(c + (size_t)i * t.R, c, (size_t)t.R * sizeof(float)) == 0;
        rc.uniform_rates = same ? 1 : 0;
    }
    cfg = &rc;
    LaunchPlan pl;
    if ((st = plan_launch(m, cfg, n, pl)) != CTL_OK) return st;
    const size_t bx = (size_t)n * t.S * 4, bc = (size_t)n * t.R * 4;
    const size_t row = (size_t)t.ns * t.s_out * 4, bo = (size_t)n * row, bi = (size_t)n * sizeof(ctl_sim_info);
    keep_pool_memory(cfg->device);
    // A pinned caller buffer that the device can address: the kernel copies
    // each finished simulation's row into it, so the copy-back runs inside
    // the sweep with no host thread in the loop.
    uint32_t* out_host = nullptr;
    {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, samples) == cudaSuccess) {
            if (pa.type == cudaMemoryTypeHost && pa.devicePointer) out_host = static_cast<uint32_t*>(pa.devicePointer);
        } else {
            cudaGetLastError();  // not a pointer CUDA knows: the copies below
        }
    }
    // Otherwise copy/compute overlap: the batch is cut into up to 16 chunks of
    // 2^shift simulations; the kernel counts finished simulations per chunk
    // (after a device-scope fence) and each complete chunk's rows are copied
    // back on a second stream while the sweep goes on.
    uint32_t shift = 0;
    while (((uint64_t)n >> shift) > 16) shift++;
    const uint32_t nch = (uint32_t)(((uint64_t)n + (1ull << shift) - 1) >> shift);
    const bool overlap = !out_host && bo >= ((size_t)64 << 20) && nch > 1;
    cudaStream_t s, cs;
    CTL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(s);
        return cuda_fail(cudaErrorMemoryAllocation, "ctl_run (copy stream)");
    }
    void *dx = nullptr, *dc = nullptr, *dout = nullptr, *dinf = nullptr, *ddone = nullptr;
    uint32_t* hdone = nullptr;
    cudaError_t e = cudaMallocAsync(&dx, bx, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dc, bc, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dout, bo, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dinf, bi, s);
    if (e == cudaSuccess && overlap) e = cudaMallocAsync(&ddone, (size_t)nch * 4, s);
    if (e == cudaSuccess && overlap) e = cudaMallocHost(reinterpret_cast<void**>(&hdone), (size_t)nch * 4);
    if (e == cudaSuccess && overlap) e = cudaMemsetAsync(ddone, 0, (size_t)nch * 4, s);
    if (e == cudaSuccess && overlap) {  // the copy stream starts after the counters are zeroed
        cudaEvent_t zeroed;
        e = cudaEventCreateWithFlags(&zeroed, cudaEventDisableTiming);
        if (e == cudaSuccess) {
            e = cudaEventRecord(zeroed, s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, zeroed, 0);
            cudaEventDestroy(zeroed);
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, X0, bx, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, c, bc, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        st = enqueue_sweep(m, cfg, n, static_cast<int32_t*>(dx), static_cast<float*>(dc),
                           static_cast<uint32_t*>(dout), static_cast<ctl_sim_info*>(dinf), s, pl, *d, nullptr, 1, 1,
                           static_cast<uint32_t*>(ddone), shift, out_host);
        if (st != CTL_OK) e = cudaErrorLaunchFailure;
    }
    std::vector<char> copied(nch, 0);
    if (e == cudaSuccess && overlap) {
        // poll the counters until the sweep ends, copying finished chunks
        while (e == cudaSuccess) {
            const cudaError_t q = cudaStreamQuery(s);
            if (q == cudaSuccess) break;  // the rest is copied below
            if (q != cudaErrorNotReady) { e = q; break; }
            if ((e = cudaMemcpyAsync(hdone, ddone, (size_t)nch * 4, cudaMemcpyDeviceToHost, cs)) != cudaSuccess) break;
            if ((e = cudaStreamSynchronize(cs)) != cudaSuccess) break;
            for (uint32_t j = 0; j < nch && e == cudaSuccess; j++) {
                const uint64_t lo = (uint64_t)j << shift, hi = std::min<uint64_t>(n, lo + (1ull << shift));
                if (!copied[j] && hdone[j] == (uint32_t)(hi - lo)) {
                    e = cudaMemcpyAsync(reinterpret_cast<unsigned char*>(samples) + lo * row,
                                        static_cast<unsigned char*>(dout) + lo * row, (hi - lo) * row,
                                        cudaMemcpyDeviceToHost, cs);
                    copied[j] = 1;
                }
            }
            if (e == cudaSuccess) std::this_thread::sleep_for(std::chrono::microseconds(200));
        }
    }
    for (uint32_t j = 0; j < nch && e == cudaSuccess && !out_host; j++) {  // chunks not yet copied, after the sweep
        const uint64_t lo = (uint64_t)j << shift, hi = std::min<uint64_t>(n, lo + (1ull << shift));
        if (!copied[j])
            e = cudaMemcpyAsync(reinterpret_cast<unsigned char*>(samples) + lo * row,
                                static_cast<unsigned char*>(dout) + lo * row, (hi - lo) * row,
                                cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(info, dinf, bi, cudaMemcpyDeviceToHost, s);
    const cudaError_t e3 = cudaStreamSynchronize(cs);  // copies in flight end before the buffers go
    if (dx) cudaFreeAsync(dx, s);
    if (dc) cudaFreeAsync(dc, s);
    if (dout) cudaFreeAsync(dout, s);
    if (dinf) cudaFreeAsync(dinf, s);
    if (ddone) cudaFreeAsync(ddone, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (hdone) cudaFreeHost(hdone);
    cudaStreamDestroy(cs);
    cudaStreamDestroy(s);
    if (st != CTL_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "ctl_run");
    if (e3 != cudaSuccess) return cuda_fail(e3, "ctl_run (copies)");
    if (e2 != cudaSuccess) return cuda_fail(e2, "ctl_run (sweep)");
    for (uint32_t i = 0; i < n; i++)
        if (info[i].status != CTL_SIM_OK) {
            set_error("simulation " + std::to_string(i) + " ended with status " + std::to_string(info[i].status));
            return CTL_ERR_STEP_LIMIT;
        }
    return CTL_OK;
}

// Measured autotuner: times the library's own plan, then candidate launch
// shapes greedily on the first `sample` simulations of the batch (results
// are identical for every shape, only the time differs) -- for tiny networks
// the register-resident sweep's simulations per warp; then lanes per
// simulation, threads per block, scheduling and register budget of the
// shared-memory sweep; then the per-round budgets -- and caches the fastest
// for this (device, batch-size bucket, rate mode, flags).  Nothing slower
// than the library's plan is cached.
extern "C" ctl_status ctl_spec_source(const ctl_model* m, int32_t group, int32_t min_blocks, char* buf, size_t cap,
                                      size_t* len) {
    if (!m || !len || group < 1 || group > 256 || (group & (group - 1)) || min_blocks < 2 || min_blocks > 4) {
        set_error("ctl_spec_source: group must be a power of two from 1 to 256 and min_blocks 2, 3 or 4");
        return CTL_ERR_ARG;
    }
    try {
        const std::string src = sweep_spec_source(m->t, std::min<int>(group, m->t.P), min_blocks);
        *len = src.size();
        if (!buf) return CTL_OK;
        if (cap <= src.size()) {
            set_error("ctl_spec_source: buffer too small");
            return CTL_ERR_SHAPE;
        }
        std::memcpy(buf, src.data(), src.size());
        buf[src.size()] = '\0';
        return CTL_OK;
    } catch (...) {
        set_error("ctl_spec_source: out of host memory");
        return CTL_ERR_OOM;
    }
}

extern "C" ctl_status ctl_autotune(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* d_X0,
                                   const float* d_c, uint32_t sample, ctl_launch_info* best) {
    if (!m || !d_X0 || !d_c || n == 0) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    const HostTables& t = m->t;
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    // The library's own plan for this batch (heuristic shape, default
    // budgets, no earlier tuning) is the incumbent every candidate must beat.
    ctl_run_cfg c0 = *cfg;
    c0.group = 0;
    c0.threads = 0;
    c0.min_blocks = 0;
    c0.sched = 0;
    c0.ssa_budget = 0;
    c0.dec_budget = 0;
    c0.warp_sims = 0;
    LaunchPlan p0;
    if ((st = plan_launch(m, &c0, n, p0, false, false)) != CTL_OK) return st;
    // A sample of about one wave of resident simulations is timed mostly by
    // its slowest simulations and favours shapes with short tails; at least
    // four waves (or the whole batch) weigh the steady state as the full
    // batch does.
    uint32_t k = sample == 0 || sample > n ? n : sample;
    k = (uint32_t)std::min<uint64_t>(n, std::max<uint64_t>(k, 4ull * (uint64_t)p0.blocks * (uint64_t)p0.NS));
    cudaStream_t s;
    CTL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *dout = nullptr, *dinf = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaError_t e = cudaMallocAsync(&dout, (size_t)k * t.ns * t.s_out * 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dinf, (size_t)k * sizeof(ctl_sim_info), s);
    struct Shape {
        int G, threads, ssa, dec, minb, sched, ws;  // ws > 0: register-resident sweep, else -1
    };
    auto time_shape = [&](const Shape& x, float& ms) -> ctl_status {
        ctl_run_cfg c = *cfg;
        c.group = x.ws > 0 ? 0 : x.G;
        c.threads = x.threads;
        c.ssa_budget = x.ssa;
        c.dec_budget = x.dec;
        c.min_blocks = x.minb;
        c.sched = x.sched;
        c.warp_sims = x.ws;
        // shared-memory candidates run the library's kernels: compiling one
        // kernel per candidate shape would cost more than the tuning itself
        // (the winner then runs compiled when the policy says so)
        if (x.ws <= 0) c.spec = -1;
        LaunchPlan pl;
        ctl_status r = plan_launch(m, &c, k, pl, false, false);
        if (r != CTL_OK) return r;
        // the faster of two runs: a kernel's first launch can include loading
        // its module (lazy loading, and every newly compiled kernel), which
        // would count against shapes that need a kernel not run before
        ms = 3.4e38f;
        for (int rep = 0; rep < 2; rep++) {
            cudaEventRecord(e0, s);
            r = enqueue_sweep(m, &c, k, d_X0, d_c, static_cast<uint32_t*>(dout), static_cast<ctl_sim_info*>(dinf), s,
                              pl, *d);
            cudaEventRecord(e1, s);
            if (r != CTL_OK) return r;
            if (cudaEventSynchronize(e1) != cudaSuccess) return CTL_ERR_CUDA;
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = t < ms ? t : ms;
        }
        return CTL_OK;
    };
    const int S0 = p0.ssa_budget;
    Shape bestx{p0.G, p0.threads, p0.ssa_budget, p0.dec_budget, p0.minb, p0.sched,
                p0.warp_sims > 0 ? p0.warp_sims : -1};
    float best_ms = 3.4e38f;
    auto consider = [&](const Shape& x) {
        float ms;
        if (time_shape(x, ms) == CTL_OK && ms < best_ms) {
            best_ms = ms;
            bestx = x;
        }
    };
    if (e == cudaSuccess) {
        consider(bestx);                                       // 0. the library's own plan
        if (tiny_eligible(t)) {                                // 1a. register-resident sweep
            for (int ws : {1, 2, 4, 8, 16, 32})                //     warp lockstep
                if (!(ws == p0.warp_sims && p0.sched == 2)) consider({1, 0, S0 > 0 ? S0 : 16, 1, 1, 2, ws});
            for (int ws : {4, 8, 12, 16})                      //     block rounds with regrouping
                if (!(ws == p0.warp_sims && p0.sched == 1)) consider({1, 0, S0 > 0 ? S0 : 16, 2, 1, 1, ws});
        }
        for (int G = 1; G <= 256 && G <= t.P; G <<= 1)        // 1b. lanes per simulation
            if (G != p0.G || p0.warp_sims > 0) consider({G, 256, S0, default_dec_budget(G), 2, 1, -1});
        const Shape b1 = bestx;
        for (int th : {64, 128, 192, 256}) {                   // 2. threads per block
            Shape x = b1;
            x.threads = th;
            if (th != b1.threads && (x.ws > 0 || (th % x.G == 0 && th >= x.G))) consider(x);
        }
        if (bestx.ws <= 0) {
            Shape x = bestx;                                   // 3. scheduling: warp-local vs block rounds
            x.sched = bestx.sched == 2 ? 1 : 2;
            consider(x);
        }
        {
            const Shape b3 = bestx;                            // 4. register budget (resident blocks); the
            for (int mb : {1, 2, 3, 4}) {                      //    register-resident kernel takes 1 or 2
                Shape y = b3;
                y.minb = mb;
                if (mb != b3.minb && (b3.ws > 0 ? mb <= 2 : mb >= 2)) consider(y);
            }
        }
        const Shape b4 = bestx;
        for (int sb : {4, 8, 16, 32}) {                        // 5. SSA steps per round
            Shape x = b4;
            x.ssa = sb;
            if (sb != b4.ssa) consider(x);
        }
        {
            const Shape b5 = bestx;
            for (int db : {1, 2, 4}) {                         // 6. decisions per round
                Shape x = b5;
                x.dec = db;
                if (db != b5.dec) consider(x);
            }
        }
    }
    if (dout) cudaFreeAsync(dout, s);
    if (dinf) cudaFreeAsync(dinf, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "ctl_autotune");
    if (e2 != cudaSuccess) return cuda_fail(e2, "ctl_autotune (sweeps)");
    {
        std::lock_guard<std::mutex> lk(m->mu);
        const uint32_t nb = n_bucket(n), uni = (uint32_t)(cfg->uniform_rates != 0);
        const ctl_model::Tuned tu{cfg->device, nb, uni, cfg->flags, bestx.ws > 0 ? 0 : bestx.G, bestx.threads,
                                  bestx.ssa, bestx.dec, bestx.minb, bestx.sched, bestx.ws};
        bool found = false;
        for (auto& x : m->tuned)
            if (x.device == cfg->device && x.nbucket == nb && x.uniform == uni && x.flags == cfg->flags) {
                x = tu;
                found = true;
            }
        if (!found) m->tuned.push_back(tu);
    }
    if (best) {
        ctl_run_cfg c = *cfg;
        c.group = 0;
        c.threads = 0;
        c.min_blocks = 0;
        c.sched = 0;
        c.warp_sims = 0;
        return ctl_launch_query(m, &c, n, best);
    }
    return CTL_OK;
}

extern "C" ctl_status ctl_graph_create(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                                       const int32_t* d_X0, const float* d_c, uint32_t* d_samples,
                                       ctl_sim_info* d_info, void* stream, ctl_graph** out) {
    if (!m || !out) return CTL_ERR_ARG;
    *out = nullptr;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    LaunchPlan pl;
    if ((st = plan_launch(m, cfg, n, pl)) != CTL_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStream_t cap = s;
    bool own = false;
    if (cap == nullptr) {
        CTL_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        own = true;
    }
    ctl_graph* g = new ctl_graph();
    g->device = cfg->device;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        st = enqueue_sweep(m, cfg, n, d_X0, d_c, d_samples, d_info, cap, pl, *d);
        cudaError_t e2 = cudaStreamEndCapture(cap, &g->graph);
        if (st == CTL_OK && e2 != cudaSuccess) e = e2;
    }
    if (e == cudaSuccess && st == CTL_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (own) cudaStreamDestroy(cap);
    if (e != cudaSuccess || st != CTL_OK) {
        ctl_graph_free(g);
        return st != CTL_OK ? st : cuda_fail(e, "ctl_graph_create");
    }
    *out = g;
    return CTL_OK;
}

// Several sweeps as parallel branches of one graph: a fork from the
// capture stream into one stream per batch, joined back at the end.  The
// persistent kernels then share the GPU: as one batch's blocks finish (its
// queue drained), the next batch's blocks take their SMs, so a batch's
// latency-bound tail overlaps the others' work (the reference runs such a
// batch as separate processes or passes, kernel.cu:242-345).
extern "C" ctl_status ctl_graph_create_multi(uint32_t count, ctl_model* const* models, const ctl_run_cfg* cfgs,
                                             const uint32_t* n, const int32_t* const* d_X0,
                                             const float* const* d_c, uint32_t* const* d_samples,
                                             ctl_sim_info* const* d_info, void* stream, ctl_graph** out) {
    if (!out) return CTL_ERR_ARG;
    *out = nullptr;
    if (count == 0 || count > 64 || !models || !cfgs || !n || !d_X0 || !d_c || !d_samples || !d_info) {
        set_error("ctl_graph_create_multi: 1 to 64 batches with every array given");
        return CTL_ERR_ARG;
    }
    const int device = cfgs[0].device;
    for (uint32_t i = 0; i < count; i++) {
        ctl_status st = check_cfg(&cfgs[i]);
        if (st != CTL_OK) return st;
        if (!models[i] || cfgs[i].device != device) {
            set_error("ctl_graph_create_multi: every batch needs a model and the same device");
            return CTL_ERR_ARG;
        }
        for (uint32_t j = 0; j < i; j++)
            if (models[j] == models[i]) {  // one work-queue ticket per model and device
                set_error("ctl_graph_create_multi: a model may appear once per graph");
                return CTL_ERR_ARG;
            }
    }
    DeviceGuard dg(device);
    if (dg.err != cudaSuccess) return cuda_fail(dg.err, "ctl_graph_create_multi (cudaSetDevice)");
    std::vector<DeviceCopy*> dcs(count, nullptr);
    std::vector<LaunchPlan> pls(count);
    for (uint32_t i = 0; i < count; i++) {
        ctl_status st = ensure_device(models[i], device, dcs[i]);
        if (st == CTL_OK) st = plan_launch(models[i], &cfgs[i], n[i], pls[i]);
        if (st != CTL_OK) return st;
    }
    cudaStream_t cap = static_cast<cudaStream_t>(stream);
    bool own = false;
    if (cap == nullptr) {
        CTL_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        own = true;
    }
    std::vector<cudaStream_t> br(count, nullptr);
    std::vector<cudaEvent_t> ev(count + 1, nullptr);
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 1; i < count && e == cudaSuccess; i++) e = cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking);
    for (uint32_t i = 0; i <= count && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    ctl_graph* g = new ctl_graph();
    g->device = device;
    ctl_status st = CTL_OK;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t ec = cudaEventRecord(ev[0], cap);  // fork
        for (uint32_t i = 0; i < count && ec == cudaSuccess && st == CTL_OK; i++) {
            cudaStream_t s = i == 0 ? cap : br[i];
            if (i > 0) ec = cudaStreamWaitEvent(s, ev[0], 0);
            if (ec == cudaSuccess)
                st = enqueue_sweep(models[i], &cfgs[i], n[i], d_X0[i], d_c[i], d_samples[i], d_info[i], s, pls[i],
                                   *dcs[i]);
            if (i > 0 && ec == cudaSuccess && st == CTL_OK) ec = cudaEventRecord(ev[i], s);
            if (i > 0 && ec == cudaSuccess && st == CTL_OK) ec = cudaStreamWaitEvent(cap, ev[i], 0);  // join
        }
        const cudaError_t e2 = cudaStreamEndCapture(cap, &g->graph);
        e = ec != cudaSuccess ? ec : e2;
    }
    if (e == cudaSuccess && st == CTL_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    for (auto s : br)
        if (s) cudaStreamDestroy(s);
    for (auto x : ev)
        if (x) cudaEventDestroy(x);
    if (own) cudaStreamDestroy(cap);
    if (e != cudaSuccess || st != CTL_OK) {
        ctl_graph_free(g);
        return st != CTL_OK ? st : cuda_fail(e, "ctl_graph_create_multi");
    }
    *out = g;
    return CTL_OK;
}

extern "C" ctl_status ctl_graph_launch(ctl_graph* g, void* stream) {
    if (!g || !g->exec) return CTL_ERR_ARG;
    DeviceGuard dg(g->device);
    CTL_CUDA(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
    return CTL_OK;
}

extern "C" void ctl_graph_free(ctl_graph* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

extern "C" ctl_status ctl_fitness_device(const uint32_t* d_samples, uint32_t ns, uint32_t s_out,
                                         const uint32_t* d_target, const uint8_t* d_experiment,
                                         uint32_t experiments, uint32_t repetitions, uint32_t threads,
                                         uint32_t blocks, uint32_t p_rep, double* d_fitness, void* stream) {
    if (!d_samples || !d_target || !d_experiment || !d_fitness || !threads || !blocks || !p_rep ||
        blocks % p_rep || !ns || !s_out) {
        set_error("ctl_fitness_device: invalid argument");
        return CTL_ERR_ARG;
    }
    const uint32_t nsets = (uint32_t)(((uint64_t)threads * blocks) / p_rep);
    dev::fitness_kernel<<<(nsets + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        d_samples, d_target, d_experiment, d_fitness, threads, nsets, p_rep, ns, s_out, experiments, repetitions);
    CTL_CUDA(cudaGetLastError());
    return CTL_OK;
}

extern "C" ctl_status ctl_fitness(ctl_model* m, const ctl_target* t, const ctl_run_cfg* cfg,
                                  const uint32_t* samples, double* fitness) {
    if (!m || !t || !cfg || !samples || !fitness) return CTL_ERR_ARG;
    const HostTables& h = m->t;
    if (t->ns != (uint32_t)h.ns || t->s_out != (uint32_t)h.s_out) {
        set_error("fitness target does not match the model's samples");
        return CTL_ERR_SHAPE;
    }
    DeviceGuard dg(cfg->device);
    const uint64_t N = (uint64_t)t->threads * t->blocks;
    const uint32_t nsets = (uint32_t)(N / t->p_rep);
    const size_t bs = (size_t)N * h.ns * h.s_out * 4, bt = t->series.size() * 4, bw = (size_t)N;
    cudaStream_t s;
    CTL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *ds = nullptr, *dt = nullptr, *dw = nullptr, *df = nullptr;
    cudaError_t e = cudaMallocAsync(&ds, bs, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dt, std::max<size_t>(bt, 4), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dw, std::max<size_t>(bw, 4), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&df, (size_t)N * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, samples, bs, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && bt) e = cudaMemcpyAsync(dt, t->series.data(), bt, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dw, t->thread2experiment.data(), bw, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(df, 0, (size_t)N * 8, s);
    if (e == cudaSuccess && nsets) {
        dev::fitness_kernel<<<(nsets + 127) / 128, 128, 0, s>>>(
            static_cast<uint32_t*>(ds), static_cast<uint32_t*>(dt), static_cast<uint8_t*>(dw),
            static_cast<double*>(df), t->threads, nsets, t->p_rep, (uint32_t)h.ns, (uint32_t)h.s_out,
            t->experiments, t->repetitions);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(fitness, df, (size_t)N * 8, cudaMemcpyDeviceToHost, s);
    if (ds) cudaFreeAsync(ds, s);
    if (dt) cudaFreeAsync(dt, s);
    if (dw) cudaFreeAsync(dw, s);
    if (df) cudaFreeAsync(df, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) return cuda_fail(e, "ctl_fitness");
    if (e2 != cudaSuccess) return cuda_fail(e2, "ctl_fitness (kernel)");
    return CTL_OK;
}

// ---------------------------------------------------------------------------
// Fitness mode without per-simulation samples
// ---------------------------------------------------------------------------

static ctl_status check_sums_shape(uint32_t n, uint32_t threads, uint32_t p_rep) {
    if (!threads || !p_rep || n % threads || (n / threads) % p_rep) {
        set_error("fitness mode needs n = threads * blocks with blocks a multiple of p_rep");
        return CTL_ERR_ARG;
    }
    return CTL_OK;
}

extern "C" ctl_status ctl_run_device_sums(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* d_X0,
                                          const float* d_c, uint32_t threads, uint32_t p_rep, uint64_t* d_sums,
                                          ctl_sim_info* d_info, void* stream) {
    if (!m) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    if (n == 0) return CTL_OK;
    if ((st = check_sums_shape(n, threads, p_rep)) != CTL_OK) return st;
    if (!d_X0 || !d_c || !d_sums || !d_info) {
        set_error("null device buffer");
        return CTL_ERR_ARG;
    }
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    LaunchPlan pl;
    if ((st = plan_launch(m, cfg, n, pl, true)) != CTL_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t words = (size_t)(n / p_rep) * m->t.ns * m->t.s_out;
    CTL_CUDA(cudaMemsetAsync(d_sums, 0, words * 8, s));
    return enqueue_sweep(m, cfg, n, d_X0, d_c, nullptr, d_info, s, pl, *d,
                         reinterpret_cast<unsigned long long*>(d_sums), threads, p_rep);
}

extern "C" ctl_status ctl_fitness_sums_device(const uint64_t* d_sums, uint32_t ns, uint32_t s_out,
                                              const uint32_t* d_target, const uint8_t* d_experiment,
                                              uint32_t experiments, uint32_t repetitions, uint32_t threads,
                                              uint32_t blocks, uint32_t p_rep, double* d_fitness, void* stream) {
    if (!d_sums || !d_target || !d_experiment || !d_fitness || !threads || !blocks || !p_rep ||
        blocks % p_rep || !ns || !s_out) {
        set_error("ctl_fitness_sums_device: invalid argument");
        return CTL_ERR_ARG;
    }
    const uint32_t nsets = (uint32_t)(((uint64_t)threads * blocks) / p_rep);
    dev::fitness_sums_kernel<<<(nsets + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const unsigned long long*>(d_sums), d_target, d_experiment, d_fitness, nsets, p_rep, ns,
        s_out, experiments, repetitions);
    CTL_CUDA(cudaGetLastError());
    return CTL_OK;
}

extern "C" ctl_status ctl_fitness_run(ctl_model* m, const ctl_target* t, const ctl_run_cfg* cfg, const int32_t* X0,
                                      const float* c, double* fitness, ctl_sim_info* info) {
    if (!m || !t || !X0 || !c || !fitness || !info) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    const HostTables& h = m->t;
    if (t->ns != (uint32_t)h.ns || t->s_out != (uint32_t)h.s_out) {
        set_error("fitness target does not match the model's samples");
        return CTL_ERR_SHAPE;
    }
    const uint64_t N64 = (uint64_t)t->threads * t->blocks;
    if (N64 == 0 || N64 > 0xffffffffull) return CTL_ERR_ARG;
    const uint32_t N = (uint32_t)N64;
    if ((st = check_sums_shape(N, t->threads, t->p_rep)) != CTL_OK) return st;
    const uint32_t nsets = N / t->p_rep;
    if ((st = check_host_rows(h, N, X0, c, cfg->uniform_rates != 0)) != CTL_OK) return st;
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    ctl_run_cfg rc = *cfg;
    if (!rc.uniform_rates) {
        bool same = true;
        for (uint32_t i = 1; i < N && same; i++)
            same = std::memcmp(c + (size_t)i * h.R, c, (size_t)h.R * sizeof(float)) == 0;
        rc.uniform_rates = same ? 1 : 0;
    }
    LaunchPlan pl;
    if ((st = plan_launch(m, &rc, N, pl, true)) != CTL_OK) return st;
    keep_pool_memory(cfg->device);
    const size_t bx = (size_t)N * h.S * 4, bc = (size_t)N * h.R * 4, bi = (size_t)N * sizeof(ctl_sim_info);
    const size_t bsum = (size_t)nsets * h.ns * h.s_out * 8, bt = t->series.size() * 4, bw = (size_t)N;
    cudaStream_t s;
    CTL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *dx = nullptr, *dc = nullptr, *dinf = nullptr, *dsum = nullptr, *dt = nullptr, *dw = nullptr, *df = nullptr;
    cudaError_t e = cudaMallocAsync(&dx, bx, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dc, bc, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dinf, bi, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dsum, bsum, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dt, std::max<size_t>(bt, 4), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dw, std::max<size_t>(bw, 4), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&df, (size_t)N * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, X0, bx, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, c, bc, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && bt) e = cudaMemcpyAsync(dt, t->series.data(), bt, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dw, t->thread2experiment.data(), bw, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dsum, 0, bsum, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(df, 0, (size_t)N * 8, s);
    if (e == cudaSuccess) {
        st = enqueue_sweep(m, &rc, N, static_cast<int32_t*>(dx), static_cast<float*>(dc), nullptr,
                           static_cast<ctl_sim_info*>(dinf), s, pl, *d, static_cast<unsigned long long*>(dsum),
                           t->threads, t->p_rep);
        if (st != CTL_OK) e = cudaErrorLaunchFailure;
    }
    if (e == cudaSuccess && nsets) {
        dev::fitness_sums_kernel<<<(nsets + 127) / 128, 128, 0, s>>>(
            static_cast<unsigned long long*>(dsum), static_cast<uint32_t*>(dt), static_cast<uint8_t*>(dw),
            static_cast<double*>(df), nsets, t->p_rep, (uint32_t)h.ns, (uint32_t)h.s_out, t->experiments,
            t->repetitions);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(fitness, df, (size_t)N * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(info, dinf, bi, cudaMemcpyDeviceToHost, s);
    for (void* p : {dx, dc, dinf, dsum, dt, dw, df})
        if (p) cudaFreeAsync(p, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (st != CTL_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "ctl_fitness_run");
    if (e2 != cudaSuccess) return cuda_fail(e2, "ctl_fitness_run (sweep)");
    for (uint32_t i = 0; i < N; i++)
        if (info[i].status != CTL_SIM_OK) {
            set_error("simulation " + std::to_string(i) + " ended with status " + std::to_string(info[i].status));
            return CTL_ERR_STEP_LIMIT;
        }
    return CTL_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free sweep
// ---------------------------------------------------------------------------
//
// Some callers cannot call cudaMalloc: an application that hands out device
// memory only through its own pool allocator, a host that has already sized
// and locked its device memory budget, or a library layer that must not grow
// device memory behind its caller's back.  ctl_run_device needs device memory
// of its own for the model tables and the work-queue ticket, which it
// allocates on first use per device.  ctl_run_device_noalloc keeps both in
// the fixed array below instead and allocates nothing.

namespace ctl {

// Holds the work-queue ticket (first 256 bytes) and the model tables of the
// call in progress.  It lives in every device that loads this library, for
// as long as the library stays loaded.
constexpr size_t NOALLOC_BYTES = (size_t)1 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_base[16];  // device address of g_noalloc_scratch, per device

}  // namespace ctl

extern "C" ctl_status ctl_run_device_noalloc(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                                             const int32_t* d_X0, const float* d_c, uint32_t* d_samples,
                                             ctl_sim_info* d_info, void* stream) {
    if (!m) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    if (cfg->device < 0 || cfg->device >= 16) {
        set_error("device ordinal out of range");
        return CTL_ERR_ARG;
    }
    const HostTables& t = m->t;
    // Same table layout as the allocating path, after a 256-byte ticket area.
    DeviceCopy d;
    size_t off = 256;
    auto place = [&](size_t bytes) {
        size_t o = off;
        off = align16(off + bytes);
        return o;
    };
    table_layout(t, d, place);
    if (off > NOALLOC_BYTES) {
        set_error("ctl_run_device_noalloc: the model tables need " + std::to_string(off) +
                  " bytes, the allocation-free path holds at most " + std::to_string(NOALLOC_BYTES) +
                  " (1 MiB); use ctl_run_device");
        return CTL_ERR_SHAPE;
    }
    if (n == 0) return CTL_OK;
    if (!d_X0 || !d_c || !d_samples || !d_info) {
        set_error("null device buffer");
        return CTL_ERR_ARG;
    }
    DeviceGuard dg(cfg->device);
    // The device must exist and be current before its copy of the array is
    // looked up, and the launch must be possible before anything is written
    // into the array: a call that fails leaves the shared array untouched.
    if (dg.err != cudaSuccess) return cuda_fail(dg.err, "ctl_run_device_noalloc (cudaSetDevice)");
    // Never a kernel compiled at run time here: loading one allocates device
    // memory for its code.  The library's own kernels run instead.
    ctl_run_cfg rc = *cfg;
    rc.spec = -1;
    cfg = &rc;
    LaunchPlan pl;
    if ((st = plan_launch(m, cfg, n, pl)) != CTL_OK) return st;
    void* base = nullptr;
    {
        // Set-up, once per device with that device current: the host-side
        // name of the array is not a device address; ask for its address.
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_base[cfg->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
            g_noalloc_base[cfg->device] = p;
        }
        base = g_noalloc_base[cfg->device];
    }
    d.device = cfg->device;
    d.buf = base;
    d.bytes = off;
    d.ctrl = static_cast<uint32_t*>(base);  // ticket: cleared by enqueue_sweep before the launch
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(base);
    auto put = [&](size_t o, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpyAsync(b + o, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
    };
    cudaError_t e = cudaSuccess;
    table_fill(t, d, [&](size_t o, const void* src, size_t bytes) {
        e = put(o, src, bytes);
        return e == cudaSuccess;
    });
    if (e != cudaSuccess) return cuda_fail(e, "ctl_run_device_noalloc (tables)");
    return enqueue_sweep(m, cfg, n, d_X0, d_c, d_samples, d_info, s, pl, d);
}

// Device side of the persistent tau-leaping / SSA sweep for sm_100a
// (shared by ctl_sweep.cu and the per-group-size kernel files
// ctl_sweep_g*.cu, which the build compiles in parallel).
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
//
// The device code is written against a model type M with the fields of
// Model below.  The library's kernels read the network's geometry (species,
// reactions, tree levels, sample counts) from that parameter block at run
// time; a kernel compiled for one network at run time by NVRTC
// (ctl_sweep.cu, sweep_spec_kernel) instantiates the same code with a type
// whose geometry fields are static constexpr members of the same names, so
// that loops over tree levels, species and samples have constant bounds and
// every level's offsets fold into the code.  Both give the same bits.
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "ctl_internal.h"
#endif
#include "ctl_devmath.cuh"

// Loops over the stored tree levels: unrolled when the geometry is a
// compile-time constant (network-compiled kernels), left to the compiler
// otherwise.
#ifdef CTL_SPEC_GEOMETRY
#define CTL_UNROLL_LEVELS _Pragma("unroll")
#else
#define CTL_UNROLL_LEVELS
#endif

namespace ctl {
namespace dev {

// The model's tables in device memory (and the end time): the part of the
// model that every kernel reads at run time.
struct Tables {
    const uint32_t* __restrict__ reac_off;
    const uint32_t* __restrict__ reac_ent;
    const uint2* __restrict__ reac_desc;  // [R] packed reactants, x == 0xffffffff: general list
    const uint32_t* __restrict__ v_off;  // V or F species-major (quirk Q5)
    const uint32_t* __restrict__ v_ent;
    const uint32_t* __restrict__ fs_off;
    const uint32_t* __restrict__ fs_ent;
    const uint32_t* __restrict__ fr_off;
    const uint32_t* __restrict__ fr_ent;
    const uint32_t* __restrict__ dep_off;
    const uint32_t* __restrict__ dep_ent;
    const uint8_t* __restrict__ hor;
    const uint8_t* __restrict__ hort;
    const double* __restrict__ tvec;
    const uint32_t* __restrict__ cs;
    double tmax;
};

// Tables plus the geometry, read at run time (the library's own kernels).
struct Model : Tables {
    int S, R, P, logP, ns, s_out;
    // Stored levels of the binary sum tree: level 3, 6, 9, ... below the
    // root, and the root.  Stored level li holds the nodes that cover 2^shift
    // leaves; each is the pairwise sum of 2^d nodes of stored level li-1
    // (li = 0: of leaves).  Intermediate levels are recomputed in registers.
    int nlev;
    int lev_shift_v[10], lev_d_v[10], lev_base_v[10], lev_count_v[10];
    __device__ __forceinline__ int lev_shift(int li) const { return lev_shift_v[li]; }
    __device__ __forceinline__ int lev_d(int li) const { return lev_d_v[li]; }
    __device__ __forceinline__ int lev_base(int li) const { return lev_base_v[li]; }
    __device__ __forceinline__ int lev_count(int li) const { return lev_count_v[li]; }
};

// Shared-memory slot layout.  G == 1: element i of slot j at i*NS + j
// (consecutive threads hit consecutive banks).  G > 1: slot-contiguous
// arrays of odd padded length (lanes of one group hit distinct banks).
struct Layout {
    uint32_t off_X, off_X1, off_a, off_K, off_tree, off_crit, off_c, off_state, off_list, off_grp, off_last;
    uint32_t len_S, len_P, len_C, len_T, len_O;  // padded lengths (G > 1)
};

// Per-slot scalars, one array each (index = slot).
struct StateArrays {
    double *T, *tl, *tnext;
    unsigned long long* fire;
    uint32_t *sim, *cursor, *n, *burst, *leaps, *ssa, *rej, *flags;
};
constexpr uint32_t ST_IN_SSA = 1u, ST_STATUS_SHIFT = 8;
constexpr uint32_t PH_EMPTY = 0u, PH_DECIDE = 1u, PH_SSA = 2u, PH_CLOSED = 3u;

// ---------------------------------------------------------------------------
// Groups and slots
// ---------------------------------------------------------------------------

// The lanes that work on one simulation.  G <= 32: a slice of one warp
// (warp-synchronous primitives).  G = 64, 128, 256: whole warps, synchronised
// by named barrier 1 + group index, cross-warp reductions through a small
// per-group scratch area in shared memory.
template <int G>
struct Grp {
    static constexpr int W = G > 32 ? G / 32 : 1;  // warps per group
    uint32_t lane, mask, bar;
    float* fs;                   // [W] per-group scratch (G > 32)
    unsigned long long* us;      // [W]
    uint32_t* ws;                // [1]
    __device__ Grp() {
        lane = threadIdx.x % G;
        const uint32_t l = threadIdx.x & 31u;
        mask = (G >= 32) ? 0xffffffffu : (((1u << G) - 1u) << (l & ~(uint32_t)(G - 1)));
        bar = 1u + threadIdx.x / G;
        fs = nullptr;
        us = nullptr;
        ws = nullptr;
    }
    __device__ __forceinline__ void scratch(unsigned char* base) {  // 16*W + 16 bytes per group
        unsigned char* b = base + (threadIdx.x / G) * (16 * W + 16);
        us = reinterpret_cast<unsigned long long*>(b);
        fs = reinterpret_cast<float*>(b + 8 * W);
        ws = reinterpret_cast<uint32_t*>(b + 16 * W);
    }
    __device__ __forceinline__ void sync() const {
        if constexpr (G > 32) asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(G) : "memory");
        else if constexpr (G > 1) __syncwarp(mask);
    }
    __device__ __forceinline__ bool any(bool p) const {
        if constexpr (G == 1) return p;
        if constexpr (G > 32) {
            uint32_t r;
            asm volatile(
                "{\n\t.reg .pred a, b;\n\t"
                "setp.ne.u32 a, %1, 0;\n\t"
                "bar.red.or.pred b, %2, %3, a;\n\t"
                "selp.u32 %0, 1, 0, b;\n\t}"
                : "=r"(r)
                : "r"((uint32_t)p), "r"(bar), "r"(G)
                : "memory");
            return r != 0;
        }
        return __any_sync(mask, p) != 0;
    }
    __device__ __forceinline__ float fmin(float v) const {
#pragma unroll
        for (int o = (G < 32 ? G : 32) / 2; o > 0; o >>= 1) {
            float t = __shfl_xor_sync(mask, v, o);
            v = t < v ? t : v;
        }
        if constexpr (G > 32) {
            sync();  // earlier readers of the scratch are done
            if ((lane & 31u) == 0) fs[lane >> 5] = v;
            sync();
            v = fs[0];
#pragma unroll
            for (int i = 1; i < W; i++) v = fs[i] < v ? fs[i] : v;
        }
        return v;
    }
    __device__ __forceinline__ unsigned long long sum(unsigned long long v) const {
#pragma unroll
        for (int o = (G < 32 ? G : 32) / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        if constexpr (G > 32) {
            sync();
            if ((lane & 31u) == 0) us[lane >> 5] = v;
            sync();
            v = us[0];
#pragma unroll
            for (int i = 1; i < W; i++) v += us[i];
        }
        return v;
    }
    __device__ __forceinline__ uint32_t bcast(uint32_t v) const {
        if constexpr (G == 1) return v;
        if constexpr (G > 32) {
            sync();
            if (lane == 0) ws[0] = v;
            sync();
            return ws[0];
        }
        return __shfl_sync(mask, v, 0, G);
    }
};

struct Slot {
    int32_t* X;
    int32_t* X1;
    float* a;
    double* tree;
    uint32_t* K;
    uint8_t* crit;
    float* c;
    uint32_t* last;  // fitness mode: the simulation's last recorded sample [s_out]
    int st;   // element stride of the slot arrays
    int cst;  // element stride of the rate constants (1 when shared by the block)
    __device__ __forceinline__ int32_t& x(int i) const { return X[i * st]; }
    __device__ __forceinline__ int32_t& x1(int i) const { return X1[i * st]; }
    __device__ __forceinline__ float& pa(int i) const { return a[i * st]; }
    __device__ __forceinline__ double& t(int i) const { return tree[i * st]; }
    __device__ __forceinline__ uint32_t& k(int i) const { return K[i * st]; }
    __device__ __forceinline__ uint8_t& cr(int i) const { return crit[i * st]; }
    __device__ __forceinline__ float& cf(int i) const { return c[i * cst]; }
    __device__ __forceinline__ uint32_t& lst(int i) const { return last[i * st]; }
};

// One reactant factor: X for coefficient 1, 0.5 X (X-1) for 2.
__device__ __forceinline__ float react_factor(int32_t x, uint32_t st) {
    const float hx = (float)x;
    return st == 1u ? hx : (0.5f * hx) * (hx - 1.0f);
}

// Mass-action propensity in FP32 (CalculatePropensity, tau.cu:1443-1470):
// c times, per reactant entry in species order, X (coefficient 1),
// 0.5 X (X-1) (coefficient 2) or the product of (X-e+1)/e (higher); zero when
// a reactant count is below its coefficient.  Reactions with at most two
// entries of coefficient <= 2 read one packed descriptor.
template <class M>
__device__ __forceinline__ float prop(const M& m, const Slot& sl, int r) {
    float v = sl.cf(r);
    const uint2 d = m.reac_desc[r];
    if (d.x != 0xffffffffu) {
        if (d.x) {
            const int32_t x = sl.x((int)(d.x >> 8));
            const uint32_t st = d.x & 0xffu;
            if (x < (int32_t)st) return 0.0f;
            v = v * react_factor(x, st);
        }
        if (d.y) {
            const int32_t x = sl.x((int)(d.y >> 8));
            const uint32_t st = d.y & 0xffu;
            if (x < (int32_t)st) return 0.0f;
            v = v * react_factor(x, st);
        }
        return v;
    }
    const uint32_t e1 = m.reac_off[r + 1];
    for (uint32_t e = m.reac_off[r]; e < e1; e++) {
        const uint32_t ent = m.reac_ent[e];
        const int32_t x = sl.x((int)(ent >> 8));
        const int st = (int)(ent & 0xffu);
        if (x < st) return 0.0f;
        if (st == 1) {
            v = v * (float)x;
        } else if (st == 2) {
            float hx = (float)x;
            v = v * ((0.5f * hx) * (hx - 1.0f));
        } else {
            for (int j = 1; j <= st; j++) v = v * ((float)(x - j + 1) / (float)j);
        }
    }
    return v;
}

// Tree leaves: mode 0 = propensity, 1 = propensity of critical reactions,
// 2 = as 1 but leaf 0 unmasked (the reference's critical pick, tau.cu:1997).
__device__ __forceinline__ double leafv(const Slot& sl, int r, int mode) {
    float v = sl.pa(r);
    if (mode == 0) return (double)v;
    bool on = sl.cr(r) != 0 || (mode == 2 && r == 0);
    return on ? (double)v : 0.0;
}

// Node i of stored level li (li < 0: leaf i).
template <class M>
__device__ __forceinline__ double tval(const M& m, const Slot& sl, int li, int i, int mode) {
    return li < 0 ? leafv(sl, i, mode) : sl.t(m.lev_base(li) + i);
}

// Value of node i of stored level li: pairwise sum of its 2^d children.
// ((c0+c1)+(c2+c3)) + ((c4+c5)+(c6+c7)) is exactly the binary-tree value.
template <class M>
__device__ __forceinline__ double group_sum(const M& m, const Slot& sl, int li, int i, int mode) {
    const int d = m.lev_d(li), c0 = i << d, lc = li - 1;
    if (d == 1) return tval(m, sl, lc, c0, mode) + tval(m, sl, lc, c0 + 1, mode);
    if (d == 2)
        return (tval(m, sl, lc, c0, mode) + tval(m, sl, lc, c0 + 1, mode)) +
               (tval(m, sl, lc, c0 + 2, mode) + tval(m, sl, lc, c0 + 3, mode));
    const double v0 = tval(m, sl, lc, c0, mode), v1 = tval(m, sl, lc, c0 + 1, mode);
    const double v2 = tval(m, sl, lc, c0 + 2, mode), v3 = tval(m, sl, lc, c0 + 3, mode);
    const double v4 = tval(m, sl, lc, c0 + 4, mode), v5 = tval(m, sl, lc, c0 + 5, mode);
    const double v6 = tval(m, sl, lc, c0 + 6, mode), v7 = tval(m, sl, lc, c0 + 7, mode);
    return ((v0 + v1) + (v2 + v3)) + ((v4 + v5) + (v6 + v7));
}

template <class M>
__device__ __forceinline__ double tree_root(const M& m, const Slot& sl) {
    return sl.t(m.lev_base(m.nlev - 1));
}

template <int G, class M>
__device__ void build_tree(const Grp<G>& g, const M& m, const Slot& sl, int mode) {
    CTL_UNROLL_LEVELS
    for (int li = 0; li < m.nlev; li++) {
        const int base = m.lev_base(li);
        for (int i = (int)g.lane; i < m.lev_count(li); i += G) sl.t(base + i) = group_sum(m, sl, li, i, mode);
        g.sync();
    }
}

// Leftmost leaf whose cumulative weight reaches x (ties go left); never a
// zero leaf.  Same decisions as a level-by-level descent of the binary tree.
template <class M>
__device__ __forceinline__ int descend(const M& m, const Slot& sl, double x, int mode) {
    int i = 0;
    CTL_UNROLL_LEVELS
    for (int li = m.nlev - 1; li >= 0; li--) {
        const int d = m.lev_d(li), c0 = i << d, lc = li - 1;
        int j;
        if (d == 1) {
            j = go_right(x, tval(m, sl, lc, c0, mode), tval(m, sl, lc, c0 + 1, mode)) ? 1 : 0;
        } else if (d == 2) {
            const double v0 = tval(m, sl, lc, c0, mode), v1 = tval(m, sl, lc, c0 + 1, mode);
            const double v2 = tval(m, sl, lc, c0 + 2, mode), v3 = tval(m, sl, lc, c0 + 3, mode);
            const bool s1 = go_right(x, v0 + v1, v2 + v3);
            const bool s2 = go_right(x, s1 ? v2 : v0, s1 ? v3 : v1);
            j = (s1 ? 2 : 0) + (s2 ? 1 : 0);
        } else {
            const double v0 = tval(m, sl, lc, c0, mode), v1 = tval(m, sl, lc, c0 + 1, mode);
            const double v2 = tval(m, sl, lc, c0 + 2, mode), v3 = tval(m, sl, lc, c0 + 3, mode);
            const double v4 = tval(m, sl, lc, c0 + 4, mode), v5 = tval(m, sl, lc, c0 + 5, mode);
            const double v6 = tval(m, sl, lc, c0 + 6, mode), v7 = tval(m, sl, lc, c0 + 7, mode);
            const bool s1 = go_right(x, (v0 + v1) + (v2 + v3), (v4 + v5) + (v6 + v7));
            const double a0 = s1 ? v4 : v0, a1 = s1 ? v5 : v1, a2 = s1 ? v6 : v2, a3 = s1 ? v7 : v3;
            const bool s2 = go_right(x, a0 + a1, a2 + a3);
            const bool s3 = go_right(x, s2 ? a2 : a0, s2 ? a3 : a1);
            j = (s1 ? 4 : 0) + (s2 ? 2 : 0) + (s3 ? 1 : 0);
        }
        i = c0 + j;
    }
    return i;
}

template <int G, class M>
__device__ __forceinline__ void all_props(const Grp<G>& g, const M& m, const Slot& sl) {
    for (int r = (int)g.lane; r < m.R; r += G) sl.pa(r) = prop(m, sl, r);
    g.sync();
    build_tree<G>(g, m, sl, 0);
}

// After firing r: new propensities for the reactions that depend on the
// changed species, then their tree paths (or a full rebuild when cheaper);
// both give the same tree.
template <int G, class M>
__device__ void update_after_fire(const Grp<G>& g, const M& m, const Slot& sl, int r) {
    const uint32_t d0 = m.dep_off[r], d1 = m.dep_off[r + 1];
    const uint32_t nd = d1 - d0;
    if (nd == 0) return;
    if (G >= 8 && nd <= 2u * G) {
        // at most two entries per lane: read them once and keep them in
        // registers for the propensity pass and the tree levels (the same
        // entries in the same order as the loops below).  One B200: 8 lanes
        // on the 64 x 128 network 1,181 -> 1,123 ms per sweep; 4 lanes on
        // the 32 x 64 network 6,620 -> 7,516 ms, so groups of fewer than 8
        // lanes keep the loops.
        const int e0 = g.lane < nd ? (int)m.dep_ent[d0 + g.lane] : -1;
        const int e1 = g.lane + G < nd ? (int)m.dep_ent[d0 + g.lane + G] : -1;
        if (e0 >= 0) sl.pa(e0) = prop(m, sl, e0);
        if (e1 >= 0) sl.pa(e1) = prop(m, sl, e1);
        g.sync();
        if (nd >= (uint32_t)m.lev_count(0)) {
            build_tree<G>(g, m, sl, 0);
            return;
        }
        CTL_UNROLL_LEVELS
        for (int li = 0; li < m.nlev; li++) {
            const int sh = m.lev_shift(li), base = m.lev_base(li);
            const int i0 = e0 >= 0 ? e0 >> sh : -1, i1 = e1 >= 0 ? e1 >> sh : -1;
            if (i0 >= 0) sl.t(base + i0) = group_sum(m, sl, li, i0, 0);
            if (i1 >= 0 && i1 != i0) sl.t(base + i1) = group_sum(m, sl, li, i1, 0);
            g.sync();
        }
        return;
    }
    for (uint32_t j = d0 + g.lane; j < d1; j += G) {
        int rr = (int)m.dep_ent[j];
        sl.pa(rr) = prop(m, sl, rr);
    }
    g.sync();
    if (nd >= (uint32_t)m.lev_count(0)) {  // touches about every bottom group: rebuild
        build_tree<G>(g, m, sl, 0);
        return;
    }
    CTL_UNROLL_LEVELS
    for (int li = 0; li < m.nlev; li++) {
        const int sh = m.lev_shift(li), base = m.lev_base(li);
        int prev = -1;  // dependency lists are sorted: equal ancestors are adjacent
        for (uint32_t j = d0 + g.lane; j < d1; j += G) {
            const int i = (int)m.dep_ent[j] >> sh;
            if (i == prev) continue;
            prev = i;
            sl.t(base + i) = group_sum(m, sl, li, i, 0);
        }
        g.sync();
    }
}

// Where a simulation's samples go: its own rows [ns][s_out] (dynamics), or,
// in fitness mode, added into the 64-bit sums [ns][s_out] of its parameter
// set (integer sums: exact and independent of the order simulations finish
// in), with the last recorded row kept in the slot for the copy-forward.
struct Out {
    uint32_t* samples;
    unsigned long long* sums;
    __device__ __forceinline__ void put(const Slot& sl, uint32_t i, int so, int k, uint32_t v) const {
        if (samples) {
            samples[(size_t)i * so + k] = v;
        } else {
            atomicAdd(sums + (size_t)i * so + k, (unsigned long long)v);
            sl.lst(k) = v;
        }
    }
    __device__ __forceinline__ uint32_t get(const Slot& sl, uint32_t i, int so, int k) const {
        return samples ? samples[(size_t)i * so + k] : sl.lst(k);
    }
};

__device__ __forceinline__ Out out_of(const Run& run, uint32_t sim, size_t row_words) {
    Out o;
    if (run.sums) {
        const uint32_t tp = run.sum_threads * run.sum_prep;
        const uint32_t set = (sim / tp) * run.sum_threads + sim % run.sum_threads;
        o.samples = nullptr;
        o.sums = run.sums + (size_t)set * row_words;
    } else {
        o.samples = run.out + (size_t)sim * row_words;
        o.sums = nullptr;
    }
    return o;
}

// A0 == 0 (tau.cu:1665-1697, 2165-2196): the reference copies the last
// recorded sample forward (writing the current state first if none exists).
template <int G, class M>
__device__ void finish_zero(const Grp<G>& g, const M& m, const Run& run, const Slot& sl,
                            const Out& out, uint32_t& cursor) {
    const int so = m.s_out;
    const uint32_t ns = (uint32_t)m.ns;
    if (!(run.flags & F_Q10_OFF)) {
        if (cursor == 0) {
            for (int k = (int)g.lane; k < so; k += G) out.put(sl, 0u, so, k, (uint32_t)sl.x((int)m.cs[k]));
            cursor = 1;
        }
        // each lane copies its own columns k, which it wrote itself
        for (uint32_t i = cursor; i < ns; i++)
            for (int k = (int)g.lane; k < so; k += G) out.put(sl, i, so, k, out.get(sl, cursor - 1, so, k));
    } else {
        for (uint32_t i = cursor; i < ns; i++)
            for (int k = (int)g.lane; k < so; k += G) out.put(sl, i, so, k, (uint32_t)sl.x((int)m.cs[k]));
    }
    cursor = ns;
}

// Scalars of one simulation while a group works on it (identical in every
// lane of the group, except `fire`, each lane's share of the firings).
struct Sim {
    double T, tl, t_next;
    unsigned long long fire;
    uint32_t sim, cursor, n, burst, leaps, ssa, rej, status;
    bool in_ssa;
    uint4 wc;         // Philox block of the current SSA step pair (not persisted)
    uint32_t wc_blk;  // its block index, or 0xffffffff
};

constexpr int CONT = 0, DONE = 1;

template <int G, class M>
__device__ void init_sim(const Grp<G>& g, const M& m, const Run& run, const Slot& sl, Sim& st,
                         uint32_t sim) {
    const int S = m.S, R = m.R, P = m.P;
    g.sync();
    for (int s = (int)g.lane; s < S; s += G) sl.x(s) = run.X0[(size_t)sim * S + s];
    for (int r = (int)g.lane; r < P; r += G) {
        if (!run.uniform_c) sl.cf(r) = r < R ? run.c[(size_t)sim * R + r] : 0.0f;
        sl.pa(r) = 0.0f;
        sl.cr(r) = 0;
    }
    g.sync();
    all_props<G>(g, m, sl);
    st.T = 0.0;
    st.tl = 0.0;
    st.t_next = m.tvec[0];
    st.fire = 0ull;
    st.sim = sim;
    st.cursor = st.n = st.burst = st.leaps = st.ssa = st.rej = 0u;
    st.status = CTL_SIM_OK;
    st.in_ssa = (run.flags & F_FORCE_SSA) != 0;
    st.wc_blk = 0xffffffffu;
}

// PreCalculations (tau.cu:1568-2093): the SSA hand-off decision and, unless
// it hands off, one Cao tau-leap with critical reactions and rejection.
template <int G, class M>
__device__ int decide_step(const Grp<G>& g, const M& m, const Run& run, const Slot& sl, Sim& st,
                           const Out& out) {
    const int S = m.S, R = m.R, so = m.s_out;
    const uint32_t ns = (uint32_t)m.ns;
    const uint32_t fl = run.flags;
    const uint32_t lane = g.lane;
    const uint32_t simg = run.sim_base + st.sim;
    if (st.T >= m.tmax) return DONE;
    if (st.n >= run.max_steps) { st.status = CTL_SIM_STEP_LIMIT; return DONE; }
    const uint32_t step = st.n++;
    const double A0 = tree_root(m, sl);
    if (A0 == 0.0) {
        finish_zero<G>(g, m, run, sl, out, st.cursor);
        st.T = m.tmax + (double)0.1f;
        return DONE;
    }
    // Critical reactions (tau.cu:1727-1733): some reactant with
    // 0 < floor(x / L) < n_c.  floor(x / L) < n_c  <=>  x < n_c * L and
    // floor(x / L) > 0  <=>  x >= L (x >= 0, L >= 1): the reference's integer
    // test without a division.  Reactions with at most two reactant entries
    // read their packed descriptor (one load), the rest their list.
    const bool q6off = (fl & F_Q6_OFF) != 0;
    auto crit_entry = [&](uint32_t ent) {
        const uint32_t x = (uint32_t)sl.x((int)(ent >> 8)), L = ent & 0xffu;
        const bool below = (uint64_t)x < (uint64_t)run.nc * L;
        return q6off ? below : (x >= L && below);
    };
    bool lany = false;
    for (int r = (int)lane; r < R; r += G) {
        bool cr = false;
        const uint2 d = m.reac_desc[r];
        if (d.x != 0xffffffffu) {
            cr = (d.x && crit_entry(d.x)) || (d.y && crit_entry(d.y));
        } else {
            const uint32_t e1 = m.reac_off[r + 1];
            for (uint32_t e = m.reac_off[r]; e < e1; e++) cr = crit_entry(m.reac_ent[e]) || cr;
        }
        sl.cr(r) = cr ? 1 : 0;
        lany |= cr;
    }
    const bool anycrit = g.any(lany);
    g.sync();
    float t1 = FLT_MAX;
    for (int s = (int)lane; s < S; s += G) {
        const uint32_t e0 = m.v_off[s], e1 = m.v_off[s + 1];
        if (e0 == e1) continue;
        float mu = 0.0f, sg = 0.0f;
        for (uint32_t e = e0; e < e1; e++) {
            // critical reactions add an exact +-0: mu and sg start at +0 and
            // are never -0, so the sums equal those that skip them
            const uint32_t ent = m.v_ent[e];
            const int r = (int)(ent >> 8);
            const float a = sl.cr(r) ? 0.0f : sl.pa(r);
            const float fv = (float)(int8_t)(ent & 0xffu);
            mu = mu + fv * a;
            sg = sg + (fv * fv) * a;
        }
        const int32_t xs = sl.x(s);
        const float gg = gfun(m.hor[s], m.hort[s], xs);
        const float tmp2 = (run.eps * (float)xs) / gg;
        const float macs = tmp2 > 1.0f ? tmp2 : 1.0f;
        const bool use = (fl & F_Q9_OFF) ? (sg != 0.0f) : (mu != 0.0f && sg != 0.0f);
        if (use) {
            const float t3 = mu != 0.0f ? macs / fabsf(mu) : __int_as_float(0x7f800000);
            const float t4 = (macs * macs) / sg;
            const float tt = t3 < t4 ? t3 : t4;
            if (tt < t1) t1 = tt;
        }
    }
    const float tau1 = g.fmin(t1);
    if ((double)tau1 < run.ssa_factor / A0) {
        st.in_ssa = true;
        st.burst = 0;
        st.tl = 0.0;
        return CONT;
    }
    double a0c = 0.0;
    if (anycrit) {
        build_tree<G>(g, m, sl, 1);
        a0c = tree_root(m, sl);
    }
    const uint4 wd = draw(run.seed, 0u, TAG_MISC, step, simg);
    double tau2 = (double)FLT_MAX;
    if (a0c > 0.0) tau2 = -dlog(u53(wd.x, wd.y)) / a0c;
    double tau = (double)tau1 < tau2 ? (double)tau1 : tau2;
    int pick = -1;
    if ((double)tau1 > tau2) {
        int mode = 1;
        if (!(fl & F_Q2_OFF) && !sl.cr(0)) {
            mode = 2;
            if (lane == 0) {  // the ancestors of leaf 0 are node 0 of every stored level
                CTL_UNROLL_LEVELS
                for (int li = 0; li < m.nlev; li++) sl.t(m.lev_base(li)) = group_sum(m, sl, li, 0, 2);
            }
            g.sync();
        }
        pick = descend(m, sl, u53(wd.z, wd.w) * a0c, mode);
    }
    uint32_t attempt = 0;
    bool ovf = false;
    for (;;) {
        const bool keep = attempt == 0 || (fl & F_Q3_OFF);
        for (uint32_t pb = lane; 2u * pb < (uint32_t)R; pb += G) {
            const int r0 = (int)(2u * pb), r1 = r0 + 1;
            const bool c0 = sl.cr(r0) != 0;
            const bool c1 = r1 < R ? sl.cr(r1) != 0 : true;
            const double l0 = c0 ? 0.0 : tau * (double)sl.pa(r0);
            const double l1 = (c1 || r1 >= R) ? 0.0 : tau * (double)sl.pa(r1);
            const uint32_t tg = tag_pois(attempt, pb);
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (l0 > 0.0 || l1 > 0.0) w = draw(run.seed, 0u, tg, step, simg);
            sl.k(r0) = c0 ? ((r0 == pick && keep) ? 1u : 0u)
                          : poisson(l0, w.x, w.y, run.seed, tg, step, simg, 0u);
            if (r1 < R)
                sl.k(r1) = c1 ? ((r1 == pick && keep) ? 1u : 0u)
                              : poisson(l1, w.z, w.w, run.seed, tg, step, simg, 1u);
        }
        g.sync();
        bool lfail = false, lovf = false;
        for (int s = (int)lane; s < S; s += G) {
            int64_t x1 = sl.x(s);
            const uint32_t e1 = m.fs_off[s + 1];
            for (uint32_t e = m.fs_off[s]; e < e1; e++) {
                const uint32_t ent = m.fs_ent[e];
                x1 += (int64_t)(int8_t)(ent & 0xffu) * (int64_t)sl.k((int)(ent >> 8));
                if (!(fl & F_Q4_OFF) && x1 < 0) { lfail = true; break; }
            }
            if (x1 < 0) lfail = true;
            if (x1 > 2147483647LL) lovf = true;
            sl.x1(s) = (int32_t)x1;
        }
        const bool fail = g.any(lfail);
        g.sync();
        if (!fail) {
            ovf = g.any(lovf);
            break;
        }
        tau = tau * 0.5;
        attempt++;
        st.rej++;
        if (attempt >= MAX_ATTEMPTS) { st.status = CTL_SIM_ATTEMPT_LIMIT; return DONE; }
    }
    if (ovf) { st.status = CTL_SIM_OVERFLOW; return DONE; }
    // check_time_instant (tau.cu:1507-1562)
    const double T = st.T;
    while (st.cursor < ns && T + tau >= st.t_next) {
        for (int k = (int)lane; k < so; k += G) {
            const int s = (int)m.cs[k];
            const int32_t xs = sl.x(s);
            const double d = (double)((int64_t)sl.x1(s) - (int64_t)xs);
            const double delta = (d * (st.t_next - T)) / tau;
            const double ri = rint(delta);
            uint32_t v;
            if (!(fl & F_Q1_OFF))
                v = (uint32_t)xs + (ri > 0.0 ? (uint32_t)ri : 0u);
            else
                v = (uint32_t)((int64_t)xs + (int64_t)ri);
            out.put(sl, st.cursor, so, k, v);
        }
        st.cursor++;
        st.t_next = st.cursor < ns ? m.tvec[st.cursor] : 0.0;
    }
    unsigned long long fs = 0;
    for (int r = (int)lane; r < R; r += G) fs += sl.k(r);
    st.fire += fs;
    st.leaps++;
    g.sync();
    for (int s = (int)lane; s < S; s += G) sl.x(s) = sl.x1(s);
    g.sync();
    st.T = T + tau;
    all_props<G>(g, m, sl);
    return st.cursor == ns ? DONE : CONT;
}

// EventualSSASteps / LightweightSSA (tau.cu:2099-2454): one direct-method step.
template <int G, class M>
__device__ int ssa_step(const Grp<G>& g, const M& m, const Run& run, const Slot& sl, Sim& st,
                        const Out& out) {
    const int so = m.s_out;
    const uint32_t ns = (uint32_t)m.ns;
    const uint32_t lane = g.lane;
    if (st.n >= run.max_steps) { st.status = CTL_SIM_STEP_LIMIT; return DONE; }
    const double A0 = tree_root(m, sl);
    if (A0 == 0.0) {
        finish_zero<G>(g, m, run, sl, out, st.cursor);
        st.T = m.tmax + (double)0.1f;
        return DONE;
    }
    const uint32_t step = st.n++;
    // one Philox block per two SSA steps: (w0,w1) for even steps, (w2,w3)
    // for odd ones; 32-bit pick uniform, FP32 waiting time
    if (st.wc_blk != (step >> 1)) {
        st.wc = draw(run.seed, 0u, TAG_SSA, step >> 1, run.sim_base + st.sim);
        st.wc_blk = step >> 1;
    }
    const uint32_t wa = (step & 1u) ? st.wc.z : st.wc.x, wb = (step & 1u) ? st.wc.w : st.wc.y;
    const int r = descend(m, sl, u32d(wa) * A0, 0);
    const float dtf = -flog(u24f(wb)) / (float)A0;
    st.tl = st.tl + (double)dtf;
    while (st.cursor < ns && st.T + st.tl > st.t_next) {
        for (int k = (int)lane; k < so; k += G) out.put(sl, st.cursor, so, k, (uint32_t)sl.x((int)m.cs[k]));
        st.cursor++;
        st.t_next = st.cursor < ns ? m.tvec[st.cursor] : 0.0;
    }
    g.sync();
    bool lovf = false;
    const uint32_t e1 = m.fr_off[r + 1];
    for (uint32_t e = m.fr_off[r] + lane; e < e1; e += G) {
        const uint32_t ent = m.fr_ent[e];
        const int s = (int)(ent >> 8);
        const int64_t nx = (int64_t)sl.x(s) + (int64_t)(int8_t)(ent & 0xffu);
        if (nx > 2147483647LL || nx < 0) lovf = true;
        sl.x(s) = (int32_t)nx;
    }
    const bool ovf = g.any(lovf);
    st.ssa++;
    if (lane == 0) st.fire += 1ull;
    if (ovf) { st.status = CTL_SIM_OVERFLOW; return DONE; }
    g.sync();
    update_after_fire<G>(g, m, sl, r);
    st.burst++;
    if (st.cursor == ns) return DONE;
    if (st.burst == run.ssa_steps) {
        st.T = st.T + st.tl;
        st.tl = 0.0;
        st.burst = 0;
        if (!(run.flags & F_FORCE_SSA)) st.in_ssa = false;
        else if (st.T >= m.tmax) return DONE;
    }
    return CONT;
}

template <int G, class M>
__device__ void finish_sim(const Grp<G>& g, const M& m, const Run& run, const Sim& st, const Out& out) {
    const int so = m.s_out;
    if (out.samples)  // rows never reached read 0 (a sum gains nothing from them)
        for (uint32_t i = st.cursor; i < (uint32_t)m.ns; i++)
            for (int k = (int)g.lane; k < so; k += G) out.samples[(size_t)i * so + k] = 0u;
    const unsigned long long ftot = g.sum(st.fire);
    if (g.lane == 0) {
        ctl_sim_info inf;
        inf.t_final = st.T + st.tl;
        inf.firings = ftot;
        inf.status = st.status;
        inf.steps = st.n;
        inf.leaps = st.leaps;
        inf.ssa_steps = st.ssa;
        inf.rejections = st.rej;
        inf.pad = 0;
        run.info[st.sim] = inf;
    }
    if (run.out_host && out.samples) {
        // the group's lanes wrote the rows; after the barrier every lane sees
        // them and the group copies the simulation's row to the caller's
        // pinned buffer (16-byte stores when the row allows)
        g.sync();
        const size_t words = (size_t)m.ns * (size_t)so;
        const uint32_t* src = out.samples;
        uint32_t* dst = run.out_host + (size_t)st.sim * words;
        if ((words & 3u) == 0u && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0u) {
            const uint4* s4 = reinterpret_cast<const uint4*>(src);
            uint4* d4 = reinterpret_cast<uint4*>(dst);
            for (size_t i = g.lane; i < words / 4; i += G) d4[i] = s4[i];
        } else {
            for (size_t i = g.lane; i < words; i += G) dst[i] = src[i];
        }
    }
    if (run.done) {  // publish: this simulation's rows and record are complete
        __threadfence();
        g.sync();
        if (g.lane == 0) atomicAdd(run.done + (st.sim >> run.done_shift), 1u);
    }
}

template <int G>
__device__ __forceinline__ void load_sim(const Grp<G>& g, const StateArrays& sa, int j, Sim& st) {
    st.T = sa.T[j];
    st.tl = sa.tl[j];
    st.t_next = sa.tnext[j];
    st.fire = g.lane == 0 ? sa.fire[j] : 0ull;
    st.sim = sa.sim[j];
    st.cursor = sa.cursor[j];
    st.n = sa.n[j];
    st.burst = sa.burst[j];
    st.leaps = sa.leaps[j];
    st.ssa = sa.ssa[j];
    st.rej = sa.rej[j];
    const uint32_t f = sa.flags[j];
    st.in_ssa = (f & ST_IN_SSA) != 0;
    st.status = f >> ST_STATUS_SHIFT;
    st.wc_blk = 0xffffffffu;
}

template <int G>
__device__ __forceinline__ void store_sim(const Grp<G>& g, const StateArrays& sa, int j, const Sim& st) {
    const unsigned long long f = g.sum(st.fire);
    if (g.lane == 0) {
        sa.T[j] = st.T;
        sa.tl[j] = st.tl;
        sa.tnext[j] = st.t_next;
        sa.fire[j] = f;
        sa.sim[j] = st.sim;
        sa.cursor[j] = st.cursor;
        sa.n[j] = st.n;
        sa.burst[j] = st.burst;
        sa.leaps[j] = st.leaps;
        sa.ssa[j] = st.ssa;
        sa.rej[j] = st.rej;
        sa.flags[j] = (st.in_ssa ? ST_IN_SSA : 0u) | (st.status << ST_STATUS_SHIFT);
    }
}

template <int G>
__device__ __forceinline__ Slot slot_of(unsigned char* smem, const Layout& lay, int j, int NS, bool uniform_c) {
    Slot sl;
    if (G == 1) {
        sl.st = NS;
        sl.X = reinterpret_cast<int32_t*>(smem + lay.off_X) + j;
        sl.X1 = reinterpret_cast<int32_t*>(smem + lay.off_X1) + j;
        sl.a = reinterpret_cast<float*>(smem + lay.off_a) + j;
        sl.K = reinterpret_cast<uint32_t*>(smem + lay.off_K) + j;
        sl.tree = reinterpret_cast<double*>(smem + lay.off_tree) + j;
        sl.crit = reinterpret_cast<uint8_t*>(smem + lay.off_crit) + j;
        sl.c = reinterpret_cast<float*>(smem + lay.off_c) + (uniform_c ? 0 : j);
        sl.last = reinterpret_cast<uint32_t*>(smem + lay.off_last) + j;
        sl.cst = uniform_c ? 1 : NS;
    } else {
        sl.st = 1;
        sl.X = reinterpret_cast<int32_t*>(smem + lay.off_X) + (size_t)j * lay.len_S;
        sl.X1 = reinterpret_cast<int32_t*>(smem + lay.off_X1) + (size_t)j * lay.len_S;
        sl.a = reinterpret_cast<float*>(smem + lay.off_a) + (size_t)j * lay.len_P;
        sl.K = reinterpret_cast<uint32_t*>(smem + lay.off_K) + (size_t)j * lay.len_P;
        sl.tree = reinterpret_cast<double*>(smem + lay.off_tree) + (size_t)j * lay.len_T;
        sl.crit = reinterpret_cast<uint8_t*>(smem + lay.off_crit) + (size_t)j * lay.len_C;
        sl.c = reinterpret_cast<float*>(smem + lay.off_c) + (uniform_c ? 0 : (size_t)j * lay.len_P);
        sl.last = reinterpret_cast<uint32_t*>(smem + lay.off_last) + (size_t)j * lay.len_O;
        sl.cst = 1;
    }
    return sl;
}

// Persistent sweep.  Every round: (1) each group refills its own slot from
// the device work queue when it is empty; (2) the block sorts the occupied
// slots into an SSA list and a decision/leap list (shared-memory atomics);
// (3) groups take list entries, so every warp executes one phase only
// (regrouping), and advance each taken simulation by a bounded amount of
// work.  The loop ends when the queue is drained and every slot is closed.
// MINB selects the register budget: compiled so that MINB blocks of 256
// threads can be resident per SM (2: up to 128 registers per thread, 3: 80,
// 4: 64, spilling to local memory as needed).  sweep_body is the kernel's
// body for either model type; sweep_kernel is the library's kernel.
template <int G, class M>
__device__ __forceinline__ void sweep_body(const M& m, const Run& run, const Layout& lay) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_cnt[2];
    const int NS = (int)(blockDim.x / G);
    const int gi = (int)(threadIdx.x / G);
    Grp<G> g;
    if constexpr (G > 32) g.scratch(smem + lay.off_grp);
    StateArrays sa;
    {
        unsigned char* b = smem + lay.off_state;
        sa.T = reinterpret_cast<double*>(b);
        sa.tl = sa.T + NS;
        sa.tnext = sa.tl + NS;
        sa.fire = reinterpret_cast<unsigned long long*>(sa.tnext + NS);
        uint32_t* u = reinterpret_cast<uint32_t*>(sa.fire + NS);
        sa.sim = u;
        sa.cursor = u + NS;
        sa.n = u + 2 * NS;
        sa.burst = u + 3 * NS;
        sa.leaps = u + 4 * NS;
        sa.ssa = u + 5 * NS;
        sa.rej = u + 6 * NS;
        sa.flags = u + 7 * NS;
    }
    uint32_t* phase = sa.flags + NS;
    uint32_t* list = reinterpret_cast<uint32_t*>(smem + lay.off_list);
    const bool uni = run.uniform_c != 0;
    if (uni) {
        float* cs = reinterpret_cast<float*>(smem + lay.off_c);
        for (int r = (int)threadIdx.x; r < m.P; r += (int)blockDim.x) cs[r] = r < m.R ? run.c[r] : 0.0f;
    }
    for (int j = (int)threadIdx.x; j < NS; j += (int)blockDim.x) phase[j] = PH_EMPTY;
    __syncthreads();
    const uint32_t ns = (uint32_t)m.ns;
    const size_t sim_stride = (size_t)ns * (size_t)m.s_out;
    if (run.warp_local) {
        // Warp-local scheduling: every group keeps its own slot and its
        // simulation's scalars in registers; the groups of a warp step in
        // lockstep per phase and no block-wide barrier is taken, so a long
        // leap decision in one warp never holds up the others.
        const Slot sl = slot_of<G>(smem, lay, gi, NS, uni);
        Sim st;
        bool live = false, closed = false;
        Out out{nullptr, nullptr};
        for (;;) {
            if (!live && !closed) {
                uint32_t sim = 0;
                if (g.lane == 0) sim = atomicAdd(run.queue, 1u);
                sim = g.bcast(sim);
                if (sim >= run.n) {
                    closed = true;
                } else {
                    init_sim<G>(g, m, run, sl, st, sim);
                    live = true;
                    out = out_of(run, st.sim, sim_stride);
                }
            }
            if (__all_sync(0xffffffffu, closed)) break;
            const bool is_ssa = live && st.in_ssa, is_dec = live && !st.in_ssa;
            const uint32_t ssa_mask = __ballot_sync(0xffffffffu, is_ssa);
            const uint32_t dec_mask = __ballot_sync(0xffffffffu, is_dec);
            int res = CONT;
            if (is_ssa) {
                for (uint32_t b = 0; b < run.ssa_budget; b++) {
                    const bool act = res == CONT && st.in_ssa;
                    if (!__any_sync(ssa_mask, act)) break;
                    if (act) res = ssa_step<G>(g, m, run, sl, st, out);
                }
            } else if (is_dec) {
                for (uint32_t b = 0; b < run.dec_budget; b++) {
                    const bool act = res == CONT && !st.in_ssa;
                    if (!__any_sync(dec_mask, act)) break;
                    if (act) res = decide_step<G>(g, m, run, sl, st, out);
                }
            }
            if (live && res == DONE) {
                finish_sim<G>(g, m, run, st, out);
                live = false;
            }
        }
        return;
    }
    for (;;) {
        if (phase[gi] == PH_EMPTY) {
            uint32_t sim = 0;
            if (g.lane == 0) sim = atomicAdd(run.queue, 1u);
            sim = g.bcast(sim);
            if (sim >= run.n) {
                if (g.lane == 0) phase[gi] = PH_CLOSED;
            } else {
                const Slot sl = slot_of<G>(smem, lay, gi, NS, uni);
                Sim st;
                init_sim<G>(g, m, run, sl, st, sim);
                store_sim<G>(g, sa, gi, st);
                if (g.lane == 0) phase[gi] = st.in_ssa ? PH_SSA : PH_DECIDE;
            }
        }
        if (threadIdx.x == 0) {
            s_cnt[0] = 0u;
            s_cnt[1] = 0u;
        }
        __syncthreads();
        for (int j = (int)threadIdx.x; j < NS; j += (int)blockDim.x) {
            const uint32_t ph = phase[j];
            if (ph == PH_SSA) list[atomicAdd(&s_cnt[0], 1u)] = (uint32_t)j;
            else if (ph == PH_DECIDE) list[NS - 1 - (int)atomicAdd(&s_cnt[1], 1u)] = (uint32_t)j;
        }
        __syncthreads();
        const uint32_t nssa = s_cnt[0], ndec = s_cnt[1];
        if (nssa + ndec == 0u) break;
        // At most one list entry per group and round (nssa + ndec <= NS).
        // The groups of a warp that work in the same phase step in lockstep:
        // before every step they agree (__any_sync over that phase's lanes)
        // whether anyone still has work, so their instruction streams merge.
        const uint32_t k = (uint32_t)gi;
        const bool has_item = k < nssa + ndec;
        const bool is_ssa = k < nssa;
        const uint32_t ssa_mask = __ballot_sync(0xffffffffu, is_ssa);
        const uint32_t dec_mask = __ballot_sync(0xffffffffu, has_item && !is_ssa);
        if (has_item) {
            const int j = (int)(is_ssa ? list[k] : list[NS - 1 - (int)(k - nssa)]);
            const Slot sl = slot_of<G>(smem, lay, j, NS, uni);
            Sim st;
            load_sim<G>(g, sa, j, st);
            const Out out = out_of(run, st.sim, sim_stride);
            int res = CONT;
            if (is_ssa) {
                for (uint32_t b = 0; b < run.ssa_budget; b++) {
                    const bool act = res == CONT && st.in_ssa;
                    if (!__any_sync(ssa_mask, act)) break;
                    if (act) res = ssa_step<G>(g, m, run, sl, st, out);
                }
            } else {
                for (uint32_t b = 0; b < run.dec_budget; b++) {
                    const bool act = res == CONT && !st.in_ssa;
                    if (!__any_sync(dec_mask, act)) break;
                    if (act) res = decide_step<G>(g, m, run, sl, st, out);
                }
            }
            if (res == DONE) {
                finish_sim<G>(g, m, run, st, out);
                if (g.lane == 0) phase[j] = PH_EMPTY;
            } else {
                store_sim<G>(g, sa, j, st);
                if (g.lane == 0) phase[j] = st.in_ssa ? PH_SSA : PH_DECIDE;
            }
        }
        __syncthreads();
    }
}

template <int G, int MINB>
__global__ void __launch_bounds__(256, MINB) sweep_kernel(Model m, Run run, Layout lay) {
    sweep_body<G>(m, run, lay);
}

#ifndef __CUDACC_RTC__
// Host-side handle of the sweep kernel for G lanes per simulation in
// register budget minb (2, 3 or 4 resident 256-thread blocks per SM).
template <int G>
const void* sweep_kernel_ptr(int minb) {
    switch (minb) {
        case 3: return reinterpret_cast<const void*>(&sweep_kernel<G, 3>);
        case 4: return reinterpret_cast<const void*>(&sweep_kernel<G, 4>);
        default: return reinterpret_cast<const void*>(&sweep_kernel<G, 2>);
    }
}

}  // namespace dev

// One translation unit per group size (ctl_sweep_g<G>.cu) instantiates these.
const void* sweep_kernel_g1(int minb);
const void* sweep_kernel_g2(int minb);
const void* sweep_kernel_g4(int minb);
const void* sweep_kernel_g8(int minb);
const void* sweep_kernel_g16(int minb);
const void* sweep_kernel_g32(int minb);
const void* sweep_kernel_g64(int minb);
const void* sweep_kernel_g128(int minb);
const void* sweep_kernel_g256(int minb);

}  // namespace ctl
#else
}  // namespace dev
}  // namespace ctl
#endif

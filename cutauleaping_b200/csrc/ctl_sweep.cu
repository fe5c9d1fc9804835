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
#include <cstdint>
#include <cstring>
#include <string>

#include "ctl_internal.h"

namespace ctl {
namespace dev {

constexpr uint32_t TAG_SSA = 0x40000000u;   // SSA steps 2b, 2b+1: block b, (w0,w1) / (w2,w3)
constexpr uint32_t TAG_MISC = 0x40000001u;  // leap: (w0,w1) tau2, (w2,w3) critical pick
constexpr uint32_t MAX_ATTEMPTS = 1024u;    // 10-bit attempt field of the Poisson tag
constexpr uint32_t PTRS_MAX_TRIALS = 256u;

enum : uint32_t {
    F_FORCE_SSA = 1u << 0, F_Q1_OFF = 1u << 1, F_Q2_OFF = 1u << 2, F_Q3_OFF = 1u << 3,
    F_Q4_OFF = 1u << 4, F_Q5_OFF = 1u << 5, F_Q6_OFF = 1u << 6, F_Q9_OFF = 1u << 7, F_Q10_OFF = 1u << 8
};

__device__ __forceinline__ uint32_t tag_pois(uint32_t attempt, uint32_t pair) {
    return 0x80000000u | (attempt << 20) | pair;
}

struct Model {
    int S, R, P, logP, ns, s_out;
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
    // Stored levels of the binary sum tree: level 3, 6, 9, ... below the
    // root, and the root.  Stored level li holds the nodes that cover 2^shift
    // leaves; each is the pairwise sum of 2^d nodes of stored level li-1
    // (li = 0: of leaves).  Intermediate levels are recomputed in registers.
    int nlev;
    int lev_shift[10], lev_d[10], lev_base[10], lev_count[10];
};

struct Run {
    uint64_t seed;
    float eps;
    uint32_t nc;
    double ssa_factor;
    uint32_t ssa_steps, flags, max_steps, sim_base, n;
    uint32_t uniform_c;              // all simulations share row 0 of c
    uint32_t ssa_budget, dec_budget; // work per slot and round (SSA steps / decisions)
    uint32_t warp_local;             // 1: warp-local scheduling (no block rounds)
    const int32_t* __restrict__ X0;  // [n][S]
    const float* __restrict__ c;     // [n][R]
    uint32_t* __restrict__ out;      // [n][ns][s_out]
    ctl_sim_info* __restrict__ info; // [n]
    uint32_t* queue;                 // work-queue ticket
};

// Shared-memory slot layout.  G == 1: element i of slot j at i*NS + j
// (consecutive threads hit consecutive banks).  G > 1: slot-contiguous
// arrays of odd padded length (lanes of one group hit distinct banks).
struct Layout {
    uint32_t off_X, off_X1, off_a, off_K, off_tree, off_crit, off_c, off_state, off_list, off_grp;
    uint32_t len_S, len_P, len_C, len_T;  // padded lengths (G > 1)
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
// Random numbers and elementary functions (bitwise identical to the oracle)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int i = 0; i < 10; i++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint4 draw(uint64_t seed, uint32_t blk, uint32_t tag, uint32_t step,
                                      uint32_t sim) {
    return philox10(make_uint4(blk, tag, step, sim), (uint32_t)seed, (uint32_t)(seed >> 32));
}

__device__ __forceinline__ double u32d(uint32_t w) { return ((double)w + 0.5) * 0x1p-32; }
__device__ __forceinline__ double u53(uint32_t wa, uint32_t wb) {
    uint64_t m = ((uint64_t)wb << 20) | (uint64_t)(wa >> 12);
    return ((double)m + 0.5) * 0x1p-52;
}

#define CTL_LN2_HI 0x1.62e42fee00000p-1
#define CTL_LN2_LO 0x1.a39ef35793c76p-33

// log(x) = e ln2 + 2 atanh(s), s = (m-1)/(m+1), m in (sqrt(1/2), sqrt(2)].
__device__ double dlog(double x) {
    if (!(x > 0.0)) return x == 0.0 ? __longlong_as_double(0xfff0000000000000ULL)
                                     : __longlong_as_double(0x7ff8000000000000ULL);
    if (x == __longlong_as_double(0x7ff0000000000000ULL)) return x;
    int eadj = 0;
    if (x < 0x1p-1022) { x = x * 0x1p54; eadj = -54; }
    uint64_t b = (uint64_t)__double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023 + eadj;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL));
    if (m > 0x1.6a09e667f3bcdp+0) { m = m * 0.5; e = e + 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double p = 0x1.8618618618618p-5;
    p = fma(p, z, 0x1.af286bca1af28p-5);
    p = fma(p, z, 0x1.e1e1e1e1e1e1ep-5);
    p = fma(p, z, 0x1.1111111111111p-4);
    p = fma(p, z, 0x1.3b13b13b13b14p-4);
    p = fma(p, z, 0x1.745d1745d1746p-4);
    p = fma(p, z, 0x1.c71c71c71c71cp-4);
    p = fma(p, z, 0x1.2492492492492p-3);
    p = fma(p, z, 0x1.999999999999ap-3);
    p = fma(p, z, 0x1.5555555555555p-2);
    double r = z * p;
    double ed = (double)e;
    double two_s = s + s;
    return fma(ed, CTL_LN2_HI, two_s + fma(two_s, r, ed * CTL_LN2_LO));
}

// exp(x): Cody-Waite reduction, degree-14 Taylor polynomial, 2^k scaling.
__device__ double dexp(double x) {
    if (x != x) return x;
    if (x > 709.0) return __longlong_as_double(0x7ff0000000000000ULL);
    if (x < -745.0) return 0.0;
    double k = rint(x * 0x1.71547652b82fep+0);
    double r = fma(-k, CTL_LN2_HI, x);
    r = fma(-k, CTL_LN2_LO, r);
    double p = 0x1.93974a8c07c9dp-37;
    p = fma(p, r, 0x1.6124613a86d09p-33);
    p = fma(p, r, 0x1.1eed8eff8d898p-29);
    p = fma(p, r, 0x1.ae64567f544e4p-26);
    p = fma(p, r, 0x1.27e4fb7789f5cp-22);
    p = fma(p, r, 0x1.71de3a556c734p-19);
    p = fma(p, r, 0x1.a01a01a01a01ap-16);
    p = fma(p, r, 0x1.a01a01a01a01ap-13);
    p = fma(p, r, 0x1.6c16c16c16c17p-10);
    p = fma(p, r, 0x1.1111111111111p-7);
    p = fma(p, r, 0x1.5555555555555p-5);
    p = fma(p, r, 0x1.5555555555555p-3);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int ki = (int)k;
    if (ki < -1000) { p = p * 0x1p-200; ki = ki + 200; }
    return p * __longlong_as_double((long long)((uint64_t)(ki + 1023) << 52));
}

// FP32 log(x) for normal x > 0: the reduction of dlog in single precision,
// series 2s(1 + s^2/3 + s^4/5 + s^6/7 + s^8/9).
__device__ __forceinline__ float flog(float x) {
    const uint32_t b = __float_as_uint(x);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 0x1.6a09e6p+0f) { m = m * 0.5f; e = e + 1; }
    const float f = m - 1.0f;
    const float sv = f / (2.0f + f);
    const float z = sv * sv;
    float p = 0x1.c71c72p-4f;
    p = fmaf(p, z, 0x1.24924ap-3f);
    p = fmaf(p, z, 0x1.99999ap-3f);
    p = fmaf(p, z, 0x1.555556p-2f);
    const float r = z * p;
    const float ef = (float)e;
    const float two_s = sv + sv;
    return fmaf(ef, 0x1.62e4p-1f, two_s + fmaf(two_s, r, ef * 0x1.7f7d1cp-20f));
}

__device__ __forceinline__ float u24f(uint32_t w) { return ((float)(w >> 8) + 0.5f) * 0x1p-24f; }

__constant__ double c_logfact[16] = {
    0.0, 0.0, 0x1.62e42fefa39efp-1, 0x1.cab0bfa2a2002p+0, 0x1.96ca77c922cf9p+1,
    0x1.326643c4479c9p+2, 0x1.a51273acf01cap+2, 0x1.10ce1f32dcc30p+3,
    0x1.5358e82fcb70dp+3, 0x1.99a8921a7f7cfp+3, 0x1.e357590954d15p+3,
    0x1.180973f3a8d74p+4, 0x1.3fcba16d50143p+4, 0x1.68d5a9c3b32cep+4,
    0x1.930f3df162a42p+4, 0x1.be636a63fd346p+4};

// log(k!) : table below 16, Stirling series above.
__device__ double dlogfact(double k) {
    if (k < 16.0) return c_logfact[(int)k];
    double x = k + 1.0;
    double ix = 1.0 / x;
    double ix2 = ix * ix;
    double ser = ix * (0x1.5555555555555p-4 -
                       ix2 * (0x1.6c16c16c16c17p-9 -
                              ix2 * (0x1.a01a01a01a01ap-11 - ix2 * 0x1.3813813813814p-11)));
    return (x - 0.5) * dlog(x) - x + 0x1.d67f1c864beb5p-1 + ser;
}

__device__ __forceinline__ uint32_t clamp_k(double k) {
    return k > 2147483647.0 ? 2147483647u : (uint32_t)k;
}

// Poisson(lam) given the reaction's primary uniform pair (wa, wb).
// lam < 10: sequential inversion.  lam >= 10: Hormann's PTRS (1993); extra
// trials read blocks 1 + 2j + odd of the same (tag, step, sim) stream.
__device__ uint32_t poisson(double lam, uint32_t wa, uint32_t wb, uint64_t seed, uint32_t tag,
                            uint32_t step, uint32_t sim, uint32_t odd) {
    if (!(lam > 0.0)) return 0u;
    if (lam < 10.0) {
        double u = u32d(wa);
        double p = dexp(-lam);
        double F = p;
        uint32_t k = 0;
        while (u > F && k < 64u) {
            k = k + 1u;
            p = (p * lam) / (double)k;
            F = F + p;
        }
        return k;
    }
    double slam = sqrt(lam);
    double loglam = dlog(lam);
    double b = 0.931 + 2.53 * slam;
    double a = -0.059 + 0.02483 * b;
    double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    double vr = 0.9277 - 3.6224 / (b - 2.0);
    uint4 w = make_uint4(0u, 0u, 0u, 0u);
    for (uint32_t t = 0; t < PTRS_MAX_TRIALS; t++) {
        if (t > 0) {
            uint32_t j = (t - 1) >> 1;
            if (((t - 1) & 1u) == 0u) w = draw(seed, 1u + 2u * j + odd, tag, step, sim);
            wa = ((t - 1) & 1u) ? w.z : w.x;
            wb = ((t - 1) & 1u) ? w.w : w.y;
        }
        double U = u32d(wa) - 0.5;
        double V = u32d(wb);
        double us = 0.5 - fabs(U);
        double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return clamp_k(k);
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        double lhs = dlog(V) + dlog(invalpha) - dlog(a / (us * us) + b);
        double rhs = -lam + k * loglam - dlogfact(k);
        if (lhs <= rhs) return clamp_k(k);
    }
    return clamp_k(floor(lam));
}

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
    int st;   // element stride of the slot arrays
    int cst;  // element stride of the rate constants (1 when shared by the block)
    __device__ __forceinline__ int32_t& x(int i) const { return X[i * st]; }
    __device__ __forceinline__ int32_t& x1(int i) const { return X1[i * st]; }
    __device__ __forceinline__ float& pa(int i) const { return a[i * st]; }
    __device__ __forceinline__ double& t(int i) const { return tree[i * st]; }
    __device__ __forceinline__ uint32_t& k(int i) const { return K[i * st]; }
    __device__ __forceinline__ uint8_t& cr(int i) const { return crit[i * st]; }
    __device__ __forceinline__ float& cf(int i) const { return c[i * cst]; }
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
__device__ __forceinline__ float prop(const Model& m, const Slot& sl, int r) {
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

// Cao's g_i (tau.cu:1741-1789) in FP32.
__device__ __forceinline__ float gfun(uint32_t hor, uint32_t hort, int32_t x) {
    float xf = (float)x;
    switch (hor) {
        case 1: return 1.0f;
        case 2: return hort == 2 ? 2.0f + 1.0f / (xf - 1.0f) : 2.0f;
        case 3:
            if (hort == 3) return 3.0f + 1.0f / (xf - 1.0f) + 2.0f / (xf - 2.0f);
            if (hort == 2) return 3.0f + 1.5f / (xf - 1.0f);
            return 3.0f;
        default: return 1.0f;
    }
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
__device__ __forceinline__ double tval(const Model& m, const Slot& sl, int li, int i, int mode) {
    return li < 0 ? leafv(sl, i, mode) : sl.t(m.lev_base[li] + i);
}

// Value of node i of stored level li: pairwise sum of its 2^d children.
// ((c0+c1)+(c2+c3)) + ((c4+c5)+(c6+c7)) is exactly the binary-tree value.
__device__ __forceinline__ double group_sum(const Model& m, const Slot& sl, int li, int i, int mode) {
    const int d = m.lev_d[li], c0 = i << d, lc = li - 1;
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

__device__ __forceinline__ double tree_root(const Model& m, const Slot& sl) {
    return sl.t(m.lev_base[m.nlev - 1]);
}

template <int G>
__device__ void build_tree(const Grp<G>& g, const Model& m, const Slot& sl, int mode) {
    for (int li = 0; li < m.nlev; li++) {
        const int base = m.lev_base[li];
        for (int i = (int)g.lane; i < m.lev_count[li]; i += G) sl.t(base + i) = group_sum(m, sl, li, i, mode);
        g.sync();
    }
}

// One binary level: left unless the target lies beyond a positive left
// weight and the right weight is positive.
__device__ __forceinline__ bool go_right(double& x, double L, double R) {
    if ((x <= L && L > 0.0) || R == 0.0) return false;
    x = x - L;
    return true;
}

// Leftmost leaf whose cumulative weight reaches x (ties go left); never a
// zero leaf.  Same decisions as a level-by-level descent of the binary tree.
__device__ __forceinline__ int descend(const Model& m, const Slot& sl, double x, int mode) {
    int i = 0;
    for (int li = m.nlev - 1; li >= 0; li--) {
        const int d = m.lev_d[li], c0 = i << d, lc = li - 1;
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

template <int G>
__device__ __forceinline__ void all_props(const Grp<G>& g, const Model& m, const Slot& sl) {
    for (int r = (int)g.lane; r < m.R; r += G) sl.pa(r) = prop(m, sl, r);
    g.sync();
    build_tree<G>(g, m, sl, 0);
}

// After firing r: new propensities for the reactions that depend on the
// changed species, then their tree paths (or a full rebuild when cheaper);
// both give the same tree.
template <int G>
__device__ void update_after_fire(const Grp<G>& g, const Model& m, const Slot& sl, int r) {
    const uint32_t d0 = m.dep_off[r], d1 = m.dep_off[r + 1];
    const uint32_t nd = d1 - d0;
    if (nd == 0) return;
    for (uint32_t j = d0 + g.lane; j < d1; j += G) {
        int rr = (int)m.dep_ent[j];
        sl.pa(rr) = prop(m, sl, rr);
    }
    g.sync();
    if (nd >= (uint32_t)m.lev_count[0]) {  // touches about every bottom group: rebuild
        build_tree<G>(g, m, sl, 0);
        return;
    }
    for (int li = 0; li < m.nlev; li++) {
        const int sh = m.lev_shift[li], base = m.lev_base[li];
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

// A0 == 0 (tau.cu:1665-1697, 2165-2196): the reference copies the last
// recorded sample forward (writing the current state first if none exists).
template <int G>
__device__ void finish_zero(const Grp<G>& g, const Model& m, const Run& run, const Slot& sl,
                            uint32_t* out, uint32_t& cursor) {
    const int so = m.s_out;
    const uint32_t ns = (uint32_t)m.ns;
    if (!(run.flags & F_Q10_OFF)) {
        if (cursor == 0) {
            for (int k = (int)g.lane; k < so; k += G) out[k] = (uint32_t)sl.x((int)m.cs[k]);
            cursor = 1;
        }
        for (uint32_t i = cursor; i < ns; i++)
            for (int k = (int)g.lane; k < so; k += G) out[(size_t)i * so + k] = out[(size_t)(cursor - 1) * so + k];
    } else {
        for (uint32_t i = cursor; i < ns; i++)
            for (int k = (int)g.lane; k < so; k += G) out[(size_t)i * so + k] = (uint32_t)sl.x((int)m.cs[k]);
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

template <int G>
__device__ void init_sim(const Grp<G>& g, const Model& m, const Run& run, const Slot& sl, Sim& st,
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
template <int G>
__device__ int decide_step(const Grp<G>& g, const Model& m, const Run& run, const Slot& sl, Sim& st,
                           uint32_t* out) {
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
    bool lany = false;
    for (int r = (int)lane; r < R; r += G) {
        uint8_t cr = 0;
        const uint32_t e1 = m.reac_off[r + 1];
        for (uint32_t e = m.reac_off[r]; e < e1; e++) {
            const uint32_t ent = m.reac_ent[e];
            const uint32_t q = (uint32_t)sl.x((int)(ent >> 8)) / (ent & 0xffu);
            if ((fl & F_Q6_OFF) ? (q < run.nc) : (q > 0u && q < run.nc)) cr = 1;
        }
        sl.cr(r) = cr;
        lany |= cr != 0;
    }
    const bool anycrit = g.any(lany);
    g.sync();
    float t1 = FLT_MAX;
    for (int s = (int)lane; s < S; s += G) {
        const uint32_t e0 = m.v_off[s], e1 = m.v_off[s + 1];
        if (e0 == e1) continue;
        float mu = 0.0f, sg = 0.0f;
        for (uint32_t e = e0; e < e1; e++) {
            const uint32_t ent = m.v_ent[e];
            const int r = (int)(ent >> 8);
            if (sl.cr(r)) continue;
            const float fv = (float)(int8_t)(ent & 0xffu);
            mu = mu + fv * sl.pa(r);
            sg = sg + (fv * fv) * sl.pa(r);
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
            if (lane == 0)  // the ancestors of leaf 0 are node 0 of every stored level
                for (int li = 0; li < m.nlev; li++) sl.t(m.lev_base[li]) = group_sum(m, sl, li, 0, 2);
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
            out[(size_t)st.cursor * so + k] = v;
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
template <int G>
__device__ int ssa_step(const Grp<G>& g, const Model& m, const Run& run, const Slot& sl, Sim& st,
                        uint32_t* out) {
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
        for (int k = (int)lane; k < so; k += G) out[(size_t)st.cursor * so + k] = (uint32_t)sl.x((int)m.cs[k]);
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

template <int G>
__device__ void finish_sim(const Grp<G>& g, const Model& m, const Run& run, const Sim& st, uint32_t* out) {
    const int so = m.s_out;
    for (uint32_t i = st.cursor; i < (uint32_t)m.ns; i++)
        for (int k = (int)g.lane; k < so; k += G) out[(size_t)i * so + k] = 0u;
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
// 4: 64, spilling to local memory as needed).
template <int G, int MINB>
__global__ void __launch_bounds__(256, MINB) sweep_kernel(Model m, Run run, Layout lay) {
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
        uint32_t* out = run.out;
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
                    out = run.out + (size_t)st.sim * sim_stride;
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
            uint32_t* out = run.out + (size_t)st.sim * sim_stride;
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
    size_t ctrl_off = place(256);
    d.bytes = off;
    std::vector<unsigned char> h(d.bytes, 0);
    auto put = [&](size_t o, const void* p, size_t bytes) {
        if (bytes) std::memcpy(h.data() + o, p, bytes);
    };
    put(d.off_reac_off, t.reac_off.data(), t.reac_off.size() * 4);
    put(d.off_reac_ent, t.reac_ent.data(), t.reac_ent.size() * 4);
    put(d.off_reac_desc, t.reac_desc.data(), t.reac_desc.size() * 4);
    put(d.off_vs_off, t.vs_off.data(), t.vs_off.size() * 4);
    put(d.off_vs_ent, t.vs_ent.data(), t.vs_ent.size() * 4);
    put(d.off_fs_off, t.fs_off.data(), t.fs_off.size() * 4);
    put(d.off_fs_ent, t.fs_ent.data(), t.fs_ent.size() * 4);
    put(d.off_fr_off, t.fr_off.data(), t.fr_off.size() * 4);
    put(d.off_fr_ent, t.fr_ent.data(), t.fr_ent.size() * 4);
    put(d.off_dep_off, t.dep_off.data(), t.dep_off.size() * 4);
    put(d.off_dep_ent, t.dep_ent.data(), t.dep_ent.size() * 4);
    put(d.off_hor, t.hor.data(), t.hor.size());
    put(d.off_hort, t.hort.data(), t.hort.size());
    put(d.off_tvec, t.tvec.data(), t.tvec.size() * 8);
    put(d.off_cs, t.cs.data(), t.cs.size() * 4);
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
};

// Stored levels of the sum tree for P = 2^k leaves: 3, 6, ... below k, then
// k (the root).  Level li is the pairwise sum of 2^d nodes of level li-1.
static void tree_levels(const HostTables& t, dev::Model& dm) {
    const int k = t.logP;
    int prev = 0, base = 0, n = 0;
    for (int l = 3; l < k; l += 3) {
        dm.lev_shift[n] = l;
        dm.lev_d[n] = l - prev;
        dm.lev_base[n] = base;
        dm.lev_count[n] = t.P >> l;
        base += t.P >> l;
        prev = l;
        n++;
    }
    dm.lev_shift[n] = k;
    dm.lev_d[n] = k - prev;
    dm.lev_base[n] = base;
    dm.lev_count[n] = 1;
    dm.nlev = n + 1;
}

static int tree_words(const HostTables& t) {
    dev::Model dm;
    tree_levels(t, dm);
    return dm.lev_base[dm.nlev - 1] + 1;
}

// Shared-memory bytes of a block with NS slots of group size G.
static size_t slot_layout(const HostTables& t, int G, int NS, bool uniform_c, dev::Layout& lay) {
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
    } else {
        lay.len_S = (uint32_t)(t.S | 1);
        lay.len_P = (uint32_t)(t.P + 1);
        lay.len_C = (uint32_t)(((t.P + 3) & ~3) + 4);
        lay.len_T = (uint32_t)(tw | 1);
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
    return off;
}

// Register budgets compiled for every group size: minimum resident
// 256-thread blocks per SM 2, 3 or 4.
template <int G>
static const void* kernel_ptr(int minb) {
    switch (minb) {
        case 3: return reinterpret_cast<const void*>(&dev::sweep_kernel<G, 3>);
        case 4: return reinterpret_cast<const void*>(&dev::sweep_kernel<G, 4>);
        default: return reinterpret_cast<const void*>(&dev::sweep_kernel<G, 2>);
    }
}
static const void* kernel_for(int G, int minb) {
    switch (G) {
        case 1: return kernel_ptr<1>(minb);
        case 2: return kernel_ptr<2>(minb);
        case 4: return kernel_ptr<4>(minb);
        case 8: return kernel_ptr<8>(minb);
        case 16: return kernel_ptr<16>(minb);
        case 32: return kernel_ptr<32>(minb);
        case 64: return kernel_ptr<64>(minb);
        case 128: return kernel_ptr<128>(minb);
        case 256: return kernel_ptr<256>(minb);
    }
    return nullptr;
}

// Lanes per simulation when the caller does not choose: about 16
// reactions per lane (measured best for 64x128: G = 8; tiny networks: 1).
static int heuristic_group(const HostTables& t) {
    int g = t.P / 16;
    int G = 1;
    while (G < g && G < 32) G <<= 1;
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
    int dev, G, minb, regs;
    size_t dyn_max;
};
static std::vector<KernAttr> g_kattr;

static ctl_status kernel_attr(int dev, int G, int minb, KernAttr& out) {
    DevAttr da;
    if (device_attr(dev, da) != CTL_OK) return CTL_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const auto& a : g_kattr)
        if (a.dev == dev && a.G == G && a.minb == minb) {
            out = a;
            return CTL_OK;
        }
    const void* k = kernel_for(G, minb);
    cudaFuncAttributes fa;
    CTL_CUDA(cudaFuncGetAttributes(&fa, k));
    if ((size_t)da.smem_optin <= fa.sharedSizeBytes) {
        set_error("sweep kernel's static shared memory exceeds the device limit");
        return CTL_ERR_SHAPE;
    }
    KernAttr a{dev, G, minb, fa.numRegs, (size_t)da.smem_optin - fa.sharedSizeBytes};
    CTL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.dyn_max));
    g_kattr.push_back(a);
    out = a;
    return CTL_OK;
}

struct OccKey {
    int dev, G, minb, threads;
    size_t smem;
    int bps;
};
static std::vector<OccKey> g_occ;

static ctl_status occupancy(int dev, int G, int minb, int threads, size_t smem, int& bps, int& regs) {
    KernAttr ka;
    ctl_status st = kernel_attr(dev, G, minb, ka);
    if (st != CTL_OK) return st;
    regs = ka.regs;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const auto& o : g_occ)
        if (o.dev == dev && o.G == G && o.minb == minb && o.threads == threads && o.smem == smem) {
            bps = o.bps;
            return CTL_OK;
        }
    CTL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel_for(G, minb), threads, smem));
    g_occ.push_back({dev, G, minb, threads, smem, bps});
    return CTL_OK;
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

static ctl_status plan_launch(ctl_model* m, const ctl_run_cfg* cfg_in, uint32_t n, LaunchPlan& pl) {
    const HostTables& t = m->t;
    ctl_run_cfg tuned_cfg = *cfg_in;
    if (cfg_in->group <= 0 && cfg_in->threads <= 0) {
        ctl_model::Tuned e;
        if (find_tuned(m, cfg_in, n, e)) {
            tuned_cfg.group = e.group;
            tuned_cfg.threads = e.threads;
            if (tuned_cfg.ssa_budget <= 0) tuned_cfg.ssa_budget = e.ssa_budget;
            if (tuned_cfg.dec_budget <= 0) tuned_cfg.dec_budget = e.dec_budget;
            if (tuned_cfg.min_blocks <= 0) tuned_cfg.min_blocks = e.min_blocks;
            if (tuned_cfg.sched <= 0) tuned_cfg.sched = e.sched;
        }
    }
    const ctl_run_cfg* cfg = &tuned_cfg;
    pl.ssa_budget = cfg->ssa_budget;
    pl.dec_budget = cfg->dec_budget;
    pl.sched = cfg->sched > 0 ? cfg->sched : 1;
    int G = cfg->group > 0 ? cfg->group : heuristic_group(t);
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
    // Register budget: as many resident blocks as the slot memory of a full
    // 256-thread block allows (2 or 3; 4 only when chosen or tuned).
    int minb = cfg->min_blocks;
    if (minb <= 0) {
        const size_t full = slot_layout(t, G, 256 / G, uni, pl.lay);
        minb = 3 * (full + 1024) <= (size_t)da.smem_optin + 1024 ? 3 : 2;
    }
    if (ctl_status st = kernel_attr(dev_id, G, minb, ka); st != CTL_OK) return st;
    const size_t smem_max = ka.dyn_max;
    if (cfg->threads <= 0) {
        while (threads > tstep && (uint64_t)n * G < (uint64_t)threads * da.sm_count) threads -= tstep;
    }
    for (;;) {
        int NS = threads / G;
        size_t bytes = slot_layout(t, G, NS, uni, pl.lay);
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
    pl.threads = threads;
    int bps = 0, regs = 0;
    if (ctl_status st = occupancy(dev_id, G, minb, threads, pl.smem, bps, regs); st != CTL_OK) return st;
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
    return CTL_OK;
}

static ctl_status enqueue_sweep(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* dX0,
                                const float* dc, uint32_t* dout, ctl_sim_info* dinfo,
                                cudaStream_t stream, const LaunchPlan& pl, const DeviceCopy& d) {
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
    run.ssa_budget = pl.ssa_budget > 0 ? (uint32_t)pl.ssa_budget : 8u;
    run.dec_budget = pl.dec_budget > 0 ? (uint32_t)pl.dec_budget : 2u;
    run.warp_local = pl.sched == 2 ? 1u : 0u;
    run.X0 = dX0;
    run.c = dc;
    run.out = dout;
    run.info = dinfo;
    run.queue = d.ctrl;
    dev::Model dm = make_dev_model(m, d, cfg->flags);
    CTL_CUDA(cudaMemsetAsync(d.ctrl, 0, sizeof(uint32_t), stream));
    void* args[] = {&dm, &run, const_cast<dev::Layout*>(&pl.lay)};
    CTL_CUDA(cudaLaunchKernel(kernel_for(pl.G, pl.minb), dim3((unsigned)pl.blocks), dim3((unsigned)pl.threads), args,
                              pl.smem, stream));
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
    if (cfg->min_blocks != 0 && (cfg->min_blocks < 2 || cfg->min_blocks > 4)) {
        set_error("min_blocks must be 0 (library choice), 2, 3 or 4");
        return CTL_ERR_ARG;
    }
    if (cfg->sched < 0 || cfg->sched > 2) {
        set_error("sched must be 0 (library choice), 1 (block regrouping) or 2 (warp-local)");
        return CTL_ERR_ARG;
    }
    return CTL_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        cudaGetDevice(&prev);
        cudaSetDevice(d);
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
    const size_t bo = (size_t)n * t.ns * t.s_out * 4, bi = (size_t)n * sizeof(ctl_sim_info);
    keep_pool_memory(cfg->device);
    cudaStream_t s;
    CTL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *dx = nullptr, *dc = nullptr, *dout = nullptr, *dinf = nullptr;
    cudaError_t e = cudaMallocAsync(&dx, bx, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dc, bc, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dout, bo, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dinf, bi, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, X0, bx, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, c, bc, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        st = enqueue_sweep(m, cfg, n, static_cast<int32_t*>(dx), static_cast<float*>(dc),
                           static_cast<uint32_t*>(dout), static_cast<ctl_sim_info*>(dinf), s, pl, *d);
        if (st != CTL_OK) e = cudaErrorLaunchFailure;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(samples, dout, bo, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(info, dinf, bi, cudaMemcpyDeviceToHost, s);
    if (dx) cudaFreeAsync(dx, s);
    if (dc) cudaFreeAsync(dc, s);
    if (dout) cudaFreeAsync(dout, s);
    if (dinf) cudaFreeAsync(dinf, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (st != CTL_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "ctl_run");
    if (e2 != cudaSuccess) return cuda_fail(e2, "ctl_run (sweep)");
    for (uint32_t i = 0; i < n; i++)
        if (info[i].status != CTL_SIM_OK) {
            set_error("simulation " + std::to_string(i) + " ended with status " + std::to_string(info[i].status));
            return CTL_ERR_STEP_LIMIT;
        }
    return CTL_OK;
}

// Measured autotuner: times candidate launch shapes on the first `sample`
// simulations of the batch (results are identical for every shape, only the
// time differs) -- group size first, then threads per block, then the
// per-round budgets -- and caches the fastest for this (device, batch-size
// bucket, rate mode, flags).
extern "C" ctl_status ctl_autotune(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* d_X0,
                                   const float* d_c, uint32_t sample, ctl_launch_info* best) {
    if (!m || !d_X0 || !d_c || n == 0) return CTL_ERR_ARG;
    ctl_status st = check_cfg(cfg);
    if (st != CTL_OK) return st;
    const HostTables& t = m->t;
    DeviceGuard dg(cfg->device);
    DeviceCopy* d = nullptr;
    if ((st = ensure_device(m, cfg->device, d)) != CTL_OK) return st;
    const uint32_t k = sample == 0 || sample > n ? n : sample;
    cudaStream_t s;
    CTL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *dout = nullptr, *dinf = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaError_t e = cudaMallocAsync(&dout, (size_t)k * t.ns * t.s_out * 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dinf, (size_t)k * sizeof(ctl_sim_info), s);
    auto time_shape = [&](int G, int threads, int sb, int db, int mb, int sc, float& ms) -> ctl_status {
        ctl_run_cfg c = *cfg;
        c.group = G;
        c.threads = threads;
        c.ssa_budget = sb;
        c.dec_budget = db;
        c.min_blocks = mb;
        c.sched = sc;
        LaunchPlan pl;
        ctl_status r = plan_launch(m, &c, k, pl);
        if (r != CTL_OK) return r;
        cudaEventRecord(e0, s);
        r = enqueue_sweep(m, &c, k, d_X0, d_c, static_cast<uint32_t*>(dout), static_cast<ctl_sim_info*>(dinf), s, pl, *d);
        cudaEventRecord(e1, s);
        if (r != CTL_OK) return r;
        if (cudaEventSynchronize(e1) != cudaSuccess) return CTL_ERR_CUDA;
        cudaEventElapsedTime(&ms, e0, e1);
        return CTL_OK;
    };
    int bestG = heuristic_group(t), bestT = 256, bestS = 8, bestD = 2, bestM = 2, bestC = 1;
    float best_ms = 3.4e38f;
    if (e == cudaSuccess) {
        for (int G = 1; G <= 256 && G <= t.P; G <<= 1) {  // 1. lanes per simulation
            float ms;
            if (time_shape(G, 256, 8, 2, 2, 1, ms) == CTL_OK && ms < best_ms) { best_ms = ms; bestG = G; }
        }
        for (int th : {64, 128, 192}) {                   // 2. threads per block
            float ms;
            if (th % bestG == 0 && th >= bestG && time_shape(bestG, th, 8, 2, 2, 1, ms) == CTL_OK && ms < best_ms) {
                best_ms = ms;
                bestT = th;
            }
        }
        {                                                  // 3. scheduling: warp-local vs block rounds
            float ms;
            if (time_shape(bestG, bestT, 8, 2, 2, 2, ms) == CTL_OK && ms < best_ms) { best_ms = ms; bestC = 2; }
        }
        for (int mb : {3, 4}) {                            // 4. register budget (resident blocks)
            float ms;
            if (time_shape(bestG, bestT, 8, 2, mb, bestC, ms) == CTL_OK && ms < best_ms) { best_ms = ms; bestM = mb; }
        }
        for (int sb : {2, 4, 16, 32}) {                    // 5. SSA steps per round
            float ms;
            if (time_shape(bestG, bestT, sb, 2, bestM, bestC, ms) == CTL_OK && ms < best_ms) { best_ms = ms; bestS = sb; }
        }
        for (int db : {1, 4, 8}) {                         // 6. decisions per round
            float ms;
            if (time_shape(bestG, bestT, bestS, db, bestM, bestC, ms) == CTL_OK && ms < best_ms) {
                best_ms = ms;
                bestD = db;
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
        bool found = false;
        for (auto& x : m->tuned)
            if (x.device == cfg->device && x.nbucket == nb && x.uniform == uni && x.flags == cfg->flags) {
                x.group = bestG; x.threads = bestT; x.ssa_budget = bestS; x.dec_budget = bestD; x.min_blocks = bestM;
                x.sched = bestC;
                found = true;
            }
        if (!found) m->tuned.push_back({cfg->device, nb, uni, cfg->flags, bestG, bestT, bestS, bestD, bestM, bestC});
    }
    if (best) {
        ctl_run_cfg c = *cfg;
        c.group = 0;
        c.threads = 0;
        c.min_blocks = 0;
        c.sched = 0;
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
    if (e == cudaSuccess) e = put(d.off_reac_off, t.reac_off.data(), t.reac_off.size() * 4);
    if (e == cudaSuccess) e = put(d.off_reac_ent, t.reac_ent.data(), t.reac_ent.size() * 4);
    if (e == cudaSuccess) e = put(d.off_reac_desc, t.reac_desc.data(), t.reac_desc.size() * 4);
    if (e == cudaSuccess) e = put(d.off_vs_off, t.vs_off.data(), t.vs_off.size() * 4);
    if (e == cudaSuccess) e = put(d.off_vs_ent, t.vs_ent.data(), t.vs_ent.size() * 4);
    if (e == cudaSuccess) e = put(d.off_fs_off, t.fs_off.data(), t.fs_off.size() * 4);
    if (e == cudaSuccess) e = put(d.off_fs_ent, t.fs_ent.data(), t.fs_ent.size() * 4);
    if (e == cudaSuccess) e = put(d.off_fr_off, t.fr_off.data(), t.fr_off.size() * 4);
    if (e == cudaSuccess) e = put(d.off_fr_ent, t.fr_ent.data(), t.fr_ent.size() * 4);
    if (e == cudaSuccess) e = put(d.off_dep_off, t.dep_off.data(), t.dep_off.size() * 4);
    if (e == cudaSuccess) e = put(d.off_dep_ent, t.dep_ent.data(), t.dep_ent.size() * 4);
    if (e == cudaSuccess) e = put(d.off_hor, t.hor.data(), t.hor.size());
    if (e == cudaSuccess) e = put(d.off_hort, t.hort.data(), t.hort.size());
    if (e == cudaSuccess) e = put(d.off_tvec, t.tvec.data(), t.tvec.size() * 8);
    if (e == cudaSuccess) e = put(d.off_cs, t.cs.data(), t.cs.size() * 4);
    if (e != cudaSuccess) return cuda_fail(e, "ctl_run_device_noalloc (tables)");
    LaunchPlan pl;
    if ((st = plan_launch(m, cfg, n, pl)) != CTL_OK) return st;
    return enqueue_sweep(m, cfg, n, d_X0, d_c, d_samples, d_info, s, pl, d);
}

// Device arithmetic shared by every sweep kernel and by the model-specialised
// kernels compiled at run time (NVRTC): the random stream, the elementary
// functions, the Poisson sampler, Cao's g_i, the sum-tree step and the run
// parameters.  Self-contained: under NVRTC it needs no host header.
//
// Determinism contract (what makes any launch shape give identical bits):
//   * every random word comes from Philox4x32-10 with key = seed and counter
//     (block, tag, step, sim): a draw depends on which simulation, which step
//     and what it is for, never on which thread computes it;
//   * every FP64 sum over reactions is the root of a fixed binary tree over
//     the reactions padded to P = 2^k leaves, and the searches descend it;
//   * the elementary functions are this file's own (no CUDA math library
//     calls on the path), so the CPU oracle (oracle/ctl_oracle.c) computes
//     the same bits.
// Built with -fmad=false: no implicit FMA contraction; fma() is called
// explicitly where it is meant.
#pragma once

#ifdef __CUDACC_RTC__
typedef unsigned char uint8_t;
typedef signed char int8_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef unsigned long size_t;
typedef unsigned long uintptr_t;
#define FLT_MAX 3.402823466e+38F
// The per-simulation record of include/ctl.h (same layout).
typedef struct {
    double t_final;
    uint64_t firings;
    uint32_t status;
    uint32_t steps, leaps, ssa_steps, rejections, pad;
} ctl_sim_info;
enum { CTL_SIM_OK = 0, CTL_SIM_STEP_LIMIT = 1, CTL_SIM_OVERFLOW = 2, CTL_SIM_ATTEMPT_LIMIT = 3 };
#else
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "../../include/ctl.h"
#endif

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

struct Run {
    uint64_t seed;
    float eps;
    uint32_t nc;
    double ssa_factor;
    uint32_t ssa_steps, flags, max_steps, sim_base, n;
    uint32_t uniform_c;              // all simulations share row 0 of c
    uint32_t ssa_budget, dec_budget; // work per slot and round (SSA steps / decisions)
    uint32_t warp_local;             // 1: warp-local scheduling (no block rounds)
    uint32_t tail_sims;              // register-resident block rounds: live simulations at or
                                     // below which a block with a closed queue finishes them in
                                     // warp lockstep (0: never)
    unsigned long long* sums;        // fitness mode: [sets][ns][s_out] sample sums, else null
    uint32_t sum_threads, sum_prep;  // simulation -> parameter set (the reference's layout)
    uint32_t* done;                  // optional: finished simulations per chunk of 2^done_shift
    uint32_t* out_host;              // optional: the caller's pinned rows [n][ns][s_out] (device view);
                                     // each finished row is copied there by the kernel
    uint32_t done_shift;
    const int32_t* __restrict__ X0;  // [n][S]
    const float* __restrict__ c;     // [n][R]
    uint32_t* __restrict__ out;      // [n][ns][s_out]
    ctl_sim_info* __restrict__ info; // [n]
    uint32_t* queue;                 // work-queue ticket
};


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
static __device__ double dlog(double x) {
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
static __device__ double dexp(double x) {
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

static __constant__ double c_logfact[16] = {
    0.0, 0.0, 0x1.62e42fefa39efp-1, 0x1.cab0bfa2a2002p+0, 0x1.96ca77c922cf9p+1,
    0x1.326643c4479c9p+2, 0x1.a51273acf01cap+2, 0x1.10ce1f32dcc30p+3,
    0x1.5358e82fcb70dp+3, 0x1.99a8921a7f7cfp+3, 0x1.e357590954d15p+3,
    0x1.180973f3a8d74p+4, 0x1.3fcba16d50143p+4, 0x1.68d5a9c3b32cep+4,
    0x1.930f3df162a42p+4, 0x1.be636a63fd346p+4};

// log(k!) : table below 16, Stirling series above.
static __device__ double dlogfact(double k) {
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

// 1/k for k = 1..64, correctly rounded: the inversion's recurrence
// multiplies by these instead of dividing (an FP64 division is a long
// instruction sequence on the GPU); the oracle holds the same literals.
static __constant__ double c_recip[64] = {
    0x1.0000000000000p+0, 0x1.0000000000000p-1, 0x1.5555555555555p-2, 0x1.0000000000000p-2,
    0x1.999999999999ap-3, 0x1.5555555555555p-3, 0x1.2492492492492p-3, 0x1.0000000000000p-3,
    0x1.c71c71c71c71cp-4, 0x1.999999999999ap-4, 0x1.745d1745d1746p-4, 0x1.5555555555555p-4,
    0x1.3b13b13b13b14p-4, 0x1.2492492492492p-4, 0x1.1111111111111p-4, 0x1.0000000000000p-4,
    0x1.e1e1e1e1e1e1ep-5, 0x1.c71c71c71c71cp-5, 0x1.af286bca1af28p-5, 0x1.999999999999ap-5,
    0x1.8618618618618p-5, 0x1.745d1745d1746p-5, 0x1.642c8590b2164p-5, 0x1.5555555555555p-5,
    0x1.47ae147ae147bp-5, 0x1.3b13b13b13b14p-5, 0x1.2f684bda12f68p-5, 0x1.2492492492492p-5,
    0x1.1a7b9611a7b96p-5, 0x1.1111111111111p-5, 0x1.0842108421084p-5, 0x1.0000000000000p-5,
    0x1.f07c1f07c1f08p-6, 0x1.e1e1e1e1e1e1ep-6, 0x1.d41d41d41d41dp-6, 0x1.c71c71c71c71cp-6,
    0x1.bacf914c1bad0p-6, 0x1.af286bca1af28p-6, 0x1.a41a41a41a41ap-6, 0x1.999999999999ap-6,
    0x1.8f9c18f9c18fap-6, 0x1.8618618618618p-6, 0x1.7d05f417d05f4p-6, 0x1.745d1745d1746p-6,
    0x1.6c16c16c16c17p-6, 0x1.642c8590b2164p-6, 0x1.5c9882b931057p-6, 0x1.5555555555555p-6,
    0x1.4e5e0a72f0539p-6, 0x1.47ae147ae147bp-6, 0x1.4141414141414p-6, 0x1.3b13b13b13b14p-6,
    0x1.3521cfb2b78c1p-6, 0x1.2f684bda12f68p-6, 0x1.29e4129e4129ep-6, 0x1.2492492492492p-6,
    0x1.1f7047dc11f70p-6, 0x1.1a7b9611a7b96p-6, 0x1.15b1e5f75270dp-6, 0x1.1111111111111p-6,
    0x1.0c9714fbcda3bp-6, 0x1.0842108421084p-6, 0x1.0410410410410p-6, 0x1.0000000000000p-6};

// Poisson(lam) given the reaction's primary uniform pair (wa, wb).
// lam < 10: sequential inversion, p_k = p_{k-1} lam (1/k) with tabulated
// reciprocals.  lam >= 10: Hormann's PTRS (1993); extra
// trials read blocks 1 + 2j + odd of the same (tag, step, sim) stream.
static __device__ uint32_t poisson(double lam, uint32_t wa, uint32_t wb, uint64_t seed, uint32_t tag,
                            uint32_t step, uint32_t sim, uint32_t odd) {
    if (!(lam > 0.0)) return 0u;
    if (lam < 10.0) {
        double u = u32d(wa);
        double p = dexp(-lam);
        double F = p;
        uint32_t k = 0;
        while (u > F && k < 64u) {
            k = k + 1u;
            p = (p * lam) * c_recip[k - 1u];
            F = F + p;
        }
        return k;
    }
    double slam = sqrt(lam);
    double b = 0.931 + 2.53 * slam;
    double a = -0.059 + 0.02483 * b;
    double vr = 0.9277 - 3.6224 / (b - 2.0);
    // log(lam) and log(1/alpha) only serve the slow acceptance test; most
    // draws are accepted before it, so they are computed on its first use
    double loglam = 0.0, log_invalpha = 0.0;
    bool slow = false;
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
        if (!slow) {
            loglam = dlog(lam);
            log_invalpha = dlog(1.1239 + 1.1328 / (b - 3.4));
            slow = true;
        }
        double lhs = dlog(V) + log_invalpha - dlog(a / (us * us) + b);
        double rhs = -lam + k * loglam - dlogfact(k);
        if (lhs <= rhs) return clamp_k(k);
    }
    return clamp_k(floor(lam));
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

// One binary level: left unless the target lies beyond a positive left
// weight and the right weight is positive.
__device__ __forceinline__ bool go_right(double& x, double L, double R) {
    if ((x <= L && L > 0.0) || R == 0.0) return false;
    x = x - L;
    return true;
}


}  // namespace dev
}  // namespace ctl

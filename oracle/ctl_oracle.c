/*
 * ctl_oracle.c -- CPU oracle for the cuTauLeaping hot path.  TEST
 * INFRASTRUCTURE ONLY (see ctl_oracle.h): the product never links it.
 *
 * Build: plain C11, -O3 -ffp-contract=off (no implicit FMA: every rounding
 * step is spelled out so that the CUDA kernels, compiled with -fmad=false,
 * produce the same bits).
 */
#include "ctl_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Canonical random stream                                                  */
/* ------------------------------------------------------------------------ */

/* Counter word 1 ("tag") of the Philox counter (block, tag, step, sim). */
#define TAG_SSA   0x40000000u /* SSA steps 2b, 2b+1: block b, (w0,w1) / (w2,w3)   */
#define TAG_MISC  0x40000001u /* leap: (w0,w1) tau2, (w2,w3) critical pick      */
#define TAG_GILL  0x20000000u /* exact Gillespie oracle                        */
#define TAG_POIS(attempt, pair) (0x80000000u | ((uint32_t)(attempt) << 20) | (uint32_t)(pair))

#define MAX_ATTEMPTS 1024u    /* 10-bit attempt field of TAG_POIS */
#define PTRS_MAX_TRIALS 256u

/* Philox4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11: ten rounds of two 32x32->64 multiplies with a
 * Weyl-sequence key schedule. */
void ctlo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int i = 0; i < 10; i++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void draw(uint64_t seed, uint32_t blk, uint32_t tag, uint32_t step, uint32_t sim,
                 uint32_t w[4]) {
    uint32_t ctr[4] = {blk, tag, step, sim};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    ctlo_philox(ctr, key, w);
}

/* (w + 1/2) / 2^32: exact in double, strictly inside (0, 1). */
static double u32d(uint32_t w) { return ((double)w + 0.5) * 0x1p-32; }
/* 52 random bits + 1/2, scaled: exact in double, strictly inside (0, 1). */
static double u53(uint32_t wa, uint32_t wb) {
    uint64_t m = ((uint64_t)wb << 20) | (uint64_t)(wa >> 12);
    return ((double)m + 0.5) * 0x1p-52;
}

/* ------------------------------------------------------------------------ */
/* Elementary functions (own implementations; identical on the GPU)         */
/* ------------------------------------------------------------------------ */

#define LN2_HI  0x1.62e42fee00000p-1   /* ln 2 rounded to 32 significant bits */
#define LN2_LO  0x1.a39ef35793c76p-33  /* ln 2 - LN2_HI                        */
#define INV_LN2 0x1.71547652b82fep+0
#define SQRT2   0x1.6a09e667f3bcdp+0

static uint64_t d2u(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static double u2d(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

/* log(x): x = m 2^e with m in (sqrt(1/2), sqrt(2)]; log m = 2 atanh(s),
 * s = (m-1)/(m+1), summed as the odd series 2s(1 + s^2/3 + ... + s^20/21). */
double ctlo_log(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    int eadj = 0;
    if (x < 0x1p-1022) { x = x * 0x1p54; eadj = -54; }
    uint64_t b = d2u(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023 + eadj;
    double m = u2d((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > SQRT2) { m = m * 0.5; e = e + 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double p = 0x1.8618618618618p-5;          /* 1/21 */
    p = fma(p, z, 0x1.af286bca1af28p-5);      /* 1/19 */
    p = fma(p, z, 0x1.e1e1e1e1e1e1ep-5);      /* 1/17 */
    p = fma(p, z, 0x1.1111111111111p-4);      /* 1/15 */
    p = fma(p, z, 0x1.3b13b13b13b14p-4);      /* 1/13 */
    p = fma(p, z, 0x1.745d1745d1746p-4);      /* 1/11 */
    p = fma(p, z, 0x1.c71c71c71c71cp-4);      /* 1/9  */
    p = fma(p, z, 0x1.2492492492492p-3);      /* 1/7  */
    p = fma(p, z, 0x1.999999999999ap-3);      /* 1/5  */
    p = fma(p, z, 0x1.5555555555555p-2);      /* 1/3  */
    double r = z * p;
    double ed = (double)e;
    double two_s = s + s;
    return fma(ed, LN2_HI, two_s + fma(two_s, r, ed * LN2_LO));
}

/* exp(x): Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, Taylor series of
 * degree 14 for exp(r), then scaling by 2^k. */
double ctlo_exp(double x) {
    if (x != x) return x;
    if (x > 709.0) return INFINITY;
    if (x < -745.0) return 0.0;
    double k = rint(x * INV_LN2);
    double r = fma(-k, LN2_HI, x);
    r = fma(-k, LN2_LO, r);
    double p = 0x1.93974a8c07c9dp-37;         /* 1/14! */
    p = fma(p, r, 0x1.6124613a86d09p-33);     /* 1/13! */
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
    return p * u2d((uint64_t)(ki + 1023) << 52);
}

/* FP32 log(x) for normal x > 0: the same reduction as ctlo_log in single
 * precision, series 2s(1 + s^2/3 + s^4/5 + s^6/7 + s^8/9). */
#define LN2_HI_F 0x1.62e4p-1f       /* ln 2 rounded to 16 significant bits */
#define LN2_LO_F 0x1.7f7d1cp-20f   /* ln 2 - LN2_HI_F, rounded */
float ctlo_logf(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    int e = (int)((b >> 23) & 0xff) - 127;
    uint32_t mb = (b & 0x007fffffu) | 0x3f800000u;
    float m;
    memcpy(&m, &mb, 4);
    if (m > 0x1.6a09e6p+0f) { m = m * 0.5f; e = e + 1; }
    float f = m - 1.0f;
    float sv = f / (2.0f + f);
    float z = sv * sv;
    float p = 0x1.c71c72p-4f;             /* 1/9 */
    p = fmaf(p, z, 0x1.24924ap-3f);       /* 1/7 */
    p = fmaf(p, z, 0x1.99999ap-3f);       /* 1/5 */
    p = fmaf(p, z, 0x1.555556p-2f);       /* 1/3 */
    float r = z * p;
    float ef = (float)e;
    float two_s = sv + sv;
    return fmaf(ef, LN2_HI_F, two_s + fmaf(two_s, r, ef * LN2_LO_F));
}

/* (w >> 8) + 1/2 over 2^24: exact in float, strictly inside (0, 1). */
static float u24f(uint32_t w) { return ((float)(w >> 8) + 0.5f) * 0x1p-24f; }

/* log(k!) for integer-valued k >= 0: table below 16, Stirling's series
 * (Bernoulli terms up to x^-7) above. */
static const double LOGFACT[16] = {
    0.0, 0.0, 0x1.62e42fefa39efp-1, 0x1.cab0bfa2a2002p+0, 0x1.96ca77c922cf9p+1,
    0x1.326643c4479c9p+2, 0x1.a51273acf01cap+2, 0x1.10ce1f32dcc30p+3,
    0x1.5358e82fcb70dp+3, 0x1.99a8921a7f7cfp+3, 0x1.e357590954d15p+3,
    0x1.180973f3a8d74p+4, 0x1.3fcba16d50143p+4, 0x1.68d5a9c3b32cep+4,
    0x1.930f3df162a42p+4, 0x1.be636a63fd346p+4};

double ctlo_logfact(double k) {
    if (k < 16.0) return LOGFACT[(int)k];
    double x = k + 1.0;
    double ix = 1.0 / x;
    double ix2 = ix * ix;
    double ser = ix * (0x1.5555555555555p-4 -
                       ix2 * (0x1.6c16c16c16c17p-9 -
                              ix2 * (0x1.a01a01a01a01ap-11 - ix2 * 0x1.3813813813814p-11)));
    return (x - 0.5) * ctlo_log(x) - x + 0x1.d67f1c864beb5p-1 + ser;
}

/* ------------------------------------------------------------------------ */
/* Poisson sampler                                                          */
/* ------------------------------------------------------------------------ */

static uint32_t clamp_k(double k) {
    if (k > 2147483647.0) return 2147483647u;
    return (uint32_t)k;
}

/* Poisson(lam) for reaction r in rejection attempt `attempt` of step `step`.
 * Stream: primary block (0, TAG_POIS(attempt, r>>1), step, sim) gives the
 * pair (w0,w1) to even r and (w2,w3) to odd r; PTRS retries read extra
 * blocks 1 + 2j + (r&1), two trials per block.
 * lam < 10: sequential inversion from k = 0 (one uniform), p_k =
 * p_{k-1} lam (1/k) with the correctly rounded reciprocals of recip_k.
 * lam >= 10: PTRS, W. Hormann, "The transformed rejection method for
 * generating Poisson random variables", Insurance: Mathematics and
 * Economics 12 (1993) 39-45. */
static const double recip_k[64] = {
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

uint32_t ctlo_poisson(double lam, uint64_t seed, uint32_t sim, uint32_t step,
                      uint32_t attempt, uint32_t r) {
    if (!(lam > 0.0)) return 0;
    uint32_t tag = TAG_POIS(attempt, r >> 1);
    uint32_t w[4];
    draw(seed, 0, tag, step, sim, w);
    uint32_t wa = (r & 1) ? w[2] : w[0];
    uint32_t wb = (r & 1) ? w[3] : w[1];
    if (lam < 10.0) {
        double u = u32d(wa);
        double p = ctlo_exp(-lam);
        double F = p;
        uint32_t k = 0;
        while (u > F && k < 64) {
            k = k + 1;
            p = (p * lam) * recip_k[k - 1];
            F = F + p;
        }
        return k;
    }
    double slam = sqrt(lam);
    double loglam = ctlo_log(lam);
    double b = 0.931 + 2.53 * slam;
    double a = -0.059 + 0.02483 * b;
    double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (uint32_t t = 0; t < PTRS_MAX_TRIALS; t++) {
        if (t > 0) {
            uint32_t j = (t - 1) >> 1;
            if (((t - 1) & 1) == 0) draw(seed, 1 + 2 * j + (r & 1), tag, step, sim, w);
            wa = ((t - 1) & 1) ? w[2] : w[0];
            wb = ((t - 1) & 1) ? w[3] : w[1];
        }
        double U = u32d(wa) - 0.5;
        double V = u32d(wb);
        double us = 0.5 - fabs(U);
        double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return clamp_k(k);
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        double lhs = ctlo_log(V) + ctlo_log(invalpha) - ctlo_log(a / (us * us) + b);
        double rhs = -lam + k * loglam - ctlo_logfact(k);
        if (lhs <= rhs) return clamp_k(k);
    }
    return clamp_k(floor(lam));
}

/* ------------------------------------------------------------------------ */
/* Model                                                                    */
/* ------------------------------------------------------------------------ */

struct ctlo_model {
    int S, R, P, ns, s_out;
    int *reac_off, *reac_s, *reac_st;    /* reactants (left > 0), reaction-major */
    int *vs_off, *vs_r, *vs_v;           /* V = right-left, species-major (RAV)  */
    int *fs_off, *fs_r, *fs_v;           /* F (feed-masked V), species-major     */
    int *fr_off, *fr_s, *fr_v;           /* F, reaction-major                    */
    uint8_t *hor, *hort;
    double* tvec;
    int* cs;
    double tmax;
    float eps;
    uint32_t nc;
    double ssa_factor;
    uint32_t ssa_steps, flags, max_steps;
    uint64_t seed;
};

void ctlo_model_free(ctlo_model* m) {
    if (!m) return;
    free(m->reac_off); free(m->reac_s); free(m->reac_st);
    free(m->vs_off); free(m->vs_r); free(m->vs_v);
    free(m->fs_off); free(m->fs_r); free(m->fs_v);
    free(m->fr_off); free(m->fr_s); free(m->fr_v);
    free(m->hor); free(m->hort); free(m->tvec); free(m->cs);
    free(m);
}

/* Compressed lists.  Entry order follows the reference flattening loops
 * (tau.cu:212-225 reactants r-major; 314-326 RAV species-major; 330-342 F
 * r-major), so that every sequential sum runs in the reference's order. */
static int build_list(int outer, int inner, int major_is_r, const int32_t* mat, int S,
                      int** off, int** idx, int** val) {
    int nnz = 0;
    for (int i = 0; i < outer * inner; i++) nnz += mat[i] != 0;
    *off = (int*)malloc(sizeof(int) * (size_t)(outer + 1));
    *idx = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    *val = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    if (!*off || !*idx || !*val) return -1;
    int n = 0;
    for (int o = 0; o < outer; o++) {
        (*off)[o] = n;
        for (int i = 0; i < inner; i++) {
            int r = major_is_r ? o : i, s = major_is_r ? i : o;
            int v = mat[r * S + s];
            if (v != 0) { (*idx)[n] = i; (*val)[n] = v; n++; }
        }
    }
    (*off)[outer] = n;
    return 0;
}

ctlo_model* ctlo_model_new(int S, int R, const int32_t* left, const int32_t* right,
                           const int32_t* feed, int ns, const double* tvec, int s_out,
                           const int32_t* cs, float eps, uint32_t nc, double ssa_factor,
                           uint32_t ssa_steps, uint32_t flags, uint64_t seed,
                           uint32_t max_steps) {
    if (S <= 0 || R <= 0 || ns <= 0 || s_out <= 0) return NULL;
    for (int i = 0; i < R * S; i++)
        if (left[i] < 0 || left[i] > 127 || right[i] < 0 || right[i] > 127) return NULL;
    for (int k = 0; k < s_out; k++)
        if (cs[k] < 0 || cs[k] >= S) return NULL;
    ctlo_model* m = (ctlo_model*)calloc(1, sizeof(ctlo_model));
    if (!m) return NULL;
    m->S = S; m->R = R; m->ns = ns; m->s_out = s_out;
    int P = 2;
    while (P < R) P <<= 1;
    m->P = P;
    int32_t* V = (int32_t*)malloc(sizeof(int32_t) * (size_t)R * S);
    int32_t* F = (int32_t*)malloc(sizeof(int32_t) * (size_t)R * S);
    for (int r = 0; r < R; r++)
        for (int s = 0; s < S; s++) {
            V[r * S + s] = right[r * S + s] - left[r * S + s];
            F[r * S + s] = (feed && feed[s]) ? 0 : V[r * S + s];
        }
    int rc = 0;
    rc |= build_list(R, S, 1, left, S, &m->reac_off, &m->reac_s, &m->reac_st);
    rc |= build_list(S, R, 0, V, S, &m->vs_off, &m->vs_r, &m->vs_v);
    rc |= build_list(S, R, 0, F, S, &m->fs_off, &m->fs_r, &m->fs_v);
    rc |= build_list(R, S, 1, F, S, &m->fr_off, &m->fr_s, &m->fr_v);
    /* HOR / HORtype exactly as the reference host code (tau.cu:402-432),
     * including its order dependence: hortype is reset whenever a higher
     * order reaction is met, then raised to any larger coefficient. */
    m->hor = (uint8_t*)calloc((size_t)S, 1);
    m->hort = (uint8_t*)calloc((size_t)S, 1);
    uint8_t* order = (uint8_t*)calloc((size_t)R, 1);
    for (int r = 0; r < R; r++) {
        uint8_t tot = 0;
        for (int s = 0; s < S; s++) tot = (uint8_t)(tot + left[r * S + s]);
        order[r] = tot;
    }
    for (int s = 0; s < S; s++)
        for (int r = 0; r < R; r++) {
            int l = left[r * S + s];
            if (l > 0 && order[r] > m->hor[s]) { m->hor[s] = order[r]; m->hort[s] = (uint8_t)l; }
            if (m->hort[s] < l) m->hort[s] = (uint8_t)l;
        }
    free(order); free(V); free(F);
    m->tvec = (double*)malloc(sizeof(double) * (size_t)ns);
    memcpy(m->tvec, tvec, sizeof(double) * (size_t)ns);
    m->cs = (int*)malloc(sizeof(int) * (size_t)s_out);
    for (int k = 0; k < s_out; k++) m->cs[k] = cs[k];
    m->tmax = tvec[ns - 1];
    m->eps = eps; m->nc = nc; m->ssa_factor = ssa_factor; m->ssa_steps = ssa_steps;
    m->flags = flags; m->seed = seed; m->max_steps = max_steps;
    if (rc) { ctlo_model_free(m); return NULL; }
    return m;
}

void ctlo_model_hor(const ctlo_model* m, uint8_t* hor, uint8_t* hort) {
    memcpy(hor, m->hor, (size_t)m->S);
    memcpy(hort, m->hort, (size_t)m->S);
}

/* ------------------------------------------------------------------------ */
/* Canonical tau-leaping simulation                                         */
/* ------------------------------------------------------------------------ */

/* Mass-action propensity in FP32 (reference CalculatePropensity, tau.cu:1443-1470:
 * order 1 multiplies by X, order 2 by 0.5*X*(X-1), higher orders by the
 * product of (X-e+1)/e). */
static float prop(const ctlo_model* m, int r, const int32_t* X, float c) {
    float v = c;
    for (int e = m->reac_off[r]; e < m->reac_off[r + 1]; e++) {
        int32_t x = X[m->reac_s[e]];
        int st = m->reac_st[e];
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

/* Cao's g_i from HOR/HORtype (tau.cu:1741-1789), in FP32. */
static float gfun(uint8_t hor, uint8_t hort, int32_t x) {
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

/* Sum tree: leaves tree[P + r] (reaction r, zero padded), node i = 2i + (2i+1). */
static void build_tree(double* tree, int P) {
    for (int i = P - 1; i >= 1; i--) tree[i] = tree[2 * i] + tree[2 * i + 1];
}
static void update_path(double* tree, int P, int r) {
    for (int i = (P + r) >> 1; i >= 1; i >>= 1) tree[i] = tree[2 * i] + tree[2 * i + 1];
}
/* Leftmost leaf whose cumulative sum reaches x (ties go left), never a
 * zero-weight leaf when the root is positive. */
static int descend(const double* tree, int P, double x) {
    int node = 1;
    while (node < P) {
        int l = 2 * node;
        double L = tree[l], Rv = tree[l + 1];
        if ((x <= L && L > 0.0) || Rv == 0.0) {
            node = l;
        } else {
            x = x - L;
            node = l + 1;
        }
    }
    return node - P;
}

typedef struct {
    int32_t *X, *X1;
    float* a;
    double *tree, *mtree;
    uint32_t* K;
    uint8_t* crit;
} work_t;

static int work_alloc(const ctlo_model* m, work_t* w) {
    w->X = (int32_t*)malloc(sizeof(int32_t) * (size_t)m->S);
    w->X1 = (int32_t*)malloc(sizeof(int32_t) * (size_t)m->S);
    w->a = (float*)calloc((size_t)m->P, sizeof(float));
    w->tree = (double*)calloc((size_t)(2 * m->P), sizeof(double));
    w->mtree = (double*)calloc((size_t)(2 * m->P), sizeof(double));
    w->K = (uint32_t*)calloc((size_t)m->P, sizeof(uint32_t));
    w->crit = (uint8_t*)calloc((size_t)m->P, 1);
    return (w->X && w->X1 && w->a && w->tree && w->mtree && w->K && w->crit) ? 0 : -1;
}
static void work_free(work_t* w) {
    free(w->X); free(w->X1); free(w->a); free(w->tree); free(w->mtree); free(w->K); free(w->crit);
}

static void all_props(const ctlo_model* m, work_t* w, const float* c) {
    for (int r = 0; r < m->R; r++) {
        w->a[r] = prop(m, r, w->X, c[r]);
        w->tree[m->P + r] = (double)w->a[r];
    }
    build_tree(w->tree, m->P);
}

/* A0 == 0 finish (tau.cu:1665-1697 and 2165-2196). */
static void finish_zero(const ctlo_model* m, const work_t* w, uint32_t* out, uint32_t* cursor) {
    int so = m->s_out;
    uint32_t c = *cursor;
    if (!(m->flags & CTLO_Q10_OFF)) {
        if (c == 0) {
            for (int k = 0; k < so; k++) out[k] = (uint32_t)w->X[m->cs[k]];
            c = 1;
        }
        for (uint32_t i = c; i < (uint32_t)m->ns; i++)
            for (int k = 0; k < so; k++) out[i * so + k] = out[(c - 1) * so + k];
    } else {
        for (uint32_t i = c; i < (uint32_t)m->ns; i++)
            for (int k = 0; k < so; k++) out[i * so + k] = (uint32_t)w->X[m->cs[k]];
    }
    *cursor = (uint32_t)m->ns;
}

int ctlo_simulate(const ctlo_model* m, uint32_t sim, const int32_t* X0, const float* c,
                  uint32_t* out, ctlo_info* info) {
    const int S = m->S, R = m->R, P = m->P, ns = m->ns, so = m->s_out;
    const uint32_t fl = m->flags;
    const int force = (fl & CTLO_FORCE_SSA) != 0;
    work_t w;
    if (work_alloc(m, &w)) { work_free(&w); return -1; }
    memset(info, 0, sizeof(*info));
    memset(out, 0, sizeof(uint32_t) * (size_t)ns * so);
    for (int s = 0; s < S; s++) w.X[s] = X0[s];
    all_props(m, &w, c);

    double T = 0.0, tl = 0.0;
    uint32_t cursor = 0, n = 0, burst = 0;
    int in_ssa = force;
    uint32_t status = CTLO_SIM_OK;
    const int* vo = (fl & CTLO_Q5_OFF) ? m->fs_off : m->vs_off;
    const int* vr = (fl & CTLO_Q5_OFF) ? m->fs_r : m->vs_r;
    const int* vv = (fl & CTLO_Q5_OFF) ? m->fs_v : m->vs_v;

    for (;;) {
        if (!in_ssa) {
            /* ---- PreCalculations: decide, then one leap ---- */
            if (T >= m->tmax) break;
            if (n >= m->max_steps) { status = CTLO_SIM_STEP_LIMIT; break; }
            uint32_t step = n++;
            double A0 = w.tree[1];
            if (A0 == 0.0) { finish_zero(m, &w, out, &cursor); T = m->tmax + (double)0.1f; break; }
            int anycrit = 0;
            for (int r = 0; r < R; r++) {
                uint8_t cr = 0;
                for (int e = m->reac_off[r]; e < m->reac_off[r + 1]; e++) {
                    uint32_t q = (uint32_t)w.X[m->reac_s[e]] / (uint32_t)m->reac_st[e];
                    if ((fl & CTLO_Q6_OFF) ? (q < m->nc) : (q > 0 && q < m->nc)) cr = 1;
                }
                w.crit[r] = cr;
                anycrit |= cr;
            }
            float tau1 = FLT_MAX;
            for (int s = 0; s < S; s++) {
                if (vo[s] == vo[s + 1]) continue;
                float mu = 0.0f, sg = 0.0f;
                for (int e = vo[s]; e < vo[s + 1]; e++) {
                    int r = vr[e];
                    if (w.crit[r]) continue;
                    float fv = (float)vv[e];
                    mu = mu + fv * w.a[r];
                    sg = sg + (fv * fv) * w.a[r];
                }
                float g = gfun(m->hor[s], m->hort[s], w.X[s]);
                float tmp2 = (m->eps * (float)w.X[s]) / g;
                float macs = tmp2 > 1.0f ? tmp2 : 1.0f;
                int use = (fl & CTLO_Q9_OFF) ? (sg != 0.0f) : (mu != 0.0f && sg != 0.0f);
                if (use) {
                    float t3 = mu != 0.0f ? macs / fabsf(mu) : INFINITY;
                    float t4 = (macs * macs) / sg;
                    float t = t3 < t4 ? t3 : t4;
                    if (t < tau1) tau1 = t;
                }
            }
            if ((double)tau1 < m->ssa_factor / A0) {
                in_ssa = 1; burst = 0; tl = 0.0;
                continue;
            }
            double a0c = 0.0;
            if (anycrit) {
                for (int i = 0; i < P; i++) w.mtree[P + i] = w.crit[i] ? (double)w.a[i] : 0.0;
                build_tree(w.mtree, P);
                a0c = w.mtree[1];
            }
            uint32_t wd[4];
            draw(m->seed, 0, TAG_MISC, step, sim, wd);
            double tau2 = (double)FLT_MAX;
            if (a0c > 0.0) tau2 = -ctlo_log(u53(wd[0], wd[1])) / a0c;
            double tau = (double)tau1 < tau2 ? (double)tau1 : tau2;
            int pick = -1;
            if ((double)tau1 > tau2) {
                if (!(fl & CTLO_Q2_OFF) && !w.crit[0]) {
                    w.mtree[P] = (double)w.a[0];
                    update_path(w.mtree, P, 0);
                }
                pick = descend(w.mtree, P, u53(wd[2], wd[3]) * a0c);
            }
            uint32_t attempt = 0;
            int overflow = 0;
            for (;;) {
                for (int r = 0; r < R; r++) {
                    if (w.crit[r])
                        w.K[r] = (r == pick && (attempt == 0 || (fl & CTLO_Q3_OFF))) ? 1u : 0u;
                    else
                        w.K[r] = ctlo_poisson(tau * (double)w.a[r], m->seed, sim, step, attempt, (uint32_t)r);
                }
                int fail = 0;
                overflow = 0;
                for (int s = 0; s < S && !fail; s++) {
                    int64_t x1 = w.X[s];
                    for (int e = m->fs_off[s]; e < m->fs_off[s + 1]; e++) {
                        x1 += (int64_t)m->fs_v[e] * (int64_t)w.K[m->fs_r[e]];
                        if (!(fl & CTLO_Q4_OFF) && x1 < 0) { fail = 1; break; }
                    }
                    if (x1 < 0) fail = 1;
                    if (x1 > 2147483647) overflow = 1;
                    w.X1[s] = (int32_t)x1;
                }
                if (!fail) break;
                tau = tau * 0.5;
                attempt++;
                info->rejections++;
                if (attempt >= MAX_ATTEMPTS) { status = CTLO_SIM_ATTEMPT_LIMIT; break; }
            }
            if (status != CTLO_SIM_OK) break;
            if (overflow) { status = CTLO_SIM_OVERFLOW; break; }
            /* check_time_instant (tau.cu:1507-1562): samples with t_i <= T+tau */
            while (cursor < (uint32_t)ns && T + tau >= m->tvec[cursor]) {
                for (int k = 0; k < so; k++) {
                    int s = m->cs[k];
                    double d = (double)((int64_t)w.X1[s] - (int64_t)w.X[s]);
                    double delta = (d * (m->tvec[cursor] - T)) / tau;
                    double ri = rint(delta);
                    uint32_t v;
                    if (!(fl & CTLO_Q1_OFF))
                        v = (uint32_t)w.X[s] + (ri > 0.0 ? (uint32_t)ri : 0u);
                    else
                        v = (uint32_t)((int64_t)w.X[s] + (int64_t)ri);
                    out[cursor * so + k] = v;
                }
                cursor++;
            }
            uint64_t fsum = 0;
            for (int r = 0; r < R; r++) fsum += w.K[r];
            info->firings += fsum;
            info->leaps++;
            for (int s = 0; s < S; s++) w.X[s] = w.X1[s];
            T = T + tau;
            all_props(m, &w, c);
            if (cursor == (uint32_t)ns) break;
        } else {
            /* ---- EventualSSASteps / LightweightSSA: one SSA step ---- */
            if (n >= m->max_steps) { status = CTLO_SIM_STEP_LIMIT; break; }
            double A0 = w.tree[1];
            if (A0 == 0.0) { finish_zero(m, &w, out, &cursor); T = m->tmax + (double)0.1f; break; }
            uint32_t step = n++;
            /* one Philox block per two SSA steps: (w0,w1) for even steps,
             * (w2,w3) for odd ones; 32-bit pick uniform, FP32 waiting time */
            uint32_t wd[4];
            draw(m->seed, 0, TAG_SSA, step >> 1, sim, wd);
            uint32_t wa = (step & 1) ? wd[2] : wd[0], wb = (step & 1) ? wd[3] : wd[1];
            int r = descend(w.tree, P, u32d(wa) * A0);
            float dtf = -ctlo_logf(u24f(wb)) / (float)A0;
            tl = tl + (double)dtf;
            while (cursor < (uint32_t)ns && T + tl > m->tvec[cursor]) {
                for (int k = 0; k < so; k++) out[cursor * so + k] = (uint32_t)w.X[m->cs[k]];
                cursor++;
            }
            int overflow = 0;
            for (int e = m->fr_off[r]; e < m->fr_off[r + 1]; e++) {
                int64_t nx = (int64_t)w.X[m->fr_s[e]] + m->fr_v[e];
                if (nx > 2147483647 || nx < 0) overflow = 1;
                w.X[m->fr_s[e]] = (int32_t)nx;
            }
            info->ssa_steps++;
            info->firings++;
            if (overflow) { status = CTLO_SIM_OVERFLOW; break; }
            all_props(m, &w, c);
            burst++;
            if (cursor == (uint32_t)ns) break;
            if (burst == m->ssa_steps) {
                T = T + tl; tl = 0.0; burst = 0;
                if (!force) in_ssa = 0;
                else if (T >= m->tmax) break;
            }
        }
    }
    info->t_final = T + tl;
    info->status = status;
    info->steps = n;
    work_free(&w);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Exact FP64 Gillespie direct method (independent oracle)                  */
/* ------------------------------------------------------------------------ */

int ctlo_gillespie(const ctlo_model* m, uint32_t sim, const int32_t* X0, const float* c,
                   uint32_t* out, ctlo_info* info) {
    const int S = m->S, R = m->R, ns = m->ns, so = m->s_out;
    int64_t* X = (int64_t*)malloc(sizeof(int64_t) * (size_t)S);
    double* a = (double*)malloc(sizeof(double) * (size_t)R);
    if (!X || !a) { free(X); free(a); return -1; }
    memset(info, 0, sizeof(*info));
    for (int s = 0; s < S; s++) X[s] = X0[s];
    uint64_t key = m->seed ^ 0x9E3779B97F4A7C15ULL;
    double T = 0.0;
    uint32_t cursor = 0, n = 0;
    while (cursor < (uint32_t)ns) {
        double a0 = 0.0;
        for (int r = 0; r < R; r++) {
            double v = (double)c[r];
            for (int e = m->reac_off[r]; e < m->reac_off[r + 1]; e++) {
                double x = (double)X[m->reac_s[e]];
                int st = m->reac_st[e];
                for (int j = 1; j <= st; j++) v *= (x - j + 1 > 0 ? (x - j + 1) : 0.0) / j;
            }
            a[r] = v;
            a0 += v;
        }
        if (a0 <= 0.0) {
            for (; cursor < (uint32_t)ns; cursor++)
                for (int k = 0; k < so; k++) out[cursor * so + k] = (uint32_t)X[m->cs[k]];
            break;
        }
        if (n >= m->max_steps) { info->status = CTLO_SIM_STEP_LIMIT; break; }
        uint32_t wd[4];
        draw(key, 0, TAG_GILL, n++, sim, wd);
        double tn = T - log(u53(wd[2], wd[3])) / a0;
        while (cursor < (uint32_t)ns && tn > m->tvec[cursor]) {
            for (int k = 0; k < so; k++) out[cursor * so + k] = (uint32_t)X[m->cs[k]];
            cursor++;
        }
        if (cursor == (uint32_t)ns) break;
        double x = u53(wd[0], wd[1]) * a0, acc = 0.0;
        int r = 0, last = -1;
        for (r = 0; r < R; r++) {
            if (a[r] > 0.0) last = r;
            acc += a[r];
            if (x <= acc && a[r] > 0.0) break;
        }
        if (r == R) r = last;
        for (int e = m->fr_off[r]; e < m->fr_off[r + 1]; e++) X[m->fr_s[e]] += m->fr_v[e];
        info->ssa_steps++;
        info->firings++;
        T = tn;
    }
    info->t_final = T;
    info->steps = n;
    free(X); free(a);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Threaded batch driver (the timed CPU baseline)                           */
/* ------------------------------------------------------------------------ */

typedef struct {
    const ctlo_model* m;
    int n, mode, err;
    uint32_t sim_base;
    const int32_t* X0;
    const float* c;
    uint32_t* out;
    ctlo_info* info;
    long next;
} job_t;

static void* worker(void* arg) {
    job_t* j = (job_t*)arg;
    const ctlo_model* m = j->m;
    for (;;) {
        long i = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (i >= j->n) break;
        const int32_t* x0 = j->X0 + (size_t)i * m->S;
        const float* c = j->c + (size_t)i * m->R;
        uint32_t* out = j->out + (size_t)i * m->ns * m->s_out;
        int rc = j->mode == 1 ? ctlo_gillespie(m, j->sim_base + (uint32_t)i, x0, c, out, j->info + i)
                              : ctlo_simulate(m, j->sim_base + (uint32_t)i, x0, c, out, j->info + i);
        if (rc) __atomic_store_n(&j->err, rc, __ATOMIC_RELAXED);
    }
    return NULL;
}

int ctlo_run_batch(const ctlo_model* m, int n, uint32_t sim_base, const int32_t* X0,
                   const float* c, uint32_t* out, ctlo_info* info, int nthreads, int mode) {
    job_t j = {m, n, mode, 0, sim_base, X0, c, out, info, 0};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > n) nthreads = n > 0 ? n : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, worker, &j);
    worker(&j);
    for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
    return j.err;
}

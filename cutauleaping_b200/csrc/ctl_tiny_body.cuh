// The register-resident sweep for tiny networks, written once for two
// kinds of model parameters N: the library's kernels read a Net parameter
// block at run time (ctl_tiny.cu), and kernels compiled at run time for one
// model by NVRTC read compile-time constants, so that every table lookup,
// coefficient branch and zero entry folds away.  Self-contained (NVRTC
// compiles it with ctl_devmath.cuh and nothing else).
//
// One thread owns one simulation and keeps everything in registers:
// populations, the proposed leap state, rate constants, propensities, the
// complete FP64 sum tree over the reactions, the Poisson counts and the last
// recorded sample.  Same arithmetic contract as the shared-memory sweep and
// the CPU oracle (oracle/ctl_oracle.c), bit for bit: Philox4x32-10 counters
// (seed, block, tag, step, sim), FP32 propensities in the reference's factor
// order, FP64 sums as the root of the binary tree over P = 2^k leaves and the
// searches as its descent, per-species sums in ascending reaction order.  It
// follows PreCalculations (2phase_n-tau-leaping.cu:1568-2093),
// EventualSSASteps (2099-2273) and LightweightSSA (2280-2454) with the
// reference's quirks switchable as in the other kernels.
//
// N provides, as const member functions: S(), R(), ns(), s_out(), tmax(),
// tvec(); ne(r) reactant entries of reaction r, es(r, e) / ec(r, e) their
// species (ascending) and coefficients; V(q, r) the tau1 table (V, or F
// when quirk Q5 is off) and vnz(q) whether species q has an entry; Fm(q, r)
// the feed-masked net change; hor(q), hort(q); cs(k) the sampled species;
// frow(r, w) word w of reaction r's F row (four signed bytes per word).
#pragma once

#include "ctl_devmath.cuh"

namespace ctl {
namespace tiny {

constexpr int MAX_E = 3;  // reactant entries per reaction
constexpr int CONT = 0, DONE = 1;

// x[s] for a warp-uniform species index s: a select chain, so that the array
// stays in registers.
template <int SM>
__device__ __forceinline__ int32_t pick(const int32_t (&x)[SM], uint32_t s) {
    int32_t v = x[0];
#pragma unroll
    for (int i = 1; i < SM; i++) v = (s == (uint32_t)i) ? x[i] : v;
    return v;
}

// Mass-action propensity of reaction r in FP32 (CalculatePropensity,
// tau.cu:1443-1470): c times, per reactant entry in species order, X
// (coefficient 1), 0.5 X (X-1) (2) or the running product of (X-j+1)/j
// (higher); zero when a reactant count is below its coefficient.  The
// factors multiply into the running value in the same order as the
// shared-memory sweep's prop().
template <class N, int SM>
__device__ __forceinline__ float propensity(const N& net, int r, float c, const int32_t (&x)[SM]) {
    float v = c;
    bool zero = false;
#pragma unroll
    for (int e = 0; e < MAX_E; e++) {
        if (e < (int)net.ne(r)) {
            const int32_t xs = pick<SM>(x, net.es(r, e));
            const int st = (int)net.ec(r, e);
            if (xs < st) zero = true;
            if (st == 1) {
                v = v * (float)xs;
            } else if (st == 2) {
                const float hx = (float)xs;
                v = v * ((0.5f * hx) * (hx - 1.0f));
            } else {
                // (x-j+1)/j: division by 1 and 2 is exact scaling, the rest divides
                v = v * (float)xs;
                v = v * ((float)(xs - 1) * 0.5f);
                for (int j = 3; j <= st; j++) v = v * ((float)(xs - j + 1) / (float)j);
            }
        }
    }
    return zero ? 0.0f : v;
}

// Complete binary sum tree over P leaves in registers: t[0..P-1] leaves,
// then each level's pairwise sums, t[2P-2] the root.
template <int P>
__device__ __forceinline__ void build(double (&t)[2 * P - 1]) {
    int in = 0, out = P;
#pragma unroll
    for (int w = P; w > 1; w >>= 1) {
#pragma unroll
        for (int i = 0; i < w / 2; i++) t[out + i] = t[in + 2 * i] + t[in + 2 * i + 1];
        in = out;
        out += w / 2;
    }
}

// Leftmost leaf whose cumulative weight reaches x (ties go left, never a
// zero leaf): one go_right per level from the root, as dev::descend.
template <int P>
__device__ __forceinline__ int descend(const double (&t)[2 * P - 1], double x) {
    int idx = 0;  // node index within the current level
#pragma unroll
    for (int w = 2; w <= P; w <<= 1) {
        const int base = 2 * P - 2 * w;  // the level of w nodes: t[2P-2w .. 2P-w-1]
        double L = t[base], R = t[base + 1];
#pragma unroll
        for (int j = 1; j < w / 2; j++) {
            const bool h = idx == j;
            L = h ? t[base + 2 * j] : L;
            R = h ? t[base + 2 * j + 1] : R;
        }
        idx = 2 * idx + (dev::go_right(x, L, R) ? 1 : 0);
    }
    return idx;
}

// The Poisson sampler out of line: the leap draws from up to 16 call sites,
// and one copy of its code keeps the kernel small enough for the
// instruction cache when many warps run different phases.
__device__ __noinline__ uint32_t poisson_draw(double lam, uint32_t wa, uint32_t wb, uint64_t seed, uint32_t tag,
                                              uint32_t step, uint32_t sim, uint32_t odd) {
    return dev::poisson(lam, wa, wb, seed, tag, step, sim, odd);
}

struct Sim {
    double T, tl, t_next;
    unsigned long long fire;
    uint32_t sim, cursor, n, burst, leaps, ssa, rej, status;
    bool in_ssa;
    // The random part of SSA step `pre`, computed during the step before (it
    // depends on the counters only, not on the state): the pick uniform and
    // the log of the waiting-time uniform.
    uint32_t pre;
    double pre_u;
    float pre_lg;
    uint4 wc;         // Philox block of SSA steps 2 wc_blk, 2 wc_blk + 1 (not carried across rounds)
    uint32_t wc_blk;
};

// Pick uniform and waiting-time log of SSA step `step`: one Philox block per
// two steps, (w0, w1) for even steps and (w2, w3) for odd ones, as
// dev::ssa_step; the block is kept for the pair's second step.
__device__ __forceinline__ void ssa_randoms(const dev::Run& run, uint32_t simg, uint32_t step, Sim& st, double& u,
                                            float& lg) {
    if (st.wc_blk != (step >> 1)) {
        st.wc = dev::draw(run.seed, 0u, dev::TAG_SSA, step >> 1, simg);
        st.wc_blk = step >> 1;
    }
    const uint32_t wa = (step & 1u) ? st.wc.z : st.wc.x, wb = (step & 1u) ? st.wc.w : st.wc.y;
    u = dev::u32d(wa);
    lg = dev::flog(dev::u24f(wb));
}

// One simulation's registers.
template <int P, int SM>
struct State {
    int32_t x[SM];
    float c[P];
    float a[P];
    double t[2 * P - 1];
    uint32_t last[SM];  // fitness mode: last recorded sample
};

template <class N, int P, int SM>
__device__ __forceinline__ void all_props(const N& net, State<P, SM>& s) {
#pragma unroll
    for (int r = 0; r < P; r++) {
        s.a[r] = r < net.R() ? propensity<N, SM>(net, r, s.c[r], s.x) : 0.0f;
        s.t[r] = (double)s.a[r];
    }
    build<P>(s.t);
}

// Where the samples go (dev::Out): the simulation's own rows, or the 64-bit
// sums of its parameter set with the last row kept in registers.
struct Out {
    uint32_t* samples;
    unsigned long long* sums;
};

template <int P, int SM>
__device__ __forceinline__ void put(const Out& o, State<P, SM>& s, uint32_t i, int so, int k, uint32_t v) {
    if (o.samples) {
        o.samples[(size_t)i * so + k] = v;
    } else {
        atomicAdd(o.sums + (size_t)i * so + k, (unsigned long long)v);
#pragma unroll
        for (int q = 0; q < SM; q++)
            if (q == k) s.last[q] = v;
    }
}

template <int P, int SM>
__device__ __forceinline__ uint32_t last_of(const Out& o, const State<P, SM>& s, uint32_t i, int so, int k) {
    if (o.samples) return o.samples[(size_t)i * so + k];
    uint32_t v = s.last[0];
#pragma unroll
    for (int q = 1; q < SM; q++) v = q == k ? s.last[q] : v;
    return v;
}

// A0 == 0 (tau.cu:1665-1697, 2165-2196): the last recorded sample is copied
// forward (the current state is written first if nothing was recorded).
template <class N, int P, int SM>
__device__ void finish_zero(const N& net, const dev::Run& run, State<P, SM>& s, const Out& o,
                            uint32_t& cursor) {
    const int so = net.s_out();
    const uint32_t ns = (uint32_t)net.ns();
    if (!(run.flags & dev::F_Q10_OFF)) {
        if (cursor == 0) {
            for (int k = 0; k < so; k++) put<P, SM>(o, s, 0u, so, k, (uint32_t)pick<SM>(s.x, net.cs(k)));
            cursor = 1;
        }
        for (uint32_t i = cursor; i < ns; i++)
            for (int k = 0; k < so; k++) put<P, SM>(o, s, i, so, k, last_of<P, SM>(o, s, cursor - 1, so, k));
    } else {
        for (uint32_t i = cursor; i < ns; i++)
            for (int k = 0; k < so; k++) put<P, SM>(o, s, i, so, k, (uint32_t)pick<SM>(s.x, net.cs(k)));
    }
    cursor = ns;
}

// PreCalculations (tau.cu:1568-2093) for one simulation in registers: the
// SSA hand-off decision and, unless it hands off, one Cao tau-leap with
// critical reactions and negative-population rejection.
template <class N, int P, int SM>
__device__ int decide_step(const N& net, const dev::Run& run, State<P, SM>& s, Sim& st, const Out& o) {
    const uint32_t fl = run.flags;
    const uint32_t ns = (uint32_t)net.ns();
    const int so = net.s_out();
    const uint32_t simg = run.sim_base + st.sim;
    if (st.T >= net.tmax()) return DONE;
    if (st.n >= run.max_steps) { st.status = CTL_SIM_STEP_LIMIT; return DONE; }
    const uint32_t step = st.n++;
    const double A0 = s.t[2 * P - 2];
    if (A0 == 0.0) {
        finish_zero<N, P, SM>(net, run, s, o, st.cursor);
        st.T = net.tmax() + (double)0.1f;
        return DONE;
    }
    // critical reactions (tau.cu:1727-1733): some reactant with
    // 0 < floor(x / L) < n_c, tested as x >= L and x < n_c L
    const bool q6off = (fl & dev::F_Q6_OFF) != 0;
    uint32_t crit = 0;
#pragma unroll
    for (int r = 0; r < P; r++) {
        bool cr = false;
#pragma unroll
        for (int e = 0; e < MAX_E; e++) {
            if (r < net.R() && e < (int)net.ne(r)) {
                const uint32_t xs = (uint32_t)pick<SM>(s.x, net.es(r, e)), L = net.ec(r, e);
                const bool below = (uint64_t)xs < (uint64_t)run.nc * L;
                cr = cr || (q6off ? below : (xs >= L && below));
            }
        }
        crit |= cr ? (1u << r) : 0u;
    }
    // tau1 (tau.cu:1741-1922): mu, sigma^2 per species over the non-critical
    // reactions in ascending order, Cao's bound with g_i
    float tau1 = FLT_MAX;
#pragma unroll
    for (int q = 0; q < SM; q++) {
        if (q < net.S() && net.vnz(q)) {
            float mu = 0.0f, sg = 0.0f;
#pragma unroll
            for (int r = 0; r < P; r++) {
                const int v = r < net.R() ? (int)net.V(q, r) : 0;
                if (v != 0) {
                    const float a = (crit >> r) & 1u ? 0.0f : s.a[r];
                    const float fv = (float)v;
                    mu = mu + fv * a;
                    sg = sg + (fv * fv) * a;
                }
            }
            const int32_t xs = s.x[q];
            const float gg = dev::gfun(net.hor(q), net.hort(q), xs);
            const float tmp2 = (run.eps * (float)xs) / gg;
            const float macs = tmp2 > 1.0f ? tmp2 : 1.0f;
            const bool use = (fl & dev::F_Q9_OFF) ? (sg != 0.0f) : (mu != 0.0f && sg != 0.0f);
            if (use) {
                const float t3 = mu != 0.0f ? macs / fabsf(mu) : __int_as_float(0x7f800000);
                const float t4 = (macs * macs) / sg;
                const float tt = t3 < t4 ? t3 : t4;
                if (tt < tau1) tau1 = tt;
            }
        }
    }
    if ((double)tau1 < run.ssa_factor / A0) {
        st.in_ssa = true;
        st.burst = 0;
        st.tl = 0.0;
        return CONT;
    }
    double tc[2 * P - 1];  // critical tree
    double a0c = 0.0;
    if (crit) {
#pragma unroll
        for (int r = 0; r < P; r++) tc[r] = (crit >> r) & 1u ? (double)s.a[r] : 0.0;
        build<P>(tc);
        a0c = tc[2 * P - 2];
    }
    double tau2 = (double)FLT_MAX;
    int pick_r = -1;
    if (a0c > 0.0) {  // the draw serves tau2 and the critical pick only
        const uint4 wd = dev::draw(run.seed, 0u, dev::TAG_MISC, step, simg);
        tau2 = -dev::dlog(dev::u53(wd.x, wd.y)) / a0c;
        if ((double)tau1 > tau2) {
            // the reference's linear search starts from PROP[0] unmasked (Q2):
            // leaf 0 joins the tree when it is not critical itself
            if (!(fl & dev::F_Q2_OFF) && !(crit & 1u)) {
                tc[0] = (double)s.a[0];
                build<P>(tc);
            }
            pick_r = descend<P>(tc, dev::u53(wd.z, wd.w) * a0c);
        }
    }
    double tau = (double)tau1 < tau2 ? (double)tau1 : tau2;
    uint32_t attempt = 0;
    uint32_t K[P];
    int32_t x1[SM];
    bool ovf = false;
    for (;;) {
        const bool keep = attempt == 0 || (fl & dev::F_Q3_OFF);
#pragma unroll
        for (int pb = 0; 2 * pb < P; pb++) {
            const int r0 = 2 * pb, r1 = r0 + 1;
            const bool c0 = r0 >= net.R() || ((crit >> r0) & 1u);
            const bool c1 = r1 >= net.R() || ((crit >> r1) & 1u);
            const double l0 = c0 ? 0.0 : tau * (double)s.a[r0];
            const double l1 = c1 ? 0.0 : tau * (double)s.a[r1];
            const uint32_t tg = dev::tag_pois(attempt, (uint32_t)pb);
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (l0 > 0.0 || l1 > 0.0) w = dev::draw(run.seed, 0u, tg, step, simg);
            K[r0] = c0 ? ((r0 == pick_r && keep) ? 1u : 0u) : poisson_draw(l0, w.x, w.y, run.seed, tg, step, simg, 0u);
            K[r1] = c1 ? ((r1 == pick_r && keep) ? 1u : 0u) : poisson_draw(l1, w.z, w.w, run.seed, tg, step, simg, 1u);
        }
        // test_update (tau.cu:1300-1351): entries of F species-major in
        // ascending reaction order, rejected at the first negative (Q4)
        bool fail = false, lovf = false;
#pragma unroll
        for (int q = 0; q < SM; q++) {
            int64_t v = s.x[q];
            bool neg = false;
#pragma unroll
            for (int r = 0; r < P; r++) {
                const int f = (q < net.S() && r < net.R()) ? (int)net.Fm(q, r) : 0;
                if (f != 0 && !neg) {
                    v += (int64_t)f * (int64_t)K[r];
                    if (!(fl & dev::F_Q4_OFF) && v < 0) neg = true;
                }
            }
            if (neg || v < 0) fail = true;
            if (v > 2147483647LL) lovf = true;
            x1[q] = (int32_t)v;
        }
        if (!fail) {
            ovf = lovf;
            break;
        }
        tau = tau * 0.5;
        attempt++;
        st.rej++;
        if (attempt >= dev::MAX_ATTEMPTS) { st.status = CTL_SIM_ATTEMPT_LIMIT; return DONE; }
    }
    if (ovf) { st.status = CTL_SIM_OVERFLOW; return DONE; }
    // check_time_instant (tau.cu:1507-1562)
    const double T = st.T;
    while (st.cursor < ns && T + tau >= st.t_next) {
        for (int k = 0; k < so; k++) {
            const uint32_t sp = net.cs(k);
            const int32_t xs = pick<SM>(s.x, sp);
            const double d = (double)((int64_t)pick<SM>(x1, sp) - (int64_t)xs);
            const double delta = (d * (st.t_next - T)) / tau;
            const double ri = rint(delta);
            uint32_t v;
            if (!(fl & dev::F_Q1_OFF)) v = (uint32_t)xs + (ri > 0.0 ? (uint32_t)ri : 0u);
            else v = (uint32_t)((int64_t)xs + (int64_t)ri);
            put<P, SM>(o, s, st.cursor, so, k, v);
        }
        st.cursor++;
        st.t_next = st.cursor < ns ? net.tvec()[st.cursor] : 0.0;
    }
    unsigned long long fs = 0;
#pragma unroll
    for (int r = 0; r < P; r++) fs += K[r];
    st.fire += fs;
    st.leaps++;
#pragma unroll
    for (int q = 0; q < SM; q++) s.x[q] = x1[q];
    st.T = T + tau;
    all_props<N, P, SM>(net, s);
    return st.cursor == ns ? DONE : CONT;
}

// EventualSSASteps / LightweightSSA (tau.cu:2099-2454): one direct-method
// step.
template <class N, int P, int SM>
__device__ __forceinline__ int ssa_step(const N& net, const dev::Run& run, State<P, SM>& s, Sim& st,
                                        const Out& o) {
    const uint32_t ns = (uint32_t)net.ns();
    const int so = net.s_out();
    if (st.n >= run.max_steps) { st.status = CTL_SIM_STEP_LIMIT; return DONE; }
    const double A0 = s.t[2 * P - 2];
    if (A0 == 0.0) {
        finish_zero<N, P, SM>(net, run, s, o, st.cursor);
        st.T = net.tmax() + (double)0.1f;
        return DONE;
    }
    const uint32_t step = st.n++;
    const uint32_t simg = run.sim_base + st.sim;
    double u;
    float lg;
    if (st.pre == step) {
        u = st.pre_u;
        lg = st.pre_lg;
    } else {
        ssa_randoms(run, simg, step, st, u, lg);
    }
    const int r = descend<P>(s.t, u * A0);
    // the next step's random part, free of the state (a leap decision in
    // between leaves it unused)
    ssa_randoms(run, simg, step + 1u, st, st.pre_u, st.pre_lg);
    st.pre = step + 1u;
    const float dtf = -lg / (float)A0;
    st.tl = st.tl + (double)dtf;
    while (st.cursor < ns && st.T + st.tl > st.t_next) {
        for (int k = 0; k < so; k++) put<P, SM>(o, s, st.cursor, so, k, (uint32_t)pick<SM>(s.x, net.cs(k)));
        st.cursor++;
        st.t_next = st.cursor < ns ? net.tvec()[st.cursor] : 0.0;
    }
    // row r of F: selects over the warp-uniform rows (no memory access)
    uint32_t f0 = net.frow(0, 0), f1 = net.frow(0, 1);
#pragma unroll
    for (int rr = 1; rr < P; rr++) {
        f0 = r == rr ? net.frow(rr, 0) : f0;
        if (SM > 4) f1 = r == rr ? net.frow(rr, 1) : f1;
    }
    bool ovf = false;
#pragma unroll
    for (int q = 0; q < SM; q++) {
        const uint32_t word = q < 4 ? f0 : f1;
        const int f = (int)(int8_t)(uint8_t)(word >> (8 * (q & 3)));
        const int64_t nx = (int64_t)s.x[q] + (int64_t)f;
        if (f != 0 && (nx > 2147483647LL || nx < 0)) ovf = true;
        s.x[q] = (int32_t)nx;
    }
    st.ssa++;
    st.fire += 1ull;
    // straight-line from the update to the new sum tree (after an overflow
    // the propensities are computed and discarded)
    all_props<N, P, SM>(net, s);
    if (ovf) { st.status = CTL_SIM_OVERFLOW; return DONE; }
    st.burst++;
    if (st.cursor == ns) return DONE;
    if (st.burst == run.ssa_steps) {
        st.T = st.T + st.tl;
        st.tl = 0.0;
        st.burst = 0;
        if (!(run.flags & dev::F_FORCE_SSA)) st.in_ssa = false;
        else if (st.T >= net.tmax()) return DONE;
    }
    return CONT;
}

// One thread per simulation, `lanes` simulations per warp (lanes 0..lanes-1
// of every warp work, the rest exit), simulations pulled from the device
// work queue.  The working lanes of a warp take their SSA steps and their
// leap decisions in lockstep phases (up to ssa_budget SSA steps, then up to
// dec_budget decisions) so that their instruction streams stay merged.
// Where simulation `sim` records its samples.
__device__ __forceinline__ Out out_for(const dev::Run& run, uint32_t sim, size_t row_words) {
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

// The simulation's rate constants from its row of c (row 0 when every row is
// the same), then its propensities and sum tree.
template <class N, int P, int SM>
__device__ __forceinline__ void load_rates(const N& net, const dev::Run& run, State<P, SM>& s, uint32_t sim) {
#pragma unroll
    for (int r = 0; r < P; r++)
        s.c[r] = r < net.R() ? run.c[(run.uniform_c ? (size_t)0 : (size_t)sim * net.R()) + r] : 0.0f;
    all_props<N, P, SM>(net, s);
}

// PrepareVariables (tau.cu:1269-1297).
template <class N, int P, int SM>
__device__ __forceinline__ void start_sim(const N& net, const dev::Run& run, State<P, SM>& s, Sim& st,
                                          uint32_t sim) {
#pragma unroll
    for (int q = 0; q < SM; q++) {
        s.x[q] = q < net.S() ? run.X0[(size_t)sim * net.S() + q] : 0;
        s.last[q] = 0u;
    }
    load_rates<N, P, SM>(net, run, s, sim);
    st.T = 0.0;
    st.tl = 0.0;
    st.t_next = net.tvec()[0];
    st.fire = 0ull;
    st.sim = sim;
    st.cursor = st.n = st.burst = st.leaps = st.ssa = st.rej = 0u;
    st.status = CTL_SIM_OK;
    st.in_ssa = (run.flags & dev::F_FORCE_SSA) != 0;
    st.pre = 0xffffffffu;
    st.wc_blk = 0xffffffffu;
}

template <class N>
__device__ __forceinline__ size_t row_words_of(const N& net) {
    return (size_t)net.ns() * (size_t)net.s_out();
}

// The record of a finished simulation; rows never reached read 0.
template <class N>
__device__ __forceinline__ void finish(const N& net, const dev::Run& run, const Sim& st, const Out& o) {
    const uint32_t ns = (uint32_t)net.ns();
    if (o.samples)
        for (uint32_t i = st.cursor; i < ns; i++)
            for (int k = 0; k < net.s_out(); k++) o.samples[(size_t)i * net.s_out() + k] = 0u;
    ctl_sim_info inf;
    inf.t_final = st.T + st.tl;
    inf.firings = st.fire;
    inf.status = st.status;
    inf.steps = st.n;
    inf.leaps = st.leaps;
    inf.ssa_steps = st.ssa;
    inf.rejections = st.rej;
    inf.pad = 0;
    run.info[st.sim] = inf;
    if (run.out_host && o.samples) {  // the row to the caller's pinned buffer
        const size_t words = row_words_of(net);
        const uint32_t* src = o.samples;
        uint32_t* dst = run.out_host + (size_t)st.sim * words;
        if ((words & 3u) == 0u && (((unsigned long long)src | (unsigned long long)dst) & 15ull) == 0ull) {
            for (size_t i = 0; i < words / 4; i++)
                reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
        } else {
            for (size_t i = 0; i < words; i++) dst[i] = src[i];
        }
    }
    if (run.done) {  // publish: this simulation's rows and record are complete
        __threadfence();
        atomicAdd(run.done + (st.sim >> run.done_shift), 1u);
    }
}

// Warp lockstep over the lanes of `mask`: each lane steps its simulation (if
// `live`) and, when it ends, takes the next one from the device work queue,
// until no lane has one.  The lanes take their SSA steps and their leap
// decisions in lockstep phases (up to ssa_budget SSA steps, then up to
// dec_budget decisions) so that their instruction streams stay merged; a
// lane in one phase waits while the others run the other.
template <class N, int P, int SM>
__device__ __forceinline__ void lockstep(const N& net, const dev::Run& run, uint32_t mask, State<P, SM>& s, Sim& st,
                                         Out& o, bool live) {
    const size_t row_words = (size_t)net.ns() * (size_t)net.s_out();
    bool closed = false;
    for (;;) {
        if (!live && !closed) {
            const uint32_t sim = atomicAdd(run.queue, 1u);
            if (sim >= run.n) {
                closed = true;
            } else {
                start_sim<N, P, SM>(net, run, s, st, sim);
                o = out_for(run, sim, row_words);
                live = true;
            }
        }
        if (__all_sync(mask, closed)) break;
        int res = CONT;
        for (uint32_t b = 0; b < run.ssa_budget; b++) {
            const bool act = live && res == CONT && st.in_ssa;
            if (!__any_sync(mask, act)) break;
            if (act) res = ssa_step<N, P, SM>(net, run, s, st, o);
        }
        for (uint32_t b = 0; b < run.dec_budget; b++) {
            const bool act = live && res == CONT && !st.in_ssa;
            if (!__any_sync(mask, act)) break;
            if (act) res = decide_step<N, P, SM>(net, run, s, st, o);
        }
        if (live && res == DONE) {
            finish<N>(net, run, st, o);
            live = false;
        }
    }
}

// Warp lockstep sweep: one thread per simulation, `lanes` simulations per
// warp (lanes 0..lanes-1 of every warp work, the rest exit), simulations
// pulled from the device work queue.
template <class N, int P, int SM>
__device__ __forceinline__ void sweep(const N& net, const dev::Run& run, uint32_t lanes) {
    const uint32_t lane = threadIdx.x & 31u;
    if (lane >= lanes) return;
    const uint32_t mask = lanes >= 32 ? 0xffffffffu : ((1u << lanes) - 1u);
    State<P, SM> s;
    Sim st;
    Out o{nullptr, nullptr};
    lockstep<N, P, SM>(net, run, mask, s, st, o, false);
}

// Words of one simulation's resumable state in the regrouping exchange:
// populations, the time and counters, the next sample instant, the prepared
// random part of the next SSA step, (fitness mode) the last recorded sample
// and the rate constants.  Propensities and the sum tree are rebuilt from
// them.
template <int P, int SM>
struct Packed {
    static constexpr int X = 0, T = SM, TL = SM + 2, FIRE = SM + 4, SIM = SM + 6, CURSOR = SM + 7, NSTEP = SM + 8,
                         BURST = SM + 9, LEAPS = SM + 10, SSA = SM + 11, REJ = SM + 12, FLAGS = SM + 13,
                         PRE = SM + 14, PREU = SM + 15, PRELG = SM + 17, TNEXT = SM + 18, LAST = SM + 20,
                         C = 2 * SM + 20, WORDS = 2 * SM + 20 + P;
};

// Word w of slot j: structure of arrays, consecutive slots in consecutive banks.
template <int P, int SM>
__device__ __forceinline__ void put_state(uint32_t* xs, uint32_t ns, uint32_t j, const State<P, SM>& s,
                                          const Sim& st) {
    using K = Packed<P, SM>;
    auto w = [&](int i, uint32_t v) { xs[(uint32_t)i * ns + j] = v; };
    auto w64 = [&](int i, unsigned long long v) {
        w(i, (uint32_t)v);
        w(i + 1, (uint32_t)(v >> 32));
    };
#pragma unroll
    for (int q = 0; q < SM; q++) {
        w(K::X + q, (uint32_t)s.x[q]);
        w(K::LAST + q, s.last[q]);
    }
    w64(K::T, (unsigned long long)__double_as_longlong(st.T));
    w64(K::TL, (unsigned long long)__double_as_longlong(st.tl));
    w64(K::FIRE, st.fire);
    w(K::SIM, st.sim);
    w(K::CURSOR, st.cursor);
    w(K::NSTEP, st.n);
    w(K::BURST, st.burst);
    w(K::LEAPS, st.leaps);
    w(K::SSA, st.ssa);
    w(K::REJ, st.rej);
    w(K::FLAGS, (st.status << 1) | (st.in_ssa ? 1u : 0u));
    w(K::PRE, st.pre);
    w64(K::PREU, (unsigned long long)__double_as_longlong(st.pre_u));
    w(K::PRELG, __float_as_uint(st.pre_lg));
    w64(K::TNEXT, (unsigned long long)__double_as_longlong(st.t_next));
#pragma unroll
    for (int r = 0; r < P; r++) w(K::C + r, __float_as_uint(s.c[r]));
}

template <class N, int P, int SM>
__device__ __forceinline__ void get_state(const N& net, const uint32_t* xs, uint32_t ns, uint32_t j, State<P, SM>& s,
                                          Sim& st) {
    using K = Packed<P, SM>;
    auto r = [&](int i) { return xs[(uint32_t)i * ns + j]; };
    auto r64 = [&](int i) { return (unsigned long long)r(i) | ((unsigned long long)r(i + 1) << 32); };
#pragma unroll
    for (int q = 0; q < SM; q++) {
        s.x[q] = (int32_t)r(K::X + q);
        s.last[q] = r(K::LAST + q);
    }
    st.T = __longlong_as_double((long long)r64(K::T));
    st.tl = __longlong_as_double((long long)r64(K::TL));
    st.fire = r64(K::FIRE);
    st.sim = r(K::SIM);
    st.cursor = r(K::CURSOR);
    st.n = r(K::NSTEP);
    st.burst = r(K::BURST);
    st.leaps = r(K::LEAPS);
    st.ssa = r(K::SSA);
    st.rej = r(K::REJ);
    const uint32_t f = r(K::FLAGS);
    st.status = f >> 1;
    st.in_ssa = (f & 1u) != 0;
    st.pre = r(K::PRE);
    st.pre_u = __longlong_as_double((long long)r64(K::PREU));
    st.pre_lg = __uint_as_float(r(K::PRELG));
    st.t_next = __longlong_as_double((long long)r64(K::TNEXT));
    st.wc_blk = 0xffffffffu;
#pragma unroll
    for (int q = 0; q < P; q++) s.c[q] = __uint_as_float(r(K::C + q));
}

// Block rounds with regrouping: at most `slots` simulations live in a block
// (threads below `slots` take the first ones from the device work queue, and
// a thread whose simulation ends takes the next one, so the count never
// grows); every round the live simulations are sorted by phase -- SSA
// first, then leap decisions from the next warp boundary -- and their state
// moves through shared memory to the thread of their new position, so that
// each warp runs one phase only (with slots <= 32 in a 64-thread block, warp
// 0 steps SSA while warp 1 decides).  Then SSA threads take up to ssa_budget
// steps and deciding threads up to dec_budget decisions, and the block meets
// at a barrier.  Once the work queue is closed and at most run.tail_sims
// simulations are live in the block, they move to the first lanes of warp 0,
// which finishes them in warp lockstep with no further barriers or state
// exchange (a lone simulation steps about a third faster so) while the other
// warps leave.  xs: dynamic shared memory of Packed<P, SM>::WORDS words per
// thread.
template <class N, int P, int SM>
__device__ __forceinline__ void sweep_rounds(const N& net, const dev::Run& run, uint32_t slots, uint32_t* xs) {
    __shared__ uint32_t s_cnt[2][32];
    // Warps that finished their share of the round, per round parity:
    // [p][0] stepping warps after ssa_budget steps, [p][1] deciding warps
    // after their decisions.
    __shared__ uint32_t s_fin[2][2];
    // set by a thread that found the work queue closed; read after a round's
    // first barrier, written only after its second
    __shared__ uint32_t s_closed;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t nt = blockDim.x, nw = nt >> 5;
    const uint32_t below = (1u << lane) - 1u;
    const size_t row_words = (size_t)net.ns() * (size_t)net.s_out();
    State<P, SM> s;
    Sim st;
    Out o{nullptr, nullptr};
    bool live = false;
    if (tid == 0) s_closed = 0u;
    __syncthreads();
    if (tid < slots) {
        const uint32_t sim = atomicAdd(run.queue, 1u);
        if (sim < run.n) {
            start_sim<N, P, SM>(net, run, s, st, sim);
            live = true;
        } else {
            s_closed = 1u;
        }
    }
    if (tid < 4) s_fin[tid >> 1][tid & 1] = 0u;
    for (uint32_t round = 0;; round++) {
        const uint32_t par = round & 1u;
        const uint32_t bs = __ballot_sync(0xffffffffu, live && st.in_ssa);
        const uint32_t bd = __ballot_sync(0xffffffffu, live && !st.in_ssa);
        if (lane == 0) {
            s_cnt[0][warp] = __popc(bs);
            s_cnt[1][warp] = __popc(bd);
        }
        __syncthreads();
        uint32_t nssa = 0, ndec = 0, offs = 0, offd = 0;
        for (uint32_t w = 0; w < nw; w++) {
            const uint32_t a = s_cnt[0][w], b = s_cnt[1][w];
            if (w < warp) {
                offs += a;
                offd += b;
            }
            nssa += a;
            ndec += b;
        }
        if (nssa + ndec == 0u) break;  // the same counts in every thread
        if (s_closed && nssa + ndec <= run.tail_sims && nssa + ndec <= 32u) {
            // the tail: the live simulations to lanes 0..k-1, SSA ones first
            if (live) {
                const uint32_t pos = st.in_ssa ? offs + __popc(bs & below) : nssa + offd + __popc(bd & below);
                put_state<P, SM>(xs, nt, pos, s, st);
            }
            __syncthreads();
            const uint32_t k = nssa + ndec;
            if (tid >= k) return;
            get_state<N, P, SM>(net, xs, nt, tid, s, st);
            all_props<N, P, SM>(net, s);
            o = out_for(run, st.sim, row_words);
            lockstep<N, P, SM>(net, run, k >= 32u ? 0xffffffffu : (1u << k) - 1u, s, st, o, true);
            return;
        }
        // the other parity's flags were last read in the round before this one
        if (tid < 2) s_fin[par ^ 1u][tid] = 0u;
        const uint32_t pad = (nssa + 31u) & ~31u;
        const uint32_t dbase = pad + ndec <= nt ? pad : nssa;
        // Elastic rounds (when no warp holds both phases): a warp that has
        // done its share keeps going while the other phase's warps still
        // work -- stepping warps take further SSA steps, and in deciding
        // warps the simulations that handed off to SSA take SSA steps --
        // instead of waiting at the round's barrier.
        const bool elastic = dbase == pad;
        const uint32_t nsw = (nssa + 31u) >> 5;
        const uint32_t ndw = ndec ? ((dbase + ndec - 1u) >> 5) - (dbase >> 5) + 1u : 0u;
        volatile uint32_t* fin = s_fin[par];
        if (live) {
            const uint32_t pos = st.in_ssa ? offs + __popc(bs & below) : dbase + offd + __popc(bd & below);
            put_state<P, SM>(xs, nt, pos, s, st);
        }
        __syncthreads();
        const bool mine_ssa = tid < nssa, mine_dec = tid >= dbase && tid < dbase + ndec;
        live = mine_ssa || mine_dec;
        if (live) {
            get_state<N, P, SM>(net, xs, nt, tid, s, st);
            all_props<N, P, SM>(net, s);
            o = out_for(run, st.sim, row_words);
        }
        const uint32_t smask = __ballot_sync(0xffffffffu, mine_ssa);
        const uint32_t dmask = __ballot_sync(0xffffffffu, mine_dec);
        int res = CONT;
        const uint32_t cap = 8u * run.ssa_budget;  // a round's longest SSA stretch
        const bool first = lane == (uint32_t)(__ffs(mine_ssa ? smask : dmask) - 1);
        if (mine_ssa) {
            bool told = false;
            for (uint32_t b = 0; b < cap; b++) {
                if (b == run.ssa_budget && first && !told) {
                    atomicAdd((uint32_t*)&fin[0], 1u);
                    told = true;
                }
                const bool more = b < run.ssa_budget || (elastic && fin[1] < ndw);
                const bool act = res == CONT && st.in_ssa && more;
                if (!__any_sync(smask, act)) break;
                if (act) res = ssa_step<N, P, SM>(net, run, s, st, o);
            }
            if (first && !told) atomicAdd((uint32_t*)&fin[0], 1u);
        } else if (mine_dec) {
            for (uint32_t b = 0; b < run.dec_budget; b++) {
                const bool act = res == CONT && !st.in_ssa;
                if (!__any_sync(dmask, act)) break;
                if (act) res = decide_step<N, P, SM>(net, run, s, st, o);
            }
            if (first) atomicAdd((uint32_t*)&fin[1], 1u);
            for (uint32_t b = 0; b < cap && elastic; b++) {
                const bool act = res == CONT && st.in_ssa && fin[0] < nsw;
                if (!__any_sync(dmask, act)) break;
                if (act) res = ssa_step<N, P, SM>(net, run, s, st, o);
            }
        }
        if (live && res == DONE) {
            finish<N>(net, run, st, o);
            live = false;
            const uint32_t sim = atomicAdd(run.queue, 1u);  // this thread's next simulation
            if (sim < run.n) {
                start_sim<N, P, SM>(net, run, s, st, sim);
                live = true;
            } else {
                s_closed = 1u;
            }
        }
    }
}

// The kernel body: warp lockstep (run.warp_local) or block rounds with
// regrouping; `lanes` is the simulations per warp of the first and the live
// simulations per block of the second.
template <class N, int P, int SM>
__device__ __forceinline__ void run_sweep(const N& net, const dev::Run& run, uint32_t lanes) {
    if (run.warp_local) {
        sweep<N, P, SM>(net, run, lanes);
    } else {
        extern __shared__ uint32_t ctl_tiny_xs[];
        sweep_rounds<N, P, SM>(net, run, lanes, ctl_tiny_xs);
    }
}

}  // namespace tiny
}  // namespace ctl

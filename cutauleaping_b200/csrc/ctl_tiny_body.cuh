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
};

// Pick uniform and waiting-time log of SSA step `step`: one Philox block per
// two steps, (w0, w1) for even steps and (w2, w3) for odd ones, as
// dev::ssa_step.
__device__ __forceinline__ void ssa_randoms(const dev::Run& run, uint32_t simg, uint32_t step, double& u, float& lg) {
    const uint4 w = dev::draw(run.seed, 0u, dev::TAG_SSA, step >> 1, simg);
    const uint32_t wa = (step & 1u) ? w.z : w.x, wb = (step & 1u) ? w.w : w.y;
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
        ssa_randoms(run, simg, step, u, lg);
    }
    const int r = descend<P>(s.t, u * A0);
    // the next step's random part, free of the state: it overlaps the
    // update below (a leap decision in between leaves it unused)
    ssa_randoms(run, simg, step + 1u, st.pre_u, st.pre_lg);
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
    if (ovf) { st.status = CTL_SIM_OVERFLOW; return DONE; }
    all_props<N, P, SM>(net, s);
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
template <class N, int P, int SM>
__device__ __forceinline__ void sweep(const N& net, const dev::Run& run, uint32_t lanes) {
    const uint32_t lane = threadIdx.x & 31u;
    if (lane >= lanes) return;
    const uint32_t mask = lanes >= 32 ? 0xffffffffu : ((1u << lanes) - 1u);
    const uint32_t ns = (uint32_t)net.ns();
    const size_t row_words = (size_t)ns * (size_t)net.s_out();
    State<P, SM> s;
    Sim st;
    Out o{nullptr, nullptr};
    bool live = false, closed = false;
    for (;;) {
        if (!live && !closed) {
            const uint32_t sim = atomicAdd(run.queue, 1u);
            if (sim >= run.n) {
                closed = true;
            } else {
                // PrepareVariables (tau.cu:1269-1297)
#pragma unroll
                for (int q = 0; q < SM; q++) {
                    s.x[q] = q < net.S() ? run.X0[(size_t)sim * net.S() + q] : 0;
                    s.last[q] = 0u;
                }
#pragma unroll
                for (int r = 0; r < P; r++)
                    s.c[r] = r < net.R() ? run.c[(run.uniform_c ? (size_t)0 : (size_t)sim * net.R()) + r] : 0.0f;
                all_props<N, P, SM>(net, s);
                st.T = 0.0;
                st.tl = 0.0;
                st.t_next = net.tvec()[0];
                st.fire = 0ull;
                st.sim = sim;
                st.cursor = st.n = st.burst = st.leaps = st.ssa = st.rej = 0u;
                st.status = CTL_SIM_OK;
                st.in_ssa = (run.flags & dev::F_FORCE_SSA) != 0;
                st.pre = 0xffffffffu;
                if (run.sums) {
                    const uint32_t tp = run.sum_threads * run.sum_prep;
                    const uint32_t set = (sim / tp) * run.sum_threads + sim % run.sum_threads;
                    o.samples = nullptr;
                    o.sums = run.sums + (size_t)set * row_words;
                } else {
                    o.samples = run.out + (size_t)sim * row_words;
                    o.sums = nullptr;
                }
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
            if (o.samples)  // rows never reached read 0
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
            if (run.done) {  // publish: this simulation's rows and record are complete
                __threadfence();
                atomicAdd(run.done + (st.sim >> run.done_shift), 1u);
            }
            live = false;
        }
    }
}

}  // namespace tiny
}  // namespace ctl

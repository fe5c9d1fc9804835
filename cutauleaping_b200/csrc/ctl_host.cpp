// Host side of cutauleaping_b200: model tables, input-folder parsers,
// output writers and fitness targets.  The device sweep lives in
// ctl_sweep.cu.
//
// Parsers follow the reference's file semantics (2phase_n-tau-leaping.cu):
// tab-separated rows, one row per reaction (left_side/right_side) or per
// simulation (MX_0/c_matrix), one value per line (t_vector/cs_vector).  The
// reference's fixed-size limits (char indices, 6400-entry constant matrix,
// 500 flattened entries, 48 KB shared memory; tau.cuh:41-98) do not apply.
// Where the reference reads out of bounds or exits, these return a status.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <memory>
#include <new>
#include <thread>

#include "ctl_internal.h"

namespace ctl {

static thread_local std::string g_last_error;
static thread_local int32_t g_last_detail = CTL_DETAIL_NONE;

void set_error(const std::string& msg) {
    g_last_error = msg;
    g_last_detail = CTL_DETAIL_NONE;
}

static ctl_status fail(ctl_status s, const std::string& msg) {
    set_error(msg);
    return s;
}

// A failure with its ctl_error_detail (what the command line maps to the
// reference's exit codes).
static ctl_status fail_d(ctl_status s, ctl_error_detail d, const std::string& msg) {
    set_error(msg);
    g_last_detail = d;
    return s;
}

// ---------------------------------------------------------------------------
// Tables
// ---------------------------------------------------------------------------

ctl_status build_tables(int S, int R, const int32_t* left, const int32_t* right,
                        const int32_t* feed, int ns, const double* tvec, int s_out,
                        const int32_t* cs, HostTables& t) {
    if (S <= 0 || R <= 0) return fail(CTL_ERR_SHAPE, "model needs at least one species and one reaction");
    if (S >= (1 << 24) || R >= (1 << 24)) return fail(CTL_ERR_SHAPE, "more than 2^24 species or reactions");
    if ((int64_t)S * R > ((int64_t)1 << 28)) return fail(CTL_ERR_SHAPE, "more than 2^28 stoichiometry entries");
    if (ns <= 0) return fail(CTL_ERR_SHAPE, "t_vector holds no sample instants");
    if (!left || !right || !tvec) return fail(CTL_ERR_ARG, "null model array");
    // A NaN or infinite instant would never be reached (the simulation would
    // run to its step cap), a negative one never compared: both are errors.
    for (int i = 0; i < ns; i++)
        if (!std::isfinite(tvec[i]) || tvec[i] < 0.0)
            return fail(CTL_ERR_SHAPE, "t_vector: instant " + std::to_string(i) + " is negative or not finite");
    for (int i = 0; i < R * S; i++) {
        if (left[i] < 0 || left[i] > 127 || right[i] < 0 || right[i] > 127)
            return fail(CTL_ERR_SHAPE, "stoichiometric coefficients must lie in [0, 127]");
    }
    t = HostTables();
    t.S = S;
    t.R = R;
    t.P = 2;
    t.logP = 1;
    while (t.P < R) { t.P <<= 1; t.logP++; }
    t.ns = ns;
    t.tvec.assign(tvec, tvec + ns);
    t.tmax = tvec[ns - 1];
    if (cs && s_out > 0) {
        for (int k = 0; k < s_out; k++) {
            if (cs[k] < 0 || cs[k] >= S) return fail(CTL_ERR_SHAPE, "cs_vector names a species that does not exist");
            t.cs.push_back((uint32_t)cs[k]);
        }
    } else {
        for (int s = 0; s < S; s++) t.cs.push_back((uint32_t)s);
    }
    t.s_out = (int)t.cs.size();

    std::vector<int> V((size_t)R * S), F((size_t)R * S);
    for (int r = 0; r < R; r++)
        for (int s = 0; s < S; s++) {
            int v = right[(size_t)r * S + s] - left[(size_t)r * S + s];
            V[(size_t)r * S + s] = v;
            F[(size_t)r * S + s] = (feed && feed[s]) ? 0 : v;
        }
    // reactants, reaction-major (tau.cu:212-225)
    t.reac_off.push_back(0);
    for (int r = 0; r < R; r++) {
        for (int s = 0; s < S; s++)
            if (left[(size_t)r * S + s] > 0) t.reac_ent.push_back(pack((uint32_t)s, left[(size_t)r * S + s]));
        t.reac_off.push_back((uint32_t)t.reac_ent.size());
    }
    // Packed reactant descriptors: the common case of at most two reactant
    // entries with coefficients 1 or 2 needs one table load per propensity.
    t.reac_desc.assign((size_t)2 * R, 0u);
    for (int r = 0; r < R; r++) {
        const uint32_t e0 = t.reac_off[r], e1 = t.reac_off[r + 1];
        bool simple = e1 - e0 <= 2;
        for (uint32_t e = e0; e < e1; e++) simple = simple && (t.reac_ent[e] & 0xffu) <= 2;
        if (!simple) {
            t.reac_desc[2 * r] = 0xffffffffu;
            continue;
        }
        for (uint32_t e = e0; e < e1; e++) t.reac_desc[2 * r + (e - e0)] = t.reac_ent[e];
    }
    // V species-major = RAV (tau.cu:314-326); F species-major and reaction-major
    t.vs_off.push_back(0);
    t.fs_off.push_back(0);
    for (int s = 0; s < S; s++) {
        for (int r = 0; r < R; r++) {
            if (V[(size_t)r * S + s]) t.vs_ent.push_back(pack((uint32_t)r, V[(size_t)r * S + s]));
            if (F[(size_t)r * S + s]) t.fs_ent.push_back(pack((uint32_t)r, F[(size_t)r * S + s]));
        }
        t.vs_off.push_back((uint32_t)t.vs_ent.size());
        t.fs_off.push_back((uint32_t)t.fs_ent.size());
    }
    t.fr_off.push_back(0);
    for (int r = 0; r < R; r++) {
        for (int s = 0; s < S; s++)
            if (F[(size_t)r * S + s]) t.fr_ent.push_back(pack((uint32_t)s, F[(size_t)r * S + s]));
        t.fr_off.push_back((uint32_t)t.fr_ent.size());
    }
    // Dependency lists: a firing of r changes the species with F[r][s] != 0;
    // every reaction that has one of them as a reactant needs a new propensity.
    std::vector<std::vector<uint32_t>> users((size_t)S);
    for (int r = 0; r < R; r++)
        for (uint32_t e = t.reac_off[r]; e < t.reac_off[r + 1]; e++) users[t.reac_ent[e] >> 8].push_back((uint32_t)r);
    t.dep_off.push_back(0);
    std::vector<uint32_t> tmp;
    for (int r = 0; r < R; r++) {
        tmp.clear();
        for (uint32_t e = t.fr_off[r]; e < t.fr_off[r + 1]; e++)
            for (uint32_t u : users[t.fr_ent[e] >> 8]) tmp.push_back(u);
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        t.dep_ent.insert(t.dep_ent.end(), tmp.begin(), tmp.end());
        t.dep_off.push_back((uint32_t)t.dep_ent.size());
    }
    // HOR / HORtype exactly as tau.cu:402-432 (order-dependent hortype).
    t.hor.assign((size_t)S, 0);
    t.hort.assign((size_t)S, 0);
    std::vector<uint8_t> order((size_t)R, 0);
    for (int r = 0; r < R; r++) {
        uint8_t tot = 0;
        for (int s = 0; s < S; s++) tot = (uint8_t)(tot + left[(size_t)r * S + s]);
        order[r] = tot;
    }
    for (int s = 0; s < S; s++)
        for (int r = 0; r < R; r++) {
            int l = left[(size_t)r * S + s];
            if (l > 0 && order[r] > t.hor[s]) { t.hor[s] = order[r]; t.hort[s] = (uint8_t)l; }
            if (t.hort[s] < l) t.hort[s] = (uint8_t)l;
        }
    return CTL_OK;
}

// ---------------------------------------------------------------------------
// Parsing helpers
// ---------------------------------------------------------------------------

static bool read_lines(const std::string& path, std::vector<std::string>& lines) {
    std::ifstream in(path.c_str());
    if (!in.is_open()) return false;
    std::string line;
    lines.clear();
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        lines.push_back(line);
    }
    return true;
}

static void split_tabs(const std::string& s, std::vector<std::string>& tok) {
    tok.clear();
    std::istringstream buf(s);
    for (std::string t; std::getline(buf, t, '\t');) tok.push_back(t);
}

// Numeric prefix of a token, like `istream >> value` in the reference.
static bool parse_double(const std::string& tok, double& v) {
    const char* p = tok.c_str();
    char* end = nullptr;
    errno = 0;
    v = std::strtod(p, &end);
    return end != p;
}
static bool parse_long(const std::string& tok, long& v) {  // out-of-range values are errors
    const char* p = tok.c_str();
    char* end = nullptr;
    errno = 0;
    v = std::strtol(p, &end, 10);
    return end != p && errno != ERANGE;
}

}  // namespace ctl

using namespace ctl;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" const char* ctl_status_str(ctl_status s) {
    switch (s) {
        case CTL_OK: return "ok";
        case CTL_ERR_IO: return "i/o error";
        case CTL_ERR_PARSE: return "parse error";
        case CTL_ERR_SHAPE: return "shape error";
        case CTL_ERR_CUDA: return "cuda error";
        case CTL_ERR_OOM: return "out of memory";
        case CTL_ERR_STEP_LIMIT: return "simulation limit reached";
        case CTL_ERR_TIMEOUT: return "timeout";
        case CTL_ERR_ARG: return "invalid argument";
    }
    return "unknown status";
}

extern "C" const char* ctl_last_error(void) { return ctl::g_last_error.c_str(); }
extern "C" int32_t ctl_last_error_detail(void) { return ctl::g_last_detail; }

static ctl_status model_create_impl(int32_t S, int32_t R, const int32_t* left,
                                       const int32_t* right, const int32_t* feed, int32_t ns,
                                       const double* tvec, int32_t s_out, const int32_t* cs,
                                       ctl_model** out) {
    if (!out) return fail(CTL_ERR_ARG, "null output handle");
    *out = nullptr;
    ctl_model* m = new (std::nothrow) ctl_model();
    if (!m) return fail(CTL_ERR_OOM, "host allocation failed");
    ctl_status st = build_tables(S, R, left, right, feed, ns, tvec, s_out, cs, m->t);
    if (st != CTL_OK) { delete m; return st; }
    *out = m;
    return CTL_OK;
}

static ctl_status model_load_impl(const char* folder, ctl_model** out) {
    if (!folder || !out) return fail(CTL_ERR_ARG, "null argument");
    *out = nullptr;
    std::string f(folder);
    std::vector<std::string> lines, tok;
    // first_pass (tau.cu:90-120): R = rows of left_side, S = tokens of row 0.
    if (!read_lines(f + "/left_side", lines)) return fail(CTL_ERR_IO, "ERROR reading left matrix: " + f + "/left_side");
    while (!lines.empty() && lines.back().empty()) lines.pop_back();
    if (lines.empty()) return fail(CTL_ERR_SHAPE, "left_side is empty");
    int R = (int)lines.size();
    split_tabs(lines[0], tok);
    int S = (int)tok.size();
    std::vector<int32_t> left((size_t)R * S), right((size_t)R * S), feed((size_t)S, 0);
    auto parse_matrix = [&](const std::vector<std::string>& rows, std::vector<int32_t>& M,
                            const char* name) -> ctl_status {
        for (int r = 0; r < R; r++) {
            split_tabs(rows[r], tok);
            if ((int)tok.size() != S)
                return fail(CTL_ERR_SHAPE, std::string(name) + ": row " + std::to_string(r) + " has " +
                                               std::to_string(tok.size()) + " entries, expected " + std::to_string(S));
            for (int s = 0; s < S; s++) {
                long v;
                if (!parse_long(tok[s], v)) return fail(CTL_ERR_PARSE, std::string(name) + ": bad entry '" + tok[s] + "'");
                M[(size_t)r * S + s] = (int32_t)v;
            }
        }
        return CTL_OK;
    };
    ctl_status st = parse_matrix(lines, left, "left_side");
    if (st != CTL_OK) return st;
    if (!read_lines(f + "/right_side", lines)) return fail(CTL_ERR_IO, "ERROR reading right matrix: " + f + "/right_side");
    while (!lines.empty() && lines.back().empty()) lines.pop_back();
    if ((int)lines.size() != R) return fail(CTL_ERR_SHAPE, "left and right matrices have different size");
    st = parse_matrix(lines, right, "right_side");
    if (st != CTL_OK) return st;
    // M_feed (optional): nonzero entries mark species held constant.
    if (read_lines(f + "/M_feed", lines) && !lines.empty()) {
        split_tabs(lines[0], tok);
        for (size_t s = 0; s < tok.size() && (int)s < S; s++) {
            long v = 0;
            if (!parse_long(tok[s], v)) return fail(CTL_ERR_PARSE, "M_feed: bad entry '" + tok[s] + "'");
            feed[s] = v != 0;
        }
    }
    // read_instants (tau.cu:932-1053)
    if (!read_lines(f + "/t_vector", lines)) return fail(CTL_ERR_IO, "ERROR reading samples vector: " + f + "/t_vector");
    while (!lines.empty() && lines.back().empty()) lines.pop_back();
    std::vector<double> tv;
    for (auto& l : lines) {
        double v;
        if (!parse_double(l, v)) return fail(CTL_ERR_PARSE, "t_vector: bad entry '" + l + "'");
        tv.push_back(v);
    }
    std::vector<int32_t> cs;
    if (read_lines(f + "/cs_vector", lines)) {
        while (!lines.empty() && lines.back().empty()) lines.pop_back();
        for (auto& l : lines) {
            long v;
            if (!parse_long(l, v)) return fail(CTL_ERR_PARSE, "cs_vector: bad entry '" + l + "'");
            cs.push_back((int32_t)v);
        }
    }
    return ctl_model_create(S, R, left.data(), right.data(), feed.data(), (int32_t)tv.size(), tv.data(),
                            (int32_t)cs.size(), cs.empty() ? nullptr : cs.data(), out);
}

extern "C" void ctl_model_free(ctl_model* m);  // defined in ctl_sweep.cu (frees device copies)

extern "C" ctl_status ctl_model_dims_get(const ctl_model* m, ctl_model_dims* d) {
    if (!m || !d) return fail(CTL_ERR_ARG, "null argument");
    d->S = m->t.S; d->R = m->t.R; d->P = m->t.P; d->ns = m->t.ns; d->s_out = m->t.s_out;
    d->nnz_left = (int32_t)m->t.reac_ent.size();
    d->nnz_var = (int32_t)m->t.vs_ent.size();
    d->nnz_feared = (int32_t)m->t.fs_ent.size();
    d->nnz_dep = (int32_t)m->t.dep_ent.size();
    d->tmax = m->t.tmax;
    return CTL_OK;
}

extern "C" ctl_status ctl_model_hor(const ctl_model* m, uint8_t* hor, uint8_t* hort) {
    if (!m || !hor || !hort) return fail(CTL_ERR_ARG, "null argument");
    std::memcpy(hor, m->t.hor.data(), m->t.hor.size());
    std::memcpy(hort, m->t.hort.data(), m->t.hort.size());
    return CTL_OK;
}

static ctl_status rows_load_impl(const char* folder, int32_t S, int32_t R, uint32_t offset,
                                    uint32_t n, int32_t* X0, float* c) {
    if (!folder || !X0 || !c) return fail(CTL_ERR_ARG, "null argument");
    std::string f(folder);
    std::vector<std::string> lines, tok;
    // read_quantities_offset (tau.cu:570-649): exit(-6) / -4 / -5 become statuses.
    if (!read_lines(f + "/MX_0", lines))
        return fail_d(CTL_ERR_IO, CTL_DETAIL_MX0_UNREADABLE, "ERROR reading quantities matrix: " + f + "/MX_0");
    if ((uint64_t)offset + n > lines.size())
        return fail_d(CTL_ERR_SHAPE, CTL_DETAIL_ROWS_SHORT,
                      "ERROR: input files rows (" + std::to_string(lines.size()) + ") and requested threads (" +
                          std::to_string(n) + ") do not fit");
    for (uint32_t i = 0; i < n; i++) {
        split_tabs(lines[offset + i], tok);
        if ((int)tok.size() != S)
            return fail_d(CTL_ERR_SHAPE, CTL_DETAIL_MX0_ROW,
                          "MX_0 row " + std::to_string(offset + i) + ": " + std::to_string(tok.size()) +
                              " quantities, expected " + std::to_string(S));
        for (int s = 0; s < S; s++) {
            double v;
            if (!parse_double(tok[s], v))
                return fail_d(CTL_ERR_PARSE, CTL_DETAIL_MX0_ROW, "MX_0: bad entry '" + tok[s] + "'");
            if (!(v >= 0.0) || v > 2147483647.0)
                return fail_d(CTL_ERR_SHAPE, CTL_DETAIL_MX0_ROW, "MX_0: quantity out of range '" + tok[s] + "'");
            X0[(size_t)i * S + s] = (int32_t)(uint32_t)v;
        }
    }
    // read_parameters_offset (tau.cu:717-782)
    if (!read_lines(f + "/c_matrix", lines)) return fail(CTL_ERR_IO, "ERROR reading parameters matrix: " + f + "/c_matrix");
    if ((uint64_t)offset + n > lines.size())
        return fail(CTL_ERR_SHAPE, "c_matrix has " + std::to_string(lines.size()) + " rows, fewer than offset + threads");
    for (uint32_t i = 0; i < n; i++) {
        split_tabs(lines[offset + i], tok);
        if ((int)tok.size() != R)
            return fail(CTL_ERR_SHAPE, "ERROR! too many parameters (" + std::to_string(tok.size()) + ") in c_matrix row " +
                                           std::to_string(offset + i));
        for (int r = 0; r < R; r++) {
            double v;
            if (!parse_double(tok[r], v)) return fail(CTL_ERR_PARSE, "c_matrix: bad entry '" + tok[r] + "'");
            if (!(v >= 0.0) || !std::isfinite(v)) return fail(CTL_ERR_SHAPE, "c_matrix: rate constants must be finite and >= 0");
            c[(size_t)i * R + r] = (float)v;
        }
    }
    return CTL_OK;
}

// ---------------------------------------------------------------------------
// Output writers (WriteDynamics2 / PrintDynamics2, tau.cu:3431-3507)
// ---------------------------------------------------------------------------

static std::vector<std::string> time_strings(const HostTables& t) {
    std::vector<std::string> ts;
    for (double v : t.tvec) {
        std::ostringstream o;
        o << v;  // iostream default formatting, as the reference writes it
        ts.push_back(o.str());
    }
    return ts;
}

static void append_sim(std::string& buf, const HostTables& t, const std::vector<std::string>& ts,
                       const uint32_t* s) {
    char num[16];
    for (int i = 0; i < t.ns; i++) {
        buf += ts[i];
        for (int k = 0; k < t.s_out; k++) {
            int len = std::snprintf(num, sizeof(num), "\t%u", s[(size_t)i * t.s_out + k]);
            buf.append(num, (size_t)len);
        }
        buf += '\n';
    }
}

static ctl_status write_dynamics_impl(const ctl_model* m, const char* path_prefix, uint32_t n,
                                         const uint32_t* samples, uint32_t first_id, int32_t nthreads) {
    if (!m || !path_prefix || (!samples && n)) return fail(CTL_ERR_ARG, "null argument");
    const HostTables& t = m->t;
    std::vector<std::string> ts = time_strings(t);
    std::string prefix(path_prefix);
    if (nthreads <= 0) nthreads = (int32_t)std::max(1u, std::thread::hardware_concurrency());
    nthreads = (int32_t)std::min<uint32_t>((uint32_t)nthreads, std::max(1u, n));
    std::atomic<uint32_t> next(0);
    std::atomic<int> err(0);
    std::string err_path;
    std::mutex err_mu;
    std::atomic<int> oom(0);
    auto work = [&]() {
        try {  // nothing may escape a worker thread
            std::string buf;
            for (;;) {
                uint32_t i = next.fetch_add(1);
                if (i >= n) break;
                buf.clear();
                append_sim(buf, t, ts, samples + (size_t)i * t.ns * t.s_out);
                std::string name = prefix + "_" + std::to_string((unsigned long long)first_id + i);
                FILE* fp = std::fopen(name.c_str(), "wb");
                if (!fp || std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) {
                    std::lock_guard<std::mutex> lk(err_mu);
                    err = 1;
                    err_path = name;
                }
                if (fp) std::fclose(fp);
            }
        } catch (...) {
            oom = 1;
            next = n;  // the other workers stop too
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int k = 1; k < nthreads; k++) pool.emplace_back(work);
    } catch (...) {  // fewer threads than asked: the ones started and this one finish the work
    }
    work();
    for (auto& th : pool) th.join();
    if (oom) return fail(CTL_ERR_OOM, "ctl_write_dynamics: host allocation failed");
    if (err) return fail(CTL_ERR_IO, "cannot write " + err_path);
    return CTL_OK;
}

static ctl_status print_dynamics_impl(const ctl_model* m, uint32_t n, const uint32_t* samples) {
    if (!m || (!samples && n)) return fail(CTL_ERR_ARG, "null argument");
    const HostTables& t = m->t;
    std::vector<std::string> ts = time_strings(t);
    std::string buf;
    for (uint32_t i = 0; i < n; i++) {
        buf.clear();
        append_sim(buf, t, ts, samples + (size_t)i * t.ns * t.s_out);
        buf += '\n';
        std::cout.write(buf.data(), (std::streamsize)buf.size());
    }
    std::cout.flush();
    return CTL_OK;
}

static ctl_status write_samples_binary_impl(const ctl_model* m, const char* path, uint32_t n,
                                               const uint32_t* samples, uint32_t first_id) {
    if (!m || !path || (!samples && n)) return fail(CTL_ERR_ARG, "null argument");
    const HostTables& t = m->t;
    std::vector<unsigned char> head;
    auto put = [&head](const void* p, size_t k) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        head.insert(head.end(), b, b + k);
    };
    put("CTLSAMP1", 8);
    const uint32_t dims[4] = {n, (uint32_t)t.ns, (uint32_t)t.s_out, first_id};
    put(dims, sizeof(dims));
    put(t.tvec.data(), t.tvec.size() * sizeof(double));
    for (int k = 0; k < t.s_out; k++) {
        const uint32_t sp = (size_t)k < t.cs.size() ? t.cs[k] : (uint32_t)k;
        put(&sp, sizeof(sp));
    }
    head.resize((head.size() + 15) & ~(size_t)15, 0);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(CTL_ERR_IO, std::string("cannot write ") + path);
    bool ok = std::fwrite(head.data(), 1, head.size(), fp) == head.size();
    const size_t bytes = (size_t)n * t.ns * t.s_out * sizeof(uint32_t);
    const size_t piece = (size_t)64 << 20;
    for (size_t off = 0; ok && off < bytes; off += piece) {
        const size_t k = std::min(piece, bytes - off);
        ok = std::fwrite(reinterpret_cast<const unsigned char*>(samples) + off, 1, k, fp) == k;
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(CTL_ERR_IO, std::string("cannot write ") + path);
    return CTL_OK;
}

static ctl_status write_run_report_impl(const ctl_model* m, const char* path, uint32_t n,
                                           const ctl_sim_info* info, double seconds,
                                           const ctl_launch_info* launch) {
    if (!m || !path || (!info && n)) return fail(CTL_ERR_ARG, "null argument");
    if (!(seconds > 0.0) || !std::isfinite(seconds)) return fail(CTL_ERR_ARG, "seconds must be positive");
    const HostTables& t = m->t;
    unsigned long long firings = 0, steps = 0, leaps = 0, ssa = 0, rej = 0, st[4] = {0, 0, 0, 0}, other = 0;
    for (uint32_t i = 0; i < n; i++) {
        firings += info[i].firings;
        steps += info[i].steps;
        leaps += info[i].leaps;
        ssa += info[i].ssa_steps;
        rej += info[i].rejections;
        if (info[i].status < 4) st[info[i].status]++;
        else other++;
    }
    // X0 (4S) + c (4R) + samples (4 ns s_out) + the 40-byte record
    const double bytes = 4.0 * t.S + 4.0 * t.R + 4.0 * t.ns * t.s_out + (double)sizeof(ctl_sim_info);
    std::ostringstream o;
    o.precision(17);
    o << "{\"simulations\": " << n << ", \"seconds\": " << seconds
      << ", \"sims_per_s\": " << n / seconds << ", \"firings\": " << firings
      << ", \"firings_per_s\": " << (double)firings / seconds << ", \"steps\": " << steps
      << ", \"leaps\": " << leaps << ", \"ssa_steps\": " << ssa << ", \"rejections\": " << rej
      << ", \"status\": {\"ok\": " << st[CTL_SIM_OK] << ", \"step_limit\": " << st[CTL_SIM_STEP_LIMIT]
      << ", \"overflow\": " << st[CTL_SIM_OVERFLOW] << ", \"attempt_limit\": " << st[CTL_SIM_ATTEMPT_LIMIT]
      << ", \"other\": " << other << "}, \"species\": " << t.S << ", \"reactions\": " << t.R
      << ", \"instants\": " << t.ns << ", \"sampled_species\": " << t.s_out
      << ", \"hbm_bytes_per_sim\": " << bytes << ", \"hbm_gb_per_s\": " << bytes * n / seconds / 1e9;
    if (launch)
        o << ", \"launch\": {\"group\": " << launch->group << ", \"threads\": " << launch->threads
          << ", \"blocks\": " << launch->blocks << ", \"min_blocks\": " << launch->min_blocks
          << ", \"sched\": " << launch->sched << ", \"ssa_budget\": " << launch->ssa_budget
          << ", \"dec_budget\": " << launch->dec_budget << "}";
    o << "}\n";
    const std::string js = o.str();
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(CTL_ERR_IO, std::string("cannot write ") + path);
    const bool ok = std::fwrite(js.data(), 1, js.size(), fp) == js.size();
    if (std::fclose(fp) != 0 || !ok) return fail(CTL_ERR_IO, std::string("cannot write ") + path);
    return CTL_OK;
}

// ---------------------------------------------------------------------------
// Fitness targets (read_time_series, tau.cu:1056-1261)
// ---------------------------------------------------------------------------

static ctl_status target_load_impl(const char* folder, const ctl_model* m, uint32_t threads,
                                      uint32_t blocks, ctl_target** out) {
    if (!folder || !m || !out) return fail(CTL_ERR_ARG, "null argument");
    *out = nullptr;
    std::string f(folder);
    std::unique_ptr<ctl_target> t(new ctl_target());
    t->threads = threads;
    t->blocks = blocks;
    t->ns = (uint32_t)m->t.ns;
    t->s_out = (uint32_t)m->t.s_out;
    uint64_t N = (uint64_t)threads * blocks;
    std::vector<std::string> lines, tok;
    auto first_int = [&](const char* name, uint32_t& v) -> ctl_status {
        if (!read_lines(f + "/" + name, lines) || lines.empty())
            return fail(CTL_ERR_IO, std::string("WARNING: cannot open ") + name + " file");
        long x = 0;
        if (!parse_long(lines[0], x) || x < 0) return fail(CTL_ERR_PARSE, std::string(name) + ": bad value");
        v = (uint32_t)x;
        return CTL_OK;
    };
    ctl_status st;
    if ((st = first_int("ts_rep", t->repetitions)) != CTL_OK) return st;
    if ((st = first_int("p_rep", t->p_rep)) != CTL_OK) return st;
    if ((st = first_int("ts_numtgt", t->target_quantities)) != CTL_OK) return st;
    if (t->p_rep == 0 || blocks % t->p_rep != 0)
        return fail(CTL_ERR_SHAPE, "p_rep must be a nonzero divisor of the number of blocks");
    if (t->target_quantities != t->s_out)
        return fail(CTL_ERR_SHAPE, "ts_numtgt must equal the number of sampled species");
    // tts_vector: cumulative simulation counts per experiment.
    if (!read_lines(f + "/tts_vector", lines)) return fail(CTL_ERR_IO, "WARNING: cannot open tts_vector file");
    t->thread2experiment.assign((size_t)N, 0);
    uint32_t pp = 0;
    uint64_t last = 0;
    for (auto& l : lines) {
        if (l.empty()) continue;
        long v;
        if (!parse_long(l, v) || v < 0 || (uint64_t)v > N) return fail(CTL_ERR_SHAPE, "tts_vector: bad boundary '" + l + "'");
        for (uint64_t k = last; k < (uint64_t)v; k++) t->thread2experiment[k] = (uint8_t)pp;
        last = (uint64_t)v;
        pp++;
    }
    if (pp > 127) return fail(CTL_ERR_SHAPE, "at most 127 experiments");
    t->experiments = pp;
    if (last != N)
        return fail_d(CTL_ERR_SHAPE, CTL_DETAIL_TARGET_ASSIGN,
                      "ERROR! cannot assign threads (" + std::to_string(N) + ") to initial conditions (" +
                          std::to_string(last) + "), aborting");
    // ts_matrix: one row per sample, first column the instant, then
    // experiments x repetitions x target_quantities counts.
    if (!read_lines(f + "/ts_matrix", lines)) return fail(CTL_ERR_IO, "WARNING: cannot open ts file (fitness unavailable)");
    const uint64_t cols64 = (uint64_t)t->experiments * t->repetitions * t->target_quantities;
    if (cols64 > ((uint64_t)1 << 24) || cols64 * t->ns > ((uint64_t)1 << 31))
        return fail(CTL_ERR_SHAPE, "ts_matrix: " + std::to_string(cols64) +
                                       " columns per instant (experiments x repetitions x quantities) is too large");
    const uint32_t cols = (uint32_t)cols64;
    t->series.assign((size_t)t->ns * cols, 0);
    uint32_t row = 0;
    for (auto& l : lines) {
        if (l.size() < 2) continue;
        if (row >= t->ns) return fail(CTL_ERR_SHAPE, "ts_matrix has more rows than t_vector");
        split_tabs(l, tok);
        if (tok.size() < (size_t)cols + 1) return fail(CTL_ERR_SHAPE, "ts_matrix row " + std::to_string(row) + " is short");
        for (uint32_t k = 1; k <= cols; k++) {
            long v;
            if (!parse_long(tok[k], v)) return fail(CTL_ERR_PARSE, "ts_matrix: bad entry '" + tok[k] + "'");
            t->series[(size_t)row * cols + k - 1] = (uint32_t)v;
        }
        row++;
    }
    *out = t.release();
    return CTL_OK;
}


// ---------------------------------------------------------------------------
// C ABI entry points of the host code: no C++ exception leaves the library
// (a failed host allocation becomes CTL_ERR_OOM, anything else CTL_ERR_ARG,
// with the message in ctl_last_error).
// ---------------------------------------------------------------------------

template <class F>
static ctl_status guarded(const char* what, F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return fail(CTL_ERR_OOM, std::string(what) + ": host allocation failed");
    } catch (const std::exception& e) {
        return fail(CTL_ERR_ARG, std::string(what) + ": " + e.what());
    } catch (...) {
        return fail(CTL_ERR_ARG, std::string(what) + ": unexpected failure");
    }
}

extern "C" ctl_status ctl_model_create(int32_t S, int32_t R, const int32_t* left, const int32_t* right,
                                       const int32_t* feed, int32_t ns, const double* tvec, int32_t s_out,
                                       const int32_t* cs, ctl_model** out) {
    return guarded("ctl_model_create",
                   [&] { return model_create_impl(S, R, left, right, feed, ns, tvec, s_out, cs, out); });
}

extern "C" ctl_status ctl_model_load(const char* folder, ctl_model** out) {
    return guarded("ctl_model_load", [&] { return model_load_impl(folder, out); });
}

extern "C" ctl_status ctl_rows_load(const char* folder, int32_t S, int32_t R, uint32_t offset, uint32_t n,
                                    int32_t* X0, float* c) {
    return guarded("ctl_rows_load", [&] { return rows_load_impl(folder, S, R, offset, n, X0, c); });
}

extern "C" ctl_status ctl_write_dynamics(const ctl_model* m, const char* path_prefix, uint32_t n,
                                         const uint32_t* samples, uint32_t first_id, int32_t nthreads) {
    return guarded("ctl_write_dynamics",
                   [&] { return write_dynamics_impl(m, path_prefix, n, samples, first_id, nthreads); });
}

extern "C" ctl_status ctl_print_dynamics(const ctl_model* m, uint32_t n, const uint32_t* samples) {
    return guarded("ctl_print_dynamics", [&] { return print_dynamics_impl(m, n, samples); });
}

extern "C" ctl_status ctl_write_samples_binary(const ctl_model* m, const char* path, uint32_t n,
                                               const uint32_t* samples, uint32_t first_id) {
    return guarded("ctl_write_samples_binary",
                   [&] { return write_samples_binary_impl(m, path, n, samples, first_id); });
}

extern "C" ctl_status ctl_write_run_report(const ctl_model* m, const char* path, uint32_t n,
                                           const ctl_sim_info* info, double seconds,
                                           const ctl_launch_info* launch) {
    return guarded("ctl_write_run_report",
                   [&] { return write_run_report_impl(m, path, n, info, seconds, launch); });
}

extern "C" ctl_status ctl_target_load(const char* folder, const ctl_model* m, uint32_t threads,
                                      uint32_t blocks, ctl_target** out) {
    return guarded("ctl_target_load", [&] { return target_load_impl(folder, m, threads, blocks, out); });
}

extern "C" void ctl_target_free(ctl_target* t) { delete t; }

extern "C" ctl_status ctl_target_dims(const ctl_target* t, uint32_t* repetitions, uint32_t* p_rep,
                                      uint32_t* target_quantities, uint32_t* experiments) {
    if (!t) return fail(CTL_ERR_ARG, "null target");
    if (repetitions) *repetitions = t->repetitions;
    if (p_rep) *p_rep = t->p_rep;
    if (target_quantities) *target_quantities = t->target_quantities;
    if (experiments) *experiments = t->experiments;
    return CTL_OK;
}

extern "C" void ctl_run_cfg_default(ctl_run_cfg* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->seed = 0;
    c->eps = 0.03f;
    c->nc = 10;
    c->ssa_factor = 10.0;
    c->ssa_steps = 100;
    c->flags = 0;
    c->max_steps = 0xFFFFFFFFu;
    c->sim_base = 0;
    c->device = 0;
    c->group = 0;
    c->threads = 0;
}

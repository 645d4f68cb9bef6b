// symbolic.cu -- the .sym rate-law files of the reference (complab3d_symbolic.hh): read on the host,
// compiled into postfix programs (symbolic.cuh), bound to a handle's species, and evaluated in the
// fused transport step (ade.cu) or on demand (clb_symbolic_eval).
//
// The file format and its rules are the reference's: keywords version / units / vars / range /
// rate / reaction / yield / biomass, '#' comments, per_second or per_hour units, rate lines that may
// use earlier rate lines, a 'growth' line (an organism's specific growth rate) or an 'extent' line
// (an abiotic reaction's rate) and, with a 'reaction' line, the species lines derived from it
// (biotic: coefficient nu_i / |nu_key| / Y times growth times the organism's biomass; abiotic:
// nu_i times extent, each coefficient written with 10 significant digits as the reference writes
// it). The expression grammar: + - (left associative) below * / below unary +- below ^ (right
// associative, its exponent a unary), numbers, variables, the constants pi and e, the functions
// exp log log10 sqrt abs tanh (one argument) and min max pow (two).
#include "clb_internal.cuh"
#include "symbolic.cuh"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace clb {

namespace {

// ------------------------------------------------------------------ expression -> postfix
struct Emitter {
    SymProg& P;
    const std::vector<std::string>& scope;  // variables, then earlier rates
    std::string s, err;
    size_t p = 0;
    int depth = 0, max_depth = 0;

    Emitter(SymProg& prog, const std::vector<std::string>& names) : P(prog), scope(names) {}

    bool fail(const std::string& m) {
        if (err.empty()) err = m + " at character " + std::to_string(p + 1);
        return false;
    }
    void skip() {
        while (p < s.size() && (s[p] == ' ' || s[p] == '\t')) ++p;
    }
    bool emit(int op, int arg, int push) {
        if (P.n_ops >= SYM_MAX_OPS) return fail("the rate lines are too long for one program");
        P.op[P.n_ops] = (int16_t)op;
        P.arg[P.n_ops] = (int16_t)arg;
        ++P.n_ops;
        depth += push;
        if (depth > max_depth) max_depth = depth;
        if (max_depth > SYM_STACK) return fail("the expression nests too deeply");
        return true;
    }
    bool constant(double v) {
        // constants are shared by value across the program's rate lines
        size_t k = 0;
        for (; k < *ncst; ++k)
            if (P.cst[k] == v && std::signbit(P.cst[k]) == std::signbit(v)) break;
        if (k == *ncst) {
            if (k >= (size_t)SYM_MAX_CONST) return fail("too many numeric constants");
            P.cst[k] = v;
            ++*ncst;
        }
        return emit(SO_CONST, (int)k, +1);
    }
    size_t* ncst = nullptr;

    bool parse(const std::string& text) {
        s = text;
        p = 0;
        depth = 0;
        if (!expr()) return false;
        skip();
        if (p != s.size()) return fail("unexpected text after the expression");
        return true;
    }
    bool expr() {
        if (!term()) return false;
        for (;;) {
            skip();
            if (p < s.size() && (s[p] == '+' || s[p] == '-')) {
                const int op = s[p] == '+' ? SO_ADD : SO_SUB;
                ++p;
                if (!term() || !emit(op, 0, -1)) return false;
            } else {
                return true;
            }
        }
    }
    bool term() {
        if (!unary()) return false;
        for (;;) {
            skip();
            if (p < s.size() && (s[p] == '*' || s[p] == '/')) {
                const int op = s[p] == '*' ? SO_MUL : SO_DIV;
                ++p;
                if (!unary() || !emit(op, 0, -1)) return false;
            } else {
                return true;
            }
        }
    }
    bool unary() {
        skip();
        if (p < s.size() && s[p] == '-') {
            ++p;
            return unary() && emit(SO_NEG, 0, 0);
        }
        if (p < s.size() && s[p] == '+') {
            ++p;
            return unary();
        }
        return power();
    }
    bool power() {
        if (!atom()) return false;
        skip();
        if (p < s.size() && s[p] == '^') {
            ++p;
            return unary() && emit(SO_POW, 0, -1);
        }
        return true;
    }
    bool atom() {
        skip();
        if (p >= s.size()) return fail("expression ended early");
        if (s[p] == '(') {
            ++p;
            if (!expr()) return false;
            skip();
            if (p >= s.size() || s[p] != ')') return fail("missing ')'");
            ++p;
            return true;
        }
        if (std::isdigit((unsigned char)s[p]) || s[p] == '.') {
            const char* b = s.c_str() + p;
            char* e = nullptr;
            const double v = std::strtod(b, &e);
            if (e == b) return fail("could not read a number");
            p += (size_t)(e - b);
            return constant(v);
        }
        if (std::isalpha((unsigned char)s[p]) || s[p] == '_') {
            const size_t st = p;
            while (p < s.size() && (std::isalnum((unsigned char)s[p]) || s[p] == '_')) ++p;
            const std::string id = s.substr(st, p - st);
            skip();
            if (p < s.size() && s[p] == '(') {
                ++p;
                const bool two = id == "min" || id == "max" || id == "pow";
                if (!expr()) return false;
                if (two) {
                    skip();
                    if (p >= s.size() || s[p] != ',') return fail("'" + id + "' takes two arguments");
                    ++p;
                    if (!expr()) return false;
                }
                skip();
                if (p >= s.size() || s[p] != ')') return fail("missing ')' after '" + id + "'");
                ++p;
                static const struct { const char* n; int op; } fn[] = {
                    {"exp", SO_EXP}, {"log", SO_LOG}, {"log10", SO_LOG10}, {"sqrt", SO_SQRT}, {"abs", SO_ABS},
                    {"tanh", SO_TANH}, {"min", SO_MIN}, {"max", SO_MAX}, {"pow", SO_POW}};
                for (const auto& f : fn)
                    if (id == f.n) return emit(f.op, 0, two ? -1 : 0);
                return fail("unknown function '" + id + "'");
            }
            if (id == "pi") return constant(3.14159265358979323846);
            if (id == "e") return constant(2.71828182845904523536);
            for (size_t i = 0; i < scope.size(); ++i)
                if (scope[i] == id) return emit(SO_VAR, (int)i, +1);
            return fail("'" + id + "' is not one of the declared variables");
        }
        return fail("unexpected character");
    }
};

std::string lower(std::string t) {
    for (char& ch : t) ch = (char)std::tolower((unsigned char)ch);
    return t;
}

std::vector<std::string> words(const std::string& t) {
    std::istringstream in(t);
    std::vector<std::string> w;
    std::string x;
    while (in >> x) w.push_back(x);
    return w;
}

}  // namespace

// A program read from `path`: the rate names in order, the variable names. Returns an empty string,
// or the reason the file was refused.
std::string sym_compile(const char* path, SymProg& P, std::vector<std::string>& vars, std::vector<std::string>& rates) {
    std::memset(&P, 0, sizeof P);
    P.unit = 1.0;
    vars.clear();
    rates.clear();
    std::ifstream f(path);
    if (!f) return std::string("cannot open '") + path + "'";
    std::vector<std::pair<std::string, double>> stoich;
    std::string yield_of, biomass;
    double yield = 0.0;
    bool saw_vars = false;
    size_t ncst = 0;
    std::vector<double> lo, hi;
    std::string line;
    int no = 0;
    auto add_rate = [&](const std::string& name, const std::string& ex) -> std::string {
        if (P.n_rates >= SYM_MAX_RATES) return "more rate lines than " + std::to_string(SYM_MAX_RATES);
        std::vector<std::string> scope = vars;
        scope.insert(scope.end(), rates.begin(), rates.end());
        Emitter E(P, scope);
        E.ncst = &ncst;
        if (!E.parse(ex)) return E.err;
        rates.push_back(name);
        P.rate_end[P.n_rates++] = (int16_t)P.n_ops;
        return "";
    };
    while (std::getline(f, line)) {
        ++no;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        while (!line.empty() && (line.back() == '\r' || line.back() == '\n')) line.pop_back();
        size_t i = 0;
        while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
        if (i >= line.size()) continue;
        size_t j = i;
        while (j < line.size() && !std::isspace((unsigned char)line[j])) ++j;
        const std::string key = line.substr(i, j - i), rest = line.substr(j);
        const std::string where = std::string("'") + path + "' line " + std::to_string(no) + ": ";
        const std::vector<std::string> w = words(rest);
        if (key == "version") continue;
        if (key == "units") {
            if (w.empty()) return where + "'units' names nothing";
            const std::string u = lower(w[0]);
            if (u == "per_second" || u == "per_sec" || u == "s") P.unit = 1.0;
            else if (u == "per_hour" || u == "per_hr" || u == "h") P.unit = 1.0 / 3600.0;
            else return where + "'units' must be per_second or per_hour, not '" + u + "'";
        } else if (key == "vars") {
            if (w.empty()) return where + "'vars' names nothing";
            if (w.size() > (size_t)SYM_MAX_VARS) return where + "more than " + std::to_string(SYM_MAX_VARS) + " variables";
            vars = w;
            lo.assign(vars.size(), 0.0);
            hi.assign(vars.size(), -1.0);
            saw_vars = true;
        } else if (key == "range") {
            if (!saw_vars) return where + "'range' appears before 'vars'";
            double a = 0, b = 0;
            char nm[256];
            if (std::sscanf(rest.c_str(), "%255s %lf %lf", nm, &a, &b) != 3)
                return where + "'range' needs a name, a low value and a high value";
            int vi = -1;
            for (size_t k = 0; k < vars.size(); ++k)
                if (vars[k] == nm) vi = (int)k;
            if (vi < 0) return where + "'" + nm + "' is not in the vars line";
            if (!(b > a)) return where + "range high must exceed range low";
            lo[vi] = a;
            hi[vi] = b;
        } else if (key == "rate") {
            if (!saw_vars) return where + "'rate' appears before 'vars'";
            const size_t eq = rest.find('=');
            if (eq == std::string::npos) return where + "a rate line needs '='";
            const std::vector<std::string> nw = words(rest.substr(0, eq));
            if (nw.size() != 1) return where + "the rate has no name";
            for (const std::string& r : rates)
                if (r == nw[0]) return where + "'" + nw[0] + "' is defined twice";
            const std::string e = add_rate(nw[0], rest.substr(eq + 1));
            if (!e.empty()) return where + e;
        } else if (key == "reaction") {
            if (!saw_vars) return where + "'reaction' appears before 'vars'";
            if (w.empty() || w.size() % 2) return where + "write the reaction in pairs: reaction acetate -1  o2 -2";
            for (size_t k = 0; k < w.size(); k += 2) {
                char* e = nullptr;
                const double nu = std::strtod(w[k + 1].c_str(), &e);
                if (e == w[k + 1].c_str() || *e) return where + "'" + w[k + 1] + "' is not a number";
                if (nu == 0.0) return where + "'" + w[k] + "' has coefficient 0";
                bool known = false;
                for (const std::string& v : vars) known |= v == w[k];
                if (!known) return where + "'" + w[k] + "' is not in the vars line";
                for (const auto& t : stoich)
                    if (t.first == w[k]) return where + "'" + w[k] + "' appears twice in the reaction";
                stoich.push_back({w[k], nu});
            }
        } else if (key == "yield") {
            if (w.size() < 2) return where + "'yield' needs a species and a number";
            yield_of = w[0];
            yield = std::strtod(w[1].c_str(), nullptr);
            if (!(yield > 0.0)) return where + "the yield must be positive";
        } else if (key == "biomass") {
            if (w.empty()) return where + "'biomass' names nothing";
            biomass = w[0];
        } else {
            return where + "unknown keyword '" + key + "'";
        }
    }
    if (!saw_vars) return std::string("'") + path + "' has no 'vars' line";
    auto has = [&](const char* n) {
        for (const std::string& r : rates)
            if (r == n) return true;
        return false;
    };
    const bool growth = has("growth"), extent = has("extent");
    const std::string ctx = std::string("'") + path + "': ";
    if (growth && extent) return ctx + "the file has both a 'growth' line and an 'extent' line";
    if (extent && stoich.empty()) return ctx + "there is an 'extent' line but no 'reaction' line";
    if (!stoich.empty()) {
        for (const auto& t : stoich)
            if (has(t.first.c_str())) return ctx + "'" + t.first + "' has both a 'rate' line and a place in the 'reaction' line";
        char buf[256];
        if (extent) {
            if (!yield_of.empty() || !biomass.empty())
                return ctx + "an 'extent' line makes this an abiotic law: a 'yield' or 'biomass' line has nothing to apply to";
            for (const auto& t : stoich) {
                std::snprintf(buf, sizeof buf, "%.10g * extent", t.second);
                const std::string e = add_rate(t.first, buf);
                if (!e.empty()) return ctx + e;
            }
        } else {
            if (yield_of.empty()) return ctx + "a 'reaction' line needs a 'yield' line to go with it";
            if (biomass.empty()) return ctx + "a 'reaction' line needs a 'biomass' line";
            bool bv = false;
            for (const std::string& v : vars) bv |= v == biomass;
            if (!bv) return ctx + "'biomass " + biomass + "' is not in the vars line";
            if (!growth) return ctx + "a 'reaction' line needs either a 'growth' or an 'extent' rate line";
            double nu_key = 0.0;
            for (const auto& t : stoich)
                if (t.first == yield_of) nu_key = t.second;
            if (nu_key == 0.0) return ctx + "the yield is quoted against '" + yield_of + "', which is not in the reaction line";
            const double mag = nu_key < 0 ? -nu_key : nu_key;
            for (const auto& t : stoich) {
                std::snprintf(buf, sizeof buf, "%.10g * growth * %s", (t.second / mag) / yield, biomass.c_str());
                const std::string e = add_rate(t.first, buf);
                if (!e.empty()) return ctx + e;
            }
        }
    } else if (!yield_of.empty() || !biomass.empty()) {
        return ctx + "'yield' or 'biomass' was given with no 'reaction' line";
    }
    if (rates.empty()) return std::string("'") + path + "' defines no rates";
    P.n_vars = (int)vars.size();
    P.kind = extent ? 1 : 0;
    for (int i = 0; i < P.n_vars; ++i) {
        P.lo[i] = lo[i];
        P.hi[i] = hi[i];
    }
    return "";
}

// ------------------------------------------------------------------ binding and the entry points

static std::string user_name(const char* const* names, int s) { return names && names[s] ? names[s] : ""; }

clb_status symbolic_set(clb_handle* h, const char* path, const char* const* species_names, int microbe,
                        const char* microbe_name) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (!path || !species_names) return fail(h, CLB_INVALID_ARG, "null argument");
    if (microbe < -1 || microbe >= CLB_MAX_MICROBES) return fail(h, CLB_INVALID_ARG, "microbe index out of range");
    SymProg P;
    std::vector<std::string> vars, rates;
    const std::string e = sym_compile(path, P, vars, rates);
    if (!e.empty()) return fail(h, CLB_INVALID_ARG, e);
    const bool abiotic = microbe < 0;
    if (abiotic != (P.kind == 1))
        return fail(h, CLB_INVALID_ARG, abiotic ? "an abiotic law needs an 'extent' line, not 'growth'"
                                                : "an organism's law needs a 'growth' line; an 'extent' line is abiotic");
    const std::string mname = microbe_name ? microbe_name : "";
    for (int v = 0; v < P.n_vars; ++v) {
        int hit = -2;
        for (int s = 0; s < h->S; ++s)
            if (user_name(species_names, s) == vars[v]) hit = h->u2i[s];
        if (hit == -2 && !abiotic && !mname.empty() && vars[v] == mname) hit = -1;
        if (hit == -2)
            return fail(h, CLB_INVALID_ARG, "the file uses variable '" + vars[v] + "', which is neither a substrate" +
                                                (abiotic ? std::string() : " nor the microbe '" + mname + "'"));
        P.var_src[v] = hit;
    }
    for (int r = 0; r < P.n_rates; ++r) {
        if (rates[r] == "growth" || rates[r] == "extent") {
            P.rate_dst[r] = -1;
            continue;
        }
        int hit = -2;
        for (int s = 0; s < h->S; ++s)
            if (user_name(species_names, s) == rates[r]) hit = h->u2i[s];
        if (hit == -2) return fail(h, CLB_INVALID_ARG, "the file defines a rate for '" + rates[r] + "', which is not a substrate");
        P.rate_dst[r] = hit;
    }
    if (!h->d_sym) {
        cudaError_t err = cudaMalloc(&h->d_sym, sizeof(SymProg) * SYM_MAX_PROGS);
        if (err != cudaSuccess) return cuda_check(h, err, "rate-law programs");
    }
    const int slot = abiotic ? CLB_MAX_MICROBES : microbe;
    cudaError_t err = cudaMemcpy(static_cast<SymProg*>(h->d_sym) + slot, &P, sizeof P, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_check(h, err, "rate-law program");
    h->sym_host[slot] = P;
    AdeParams& A = h->ap;
    A.sym = static_cast<const SymProg*>(h->d_sym);
    if (abiotic) {
        A.law2 = CLB_LAW_SYMBOLIC;
        A.gnn_abiotic = 0;
    } else {
        A.law = CLB_LAW_SYMBOLIC;
        A.sym_mask |= 1u << microbe;
        A.gnn_mask &= ~(1u << microbe);  // an organism has one run-time law
        A.srg_mask &= ~(1u << microbe);
    }
    return geometry_refresh(h);
}

clb_status symbolic_eval(clb_handle* h, int which, const double* vars, int n, double* rates, int* n_rates) {
    const int slot = which < 0 ? CLB_MAX_MICROBES : which;
    if (which >= CLB_MAX_MICROBES || (which >= 0 && !(h->ap.sym_mask >> which & 1u)) ||
        (which < 0 && (h->ap.law2 != CLB_LAW_SYMBOLIC || h->ap.gnn_abiotic)))
        return fail(h, CLB_INVALID_ARG, "no rate-law file is bound there");
    const SymProg& P = h->sym_host[slot];
    if (n_rates) *n_rates = P.n_rates;
    if (n <= 0) return CLB_OK;
    double *dv = nullptr, *dr = nullptr;
    cudaError_t e = cudaMalloc(&dv, sizeof(double) * (size_t)n * P.n_vars);
    if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(double) * (size_t)n * P.n_rates);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dv, vars, sizeof(double) * (size_t)n * P.n_vars, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        sym_eval_batch(h, slot, dv, n, dr);
        e = cudaMemcpyAsync(rates, dr, sizeof(double) * (size_t)n * P.n_rates, cudaMemcpyDeviceToHost, h->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dv);
    cudaFree(dr);
    return cuda_check(h, e, "rate-law evaluation");
}

__global__ void k_sym_eval(const SymProg* __restrict__ progs, int slot, const double* __restrict__ vars, int n,
                           double* __restrict__ out) {
    const SymProg& P = progs[slot];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x[SYM_MAX_VARS], y[SYM_MAX_RATES];
        for (int v = 0; v < P.n_vars; ++v) x[v] = vars[(int64_t)i * P.n_vars + v];
        sym_eval(P, x, y);
        for (int r = 0; r < P.n_rates; ++r) out[(int64_t)i * P.n_rates + r] = y[r];
    }
}

void sym_eval_batch(clb_handle* h, int slot, const double* dvars, int n, double* drates) {
    ++h->launches;
    k_sym_eval<<<std::max(1, std::min(h->num_sms * 4, (n + 127) / 128)), 128, 0, h->stream>>>(
        static_cast<const SymProg*>(h->d_sym), slot, dvars, n, drates);
}

}  // namespace clb

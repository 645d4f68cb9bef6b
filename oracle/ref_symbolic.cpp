// Thin C entry points around the reference's own run-time rate-law reader and evaluator
// (complab3d_symbolic.hh: the .sym file loader with its derived reaction lines, and evaluate()
// with the range clamp and the unit scale), compiled from the reference sources where they lie
// (Makefile target `ref`). TEST INFRASTRUCTURE ONLY: used to pin the oracle's restatement and
// the GPU interpreter of the same language to the reference's values.
#include "complab3d_symbolic.hh"

#include <cstring>
#include <string>
#include <vector>

// Loads `path`; returns 0 and the variable and rate counts and the rate names (space separated in
// names, at most names_len bytes), or -1 with the reference's message in names.
extern "C" int ref_sym_info(const char* path, int* n_vars, int* n_rates, char* names, int names_len) {
    complab_sym::Program P;
    std::string err;
    if (!complab_sym::load(P, path, &err)) {
        std::strncpy(names, err.c_str(), (size_t)names_len - 1);
        names[names_len - 1] = 0;
        return -1;
    }
    *n_vars = (int)P.vars.size();
    *n_rates = (int)P.rates.size();
    std::string s;
    for (const auto& r : P.rates) s += (s.empty() ? "" : " ") + r.name;
    std::strncpy(names, s.c_str(), (size_t)names_len - 1);
    names[names_len - 1] = 0;
    return 0;
}

// evaluate() (clamped to the file's ranges) of n rows of variable values [n][n_vars] into
// out [n][n_rates]; clamped receives the number of rows the range clamp changed.
extern "C" int ref_sym_eval(const char* path, int n, const double* vars, double* out, long* clamped) {
    complab_sym::Program P;
    std::string err;
    if (!complab_sym::load(P, path, &err)) return -1;
    const size_t nv = P.vars.size(), nr = P.rates.size();
    std::vector<double> v(nv), o;
    long c = 0;
    for (int i = 0; i < n; ++i) {
        v.assign(vars + (size_t)i * nv, vars + (size_t)(i + 1) * nv);
        complab_sym::evaluate(P, v, o, true, &c);
        for (size_t r = 0; r < nr; ++r) out[(size_t)i * nr + r] = o[r];
    }
    *clamped = c;
    return 0;
}

// Thin C entry points around the reference's own graph-network reader and evaluator
// (complab3d_graphnet.hh: load() of the .gnn file and Network::eval() with the training-box clamp
// and the unit scale), compiled from the reference sources where they lie (Makefile target `ref`).
// TEST INFRASTRUCTURE ONLY: used to pin the oracle's restatement and the GPU evaluator of the same
// networks to the reference's values.
#include "complab3d_graphnet.hh"

#include <cstring>
#include <string>
#include <vector>

// Loads `path`; returns 0 with the species count and the output count (species rates, then growth),
// or -1 with the reference's message in msg.
extern "C" int ref_gnn_info(const char* path, int* n_species, int* n_out, char* msg, int msg_len) {
    complab_gnn::Network N;
    std::string err;
    if (!complab_gnn::load(N, path, &err)) {
        std::strncpy(msg, err.c_str(), (size_t)msg_len - 1);
        msg[msg_len - 1] = 0;
        return -1;
    }
    *n_species = N.nS;
    *n_out = N.nOut();
    msg[0] = 0;
    return 0;
}

// eval() with the clamp of n rows of concentrations [n][nS] into out [n][nOut]; clamped receives the
// number of rows the clamp changed.
extern "C" int ref_gnn_eval(const char* path, int n, const double* conc, double* out, long* clamped) {
    complab_gnn::Network N;
    std::string err;
    if (!complab_gnn::load(N, path, &err)) return -1;
    const size_t ns = (size_t)N.nS, no = (size_t)N.nOut();
    std::vector<double> c, o;
    complab_gnn::Network::Scratch sc;
    long k = 0;
    for (int i = 0; i < n; ++i) {
        c.assign(conc + (size_t)i * ns, conc + (size_t)(i + 1) * ns);
        N.eval(c, o, sc, true, &k);
        for (size_t j = 0; j < no; ++j) out[(size_t)i * no + j] = o[j];
    }
    *clamped = k;
    return 0;
}

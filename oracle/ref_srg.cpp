// Thin C entry points around the reference's own surrogate-network reader and evaluator
// (complab3d_surrogate.hh: load() of the .srg file, Network::evalAll()), compiled from the reference
// sources where they lie (Makefile target `ref`). TEST INFRASTRUCTURE ONLY: used to pin the oracle's
// restatement and the GPU evaluator of the same networks to the reference's values.
#include "complab3d_surrogate.hh"

#include <cstring>
#include <string>
#include <vector>

// Loads `path`; returns 0 with the input and output counts, or -1 with the reference's message.
extern "C" int ref_srg_info(const char* path, int* n_in, int* n_out, char* msg, int msg_len) {
    complab_srg::Network N;
    std::string err;
    if (!complab_srg::load(N, path, &err)) {
        std::strncpy(msg, err.c_str(), (size_t)msg_len - 1);
        msg[msg_len - 1] = 0;
        return -1;
    }
    *n_in = N.nIn;
    *n_out = N.nOut();
    msg[0] = 0;
    return 0;
}

// evalAll() of n rows [n][nIn] into out [n][nOut]; with clamp != 0 each input is first held to the
// training box as evalBound() holds it (clamped receives the rows it changed).
extern "C" int ref_srg_eval(const char* path, int n, const double* x, int clamp, double* out, long* clamped) {
    complab_srg::Network N;
    std::string err;
    if (!complab_srg::load(N, path, &err)) return -1;
    const size_t ni = (size_t)N.nIn, no = (size_t)N.nOut();
    std::vector<double> v, o;
    long k = 0;
    for (int i = 0; i < n; ++i) {
        v.assign(x + (size_t)i * ni, x + (size_t)(i + 1) * ni);
        bool outside = false;
        if (clamp)
            for (size_t j = 0; j < ni; ++j) {
                if (v[j] < N.trainMin[j]) { v[j] = N.trainMin[j]; outside = true; }
                else if (v[j] > N.trainMax[j]) { v[j] = N.trainMax[j]; outside = true; }
            }
        k += outside ? 1 : 0;
        N.evalAll(v, o);
        for (size_t j = 0; j < no; ++j) out[(size_t)i * no + j] = o[j];
    }
    *clamped = k;
    return 0;
}

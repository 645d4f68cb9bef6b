// srgnet.cu -- surrogate organisms (srgnet.cuh): the reference's .srg network files
// (complab3d_surrogate.hh) read on the host, bound to an organism of a handle with its uptake
// parameters, and evaluated in the fused transport step (ade.cu, under the run-time laws' shared
// budget) or on demand (clb_surrogate_eval).
//
// The file format is the reference's: '#' comments to the end of the line; `version`, `inputs n`,
// `layers n h1 ... out` (the rest of the line), `logoutput 0|1`, `inputnames` and `outputnames`
// (names on the rest of the line), `xoffset` / `xgain` / `trainmin` / `trainmax` (one per input),
// `xymin`, `outputs n`, `yoffset` / `ygain` (one per output; the missing ones read 0 and 1),
// `yymin`, `outrange` (pairs on the rest of the line, not used here), then `W l` (rows x cols, row
// major) and `B l` per layer. A file whose layers are incomplete, whose declared outputs disagree
// with its last layer or that has no training box is refused.
#include "clb_internal.cuh"
#include "srgnet.cuh"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace clb {

namespace {

// token and line reading over the file's text
struct SrgText {
    std::string s;
    size_t p = 0;
    bool token(std::string& t) {
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
        if (p >= s.size()) return false;
        const size_t b = p;
        while (p < s.size() && !std::isspace((unsigned char)s[p])) ++p;
        t = s.substr(b, p - b);
        return true;
    }
    std::string line() {
        const size_t b = p;
        while (p < s.size() && s[p] != '\n') ++p;
        return s.substr(b, p - b);
    }
    bool num(double& v) {
        std::string t;
        if (!token(t)) return false;
        char* end = nullptr;
        v = std::strtod(t.c_str(), &end);
        return end && *end == 0 && end != t.c_str();
    }
};

std::vector<std::string> split_words(const std::string& l) {
    std::vector<std::string> w;
    std::istringstream in(l);
    std::string t;
    while (in >> t) w.push_back(t);
    return w;
}

// Reads `path` into N (input names into names); "" on success, else the reason.
std::string srg_read(const char* path, SrgNet& N, std::vector<std::string>& names) {
    std::ifstream f(path);
    if (!f) return std::string("cannot open '") + path + "'";
    std::stringstream ss;
    ss << f.rdbuf();
    SrgText T;
    T.s = ss.str();
    N = SrgNet();
    N.xymin = -1.0;
    N.yymin = -1.0;
    const std::string where = std::string("'") + path + "'";
    std::vector<int> sizes;
    std::vector<std::vector<double>> W, B;
    std::vector<double> xoff, xgain, tmin, tmax, yoff, ygain;
    int declared_out = 0, n_out_names = -1;
    auto read_n = [&](std::vector<double>& v, int n) {
        v.assign((size_t)std::max(n, 0), 0.0);
        for (auto& x : v)
            if (!T.num(x)) return false;
        return true;
    };
    std::string k;
    while (T.token(k)) {
        if (k[0] == '#') {
            T.line();
            continue;
        }
        bool ok = true;
        if (k == "version") {
            double v;
            ok = T.num(v);
        } else if (k == "inputs") {
            double v;
            ok = T.num(v);
            N.nIn = (int)v;
        } else if (k == "layers") {
            sizes.clear();
            for (const std::string& w : split_words(T.line())) sizes.push_back(std::atoi(w.c_str()));
        } else if (k == "logoutput") {
            double v;
            ok = T.num(v);
            N.logout = v != 0.0;
        } else if (k == "inputnames") {
            names = split_words(T.line());
        } else if (k == "outputnames") {
            n_out_names = (int)split_words(T.line()).size();
        } else if (k == "xoffset") ok = read_n(xoff, N.nIn);
        else if (k == "xgain") ok = read_n(xgain, N.nIn);
        else if (k == "trainmin") ok = read_n(tmin, N.nIn);
        else if (k == "trainmax") ok = read_n(tmax, N.nIn);
        else if (k == "xymin") ok = T.num(N.xymin);
        else if (k == "yymin") ok = T.num(N.yymin);
        else if (k == "outputs") {
            double v;
            ok = T.num(v);
            declared_out = (int)v;
        } else if (k == "yoffset" || k == "ygain") {
            std::vector<double> v;
            for (const std::string& w : split_words(T.line())) v.push_back(std::strtod(w.c_str(), nullptr));
            (k == "yoffset" ? yoff : ygain) = v;
        } else if (k == "outrange") {
            T.line();
        } else if (k == "W" || k == "B") {
            double lv;
            if (!T.num(lv)) return where + ": '" + k + "' needs a layer index";
            const int L = (int)lv;
            if (sizes.size() < 2 || L < 0 || L + 1 >= (int)sizes.size())
                return where + ": '" + k + " " + std::to_string(L) + "' outside the declared layers";
            if ((int)W.size() < L + 1) {
                W.resize((size_t)L + 1);
                B.resize((size_t)L + 1);
            }
            const int rows = sizes[(size_t)L + 1], cols = sizes[(size_t)L];
            if (!read_n(k == "W" ? W[(size_t)L] : B[(size_t)L], k == "W" ? rows * cols : rows))
                return where + " is truncated: not enough numbers for layer " + std::to_string(L);
        } else {
            return where + ": unknown keyword '" + k + "'";
        }
        if (!ok) return where + ": '" + k + "' is short or not numeric";
    }
    const int nL = (int)sizes.size() - 1;
    bool valid = N.nIn > 0 && nL >= 1 && sizes[0] == N.nIn && (int)W.size() == nL && (int)B.size() == nL;
    for (int l = 0; valid && l < nL; ++l)
        valid = (int)W[(size_t)l].size() == sizes[(size_t)l + 1] * sizes[(size_t)l] &&
                (int)B[(size_t)l].size() == sizes[(size_t)l + 1];
    if (!valid) return where + " is not a usable surrogate file";
    if (N.nIn > SRG_MAX_IN || nL > SRG_MAX_LAYERS ||
        *std::max_element(sizes.begin(), sizes.end()) > SRG_MAX_W)
        return where + ": the network exceeds what this library evaluates (" + std::to_string(SRG_MAX_IN) +
               " inputs, " + std::to_string(SRG_MAX_LAYERS) + " layers, " + std::to_string(SRG_MAX_W) +
               " units a layer)";
    const int nO = sizes.back();
    if (declared_out > 0 && declared_out != nO)
        return where + " declares outputs " + std::to_string(declared_out) + " but its last layer has " +
               std::to_string(nO);
    if (n_out_names >= 0 && n_out_names != nO)
        return where + " names " + std::to_string(n_out_names) + " output(s) but returns " + std::to_string(nO);
    const char* missing = nullptr;
    if ((int)tmin.size() < N.nIn) missing = "trainmin";
    else if ((int)tmax.size() < N.nIn) missing = "trainmax";
    else if ((int)xoff.size() < N.nIn) missing = "xoffset";
    else if ((int)xgain.size() < N.nIn) missing = "xgain";
    if (missing)
        return where + " has no complete '" + missing + "' line, so the range it was fitted over is unknown";
    N.nL = nL;
    for (int l = 0; l <= nL; ++l) N.sizes[l] = sizes[(size_t)l];
    for (int i = 0; i < N.nIn; ++i) {
        N.xoff[i] = xoff[(size_t)i];
        N.xgain[i] = xgain[(size_t)i];
        N.tmin[i] = tmin[(size_t)i];
        N.tmax[i] = tmax[(size_t)i];
    }
    for (int o = 0; o < nO; ++o) {
        N.yoff[o] = o < (int)yoff.size() ? yoff[(size_t)o] : 0.0;
        N.ygain[o] = o < (int)ygain.size() ? ygain[(size_t)o] : 1.0;
    }
    for (int l = 0; l < nL; ++l) {
        std::copy(W[(size_t)l].begin(), W[(size_t)l].end(), N.W[l]);
        std::copy(B[(size_t)l].begin(), B[(size_t)l].end(), N.B[l]);
    }
    return "";
}

std::string user_name(const char* const* names, int s) { return names && names[s] ? names[s] : ""; }

}  // namespace

clb_status srg_set(clb_handle* h, const char* path, const char* const* species_names, int microbe,
                   const clb_surrogate_desc* d) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (!path || !species_names || !d) return fail(h, CLB_INVALID_ARG, "null argument");
    if (microbe < 0 || microbe >= CLB_MAX_MICROBES)
        return fail(h, CLB_INVALID_ARG, "a surrogate belongs to an organism: microbe index out of range");
    if (!(d->biomass_molar_mass > 0)) return fail(h, CLB_INVALID_ARG, "biomass_molar_mass must be positive");
    SrgNet N;
    std::vector<std::string> names;
    const std::string e = srg_read(path, N, names);
    if (!e.empty()) return fail(h, CLB_INVALID_ARG, e);
    // inputs by name (inputnames); a file without names feeds the substrates in order
    for (int i = 0; i < N.nIn; ++i) {
        int hit = -1;
        if (!names.empty()) {
            if ((int)names.size() != N.nIn)
                return fail(h, CLB_INVALID_ARG, "the file names " + std::to_string(names.size()) +
                                                    " inputs but has " + std::to_string(N.nIn));
            for (int s = 0; s < h->S && hit < 0; ++s)
                if (user_name(species_names, s) == names[(size_t)i]) hit = h->u2i[s];
            if (hit < 0)
                return fail(h, CLB_INVALID_ARG,
                            "the network's input '" + names[(size_t)i] + "' is not one of the handle's species");
        } else {
            if (i >= h->S) return fail(h, CLB_INVALID_ARG, "the network has more inputs than the handle has species");
            hit = h->u2i[i];
        }
        N.subs[i] = hit;
    }
    for (int s = 0; s < h->S; ++s) {
        N.kc[h->u2i[s]] = d->half_saturation[s];
        N.vmax[h->u2i[s]] = d->max_uptake_flux[s];
    }
    N.mw = d->biomass_molar_mass;
    N.kd = d->decay;
    if (!h->d_srg) {
        cudaError_t err = cudaMalloc(&h->d_srg, sizeof(SrgNet) * CLB_MAX_MICROBES);
        if (err != cudaSuccess) return cuda_check(h, err, "surrogate networks");
    }
    cudaError_t err = cudaMemcpy(static_cast<SrgNet*>(h->d_srg) + microbe, &N, sizeof N, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_check(h, err, "surrogate network");
    if (!h->srg_host) h->srg_host = new SrgNet[CLB_MAX_MICROBES];
    h->srg_host[microbe] = N;
    AdeParams& A = h->ap;
    A.srg = static_cast<const SrgNet*>(h->d_srg);
    A.law = CLB_LAW_SYMBOLIC;
    A.srg_mask |= 1u << microbe;
    A.sym_mask &= ~(1u << microbe);  // an organism has one run-time law
    A.gnn_mask &= ~(1u << microbe);
    return geometry_refresh(h);
}

__global__ void k_srg_eval(const SrgNet* __restrict__ nets, int slot, const double* __restrict__ x, int n,
                           double* __restrict__ out, unsigned int* __restrict__ clamped) {
    const SrgNet& N = nets[slot];
    const int nO = N.sizes[N.nL];
    unsigned int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double xi[SRG_MAX_IN], y[SRG_MAX_W];
        for (int k = 0; k < N.nIn; ++k) xi[k] = x[(int64_t)i * N.nIn + k];
        c += srg_eval(N, xi, y) ? 1u : 0u;
        for (int o = 0; o < nO; ++o) out[(int64_t)i * nO + o] = y[o];
    }
    if (c) atomicAdd(clamped, c);
}

clb_status srg_eval_host(clb_handle* h, int microbe, const double* x, int n, double* out, int* n_out,
                         long* n_clamped) {
    if (microbe < 0 || microbe >= CLB_MAX_MICROBES || !(h->ap.srg_mask >> microbe & 1u))
        return fail(h, CLB_INVALID_ARG, "no surrogate network is bound there");
    const SrgNet& N = h->srg_host[microbe];
    const int nO = N.sizes[N.nL];
    if (n_out) *n_out = nO;
    if (n_clamped) *n_clamped = 0;
    if (n <= 0) return CLB_OK;
    double *dx = nullptr, *dout = nullptr;
    unsigned int* dcl = nullptr;
    cudaError_t e = cudaMalloc(&dx, sizeof(double) * (size_t)n * N.nIn);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * (size_t)n * nO);
    if (e == cudaSuccess) e = cudaMalloc(&dcl, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(dcl, 0, sizeof(unsigned int), h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, sizeof(double) * (size_t)n * N.nIn, cudaMemcpyHostToDevice, h->stream);
    unsigned int cl = 0;
    if (e == cudaSuccess) {
        ++h->launches;
        k_srg_eval<<<std::max(1, std::min(h->num_sms * 4, (n + 127) / 128)), 128, 0, h->stream>>>(
            static_cast<const SrgNet*>(h->d_srg), microbe, dx, n, dout, dcl);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(double) * (size_t)n * nO, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&cl, dcl, sizeof cl, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dx);
    cudaFree(dout);
    cudaFree(dcl);
    if (n_clamped) *n_clamped = (long)cl;
    return cuda_check(h, e, "surrogate evaluation");
}

}  // namespace clb

// graphnet.cu -- the reference's .gnn graph-network rate laws (complab3d_graphnet.hh): read on the
// host into a GnnNet (graphnet.cuh), bound to a handle's species, and evaluated in the fused
// transport step (ade.cu, with the .sym laws' budget rules) or on demand (clb_graph_network_eval).
//
// The file format is the reference's: whitespace-separated keywords, each followed by its numbers;
// '#' starts a comment to the end of the line; `provenance` takes the rest of its line, `species`
// and `reactions` the names on the rest of theirs; `version`, `units` (per_second or per_hour),
// `rounds`, `width`, `growth`, `readout` (species or extent) and the `stoich nS nR` block come
// first, then the per-species, per-reaction and per-layer arrays (`da`, `xoffset`, `xgain`,
// `xymin`, `yoffset`, `ygain`, `xiscale`, `yymin`, `trainmin`, `trainmax`, `Wenc`, `benc`,
// `layer l` followed by its `Wsr` `Wss` `Wrs` `Wda` `bR` `bS`, `Wout`, `bout`). Matrices are row
// major. A file that is incomplete, names an unknown keyword or has no training box is refused.
#include "clb_internal.cuh"
#include "graphnet.cuh"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace clb {

namespace {

// A cursor over the file's text with the two reading modes the format uses: the next
// whitespace-separated token, or the rest of the current line.
struct GnnText {
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
    std::string rest_of_line() {
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
    bool integer(int& v) {
        double d;
        if (!num(d) || d != (double)(int)d) return false;
        v = (int)d;
        return true;
    }
    bool nums(double* out, int n) {
        for (int i = 0; i < n; ++i)
            if (!num(out[i])) return false;
        return true;
    }
};

std::vector<std::string> words(const std::string& line) {
    std::vector<std::string> w;
    std::istringstream in(line);
    std::string t;
    while (in >> t) w.push_back(t);
    return w;
}

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Reads `path` into N (names into species); "" on success, else the reason.
std::string gnn_read(const char* path, GnnNet& N, std::vector<std::string>& species) {
    std::ifstream f(path);
    if (!f) return std::string("cannot open '") + path + "'";
    std::stringstream ss;
    ss << f.rdbuf();
    GnnText T;
    T.s = ss.str();
    N = GnnNet();
    N.unit = 1.0;
    N.xymin = -1.0;
    N.yymin = -1.0;
    bool shape = false;
    int cur = -1;
    // which arrays appeared (a network missing one is incomplete)
    bool got_da = false, got_xoff = false, got_xgain = false, got_yoff = false, got_ygain = false, got_xi = false;
    bool got_tmin = false, got_tmax = false, got_wenc = false, got_benc = false, got_wout = false, got_bout = false;
    bool layer_got[GNN_MAX_ROUNDS][6] = {};
    int n_species_names = -1;
    const std::string where = std::string("'") + path + "'";
    auto nyscale = [&]() { return N.extent ? (N.growth ? 1 : 0) : N.nS + (N.growth ? 1 : 0); };
    auto nhead = [&]() { return N.growth ? 2 : 1; };
    std::string k;
    while (T.token(k)) {
        if (k[0] == '#' || k == "provenance") {
            T.rest_of_line();
            continue;
        }
        if (k == "version") {
            int v;
            if (!T.integer(v)) return where + ": 'version' needs a number";
            continue;
        }
        if (k == "units") {
            std::string u;
            if (!T.token(u)) return where + ": 'units' needs a value";
            u = lower(u);
            if (u == "per_second") N.unit = 1.0;
            else if (u == "per_hour") N.unit = 1.0 / 3600.0;
            else return "'units' must be per_second or per_hour";
            continue;
        }
        if (k == "species" || k == "reactions") {
            const std::vector<std::string> w = words(T.rest_of_line());
            if (k == "species") {
                species = w;
                n_species_names = (int)w.size();
            }
            continue;
        }
        if (k == "rounds" || k == "width" || k == "growth") {
            int v;
            if (!T.integer(v)) return where + ": '" + k + "' needs an integer";
            if (k == "rounds") N.rounds = v;
            else if (k == "width") N.W = v;
            else N.growth = v != 0;
            continue;
        }
        if (k == "readout") {
            std::string m;
            if (!T.token(m)) return where + ": 'readout' needs a value";
            m = lower(m);
            if (m == "species") N.extent = 0;
            else if (m == "extent") N.extent = 1;
            else return "'readout' must be species or extent, not '" + m + "'";
            continue;
        }
        if (k == "stoich") {
            if (!T.integer(N.nS) || !T.integer(N.nR)) return where + ": 'stoich' needs nS and nR";
            if (N.nS < 1 || N.nR < 1) return where + ": 'stoich' needs at least one species and one reaction";
            if (N.nS > GNN_MAX_S || N.nR > GNN_MAX_R)
                return where + ": the network has " + std::to_string(N.nS) + " species and " + std::to_string(N.nR) +
                       " reactions; this library evaluates networks of up to " + std::to_string(GNN_MAX_S) +
                       " species and " + std::to_string(GNN_MAX_R) + " reactions";
            for (int i = 0; i < N.nS; ++i)
                for (int r = 0; r < N.nR; ++r)
                    if (!T.num(N.S[i * GNN_MAX_R + r])) return where + ": the stoich block is short";
            shape = true;
            continue;
        }
        if (!shape) return where + ": '" + k + "' appears before the stoich block";
        const bool sized = k == "Wenc" || k == "benc" || k == "layer" || k == "Wsr" || k == "Wss" || k == "Wrs" ||
                           k == "Wda" || k == "bR" || k == "bS" || k == "Wout";
        if (sized && (N.W < 1 || N.W > GNN_MAX_W))
            return where + ": width " + std::to_string(N.W) + " (declared before the weights) must be 1.." +
                   std::to_string(GNN_MAX_W) + " for this library";
        if (k == "layer" && (N.rounds < 1 || N.rounds > GNN_MAX_ROUNDS))
            return where + ": rounds " + std::to_string(N.rounds) + " (declared before the layers) must be 1.." +
                   std::to_string(GNN_MAX_ROUNDS) + " for this library";
        bool ok = true;
        if (k == "da") ok = got_da = T.nums(N.da, N.nR);
        else if (k == "xoffset") ok = got_xoff = T.nums(N.xoff, N.nS);
        else if (k == "xgain") ok = got_xgain = T.nums(N.xgain, N.nS);
        else if (k == "xymin") ok = T.num(N.xymin);
        else if (k == "yoffset") ok = got_yoff = T.nums(N.yoff, nyscale());
        else if (k == "ygain") ok = got_ygain = T.nums(N.ygain, nyscale());
        else if (k == "xiscale") ok = got_xi = T.nums(N.xiscale, N.nR);
        else if (k == "yymin") ok = T.num(N.yymin);
        else if (k == "trainmin") ok = got_tmin = T.nums(N.tmin, N.nS);
        else if (k == "trainmax") ok = got_tmax = T.nums(N.tmax, N.nS);
        else if (k == "Wenc") ok = got_wenc = T.nums(N.Wenc, N.W);
        else if (k == "benc") ok = got_benc = T.nums(N.benc, N.W);
        else if (k == "layer") {
            ok = T.integer(cur) && cur >= 0 && cur < N.rounds;
            if (!ok) return where + ": a 'layer' index outside 0.." + std::to_string(N.rounds - 1);
        } else if (k == "Wsr" || k == "Wss" || k == "Wrs" || k == "Wda" || k == "bR" || k == "bS") {
            if (cur < 0) return where + ": '" + k + "' outside any layer block";
            GnnLayer& L = N.layer[cur];
            const int W = N.W;
            auto mat = [&](double* a, int slot) {
                for (int h = 0; h < W; ++h)
                    for (int j = 0; j < W; ++j)
                        if (!T.num(a[h * GNN_MAX_W + j])) return false;
                layer_got[cur][slot] = true;
                return true;
            };
            if (k == "Wsr") ok = mat(L.Wsr, 0);
            else if (k == "Wss") ok = mat(L.Wss, 1);
            else if (k == "Wrs") ok = mat(L.Wrs, 2);
            else if (k == "Wda") ok = layer_got[cur][3] = T.nums(L.Wda, W);
            else if (k == "bR") ok = layer_got[cur][4] = T.nums(L.bR, W);
            else ok = layer_got[cur][5] = T.nums(L.bS, W);
        } else if (k == "Wout") {
            ok = true;
            for (int o = 0; o < nhead() && ok; ++o) ok = T.nums(N.Wout + o * GNN_MAX_W, N.W);
            got_wout = ok;
        } else if (k == "bout") {
            ok = got_bout = T.nums(N.bout, nhead());
        } else {
            return where + ": unknown keyword '" + k + "'";
        }
        if (!ok) return where + ": '" + k + "' is short or not numeric";
    }
    bool complete = shape && N.W >= 1 && N.rounds >= 1 && N.rounds <= GNN_MAX_ROUNDS && got_da && got_xoff && got_xgain && got_tmin && got_tmax && got_wenc && got_benc &&
                    got_wout && got_bout && (N.extent ? got_xi : true) &&
                    (nyscale() == 0 || (got_yoff && got_ygain));
    for (int l = 0; l < N.rounds && complete; ++l)
        for (int j = 0; j < 6; ++j) complete = complete && layer_got[l][j];
    if (!complete)
        return where + " is incomplete or inconsistent: it should declare stoich, rounds, width, one layer block per "
                       "round, Wenc/benc, Wout/bout, the scalings and trainmin/trainmax";
    if (n_species_names != N.nS)
        return "the file names " + std::to_string(std::max(0, n_species_names)) + " species but declares " +
               std::to_string(N.nS) + ".";
    return "";
}

std::string user_name(const char* const* names, int s) { return names && names[s] ? names[s] : ""; }

}  // namespace

clb_status graphnet_set(clb_handle* h, const char* path, const char* const* species_names, int microbe) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (!path || !species_names) return fail(h, CLB_INVALID_ARG, "null argument");
    if (microbe < -1 || microbe >= CLB_MAX_MICROBES) return fail(h, CLB_INVALID_ARG, "microbe index out of range");
    GnnNet N;
    std::vector<std::string> names;
    const std::string e = gnn_read(path, N, names);
    if (!e.empty()) return fail(h, CLB_INVALID_ARG, e);
    const bool abiotic = microbe < 0;
    if (abiotic && N.growth)
        return fail(h, CLB_INVALID_ARG,
                    "the abiotic network declares a growth output; an abiotic network belongs to no organism, so "
                    "there is no biomass for it to apply to");
    for (int i = 0; i < N.nS; ++i) {
        int hit = -1;
        for (int s = 0; s < h->S && hit < 0; ++s)
            if (user_name(species_names, s) == names[i]) hit = h->u2i[s];
        if (hit < 0)
            return fail(h, CLB_INVALID_ARG,
                        "the network was trained on species '" + names[i] + "', which is not one of the handle's species");
        N.sp[i] = hit;
    }
    if (!h->d_gnn) {
        cudaError_t err = cudaMalloc(&h->d_gnn, sizeof(GnnNet) * SYM_MAX_PROGS);
        if (err != cudaSuccess) return cuda_check(h, err, "graph networks");
    }
    const int slot = abiotic ? CLB_MAX_MICROBES : microbe;
    cudaError_t err = cudaMemcpy(static_cast<GnnNet*>(h->d_gnn) + slot, &N, sizeof N, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_check(h, err, "graph network");
    if (!h->gnn_host) h->gnn_host = new GnnNet[SYM_MAX_PROGS];
    h->gnn_host[slot] = N;
    AdeParams& A = h->ap;
    A.gnn = static_cast<const GnnNet*>(h->d_gnn);
    if (abiotic) {
        A.law2 = CLB_LAW_SYMBOLIC;
        A.gnn_abiotic = 1;
    } else {
        A.law = CLB_LAW_SYMBOLIC;
        A.gnn_mask |= 1u << microbe;
        A.sym_mask &= ~(1u << microbe);  // an organism has one run-time law
        A.srg_mask &= ~(1u << microbe);
    }
    return geometry_refresh(h);
}

__global__ void k_gnn_eval(const GnnNet* __restrict__ nets, int slot, const double* __restrict__ conc, int n,
                           double* __restrict__ out, unsigned int* __restrict__ clamped) {
    const GnnNet& N = nets[slot];
    const int nout = N.nS + (N.growth ? 1 : 0);
    unsigned int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x[GNN_MAX_S], y[GNN_MAX_S + 1];
        for (int s = 0; s < N.nS; ++s) x[s] = conc[(int64_t)i * N.nS + s];
        c += gnn_eval(N, x, y) ? 1u : 0u;
        for (int o = 0; o < nout; ++o) out[(int64_t)i * nout + o] = y[o];
    }
    if (c) atomicAdd(clamped, c);
}

clb_status graphnet_eval(clb_handle* h, int which, const double* conc, int n, double* out, int* n_out,
                         long* n_clamped) {
    const int slot = which < 0 ? CLB_MAX_MICROBES : which;
    if (which >= CLB_MAX_MICROBES || (which >= 0 && !(h->ap.gnn_mask >> which & 1u)) ||
        (which < 0 && !(h->ap.law2 == CLB_LAW_SYMBOLIC && h->ap.gnn_abiotic)))
        return fail(h, CLB_INVALID_ARG, "no graph network is bound there");
    const GnnNet& N = h->gnn_host[slot];
    const int nout = N.nS + (N.growth ? 1 : 0);
    if (n_out) *n_out = nout;
    if (n_clamped) *n_clamped = 0;
    if (n <= 0) return CLB_OK;
    double *dc = nullptr, *dout = nullptr;
    unsigned int* dcl = nullptr;
    cudaError_t e = cudaMalloc(&dc, sizeof(double) * (size_t)n * N.nS);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * (size_t)n * nout);
    if (e == cudaSuccess) e = cudaMalloc(&dcl, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(dcl, 0, sizeof(unsigned int), h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, conc, sizeof(double) * (size_t)n * N.nS, cudaMemcpyHostToDevice, h->stream);
    unsigned int cl = 0;
    if (e == cudaSuccess) {
        ++h->launches;
        k_gnn_eval<<<std::max(1, std::min(h->num_sms * 4, (n + 127) / 128)), 128, 0, h->stream>>>(
            static_cast<const GnnNet*>(h->d_gnn), slot, dc, n, dout, dcl);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(double) * (size_t)n * nout, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&cl, dcl, sizeof cl, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dc);
    cudaFree(dout);
    cudaFree(dcl);
    if (n_clamped) *n_clamped = (long)cl;
    return cuda_check(h, e, "graph network evaluation");
}

}  // namespace clb

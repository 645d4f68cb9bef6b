// graphnet.cuh -- rate laws given as a bipartite graph network over the reaction network (the
// reference's .gnn files, complab3d_graphnet.hh), evaluated per voxel in FP64 on the device.
//
// The graph has one node per species and one per reaction, with the stoichiometric coefficient
// S(i, r) as the weight of the edge between species i and reaction r. A species node starts from
// its scaled concentration; each round of message passing updates every reaction node from the
// stoichiometry-weighted sum of the species states (and the reaction's Damkohler number), then
// every species node from its own state and the weighted sum of the reaction states; every update
// is a dense W x W layer with tanh. The rates are read off the last states: per species from its
// node (readout SPECIES, each rate unscaled by its own offset and gain), or as one extent per
// reaction from its node with the species rates formed as sum_r S(i, r) xi_r (readout EXTENT);
// a growth rate, when the file has one, is read off the mean species node. Inputs are clamped to
// the training box first; a NaN output reads as 0; the file's unit (per_hour) scales every output.
//
// Sums are formed in the order the reference forms them and every product and sum is rounded on
// its own (no fused multiply-add), so the device computes what the reference computes up to the
// last bits of tanh.
#pragma once

#include <cstdint>

namespace clb {

constexpr int GNN_MAX_S = 8;       // species a network reads and rates
constexpr int GNN_MAX_R = 8;       // reactions
constexpr int GNN_MAX_W = 16;      // hidden width
constexpr int GNN_MAX_ROUNDS = 4;  // message-passing rounds

struct GnnLayer {
    double Wsr[GNN_MAX_W * GNN_MAX_W], Wss[GNN_MAX_W * GNN_MAX_W], Wrs[GNN_MAX_W * GNN_MAX_W];  // [h][k]
    double Wda[GNN_MAX_W], bR[GNN_MAX_W], bS[GNN_MAX_W];
};

struct GnnNet {
    int nS, nR, W, rounds;
    int extent;                   // readout: 0 SPECIES, 1 EXTENT
    int growth;                   // 1: a growth rate after the nS species rates
    double unit;                  // 1, or 1/3600 for per_hour
    double xymin, yymin;
    double S[GNN_MAX_S * GNN_MAX_R];          // [i][r]
    double da[GNN_MAX_R], xiscale[GNN_MAX_R];
    double xoff[GNN_MAX_S], xgain[GNN_MAX_S], tmin[GNN_MAX_S], tmax[GNN_MAX_S];
    double yoff[GNN_MAX_S + 1], ygain[GNN_MAX_S + 1];  // SPECIES: nS (+ growth); EXTENT: growth only
    double Wenc[GNN_MAX_W], benc[GNN_MAX_W];
    GnnLayer layer[GNN_MAX_ROUNDS];
    double Wout[2 * GNN_MAX_W], bout[2];      // row 0 the species (or reaction) head, row 1 growth
    // binding to the handle: internal species index of each network species
    int sp[GNN_MAX_S];
};

namespace gnn_detail {
#ifdef __CUDA_ARCH__
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
#else
inline double mul(double a, double b) { return a * b; }
inline double add(double a, double b) { return a + b; }
inline double sub(double a, double b) { return a - b; }
inline double div(double a, double b) { return a / b; }
#endif
}  // namespace gnn_detail

// Rates of network N for the concentrations c[0..nS) (the network's species order): out[0..nS) the
// species rates, out[nS] the growth rate when N.growth. Returns true when the training-box clamp
// changed an input.
// Not inlined: on the device one frame serves the organisms' and the abiotic call sites.
__host__ __device__ inline __noinline__ bool gnn_eval(const GnnNet& N, const double* c, double* out) {
    using namespace gnn_detail;
    const int W = N.W, nS = N.nS, nR = N.nR;
    double hS[GNN_MAX_S * GNN_MAX_W], hR[GNN_MAX_R * GNN_MAX_W], m[GNN_MAX_W], hn[GNN_MAX_W];
    bool clamped = false;
    for (int i = 0; i < nS; ++i) {
        double ci = c[i];
        if (ci < N.tmin[i]) { ci = N.tmin[i]; clamped = true; }
        else if (ci > N.tmax[i]) { ci = N.tmax[i]; clamped = true; }
        const double x = add(mul(sub(ci, N.xoff[i]), N.xgain[i]), N.xymin);
        for (int h = 0; h < W; ++h) hS[i * W + h] = tanh(add(mul(x, N.Wenc[h]), N.benc[h]));
    }
    for (int l = 0; l < N.rounds; ++l) {
        const GnnLayer& L = N.layer[l];
        // species -> reactions, weighted by the stoichiometry
        for (int r = 0; r < nR; ++r) {
            for (int k = 0; k < W; ++k) m[k] = 0.0;
            for (int i = 0; i < nS; ++i) {
                const double s = N.S[i * GNN_MAX_R + r];
                if (s == 0.0) continue;  // no edge
                for (int k = 0; k < W; ++k) m[k] = add(m[k], mul(s, hS[i * W + k]));
            }
            for (int h = 0; h < W; ++h) {
                double acc = add(L.bR[h], mul(N.da[r], L.Wda[h]));
                for (int k = 0; k < W; ++k) acc = add(acc, mul(L.Wsr[h * GNN_MAX_W + k], m[k]));
                hR[r * W + h] = tanh(acc);
            }
        }
        // reactions -> species; a species' new state reads only its own old state, so the update
        // is made in place species by species
        for (int i = 0; i < nS; ++i) {
            for (int k = 0; k < W; ++k) m[k] = 0.0;
            for (int r = 0; r < nR; ++r) {
                const double s = N.S[i * GNN_MAX_R + r];
                if (s == 0.0) continue;
                for (int k = 0; k < W; ++k) m[k] = add(m[k], mul(s, hR[r * W + k]));
            }
            for (int h = 0; h < W; ++h) {
                double acc = L.bS[h];
                for (int k = 0; k < W; ++k)
                    acc = add(acc, add(mul(L.Wss[h * GNN_MAX_W + k], hS[i * W + k]), mul(L.Wrs[h * GNN_MAX_W + k], m[k])));
                hn[h] = tanh(acc);
            }
            for (int h = 0; h < W; ++h) hS[i * W + h] = hn[h];
        }
    }
    if (N.extent) {
        double xi[GNN_MAX_R];
        for (int r = 0; r < nR; ++r) {
            double y = N.bout[0];
            for (int h = 0; h < W; ++h) y = add(y, mul(N.Wout[h], hR[r * W + h]));
            if (y != y) y = 0.0;
            xi[r] = mul(y, N.xiscale[r]);
        }
        for (int i = 0; i < nS; ++i) {
            double v = 0.0;
            for (int r = 0; r < nR; ++r) v = add(v, mul(N.S[i * GNN_MAX_R + r], xi[r]));
            out[i] = mul(v, N.unit);
        }
    } else {
        for (int i = 0; i < nS; ++i) {
            double y = N.bout[0];
            for (int h = 0; h < W; ++h) y = add(y, mul(N.Wout[h], hS[i * W + h]));
            double v = add(div(sub(y, N.yymin), N.ygain[i]), N.yoff[i]);
            if (v != v) v = 0.0;
            out[i] = mul(v, N.unit);
        }
    }
    if (N.growth) {
        const int gs = N.extent ? 0 : nS;
        double y = N.bout[1];
        for (int h = 0; h < W; ++h) {
            double s = 0.0;
            for (int i = 0; i < nS; ++i) s = add(s, hS[i * W + h]);
            y = add(y, mul(N.Wout[GNN_MAX_W + h], div(s, (double)nS)));
        }
        double v = add(div(sub(y, N.yymin), N.ygain[gs]), N.yoff[gs]);
        if (v != v) v = 0.0;
        out[nS] = mul(v, N.unit);
    }
    return clamped;
}

}  // namespace clb

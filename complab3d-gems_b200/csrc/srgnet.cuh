// srgnet.cuh -- surrogate organisms: a growth rate from a feed-forward network (the reference's
// .srg files, complab3d_surrogate.hh) fed with the organism's Michaelis-Menten uptake estimates, as
// run_surrogate3D drives it with the reference's default model (complab3d_processors_surrogate.hh,
// surrogateModel.hh: a run-time network bound to the organism), evaluated per voxel in FP64.
//
// The network: inputs clamped to the training box, scaled by mapminmax ((x - xoffset) xgain +
// xymin), dense layers with tansig (2 / (1 + exp(-2 n)) - 1) on every layer but the last, which is
// linear; each output unscaled ((a - yymin) / ygain + yoffset), output 0 is the specific growth
// rate (1/h), raised to 10^ when the file says logoutput, and floored: anything not above 1e-8
// (NaN included) is no growth. Sums run in the file's order and every operation is rounded on its
// own, so the device computes what the reference computes up to the last bits of exp.
//
// The organism around it (per voxel where its biomass B exceeds 1e-12, C the floored
// concentrations, dt the kinetics time step in seconds): the uptake estimate of every substrate
// v = vmax C / (Kc + C) where a maximum uptake flux is given, else the flux that would exhaust the
// voxel in one step, -exhaustion = C 3.6e6 / (B MW dt) (capped at 1e4 mmol/gDW/h), times the same
// Michaelis-Menten factor, and never above that exhaustion flux; the network's inputs are the
// estimates of the substrates it names; the growth rate mu grows the biomass by mu B dt / 3600, or
// where |mu| < 1e-12 the decay kd B dt takes it; the substrates are drawn by v B MW dt / 3.6e6
// (mmol/gDW/h to mol/L), shared with the voxel's other organisms under one headroom budget.
#pragma once

#include <cmath>
#include <cstdint>

namespace clb {

constexpr int SRG_MAX_IN = 8;      // network inputs
constexpr int SRG_MAX_LAYERS = 4;  // weight layers
constexpr int SRG_MAX_W = 32;      // widest layer (outputs included)

struct SrgNet {
    int nIn, nL;                         // inputs, weight layers
    int sizes[SRG_MAX_LAYERS + 1];       // nIn, hidden..., outputs
    int logout;                          // 1: output 0 is log10 of the growth rate
    double xoff[SRG_MAX_IN], xgain[SRG_MAX_IN], tmin[SRG_MAX_IN], tmax[SRG_MAX_IN], xymin;
    double yoff[SRG_MAX_W], ygain[SRG_MAX_W], yymin;
    double W[SRG_MAX_LAYERS][SRG_MAX_W * SRG_MAX_W];  // [layer][row][col], rows = sizes[l + 1]
    double B[SRG_MAX_LAYERS][SRG_MAX_W];
    // binding to the handle (internal species indices) and the organism's uptake parameters
    int subs[SRG_MAX_IN];                // species of each input
    double kc[CLB_MAX_SPECIES];          // half-saturation constants (mol/L)
    double vmax[CLB_MAX_SPECIES];        // maximum uptake fluxes (mmol/gDW/h); not above 1e-12: none
    double mw;                           // biomass molar mass (gDW/mol)
    double kd;                           // decay coefficient (1/s)
};

namespace srg_detail {
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
}  // namespace srg_detail

// Every output of network N on inputs x[0..nIn) after the training-box clamp (out[0] the growth
// rate with its log and floor, the others unscaled with a NaN read as 0). Returns true when the
// clamp changed an input.
__host__ __device__ inline __noinline__ bool srg_eval(const SrgNet& N, const double* x, double* out) {
    using namespace srg_detail;
    double a[SRG_MAX_W], o[SRG_MAX_W];
    bool clamped = false;
    for (int i = 0; i < N.nIn; ++i) {
        double v = x[i];
        if (v < N.tmin[i]) { v = N.tmin[i]; clamped = true; }
        else if (v > N.tmax[i]) { v = N.tmax[i]; clamped = true; }
        a[i] = add(mul(sub(v, N.xoff[i]), N.xgain[i]), N.xymin);
    }
    for (int l = 0; l < N.nL; ++l) {
        const int rows = N.sizes[l + 1], cols = N.sizes[l];
        const bool last = l + 1 == N.nL;
        for (int r = 0; r < rows; ++r) {
            double s = N.B[l][r];
            for (int c = 0; c < cols; ++c) s = add(s, mul(N.W[l][r * cols + c], a[c]));
            o[r] = last ? s : sub(div(2.0, add(1.0, exp(mul(-2.0, s)))), 1.0);
        }
        for (int r = 0; r < rows; ++r) a[r] = o[r];
    }
    const int nO = N.sizes[N.nL];
    for (int k = 0; k < nO; ++k) {
        const double gain = N.ygain[k] != 0.0 ? N.ygain[k] : 1.0;
        out[k] = add(div(sub(a[k], N.yymin), gain), N.yoff[k]);
    }
    if (N.logout) out[0] = pow(10.0, out[0]);
    if (!(out[0] > 1e-8)) out[0] = 0.0;
    for (int k = 1; k < nO; ++k)
        if (out[k] != out[k]) out[k] = 0.0;
    return clamped;
}

// The exhaustion flux of concentration c for biomass b (mmol/gDW/h, negative: uptake), 0 where
// B MW dt is not above 1e-30 (MetabolicConfig::exhaustionFlux, complab3d_metabolic.hh:577-595).
__host__ __device__ inline double srg_exhaustion(double c, double b, double mw, double dt) {
    using namespace srg_detail;
    const double denom = mul(mul(b, mw), dt);
    if (!(denom > 1e-30)) return 0.0;
    double v = div(mul(-c, 3.6e6), denom);
    if (v < -1e4) v = -1e4;
    return v;
}

}  // namespace clb

// Thin C entry points around the reference's own kinetics processors: run_kinetics and
// run_abiotic_kinetics (complab3d_processors_part1.hh) and surfaceAbioticKinetics3D
// (precipitationVOP.hh), compiled from the reference sources where they lie against the minimal
// lattice stand-ins of palabos_shim.hh (see Makefile target `ref`). TEST INFRASTRUCTURE ONLY:
// used to pin the oracle's kinetics passes to the reference.
//
// The rate laws are the reference's compile-time hooks. The abiotic one is the reference's own
// FeS precipitation law of examples/15_precip_and_dissolution (found on the include path); the
// biotic one is the library's decay / Monod / dual-Monod law, supplied here the way a user's
// defineKinetics.hh supplies it. part1 includes "../defineKinetics.hh" and
// "../defineAbioticKinetics.hh"; the Makefile points those at empty files, since both hooks are
// already defined when part1 is read.
#include "palabos_shim.hh"

#include <algorithm>
#include <cmath>
#include <iostream>
#include <vector>

using namespace plb;
typedef double T;
const T thrd = 1e-12;  // the reference's threshold (complab3d_processors.hh)

static int g_law = 0;
static std::vector<double> g_prm;

// CLB_LAW_DECAY (1): R_s = -k_s C_s; CLB_LAW_MONOD (2): R_s = -k_s C_s / (Ks_s + C_s);
// CLB_LAW_DUAL_MONOD (3): microbe m grows on species 0 and 1 + m (params mu_max, Ks, Y, kd).
void defineRxnKinetics(std::vector<double> B, std::vector<double> C, std::vector<double>& subsR,
                       std::vector<double>& bioR, plint) {
    const size_t S = subsR.size(), M = bioR.size();
    for (auto& r : subsR) r = 0.0;
    for (auto& r : bioR) r = 0.0;
    const std::vector<double>& p = g_prm;
    if (g_law == 1) {
        for (size_t s = 0; s < S; ++s) subsR[s] = -p[s] * C[s];
    } else if (g_law == 2) {
        for (size_t s = 0; s < S; ++s) subsR[s] = -p[s] * C[s] / (p[S + s] + C[s]);
    } else if (g_law == 3) {
        for (size_t m = 0; m < M; ++m) {
            const size_t a = 1 + m;
            if (a >= S) break;
            if (B[m] <= 0.0) continue;
            const double growth = p[0] * (C[0] / (p[1] + C[0])) * (C[a] / (p[1] + C[a])) * B[m];
            bioR[m] += growth - p[3] * B[m];
            subsR[0] -= growth / p[2];
            subsR[a] -= growth / p[2];
        }
    }
}

#include "defineAbioticKinetics.hh"  // examples/15_precip_and_dissolution/kinetics
#include "complab3d_processors_part1.hh"
#include "precipitationVOP.hh"

typedef BlockLattice3D<T, D3Q7Descriptor> Lat;

// lattices with the given densities, in the reference's lattice order
static void fill(std::vector<Lat>& L, size_t first, int count, const double* v, size_t N) {
    for (int k = 0; k < count; ++k)
        for (size_t n = 0; n < N; ++n) L[first + k].cells[n].setDensity(v ? v[(size_t)k * N + n] : 0.0);
}

static void read(const std::vector<Lat>& L, size_t first, int count, double* out, size_t N) {
    for (int k = 0; k < count; ++k)
        for (size_t n = 0; n < N; ++n) out[(size_t)k * N + n] = L[first + k].cells[n].computeDensity();
}

/* run_kinetics over the whole box: lattices = S substrates, M biomass, S dC, M dB, the mask.
 * Returns the dC [S][N] and dB [M][N] it leaves (update_rxnLattices then adds them). */
extern "C" void ref_biotic_increments(int nx, int ny, int nz, int S, int M, double dt, int law, const double* prm,
                                      int nprm, const int8_t* mat, int solid, int bb, const double* C,
                                      const double* B, double* dC, double* dB) {
    g_law = law;
    g_prm.assign(prm, prm + nprm);
    const size_t N = (size_t)nx * ny * nz;
    std::vector<Lat> L;
    L.reserve(2 * (S + M) + 1);
    for (int i = 0; i < 2 * (S + M) + 1; ++i) L.emplace_back(nx, ny, nz);
    fill(L, 0, S, C, N);
    fill(L, S, M, B, N);
    fill(L, S + M, S + M, nullptr, N);
    for (size_t n = 0; n < N; ++n) L[2 * (S + M)].cells[n].setDensity((T)mat[n]);
    std::vector<Lat*> ptr;
    for (auto& l : L) ptr.push_back(&l);
    run_kinetics<T, D3Q7Descriptor> f(nx, S, M, dt, std::vector<std::vector<T>>(), std::vector<T>(), solid, bb);
    f.process(Box3D{0, nx - 1, 0, ny - 1, 0, nz - 1}, ptr);
    read(L, S + M, S, dC, N);
    read(L, 2 * S + M, M, dB, N);
}

/* run_abiotic_kinetics (surface_only 0) or surfaceAbioticKinetics3D (surface_only 1) with the FeS
 * law of examples/15: lattices = S substrates, S dC, the mask. Returns the dC [S][N] it leaves. */
extern "C" void ref_abiotic_increments(int nx, int ny, int nz, int S, double dt, int surface_only,
                                       const int8_t* mat, int solid, int bb, const double* C, double* dC) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<Lat> L;
    L.reserve(2 * S + 1);
    for (int i = 0; i < 2 * S + 1; ++i) L.emplace_back(nx, ny, nz);
    fill(L, 0, S, C, N);
    fill(L, S, S, nullptr, N);
    for (size_t n = 0; n < N; ++n) L[2 * S].cells[n].setDensity((T)mat[n]);
    std::vector<Lat*> ptr;
    for (auto& l : L) ptr.push_back(&l);
    const Box3D box{0, nx - 1, 0, ny - 1, 0, nz - 1};
    if (surface_only) {
        surfaceAbioticKinetics3D<T, D3Q7Descriptor> f(nx, ny, nz, S, dt, solid, bb, 1);
        f.process(box, ptr);
    } else {
        run_abiotic_kinetics<T, D3Q7Descriptor> f(nx, S, dt, solid, bb);
        f.process(box, ptr);
    }
    read(L, S, S, dC, N);
}

/* The thermodynamic gate (complab3d_thermo.hh): one reaction block (terms sp/nu; v = dG0, atp,
 * dGatp, chi, cmin, dGloss, temperature, gas constant, concentration scale, energies in kJ/mol),
 * registered for n_microbes organisms as the kinetics path registers it, so run_kinetics gates its
 * rates through gateFor(0, ...). n = 0 clears it. */
extern "C" void ref_set_thermo(int n, const int32_t* sp, const double* nu, const double* v, int n_microbes) {
    complab_thermo::Runtime& R = complab_thermo::runtime();
    R = complab_thermo::Runtime();
    if (n <= 0) return;
    complab_thermo::Spec s;
    s.name = "gate";
    s.microbe = -1;
    for (int i = 0; i < n; ++i) {
        s.species.push_back("s" + std::to_string(sp[i]));
        s.nu.push_back(nu[i]);
        s.subsOfSpecies.push_back(sp[i]);
    }
    s.dG0 = v[0]; s.atp = v[1]; s.dGatp = v[2]; s.chi = v[3]; s.cmin = v[4]; s.dGloss = v[5];
    R.model.Tkelvin = v[6];
    R.model.Rgas = v[7];
    R.model.concScale = v[8];
    R.model.specs.push_back(s);
    complab_thermo::registerModel(n_microbes);
}

// complab_thermo::factor on one concentration vector of S species (scaled as fillConc scales it)
extern "C" double ref_thermo_factor(int S, const double* C) {
    std::vector<double> conc;
    complab_thermo::fillConc(C, S, conc);
    return complab_thermo::gateFor(0, conc);
}

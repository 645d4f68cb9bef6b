// Thin C entry points around the reference's own dissolution processors (surfaceDissolutionKinetics3D
// and dissolutionGather3D, dissolutionVOP.hh) and the deterministic passes of its biofilm automaton
// (updateLocalMaskNtotalLattices3D, updateAgeDistance3D, complab3d_processors_part2.hh), compiled
// from the reference sources where they lie against the minimal lattice stand-ins of
// palabos_shim.hh (see Makefile target `ref`). TEST INFRASTRUCTURE ONLY: used to pin the oracle's
// restatement of these passes to the reference.
#include "palabos_shim.hh"

#include <algorithm>
#include <iostream>
#include <random>
#include <string>
#include <vector>

using namespace plb;
typedef double T;
const T thrd = 1e-12;  // the reference's threshold (complab3d_processors.hh)

// The dissolution law is the user's compile-time hook in the reference; here it is the library's
// first-order law (params kd, h, sigma[S]) or its saturation-index law (params k, log10 Ksp, nu[S]).
static int g_law = 0, g_sM = -1;
static std::vector<double> g_prm;

inline void defineDissolutionRate(plint, const std::vector<double>& C, double mineral, std::vector<double>& subsR,
                                  double& mineralR, plint) {
    const size_t S = subsR.size();
    mineralR = 0.0;
    for (size_t i = 0; i < S; ++i) subsR[i] = 0.0;
    const std::vector<double>& p = g_prm;
    if (g_law == 1) {
        const int h = (int)p[1];
        const double rate = p[0] * (h >= 0 ? std::max(C[(size_t)h], 0.0) : 1.0) * std::max(mineral, 0.0);
        mineralR = -rate;
        for (size_t j = 0; j < S; ++j) subsR[j] = p[2 + j] * rate;
    } else if (g_law == 2) {
        double la = 0;
        for (size_t j = 0; j < S; ++j)
            if ((int)j != g_sM && p[2 + j] != 0.0) la += p[2 + j] * std::log10(std::max(C[j], 1e-30));
        const double om = std::pow(10.0, la - p[1]);
        if (om < 1.0) {
            mineralR = p[0] * (om - 1.0);
            for (size_t j = 0; j < S; ++j)
                if ((int)j != g_sM) subsR[j] = -p[2 + j] * mineralR;
        }
    }
}

double g_abioticRateScale = 1.0;  // the reference's global rate scale (1: no scaling)

inline void defineAbioticRxnKinetics(std::vector<double>, std::vector<double>& subsR, plint) {
    for (size_t i = 0; i < subsR.size(); ++i) subsR[i] = 0.0;
}

#define COMPLAB_THRD 1e-14  // complab_functions.hh

#include "precipitationVOP.hh"
#include "dissolutionVOP.hh"
#include "complab3d_processors_part2.hh"

typedef BlockLattice3D<T, D3Q7Descriptor> Lat;

extern "C" int ref_dissolution_increments(int nx, int ny, int nz, int S, int sM, double dt, int law, const double* prm,
                                          int nprm, int surface_only, const int8_t* mat, int solid, int bb,
                                          const uint8_t* stamp, const double* C, double* dC) {
    const size_t N = (size_t)nx * ny * nz;
    g_law = law;
    g_sM = sM;
    g_prm.assign(prm, prm + nprm);
    std::vector<Lat> lat;
    lat.reserve((size_t)2 * S + 2);
    for (int i = 0; i < 2 * S + 2; ++i) lat.emplace_back(nx, ny, nz);
    for (size_t n = 0; n < N; ++n) {
        for (int s = 0; s < S; ++s) {
            lat[(size_t)s].cells[n].setDensity(C[(size_t)s * N + n]);
            lat[(size_t)(S + s)].cells[n].setDensity(dC[(size_t)s * N + n]);
        }
        lat[(size_t)(2 * S)].cells[n].setDensity((T)mat[n]);
        lat[(size_t)(2 * S + 1)].cells[n].setDensity(stamp[n] ? (T)1 : (T)0);
    }
    std::vector<Lat*> ptr;
    for (auto& l : lat) ptr.push_back(&l);
    DissolutionConfig cfg;
    cfg.enabled = true;
    cfg.surface_only = surface_only;
    SolidPhase ph;
    ph.id = 1;
    ph.substrate = sM;
    ph.full_density = 1;
    ph.is_precipitate = true;
    cfg.phases.push_back(ph);
    const Box3D box{0, nx - 1, 0, ny - 1, 0, nz - 1};
    std::vector<plint> pore{2};
    surfaceDissolutionKinetics3D<T, D3Q7Descriptor> park(nx, ny, nz, S, dt, solid, bb, pore, &cfg);
    park.process(box, ptr);
    dissolutionGather3D<T, D3Q7Descriptor> gather(nx, ny, nz, S, solid, bb, &cfg);
    gather.process(box, ptr);
    for (int s = 0; s < S; ++s)
        for (size_t n = 0; n < N; ++n) dC[(size_t)s * N + n] = lat[(size_t)(S + s)].cells[n].computeDensity();
    return 0;
}

// updateLocalMaskNtotalLattices3D over the whole box: biomass bio[M][N], total[N] and mask[N]
// (material codes) in, total and mask out.
extern "C" int ref_ca_mask_total(int nx, int ny, int nz, int M, const double* bio, double* total, int* mask, int bb,
                                 int solid, const int* bio_codes, int n_pore, const int* pore, double frac,
                                 double Bmax) {
    const size_t N = (size_t)nx * ny * nz;
    const int len = 2 * M + 3;
    std::vector<Lat> lat;
    lat.reserve((size_t)len);
    for (int i = 0; i < len; ++i) lat.emplace_back(nx, ny, nz);
    for (size_t n = 0; n < N; ++n) {
        for (int m = 0; m < M; ++m) {
            lat[(size_t)m].cells[n].setDensity(bio[(size_t)m * N + n]);
            lat[(size_t)(M + m)].cells[n].setDensity(bio[(size_t)m * N + n]);
        }
        lat[(size_t)(len - 3)].cells[n].setDensity(total[n]);
        lat[(size_t)(len - 2)].cells[n].setDensity((T)mask[n]);
        lat[(size_t)(len - 1)].cells[n].setDensity(0);
    }
    std::vector<Lat*> ptr;
    for (auto& l : lat) ptr.push_back(&l);
    std::vector<std::vector<plint>> bv;
    for (int m = 0; m < M; ++m) bv.push_back(std::vector<plint>{bio_codes[m]});
    std::vector<plint> pv(pore, pore + n_pore);
    updateLocalMaskNtotalLattices3D<T, D3Q7Descriptor> f(nx, ny, nz, len, bb, solid, bv, pv, frac, Bmax);
    f.process(Box3D{0, nx - 1, 0, ny - 1, 0, nz - 1}, ptr);
    for (size_t n = 0; n < N; ++n) {
        total[n] = lat[(size_t)(len - 3)].cells[n].computeDensity();
        mask[n] = (int)util::roundToInt(lat[(size_t)(len - 2)].cells[n].computeDensity());
    }
    return 0;
}

// updateAgeDistance3D over the whole box, applied until no age changes (at most max_sweeps):
// age[N] in/out, dist[N] (the distance field's sign: > 0 inside the open region), total[N].
// Returns the number of sweeps that changed something.
extern "C" int ref_ca_age_relax(int nx, int ny, int nz, int* age, const int* dist, const double* total, double Bmax,
                                int max_sweeps) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<Lat> lat;
    lat.reserve(3);
    for (int i = 0; i < 3; ++i) lat.emplace_back(nx, ny, nz);
    for (size_t n = 0; n < N; ++n) {
        lat[0].cells[n].setDensity((T)age[n]);
        lat[1].cells[n].setDensity((T)dist[n]);
        lat[2].cells[n].setDensity(total[n]);
    }
    std::vector<Lat*> ptr{&lat[0], &lat[1], &lat[2]};
    updateAgeDistance3D<T, D3Q7Descriptor> f(Bmax, nx, ny, nz);
    int sweeps = 0;
    for (; sweeps < max_sweeps; ++sweeps) {
        std::vector<int> before(N);
        for (size_t n = 0; n < N; ++n) before[n] = (int)util::roundToInt(lat[0].cells[n].computeDensity());
        f.process(Box3D{0, nx - 1, 0, ny - 1, 0, nz - 1}, ptr);
        bool changed = false;
        for (size_t n = 0; n < N; ++n)
            if ((int)util::roundToInt(lat[0].cells[n].computeDensity()) != before[n]) changed = true;
        if (!changed) break;
    }
    for (size_t n = 0; n < N; ++n) age[n] = (int)util::roundToInt(lat[0].cells[n].computeDensity());
    return sweeps;
}

/* precipNodeConversion3D over Box3D(1, nx-2, 0, ny-1, 0, nz-1) (complab.cpp:3139-3146) with
 * lattices [mineral, mask, phase] and the precipitate's phase id 1, then, when dissolution is on,
 * dissolNodeConversion3D over the same box with lattices [S substrates, mask, phase] and one
 * declared phase (id 1, the precipitate: material precip_code, substrate sM, full density full).
 * mat and phase (0 or 1 per voxel) are updated in place. */
extern "C" void ref_node_conversion(int nx, int ny, int nz, int S, int sM, double full, double reopen,
                                    int precip_code, int pore_code, int solid, int bb, int dissolution,
                                    const double* C, int8_t* mat, uint8_t* phase) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<Lat> L;
    L.reserve(S + 2);
    for (int i = 0; i < S + 2; ++i) L.emplace_back(nx, ny, nz);
    for (int s = 0; s < S; ++s)
        for (size_t n = 0; n < N; ++n) L[s].cells[n].setDensity(C[(size_t)s * N + n]);
    for (size_t n = 0; n < N; ++n) {
        L[S].cells[n].setDensity((T)mat[n]);
        L[S + 1].cells[n].setDensity((T)phase[n]);
    }
    const Box3D box{1, nx - 2, 0, ny - 1, 0, nz - 1};
    {
        std::vector<Lat*> ptr{&L[sM], &L[S], &L[S + 1]};
        precipNodeConversion3D<T, D3Q7Descriptor> f(nx, ny, nz, full, solid, bb, precip_code, dissolution ? 1 : 0);
        f.process(box, ptr);
    }
    if (dissolution) {
        DissolutionConfig cfg;
        cfg.enabled = true;
        cfg.reopen_fraction = reopen;
        SolidPhase ph;
        ph.id = 1;
        ph.material_number = precip_code;
        ph.substrate = sM;
        ph.full_density = full;
        ph.is_precipitate = true;
        cfg.phases.push_back(ph);
        std::vector<Lat*> ptr;
        for (auto& l : L) ptr.push_back(&l);
        dissolNodeConversion3D<T, D3Q7Descriptor> f(S, pore_code, solid, bb, &cfg);
        f.process(box, ptr);
    }
    for (size_t n = 0; n < N; ++n) {
        mat[n] = (int8_t)util::roundToInt(L[S].cells[n].computeDensity());
        phase[n] = (uint8_t)util::roundToInt(L[S + 1].cells[n].computeDensity());
    }
}

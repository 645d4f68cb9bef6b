/* lbm_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * An FP64 CPU restatement of CompLaB3D's coupled reactive-transport step (flow lattice,
 * per-species advection-diffusion lattices, kinetics increments), used only to check parity
 * in tests/ and __graft_entry__.smoke(), and as the timed CPU baseline by bench.py.
 * It is never linked into, called by, or shipped with the product library.
 *
 * The LBM arithmetic itself lives in Palabos 2.3.0 (not vendored with the reference). What
 * is restated here follows the reference's call sites and the published Palabos algorithms:
 *
 *   flow lattice  (complab_functions.hh:296-345 NSdomainSetup)
 *     - IncBGKdynamics: f_i <- (1-w) f_i + w t_i (rb + 3 c.j + 4.5 (c.j)^2 - 1.5 j^2),
 *       populations stored shifted by t_i, u = j (incompressible, rho0 = 1).
 *     - BounceBack: the collision swaps opposite populations (full-way bounce-back;
 *       populations are held one step inside the wall node).
 *     - NoDynamics: no collision; populations still stream.
 *     - pressure planes x=0 (rho=1) and x=nx-1 (rho=1-3 dP): Palabos' local regularized
 *       density boundary (createLocalBoundaryCondition3D + addPressureBoundary0N/0P):
 *       j_x = orient (rb_0 + 2 rb_n - rb), j_y = j_z = 0, Pi_neq from the known
 *       populations with bounce-back of off-equilibrium parts, f_i = feq_i + fneq_i(Pi),
 *       then the wrapped IncBGK collision.  Wrapping a bounce-back or no-dynamics node is a
 *       no-op in Palabos (their equilibrium is zero and regularize() does nothing), so the
 *       boundary acts on BGK nodes only.
 *     - edges of the box along y and z: Palabos' swap streaming leaves a population whose
 *       source lies outside the block in the node's own opposite slot (reflection).
 *     - PressureGradient initial state (complab_functions.hh:82-94).
 *     - statistics: the mean of |u|^2 over BGK nodes gathered during the collision;
 *       getStoredAverageEnergy returns half that mean.
 *     - util::ValueTracer(u=1, L=1000, eps): window deltaT = L/u/2 = 500 values,
 *       converged when the window is full and stddev/mean < eps (sample stddev, n-1).
 *       Driven exactly as complab.cpp:1120-1124 does.
 *
 *   advection-diffusion lattices  (complab_functions.hh:347-442 soluteDomainSetup,
 *   complab.cpp:1380-1393, 1506-1656)
 *     - AdvectionDiffusionBGKdynamics (D3Q7, t0=1/4, ti=1/8, cs2=1/4):
 *       g_i <- (1-w) g_i + w t_i (rb + 4 c_i.(rho u)), u the external (flow) velocity.
 *     - per-voxel omega: pore vs biofilm (complab.cpp:1244-1253).
 *     - solid and wall voxels of a mobile species are BounceBack seeded at c0
 *       (complab.cpp:1589-1656, stabilizeADElattice3D part3.hh:261-311).
 *     - x faces: 0 Dirichlet, 1 Neumann, 2 closed (complab_functions.hh:404-438).
 *       Dirichlet/Neumann: the single unknown population is completed so the node's
 *       density equals the stored value (Palabos AdvectionDiffusionBoundaryDynamics);
 *       Neumann stores the inner neighbour's density after every stream
 *       (FlatAdiabaticBoundaryFunctional3D, an integrated processor run by stream()).
 *       Closed: the whole plane becomes BounceBack after initialisation.
 *     - step order (complab.cpp:2307-2315, 2340-2452, 3251-3259): collide all mobile
 *       species, kinetics on the post-collision densities, deposit dC*t_i, stream.
 *     - kinetics (part1.hh:85-187, 406-497): x in 1..nx-2, mask not solid/wall;
 *       C < 1e-12 is read as 0; dC = R dt; clamp dC = max(R dt, -C)
 *       (complab3d_processors_symbolic.hh:165-180); applied only if |dC| > 1e-12;
 *       biomass never negative (ibid. :193).
 */
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- D3Q19 (Palabos order)
const int Q19 = 19;
const int C19[19][3] = {
    {0, 0, 0},
    {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {-1, -1, 0}, {-1, 1, 0}, {-1, 0, -1},
    {-1, 0, 1}, {0, -1, -1}, {0, -1, 1},
    {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, -1, 0}, {1, 0, 1},
    {1, 0, -1}, {0, 1, 1}, {0, 1, -1}};
const double T19[19] = {
    1.0 / 3,
    1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36,
    1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
inline int opp19(int i) { return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9); }

// ---------------------------------------------------------------- D3Q7 (Palabos order)
const int Q7 = 7;
const int C7[7][3] = {{0, 0, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
const double T7[7] = {0.25, 0.125, 0.125, 0.125, 0.125, 0.125, 0.125};
inline int opp7(int i) { return i == 0 ? 0 : (i <= 3 ? i + 3 : i - 3); }

const double THRD = 1e-12;  // complab3d_processors.hh:60

enum { DYN_BB = 0, DYN_NONE = 1, DYN_BGK = 2 };

inline double feq19(int i, double rb, const double j[3], double jsq) {
    double cj = C19[i][0] * j[0] + C19[i][1] * j[1] + C19[i][2] * j[2];
    return T19[i] * (rb + 3.0 * cj + 1.5 * (3.0 * cj * cj - jsq));
}

int g_threads = 1;

struct Tracer {  // util::ValueTracer<T>(1, 1000, eps)
    int deltaT = 500;
    double eps = 1e-6;
    std::vector<double> v;
    void take(double x) {
        v.push_back(x);
        if ((int)v.size() > deltaT) v.erase(v.begin());
    }
    bool converged() const {
        if ((int)v.size() < deltaT) return false;
        double s = 0;
        for (double x : v) s += x;
        double avg = s / (double)v.size();
        double sq = 0;
        for (double x : v) sq += (x - avg) * (x - avg);
        double sd = std::sqrt(sq / (double)(v.size() - 1));
        double r = sd / avg;
        if (std::isnan(r)) return true;  // "simulation diverged" also ends the loop
        return std::fabs(r) < eps;
    }
};

}  // namespace

// =====================================================================================
//                                   FLOW LATTICE
// =====================================================================================
struct OrcFlow {
    int nx, ny, nz;
    size_t N;
    std::vector<double> f, fp;  // [N][19]
    std::vector<int8_t> mat;
    int dyn[256];
    double omega[256];
    double rho_w, rho_e;
    double energy = 0;
    long iters = 0;
    Tracer tr;
    size_t id(int x, int y, int z) const { return ((size_t)x * ny + y) * nz + z; }
};

extern "C" {

void orc_set_threads(int n) {
    g_threads = n > 0 ? n : 1;
#ifdef _OPENMP
    omp_set_num_threads(g_threads);
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

OrcFlow* orc_flow_create(int nx, int ny, int nz, const int8_t* mat, const int32_t* dyn_by_code,
                         const double* omega_by_code, double delta_p) {
    OrcFlow* F = new OrcFlow();
    F->nx = nx; F->ny = ny; F->nz = nz;
    F->N = (size_t)nx * ny * nz;
    F->mat.assign(mat, mat + F->N);
    for (int k = 0; k < 256; ++k) { F->dyn[k] = dyn_by_code[k]; F->omega[k] = omega_by_code[k]; }
    F->rho_w = 1.0;
    F->rho_e = 1.0 - delta_p * 3.0;
    F->f.assign(F->N * Q19, 0.0);
    F->fp.assign(F->N * Q19, 0.0);
    // initializeAtEquilibrium(PressureGradient): rho(x) = 1 - dP*invCs2/(nx-1)*x, u = 0.
    // BounceBack / NoDynamics return a zero equilibrium, i.e. shifted populations 0.
    for (int x = 0; x < nx; ++x) {
        double rho = 1.0 - delta_p * 3.0 / (double)(nx - 1) * (double)x;
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = F->id(x, y, z);
                if (F->dyn[(uint8_t)F->mat[n]] != DYN_BGK) continue;
                for (int i = 0; i < Q19; ++i) F->f[n * Q19 + i] = T19[i] * (rho - 1.0);
            }
    }
    return F;
}

void orc_flow_destroy(OrcFlow* F) { delete F; }

static void flow_collide_stream(OrcFlow* F) {
    const int nx = F->nx, ny = F->ny, nz = F->nz;
    double esum = 0;
    long ecnt = 0;
    // ---- collision (all nodes)
#pragma omp parallel for reduction(+ : esum, ecnt) schedule(static)
    for (int x = 0; x < nx; ++x) {
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = F->id(x, y, z);
                double* c = &F->f[n * Q19];
                double* o = &F->fp[n * Q19];
                int d = F->dyn[(uint8_t)F->mat[n]];
                if (d == DYN_NONE) {
                    for (int i = 0; i < Q19; ++i) o[i] = c[i];
                    continue;
                }
                if (d == DYN_BB) {
                    for (int i = 0; i < Q19; ++i) o[i] = c[opp19(i)];
                    continue;
                }
                double w = F->omega[(uint8_t)F->mat[n]];
                double g[19];
                for (int i = 0; i < Q19; ++i) g[i] = c[i];
                if (x == 0 || x == nx - 1) {
                    // regularized density boundary, direction 0, orientation -1 (west) / +1 (east)
                    int orient = (x == 0) ? -1 : 1;
                    double rb = ((x == 0) ? F->rho_w : F->rho_e) - 1.0;
                    double r0 = 0, rn = 0;
                    for (int i = 0; i < Q19; ++i) {
                        if (C19[i][0] == 0) r0 += g[i];
                        else if (C19[i][0] == orient) rn += g[i];
                    }
                    double j[3] = {orient * (r0 + 2.0 * rn - rb), 0.0, 0.0};
                    double jsq = j[0] * j[0];
                    double pi[6] = {0, 0, 0, 0, 0, 0};  // xx xy xz yy yz zz
                    for (int i = 0; i < Q19; ++i) {
                        double fac;
                        if (C19[i][0] == 0) fac = 1.0;
                        else if (C19[i][0] == orient) fac = 2.0;
                        else continue;
                        double fneq = (i == 0 && C19[i][0] == orient) ? 0.0 : g[i] - feq19(i, rb, j, jsq);
                        int p = 0;
                        for (int a = 0; a < 3; ++a)
                            for (int b = a; b < 3; ++b) pi[p++] += fac * C19[i][a] * C19[i][b] * fneq;
                    }
                    for (int i = 0; i < Q19; ++i) {
                        double s = 0;
                        int p = 0;
                        for (int a = 0; a < 3; ++a)
                            for (int b = a; b < 3; ++b) {
                                double q = C19[i][a] * C19[i][b];
                                if (a == b) q -= 1.0 / 3.0;
                                else q *= 2.0;
                                s += q * pi[p++];
                            }
                        g[i] = feq19(i, rb, j, jsq) + T19[i] * 9.0 / 2.0 * s;
                    }
                }
                double rb = 0, j[3] = {0, 0, 0};
                for (int i = 0; i < Q19; ++i) {
                    rb += g[i];
                    j[0] += C19[i][0] * g[i];
                    j[1] += C19[i][1] * g[i];
                    j[2] += C19[i][2] * g[i];
                }
                double jsq = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
                for (int i = 0; i < Q19; ++i) o[i] = g[i] * (1.0 - w) + w * feq19(i, rb, j, jsq);
                esum += jsq;
                ecnt += 1;
            }
    }
    // ---- streaming (pull form of Palabos' swap streaming; out-of-block sources reflect)
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x) {
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = F->id(x, y, z);
                double* dst = &F->f[n * Q19];
                dst[0] = F->fp[n * Q19];
                for (int i = 1; i < Q19; ++i) {
                    int sx = x - C19[i][0], sy = y - C19[i][1], sz = z - C19[i][2];
                    if (sx < 0 || sy < 0 || sz < 0 || sx >= nx || sy >= ny || sz >= nz)
                        dst[i] = F->fp[n * Q19 + opp19(i)];
                    else
                        dst[i] = F->fp[F->id(sx, sy, sz) * Q19 + i];
                }
            }
    }
    F->energy = ecnt > 0 ? 0.5 * esum / (double)ecnt : 0.0;
    F->iters += 1;
}

void orc_flow_set_material(OrcFlow* F, const int8_t* mat) { F->mat.assign(mat, mat + F->N); }
void orc_flow_set_dynamics(OrcFlow* F, int code, int dyn, double omega) {
    F->dyn[code & 255] = dyn;
    F->omega[code & 255] = omega;
}

void orc_flow_step(OrcFlow* F, int n) {
    for (int k = 0; k < n; ++k) flow_collide_stream(F);
}

double orc_flow_energy(OrcFlow* F) { return F->energy; }
long orc_flow_iterations(OrcFlow* F) { return F->iters; }

/* complab.cpp:1120-1124: for (; iT < max; ++iT) { collideAndStream(); takeValue(energy);
 * if (hasConverged()) break; }.  Returns the number of collideAndStream calls made. */
int orc_flow_solve(OrcFlow* F, int max_it, double eps) {
    F->tr = Tracer();
    F->tr.eps = eps;
    int k = 0;
    for (; k < max_it;) {
        flow_collide_stream(F);
        ++k;
        F->tr.take(F->energy);
        if (F->tr.converged()) break;
    }
    return k;
}

/* computeVelocity: BGK nodes u = j; density-boundary nodes u = (j_x from the known
 * populations, 0, 0); BounceBack and NoDynamics nodes report zero. */
void orc_flow_velocity(OrcFlow* F, double* u) {
    const int nx = F->nx, ny = F->ny, nz = F->nz;
    const size_t N = F->N;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = F->id(x, y, z);
                const double* g = &F->f[n * Q19];
                double j[3] = {0, 0, 0};
                if (F->dyn[(uint8_t)F->mat[n]] == DYN_BGK) {
                    if (x == 0 || x == nx - 1) {
                        int orient = (x == 0) ? -1 : 1;
                        double rb = ((x == 0) ? F->rho_w : F->rho_e) - 1.0;
                        double r0 = 0, rn = 0;
                        for (int i = 0; i < Q19; ++i) {
                            if (C19[i][0] == 0) r0 += g[i];
                            else if (C19[i][0] == orient) rn += g[i];
                        }
                        j[0] = orient * (r0 + 2.0 * rn - rb);
                    } else {
                        for (int i = 0; i < Q19; ++i)
                            for (int a = 0; a < 3; ++a) j[a] += C19[i][a] * g[i];
                    }
                }
                u[n] = j[0];
                u[N + n] = j[1];
                u[2 * N + n] = j[2];
            }
}

/* Palabos populations as stored (shifted by t_i), direction-major [19][N]. */
void orc_flow_populations(OrcFlow* F, double* out) {
    for (size_t n = 0; n < F->N; ++n)
        for (int i = 0; i < Q19; ++i) out[(size_t)i * F->N + n] = F->f[n * Q19 + i];
}

void orc_flow_set_populations(OrcFlow* F, const double* in) {
    for (size_t n = 0; n < F->N; ++n)
        for (int i = 0; i < Q19; ++i) F->f[n * Q19 + i] = in[(size_t)i * F->N + n];
}

}  // extern "C"

// =====================================================================================
//                           ADVECTION-DIFFUSION LATTICES
// =====================================================================================
enum { ADE_BB = 0, ADE_NONE = 1, ADE_PORE = 2, ADE_BIO = 3 };
enum { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_CLOSED = 2 };
enum { LAW_NONE = 0, LAW_DECAY = 1, LAW_MONOD = 2, LAW_DUAL_MONOD = 3, LAW_PRECIP = 4, LAW_MINERAL = 5, LAW_SYMBOLIC = 6 };
enum { DISSOL_NONE = 0, DISSOL_FIRST_ORDER = 1, DISSOL_MINERAL = 2 };

// ---- rate laws read from a .sym file (complab3d_symbolic.hh restated; see the section below)
struct SymNode {
    int kind;         // 0 const, 1 var, 2 neg, 3 add, 4 sub, 5 mul, 6 div, 7 pow, 8 exp, 9 log, 10 log10,
                      // 11 sqrt, 12 abs, 13 tanh, 14 min, 15 max
    double value;
    int a, b;
};
struct SymLaw {
    std::vector<std::string> vars, rates;
    std::vector<SymNode> nodes;
    std::vector<int> roots;
    std::vector<double> lo, hi;
    double unit = 1.0;
    bool extent = false;
    std::vector<int> var_src, rate_dst;  // binding: species index (-1 biomass / growth / extent)
};

// ---- graph networks read from a .gnn file (complab3d_graphnet.hh restated; section below)
struct GnnLaw {
    int nS = 0, nR = 0, W = 0, rounds = 0;
    bool extent = false, growth = false;
    double unit = 1.0, xymin = -1.0, yymin = -1.0;
    std::vector<std::string> species;
    std::vector<double> S;  // nS x nR
    std::vector<double> da, xiscale, xoff, xgain, yoff, ygain, tmin, tmax, Wenc, benc, Wout, bout;
    std::vector<std::vector<double>> Wsr, Wss, Wrs, Wda, bR, bS;  // per round
    std::vector<int> sp;  // binding: species index of each network species
};

// ---- surrogate organisms: .srg networks (complab3d_surrogate.hh restated; section below)
struct SrgLaw {
    int nIn = 0;
    std::vector<int> sizes;
    std::vector<std::vector<double>> W, B;
    std::vector<double> xoff, xgain, tmin, tmax, yoff, ygain;
    double xymin = -1.0, yymin = -1.0;
    bool logout = false;
    std::vector<std::string> inputs;
    std::vector<int> subs;            // binding: species index of each input
    std::vector<double> kc, vmax;     // per species
    double mw = 1.0, kd = 0.0;
};

struct OrcAde {
    int nx, ny, nz, S, M;
    size_t N;
    std::vector<int8_t> mat;
    int dyn[256];       // ADE_* per material code (mobile species)
    int react[256];     // 1 where kinetics runs (mask not solid / wall)
    std::vector<double> wpore, wbio, c0, lbc, rbc;
    std::vector<int> mobile, ltype, rtype;
    std::vector<double> u;                 // [3][N]
    std::vector<std::vector<double>> g, gp;  // per species [N][7]
    std::vector<std::vector<double>> imm;   // immobile species: concentration [N]
    std::vector<double> bio;                // biomass [M][N]
    std::vector<double> lstore, rstore;     // stored boundary densities [S][ny*nz]
    int law = LAW_NONE;
    std::vector<double> prm;
    // thermodynamic gate of the biotic rates (complab3d_thermo.hh; one reaction block)
    int gate_on = 0;
    std::vector<int> gate_sp;
    std::vector<double> gate_nu;
    double gate_dG0 = 0, gate_atp = 0, gate_dGatp = 50, gate_chi = 1, gate_cmin = 1e-9, gate_dGloss = 0;
    double gate_T = 298.15, gate_R = 8.314462618e-3, gate_cscale = 1;
    double dt = 1.0;
    long iters = 0;
    void* spec = nullptr;  // EqTableau of the speciation step, or none
    // abiotic rate law (run_abiotic_kinetics / surfaceAbioticKinetics3D)
    int law2 = LAW_NONE;
    std::vector<SymLaw> sym;             // [microbe] then the abiotic law at index 8
    unsigned sym_mask = 0;
    std::vector<GnnLaw> gnn;             // graph networks in the same slots
    unsigned gnn_mask = 0;
    int gnn_abiotic = 0;
    std::vector<SrgLaw> srg;             // surrogate organisms [microbe]
    unsigned srg_mask = 0;
    std::vector<double> prm2;
    int surf = 0;
    // precipitation sealing and dissolution (precipitationVOP.hh, dissolutionVOP.hh)
    int pr_on = 0, sM = -1, pcode = 0, porecode = 2, dis_on = 0, dis_law = DISSOL_NONE, dis_surf = 1;
    double full = 0, reopen = 0.9;
    std::vector<double> dprm;
    std::vector<uint8_t> stamp;  // 1 where the voxel was sealed by precipitation (phase id)
    // species dynamics map (the material each species lattice's dynamics were last chosen from);
    // `mat` is the mask lattice. They differ only between a CA mask change and the next
    // updateSoluteDynamics3D.
    std::vector<int8_t> dmat;
    // biofilm cellular automaton (complab3d_processors_part1.hh:499-732, part2.hh:71-259, :840-965)
    int ca_on = 0;
    int half = 0;       // push mode: 0 'fraction' (pushExcessBiomass3D), 1 'half' (halfPushExcessBiomass3D)
    double Bmax = 0, bfrac = 0;
    uint64_t seed = 0, sweeps = 0;
    std::vector<int> pore_codes, bio_code;
    int bbc = -1, solc = -1;
    std::vector<double> total;
    std::vector<int> age;
    std::vector<int8_t> distp;  // 1 where the distance field is positive
    long long old_mask_sum = 0;
    size_t id(int x, int y, int z) const { return ((size_t)x * ny + y) * nz + z; }
    // the lattice dynamics of species s at node n
    int node_dyn(int s, int x, size_t n) const {
        if ((x == 0 && ltype[s] == BC_CLOSED) || (x == nx - 1 && rtype[s] == BC_CLOSED)) return ADE_BB;
        return dyn[(uint8_t)(dmat.empty() ? mat[n] : dmat[n])];
    }
};

extern "C" {

OrcAde* orc_ade_create(int nx, int ny, int nz, const int8_t* mat, int S, const int32_t* dyn_by_code,
                       const int32_t* react_by_code, const double* omega_pore, const double* omega_bio,
                       const int32_t* mobile, const int32_t* left_type, const int32_t* right_type,
                       const double* left_bc, const double* right_bc, const double* c0, const double* u) {
    OrcAde* A = new OrcAde();
    A->nx = nx; A->ny = ny; A->nz = nz; A->S = S; A->M = 0;
    A->N = (size_t)nx * ny * nz;
    A->mat.assign(mat, mat + A->N);
    for (int k = 0; k < 256; ++k) { A->dyn[k] = dyn_by_code[k]; A->react[k] = react_by_code[k]; }
    A->wpore.assign(omega_pore, omega_pore + S);
    A->wbio.assign(omega_bio, omega_bio + S);
    A->mobile.assign(mobile, mobile + S);
    A->ltype.assign(left_type, left_type + S);
    A->rtype.assign(right_type, right_type + S);
    A->lbc.assign(left_bc, left_bc + S);
    A->rbc.assign(right_bc, right_bc + S);
    A->c0.assign(c0, c0 + S);
    A->u.assign(u, u + 3 * A->N);
    A->g.resize(S);
    A->gp.resize(S);
    A->imm.resize(S);
    const size_t P = (size_t)ny * nz;
    A->lstore.assign((size_t)S * P, 0.0);
    A->rstore.assign((size_t)S * P, 0.0);
    for (int s = 0; s < S; ++s) {
        double c = c0[s];
        if (c < THRD && c > -THRD) c = 0;  // stabilizeADElattice3D
        if (!mobile[s]) {
            A->imm[s].assign(A->N, c0[s]);
            continue;
        }
        // every node at equilibrium at c0 with u = 0 (initializeAtEquilibrium for BGK nodes,
        // stabilizeADElattice3D for wall and solid nodes); closed planes keep these values.
        A->g[s].assign(A->N * Q7, 0.0);
        A->gp[s].assign(A->N * Q7, 0.0);
        for (size_t n = 0; n < A->N; ++n)
            for (int i = 0; i < Q7; ++i) A->g[s][n * Q7 + i] = T7[i] * (c - 1.0);
        for (size_t p = 0; p < P; ++p) {
            A->lstore[(size_t)s * P + p] = left_type[s] == BC_DIRICHLET ? left_bc[s] : c0[s];
            A->rstore[(size_t)s * P + p] = right_type[s] == BC_DIRICHLET ? right_bc[s] : c0[s];
        }
    }
    return A;
}

void orc_ade_destroy(OrcAde* A) { delete A; }

/* law parameters:
 *   LAW_DECAY:      k[S]                      R_s = -k_s C_s
 *   LAW_MONOD:      k[S], Ks[S]               R_s = -k_s C_s / (Ks_s + C_s)
 *   LAW_DUAL_MONOD: mu_max, Ks, Y, kd         per microbe m (biomass field m):
 *                   growth = mu_max * C0/(Ks+C0) * Ca/(Ks+Ca) * B_m,  a = 1 + m
 *                   R_B = growth - kd B_m;  R_0 -= growth / Y;  R_a -= growth / Y */
void orc_ade_set_kinetics(OrcAde* A, int law, const double* prm, int nprm, double dt) {
    A->law = law;
    A->prm.assign(prm, prm + nprm);
    A->dt = dt;
}

/* One reaction block of a .thm file, energies in kJ/mol: n terms (species, nu), dG0, atp, dGatp,
 * chi, cmin, dGloss, temperature, gas constant, concentration scale. n = 0 turns the gate off. */
void orc_ade_set_thermo(OrcAde* A, int n, const int32_t* sp, const double* nu, const double* v) {
    A->gate_on = n > 0;
    A->gate_sp.assign(sp, sp + n);
    A->gate_nu.assign(nu, nu + n);
    A->gate_dG0 = v[0]; A->gate_atp = v[1]; A->gate_dGatp = v[2]; A->gate_chi = v[3];
    A->gate_cmin = v[4]; A->gate_dGloss = v[5]; A->gate_T = v[6]; A->gate_R = v[7]; A->gate_cscale = v[8];
}

static double thermo_factor(const OrcAde* A, const double* C);
double orc_thermo_factor(OrcAde* A, const double* C) { return thermo_factor(A, C); }

void orc_ade_set_biomass(OrcAde* A, int M, const double* b) {
    A->M = M;
    A->bio.assign(b, b + (size_t)M * A->N);
}


// =====================================================================================
//          RATE LAWS READ FROM A .sym FILE (complab3d_symbolic.hh, restated)
// =====================================================================================
// The file's keywords, the expression grammar and the evaluation rules of the reference's run-time
// rate laws: a tree per rate line evaluated recursively; division by a number below 1e-300 gives 0,
// a negative base to a fractional power 0, log / log10 / sqrt of a non-positive number 0; a NaN rate
// is 0 and a rate is held within +-1e300; variables are clamped to their ranges; rates are scaled
// by the unit (per_hour / 3600) but later lines see the unscaled values; a 'reaction' line derives
// the species lines (nu / |nu_key| / Y * growth * biomass, or nu * extent, coefficients written with
// 10 significant digits).
namespace {
struct SymParser {
    const std::vector<std::string>& scope;
    std::vector<SymNode>& nodes;
    std::string s;
    size_t p = 0;
    bool ok = true;
    SymParser(const std::vector<std::string>& sc, std::vector<SymNode>& n) : scope(sc), nodes(n) {}
    int mk(int k, int a = -1, int b = -1, double v = 0.0) {
        nodes.push_back(SymNode{k, v, a, b});
        return (int)nodes.size() - 1;
    }
    void sk() {
        while (p < s.size() && (s[p] == ' ' || s[p] == '\t')) ++p;
    }
    int expr() {
        int l = term();
        for (;;) {
            sk();
            if (!ok || p >= s.size()) return l;
            if (s[p] == '+') { ++p; l = mk(3, l, term()); }
            else if (s[p] == '-') { ++p; l = mk(4, l, term()); }
            else return l;
        }
    }
    int term() {
        int l = unary();
        for (;;) {
            sk();
            if (!ok || p >= s.size()) return l;
            if (s[p] == '*') { ++p; l = mk(5, l, unary()); }
            else if (s[p] == '/') { ++p; l = mk(6, l, unary()); }
            else return l;
        }
    }
    int unary() {
        sk();
        if (p < s.size() && s[p] == '-') { ++p; return mk(2, unary()); }
        if (p < s.size() && s[p] == '+') { ++p; return unary(); }
        int b = atom();
        sk();
        if (p < s.size() && s[p] == '^') { ++p; return mk(7, b, unary()); }
        return b;
    }
    int atom() {
        sk();
        if (p >= s.size()) { ok = false; return mk(0); }
        if (s[p] == '(') {
            ++p;
            int e = expr();
            sk();
            if (p < s.size() && s[p] == ')') ++p; else ok = false;
            return e;
        }
        if (std::isdigit((unsigned char)s[p]) || s[p] == '.') {
            char* e = nullptr;
            const double v = std::strtod(s.c_str() + p, &e);
            if (e == s.c_str() + p) { ok = false; return mk(0); }
            p = (size_t)(e - s.c_str());
            return mk(0, -1, -1, v);
        }
        if (std::isalpha((unsigned char)s[p]) || s[p] == '_') {
            size_t q = p;
            while (p < s.size() && (std::isalnum((unsigned char)s[p]) || s[p] == '_')) ++p;
            const std::string id = s.substr(q, p - q);
            sk();
            if (p < s.size() && s[p] == '(') {
                ++p;
                int a = expr(), b = -1;
                const bool two = id == "min" || id == "max" || id == "pow";
                sk();
                if (two) { if (p < s.size() && s[p] == ',') { ++p; b = expr(); } else ok = false; }
                sk();
                if (p < s.size() && s[p] == ')') ++p; else ok = false;
                static const char* f1[] = {"exp", "log", "log10", "sqrt", "abs", "tanh"};
                for (int k = 0; k < 6; ++k) if (id == f1[k]) return mk(8 + k, a);
                if (id == "min") return mk(14, a, b);
                if (id == "max") return mk(15, a, b);
                if (id == "pow") return mk(7, a, b);
                ok = false;
                return mk(0);
            }
            if (id == "pi") return mk(0, -1, -1, 3.14159265358979323846);
            if (id == "e") return mk(0, -1, -1, 2.71828182845904523536);
            for (size_t i = 0; i < scope.size(); ++i) if (scope[i] == id) return mk(1, (int)i);
            ok = false;
            return mk(0);
        }
        ok = false;
        return mk(0);
    }
};

double sym_node(const std::vector<SymNode>& n, int i, const std::vector<double>& v) {
    const SymNode& d = n[(size_t)i];
    switch (d.kind) {
        case 0: return d.value;
        case 1: return v[(size_t)d.a];
        case 2: return -sym_node(n, d.a, v);
        case 3: return sym_node(n, d.a, v) + sym_node(n, d.b, v);
        case 4: return sym_node(n, d.a, v) - sym_node(n, d.b, v);
        case 5: return sym_node(n, d.a, v) * sym_node(n, d.b, v);
        case 6: { const double q = sym_node(n, d.b, v); return std::fabs(q) < 1e-300 ? 0.0 : sym_node(n, d.a, v) / q; }
        case 7: { const double b = sym_node(n, d.a, v), e = sym_node(n, d.b, v);
                  return (b < 0.0 && e != std::floor(e)) ? 0.0 : std::pow(b, e); }
        case 8: return std::exp(sym_node(n, d.a, v));
        case 9: { const double x = sym_node(n, d.a, v); return x > 0.0 ? std::log(x) : 0.0; }
        case 10: { const double x = sym_node(n, d.a, v); return x > 0.0 ? std::log10(x) : 0.0; }
        case 11: { const double x = sym_node(n, d.a, v); return x > 0.0 ? std::sqrt(x) : 0.0; }
        case 12: return std::fabs(sym_node(n, d.a, v));
        case 13: return std::tanh(sym_node(n, d.a, v));
        case 14: { const double x = sym_node(n, d.a, v), y = sym_node(n, d.b, v); return x < y ? x : y; }
        case 15: { const double x = sym_node(n, d.a, v), y = sym_node(n, d.b, v); return x > y ? x : y; }
    }
    return 0.0;
}

bool sym_add(SymLaw& L, const std::string& name, const std::string& ex) {
    std::vector<std::string> scope = L.vars;
    scope.insert(scope.end(), L.rates.begin(), L.rates.end());
    SymParser P(scope, L.nodes);
    P.s = ex;
    const int root = P.expr();
    P.sk();
    if (!P.ok || P.p != P.s.size()) return false;
    L.rates.push_back(name);
    L.roots.push_back(root);
    return true;
}

bool sym_load(const char* path, SymLaw& L) {
    L = SymLaw();
    FILE* f = std::fopen(path, "r");
    if (!f) return false;
    char buf[4096];
    std::vector<std::pair<std::string, double>> st;
    std::string yof, bio;
    double y = 0;
    bool ok = true;
    while (ok && std::fgets(buf, sizeof buf, f)) {
        std::string l(buf);
        const size_t h = l.find('#');
        if (h != std::string::npos) l = l.substr(0, h);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
        std::istringstream in(l);
        std::string key;
        if (!(in >> key)) continue;
        const std::string rest = l.substr(l.find(key) + key.size());
        if (key == "version") continue;
        if (key == "units") {
            std::string u;
            in >> u;
            for (char& c : u) c = (char)std::tolower((unsigned char)c);
            if (u == "per_hour" || u == "per_hr" || u == "h") L.unit = 1.0 / 3600.0;
        } else if (key == "vars") {
            std::string w;
            while (in >> w) L.vars.push_back(w);
            L.lo.assign(L.vars.size(), 0.0);
            L.hi.assign(L.vars.size(), -1.0);
        } else if (key == "range") {
            std::string nm;
            double a, b;
            in >> nm >> a >> b;
            for (size_t i = 0; i < L.vars.size(); ++i) if (L.vars[i] == nm) { L.lo[i] = a; L.hi[i] = b; }
        } else if (key == "rate") {
            const size_t eq = rest.find('=');
            std::istringstream nn(rest.substr(0, eq));
            std::string nm;
            nn >> nm;
            ok = sym_add(L, nm, rest.substr(eq + 1));
        } else if (key == "reaction") {
            std::string nm;
            double nu;
            while (in >> nm >> nu) st.push_back({nm, nu});
        } else if (key == "yield") {
            in >> yof >> y;
        } else if (key == "biomass") {
            in >> bio;
        }
    }
    std::fclose(f);
    if (!ok) return false;
    for (const std::string& r : L.rates) L.extent |= r == "extent";
    char b2[256];
    if (!st.empty() && L.extent) {
        for (const auto& t : st) { std::snprintf(b2, sizeof b2, "%.10g * extent", t.second); if (!sym_add(L, t.first, b2)) return false; }
    } else if (!st.empty()) {
        double key = 0;
        for (const auto& t : st) if (t.first == yof) key = t.second;
        const double mag = key < 0 ? -key : key;
        for (const auto& t : st) {
            std::snprintf(b2, sizeof b2, "%.10g * growth * %s", (t.second / mag) / y, bio.c_str());
            if (!sym_add(L, t.first, b2)) return false;
        }
    }
    return !L.rates.empty();
}

void sym_rates(const SymLaw& L, const double* x, double* out) {
    const size_t nv = L.vars.size();
    std::vector<double> v(nv + L.rates.size(), 0.0);
    for (size_t i = 0; i < nv; ++i) {
        double a = x[i];
        if (L.hi[i] > L.lo[i]) a = a < L.lo[i] ? L.lo[i] : (a > L.hi[i] ? L.hi[i] : a);
        v[i] = a;
    }
    for (size_t r = 0; r < L.rates.size(); ++r) {
        double y = sym_node(L.nodes, L.roots[r], v);
        if (y != y) y = 0.0;
        if (y > 1e300) y = 1e300; else if (y < -1e300) y = -1e300;
        v[nv + r] = y;
        out[r] = y * L.unit;
    }
}
}  // namespace

// Reads a .gnn file: keywords then their numbers; '#' comments and `provenance` to the end of the
// line; `species` / `reactions` with their names on the rest of the line; the per-round arrays
// after `layer l`. False on anything missing or unknown.
bool gnn_load(const char* path, GnnLaw& G) {
    G = GnnLaw();
    std::FILE* f = std::fopen(path, "r");
    if (!f) return false;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    std::istringstream in(text);
    auto read_n = [&](std::vector<double>& v, int n) {
        v.assign((size_t)std::max(n, 0), 0.0);
        for (auto& x : v)
            if (!(in >> x)) return false;
        return true;
    };
    int cur = -1;
    bool stoich = false;
    std::string k;
    while (in >> k) {
        if (k[0] == '#' || k == "provenance") {
            std::string rest;
            std::getline(in, rest);
        } else if (k == "species" || k == "reactions") {
            std::string rest, w;
            std::getline(in, rest);
            if (k == "species") {
                std::istringstream ws(rest);
                while (ws >> w) G.species.push_back(w);
            }
        } else if (k == "version") {
            int v;
            if (!(in >> v)) return false;
        } else if (k == "units") {
            std::string u;
            in >> u;
            for (auto& c : u) c = (char)std::tolower((unsigned char)c);
            if (u == "per_hour") G.unit = 1.0 / 3600.0;
            else if (u != "per_second") return false;
        } else if (k == "rounds") {
            if (!(in >> G.rounds)) return false;
        } else if (k == "width") {
            if (!(in >> G.W)) return false;
        } else if (k == "growth") {
            int v;
            if (!(in >> v)) return false;
            G.growth = v != 0;
        } else if (k == "readout") {
            std::string m;
            in >> m;
            for (auto& c : m) c = (char)std::tolower((unsigned char)c);
            if (m == "extent") G.extent = true;
            else if (m != "species") return false;
        } else if (k == "stoich") {
            if (!(in >> G.nS >> G.nR) || !read_n(G.S, G.nS * G.nR)) return false;
            stoich = true;
        } else if (!stoich) {
            return false;
        } else {
            const int nys = G.extent ? (G.growth ? 1 : 0) : G.nS + (G.growth ? 1 : 0);
            const int nh = G.growth ? 2 : 1;
            bool ok = true;
            if (k == "da") ok = read_n(G.da, G.nR);
            else if (k == "xoffset") ok = read_n(G.xoff, G.nS);
            else if (k == "xgain") ok = read_n(G.xgain, G.nS);
            else if (k == "xymin") ok = (bool)(in >> G.xymin);
            else if (k == "yoffset") ok = read_n(G.yoff, nys);
            else if (k == "ygain") ok = read_n(G.ygain, nys);
            else if (k == "xiscale") ok = read_n(G.xiscale, G.nR);
            else if (k == "yymin") ok = (bool)(in >> G.yymin);
            else if (k == "trainmin") ok = read_n(G.tmin, G.nS);
            else if (k == "trainmax") ok = read_n(G.tmax, G.nS);
            else if (k == "Wenc") ok = read_n(G.Wenc, G.W);
            else if (k == "benc") ok = read_n(G.benc, G.W);
            else if (k == "Wout") ok = read_n(G.Wout, nh * G.W);
            else if (k == "bout") ok = read_n(G.bout, nh);
            else if (k == "layer") {
                ok = (bool)(in >> cur) && cur >= 0 && cur < G.rounds;
                if (ok && G.Wsr.size() < (size_t)G.rounds) {
                    G.Wsr.resize(G.rounds); G.Wss.resize(G.rounds); G.Wrs.resize(G.rounds);
                    G.Wda.resize(G.rounds); G.bR.resize(G.rounds); G.bS.resize(G.rounds);
                }
            } else if (cur >= 0 && k == "Wsr") ok = read_n(G.Wsr[cur], G.W * G.W);
            else if (cur >= 0 && k == "Wss") ok = read_n(G.Wss[cur], G.W * G.W);
            else if (cur >= 0 && k == "Wrs") ok = read_n(G.Wrs[cur], G.W * G.W);
            else if (cur >= 0 && k == "Wda") ok = read_n(G.Wda[cur], G.W);
            else if (cur >= 0 && k == "bR") ok = read_n(G.bR[cur], G.W);
            else if (cur >= 0 && k == "bS") ok = read_n(G.bS[cur], G.W);
            else return false;
            if (!ok) return false;
        }
    }
    if (!stoich || G.W < 1 || G.rounds < 1 || (int)G.species.size() != G.nS) return false;
    if ((int)G.Wsr.size() != G.rounds) return false;
    for (int l = 0; l < G.rounds; ++l)
        if (G.Wsr[l].empty() || G.Wss[l].empty() || G.Wrs[l].empty() || G.Wda[l].empty() || G.bR[l].empty() ||
            G.bS[l].empty())
            return false;
    return (int)G.da.size() == G.nR && (int)G.tmin.size() == G.nS && (int)G.tmax.size() == G.nS &&
           !G.Wenc.empty() && !G.bout.empty() && (!G.extent || (int)G.xiscale.size() == G.nR);
}

// The forward pass of complab_gnn::Network::eval (complab3d_graphnet.hh:215-332), restated: encode
// each species node from its clamped, scaled concentration; per round, reaction nodes from the
// stoichiometry-weighted species states, then species nodes from their own state and the weighted
// reaction states; read the rates off the species nodes (SPECIES) or as extents off the reaction
// nodes (EXTENT), and growth off the mean species node. Returns whether the clamp acted.
bool gnn_rates(const GnnLaw& G, const double* c, double* out) {
    const int W = G.W, nS = G.nS, nR = G.nR;
    auto S = [&](int i, int r) { return G.S[(size_t)i * nR + r]; };
    std::vector<std::vector<double>> hs(nS, std::vector<double>(W)), hr(nR, std::vector<double>(W));
    bool clamped = false;
    for (int i = 0; i < nS; ++i) {
        const double ci = c[i] < G.tmin[i] ? G.tmin[i] : (c[i] > G.tmax[i] ? G.tmax[i] : c[i]);
        clamped = clamped || ci != c[i];
        const double x = (ci - G.xoff[i]) * G.xgain[i] + G.xymin;
        for (int h = 0; h < W; ++h) hs[i][h] = std::tanh(x * G.Wenc[h] + G.benc[h]);
    }
    std::vector<double> msg(W);
    for (int l = 0; l < G.rounds; ++l) {
        for (int r = 0; r < nR; ++r) {
            std::fill(msg.begin(), msg.end(), 0.0);
            for (int i = 0; i < nS; ++i)
                if (S(i, r) != 0.0)
                    for (int k = 0; k < W; ++k) msg[k] += S(i, r) * hs[i][k];
            for (int h = 0; h < W; ++h) {
                double a = G.bR[l][h] + G.da[r] * G.Wda[l][h];
                for (int k = 0; k < W; ++k) a += G.Wsr[l][(size_t)h * W + k] * msg[k];
                hr[r][h] = std::tanh(a);
            }
        }
        std::vector<std::vector<double>> next(nS, std::vector<double>(W));
        for (int i = 0; i < nS; ++i) {
            std::fill(msg.begin(), msg.end(), 0.0);
            for (int r = 0; r < nR; ++r)
                if (S(i, r) != 0.0)
                    for (int k = 0; k < W; ++k) msg[k] += S(i, r) * hr[r][k];
            for (int h = 0; h < W; ++h) {
                double a = G.bS[l][h];
                for (int k = 0; k < W; ++k)
                    a += G.Wss[l][(size_t)h * W + k] * hs[i][k] + G.Wrs[l][(size_t)h * W + k] * msg[k];
                next[i][h] = std::tanh(a);
            }
        }
        hs.swap(next);
    }
    if (G.extent) {
        std::vector<double> xi(nR);
        for (int r = 0; r < nR; ++r) {
            double y = G.bout[0];
            for (int h = 0; h < W; ++h) y += G.Wout[h] * hr[r][h];
            xi[r] = (y == y ? y : 0.0) * G.xiscale[r];
        }
        for (int i = 0; i < nS; ++i) {
            double v = 0.0;
            for (int r = 0; r < nR; ++r) v += S(i, r) * xi[r];
            out[i] = v * G.unit;
        }
    } else {
        for (int i = 0; i < nS; ++i) {
            double y = G.bout[0];
            for (int h = 0; h < W; ++h) y += G.Wout[h] * hs[i][h];
            const double v = (y - G.yymin) / G.ygain[i] + G.yoff[i];
            out[i] = (v == v ? v : 0.0) * G.unit;
        }
    }
    if (G.growth) {
        const int gs = G.extent ? 0 : nS;
        double y = G.bout[1];
        for (int h = 0; h < W; ++h) {
            double sum = 0.0;
            for (int i = 0; i < nS; ++i) sum += hs[i][h];
            y += G.Wout[(size_t)W + h] * (sum / (double)nS);
        }
        const double v = (y - G.yymin) / G.ygain[gs] + G.yoff[gs];
        out[nS] = (v == v ? v : 0.0) * G.unit;
    }
    return clamped;
}

// Reads a .srg file (keywords, '#' comments, `layers` / `inputnames` / `outputnames` / `yoffset` /
// `ygain` / `outrange` on the rest of their line, `W l` and `B l` blocks); false on anything
// missing.
bool srg_load(const char* path, SrgLaw& Q) {
    Q = SrgLaw();
    std::FILE* f = std::fopen(path, "r");
    if (!f) return false;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    std::istringstream in(text);
    auto rest = [&]() {
        std::string r;
        std::getline(in, r);
        std::istringstream ws(r);
        std::vector<std::string> w;
        std::string t;
        while (ws >> t) w.push_back(t);
        return w;
    };
    auto nums = [&](std::vector<double>& v, int n) {
        v.assign((size_t)std::max(n, 0), 0.0);
        for (auto& x : v)
            if (!(in >> x)) return false;
        return true;
    };
    std::string k;
    while (in >> k) {
        if (k[0] == '#') { rest(); continue; }
        if (k == "version") { int v; if (!(in >> v)) return false; }
        else if (k == "inputs") { if (!(in >> Q.nIn)) return false; }
        else if (k == "layers") { Q.sizes.clear(); for (auto& w : rest()) Q.sizes.push_back(std::atoi(w.c_str())); }
        else if (k == "logoutput") { int v; if (!(in >> v)) return false; Q.logout = v != 0; }
        else if (k == "inputnames") Q.inputs = rest();
        else if (k == "outputnames" || k == "outrange") rest();
        else if (k == "xoffset") { if (!nums(Q.xoff, Q.nIn)) return false; }
        else if (k == "xgain") { if (!nums(Q.xgain, Q.nIn)) return false; }
        else if (k == "trainmin") { if (!nums(Q.tmin, Q.nIn)) return false; }
        else if (k == "trainmax") { if (!nums(Q.tmax, Q.nIn)) return false; }
        else if (k == "xymin") { if (!(in >> Q.xymin)) return false; }
        else if (k == "yymin") { if (!(in >> Q.yymin)) return false; }
        else if (k == "outputs") { int v; if (!(in >> v)) return false; }
        else if (k == "yoffset" || k == "ygain") {
            std::vector<double>& v = k == "yoffset" ? Q.yoff : Q.ygain;
            v.clear();
            for (auto& w : rest()) v.push_back(std::atof(w.c_str()));
        } else if (k == "W" || k == "B") {
            int L;
            if (!(in >> L) || L < 0 || L + 1 >= (int)Q.sizes.size()) return false;
            if ((int)Q.W.size() < L + 1) { Q.W.resize(L + 1); Q.B.resize(L + 1); }
            const int rows = Q.sizes[L + 1], cols = Q.sizes[L];
            if (!nums(k == "W" ? Q.W[L] : Q.B[L], k == "W" ? rows * cols : rows)) return false;
        } else return false;
    }
    const int nL = (int)Q.sizes.size() - 1;
    if (Q.nIn <= 0 || nL < 1 || (int)Q.W.size() != nL || (int)Q.B.size() != nL) return false;
    for (int l = 0; l < nL; ++l)
        if ((int)Q.W[l].size() != Q.sizes[l + 1] * Q.sizes[l] || (int)Q.B[l].size() != Q.sizes[l + 1]) return false;
    if ((int)Q.tmin.size() < Q.nIn || (int)Q.tmax.size() < Q.nIn) return false;
    const int nO = Q.sizes.back();
    Q.yoff.resize((size_t)nO, 0.0);
    if ((int)Q.ygain.size() < nO) Q.ygain.resize((size_t)nO, 1.0);
    return true;
}

// Network::evalAll (complab3d_surrogate.hh:200-235) after evalBound's clamp (:1029-1049), restated:
// every output; returns whether the clamp acted
bool srg_outputs(const SrgLaw& Q, const double* x, double* out) {
    std::vector<double> a((size_t)Q.nIn);
    bool clamped = false;
    for (int i = 0; i < Q.nIn; ++i) {
        double v = x[i];
        if (v < Q.tmin[i]) { v = Q.tmin[i]; clamped = true; }
        else if (v > Q.tmax[i]) { v = Q.tmax[i]; clamped = true; }
        a[(size_t)i] = (v - Q.xoff[i]) * Q.xgain[i] + Q.xymin;
    }
    const size_t nL = Q.W.size();
    for (size_t l = 0; l < nL; ++l) {
        const int rows = Q.sizes[l + 1], cols = Q.sizes[l];
        std::vector<double> o((size_t)rows);
        for (int r = 0; r < rows; ++r) {
            double t = Q.B[l][(size_t)r];
            for (int c = 0; c < cols; ++c) t += Q.W[l][(size_t)r * cols + c] * a[(size_t)c];
            o[(size_t)r] = (l + 1 == nL) ? t : 2.0 / (1.0 + std::exp(-2.0 * t)) - 1.0;
        }
        a.swap(o);
    }
    const int nO = Q.sizes.back();
    for (int k = 0; k < nO; ++k) {
        const double gain = Q.ygain[k] != 0.0 ? Q.ygain[k] : 1.0;
        out[k] = (a[(size_t)k] - Q.yymin) / gain + Q.yoff[k];
    }
    if (Q.logout) out[0] = std::pow(10.0, out[0]);
    if (!(out[0] > 1e-8)) out[0] = 0.0;
    for (int k = 1; k < nO; ++k)
        if (out[k] != out[k]) out[k] = 0.0;
    return clamped;
}

extern "C" {

// standalone evaluation of a .srg file on n rows of its inputs, clamped to its training box
int orc_srg_eval(const char* path, int n, const double* x, double* out, int* n_out) {
    SrgLaw Q;
    if (!srg_load(path, Q)) return -1;
    const int no = Q.sizes.back();
    *n_out = no;
    for (int i = 0; i < n; ++i) srg_outputs(Q, x + (size_t)i * Q.nIn, out + (size_t)i * no);
    return 0;
}

// binds a .srg file to the species (names: S newline-separated) as microbe m's surrogate, with its
// uptake parameters per species (kc, vmax), biomass molar mass and decay coefficient
int orc_ade_set_surrogate(OrcAde* A, const char* path, const char* names, int m, const double* kc,
                          const double* vmax, double mw, double kd) {
    SrgLaw Q;
    if (!srg_load(path, Q) || m < 0) return -1;
    std::vector<std::string> sp;
    std::istringstream in(names);
    std::string w;
    while (std::getline(in, w)) sp.push_back(w);
    for (int i = 0; i < Q.nIn; ++i) {
        int hit = -1;
        if (Q.inputs.empty()) hit = i < (int)sp.size() ? i : -1;
        else
            for (size_t s = 0; s < sp.size(); ++s) if (sp[s] == Q.inputs[(size_t)i]) hit = (int)s;
        if (hit < 0) return -2;
        Q.subs.push_back(hit);
    }
    Q.kc.assign(kc, kc + A->S);
    Q.vmax.assign(vmax, vmax + A->S);
    Q.mw = mw;
    Q.kd = kd;
    if ((int)A->srg.size() < 8) A->srg.resize(8);
    A->srg[(size_t)m] = Q;
    A->srg_mask |= 1u << m;
    A->sym_mask &= ~(1u << m);
    A->gnn_mask &= ~(1u << m);
    A->law = LAW_SYMBOLIC;
    return 0;
}

}  // extern "C"

extern "C" {

// standalone evaluation of a .gnn file on n rows of concentrations (the pinning test's entry point)
int orc_gnn_eval(const char* path, int n, const double* conc, double* out, int* n_out) {
    GnnLaw G;
    if (!gnn_load(path, G)) return -1;
    const int no = G.nS + (G.growth ? 1 : 0);
    *n_out = no;
    for (int i = 0; i < n; ++i) gnn_rates(G, conc + (size_t)i * G.nS, out + (size_t)i * no);
    return 0;
}

// binds a .gnn file to the species (names: S newline-separated names) as microbe m's law (m >= 0)
// or the abiotic law (m = -1)
int orc_ade_set_graph_network(OrcAde* A, const char* path, const char* names, int m) {
    GnnLaw G;
    if (!gnn_load(path, G)) return -1;
    std::vector<std::string> sp;
    std::istringstream in(names);
    std::string w;
    while (std::getline(in, w)) sp.push_back(w);
    for (const std::string& v : G.species) {
        int hit = -1;
        for (size_t s = 0; s < sp.size(); ++s) if (sp[s] == v) hit = (int)s;
        if (hit < 0) return -2;
        G.sp.push_back(hit);
    }
    if (m < 0 && G.growth) return -3;
    if (A->gnn.size() < 9) A->gnn.resize(9);
    if (m >= 0) {
        A->gnn[(size_t)m] = G;
        A->gnn_mask |= 1u << m;
        A->sym_mask &= ~(1u << m);
        A->srg_mask &= ~(1u << m);
        A->law = LAW_SYMBOLIC;
    } else {
        A->gnn[8] = G;
        A->gnn_abiotic = 1;
        A->law2 = LAW_SYMBOLIC;
    }
    return 0;
}

}  // extern "C"

extern "C" {

// standalone evaluation of a file on n rows of its variables (the pinning test's entry point)
int orc_sym_eval(const char* path, int n, const double* vars, double* out, int* n_rates) {
    SymLaw L;
    if (!sym_load(path, L)) return -1;
    const size_t nv = L.vars.size(), nr = L.rates.size();
    *n_rates = (int)nr;
    for (int i = 0; i < n; ++i) sym_rates(L, vars + (size_t)i * nv, out + (size_t)i * nr);
    return 0;
}

// binds a file to the species (names: S newline-separated names) as microbe m's law (m >= 0) or the
// abiotic law (m = -1)
int orc_ade_set_symbolic(OrcAde* A, const char* path, const char* names, int m, const char* microbe_name) {
    SymLaw L;
    if (!sym_load(path, L)) return -1;
    std::vector<std::string> sp;
    std::istringstream in(names);
    std::string w;
    while (std::getline(in, w)) sp.push_back(w);
    for (const std::string& v : L.vars) {
        int hit = -2;
        for (size_t s = 0; s < sp.size(); ++s) if (sp[s] == v) hit = (int)s;
        if (hit == -2 && m >= 0 && v == microbe_name) hit = -1;
        if (hit == -2) return -2;
        L.var_src.push_back(hit);
    }
    for (const std::string& r : L.rates) {
        int hit = -1;
        for (size_t s = 0; s < sp.size(); ++s) if (sp[s] == r) hit = (int)s;
        L.rate_dst.push_back(hit);
    }
    if (A->sym.size() < 9) A->sym.resize(9);
    if (m >= 0) {
        A->sym[(size_t)m] = L;
        A->sym_mask |= 1u << m;
        A->gnn_mask &= ~(1u << m);
        A->srg_mask &= ~(1u << m);
        A->law = LAW_SYMBOLIC;
    } else {
        A->sym[8] = L;
        A->gnn_abiotic = 0;
        A->law2 = LAW_SYMBOLIC;
    }
    return 0;
}

}  // extern "C"

static void rates(const OrcAde* A, const double* C, const double* B, double* R, double* RB) {
    const int S = A->S;
    for (int s = 0; s < S; ++s) R[s] = 0;
    for (int m = 0; m < A->M; ++m) RB[m] = 0;
    switch (A->law) {
        case LAW_DECAY:
            for (int s = 0; s < S; ++s) R[s] = -A->prm[s] * C[s];
            break;
        case LAW_MONOD:
            for (int s = 0; s < S; ++s) R[s] = -A->prm[s] * C[s] / (A->prm[S + s] + C[s]);
            break;
        case LAW_DUAL_MONOD: {
            double mu = A->prm[0], ks = A->prm[1], Y = A->prm[2], kd = A->prm[3];
            for (int m = 0; m < A->M; ++m) {
                int a = 1 + m;
                if (a >= S) break;
                double Bm = B[m];
                if (Bm <= 0.0) continue;
                double growth = mu * (C[0] / (ks + C[0])) * (C[a] / (ks + C[a])) * Bm;
                RB[m] += growth - kd * Bm;
                R[0] -= growth / Y;
                R[a] -= growth / Y;
            }
            break;
        }
        default:
            break;
    }
}

/* abiotic laws:
 *   LAW_PRECIP:  kp, a, b, p            A + B -> P,  R = kp max(C_a,0) max(C_b,0): R_a = R_b = -R, R_p = +R
 *                                       (defineAbioticRxnKinetics of examples/13_precipitation)
 *   LAW_MINERAL: k, log10 Ksp, p, nu[S] Omega = 10^(sum_j nu_j log10 C_j - log10 Ksp) over the dissolved
 *                                       species j != p; R_p = k (Omega - 1), R_j = -nu_j R_p */
static void rates2(const OrcAde* A, const double* C, double* R) {
    const int S = A->S;
    for (int s = 0; s < S; ++s) R[s] = 0;
    const std::vector<double>& p = A->prm2;
    if (A->law2 == LAW_PRECIP) {
        const int a = (int)p[1], b = (int)p[2], q = (int)p[3];
        const double r = p[0] * std::max(C[a], 0.0) * std::max(C[b], 0.0);
        R[a] -= r;
        R[b] -= r;
        R[q] += r;
    } else if (A->law2 == LAW_SYMBOLIC && A->gnn_abiotic) {
        // run_graphnet_abiotic3D (complab3d_processors_abiotic_learned.hh:200-235)
        const GnnLaw& G = A->gnn[8];
        std::vector<double> x((size_t)G.nS), y((size_t)G.nS + 1);
        for (int i = 0; i < G.nS; ++i) x[(size_t)i] = C[G.sp[(size_t)i]];
        gnn_rates(G, x.data(), y.data());
        for (int i = 0; i < G.nS; ++i) R[G.sp[(size_t)i]] += y[(size_t)i];
    } else if (A->law2 == LAW_SYMBOLIC) {
        const SymLaw& L = A->sym[8];
        std::vector<double> x(L.vars.size()), y(L.rates.size());
        for (size_t v = 0; v < x.size(); ++v) x[v] = C[L.var_src[v]];
        sym_rates(L, x.data(), y.data());
        for (size_t r = 0; r < y.size(); ++r)
            if (L.rate_dst[r] >= 0) R[L.rate_dst[r]] += y[r];
    } else if (A->law2 == LAW_MINERAL) {
        const int q = (int)p[2];
        double la = 0;
        for (int j = 0; j < S; ++j)
            if (j != q && p[3 + j] != 0.0) la += p[3 + j] * std::log10(std::max(C[j], 1e-30));
        const double rm = p[0] * (std::pow(10.0, la - p[1]) - 1.0);
        R[q] += rm;
        for (int j = 0; j < S; ++j)
            if (j != q) R[j] -= p[3 + j] * rm;
    }
}

/* dissolution laws of a sealed mineral voxel (defineDissolutionRate):
 *   DISSOL_FIRST_ORDER: kd, h, sigma[S]  rate = kd max(water_h,0) max(mineral,0) (h < 0: no water factor);
 *                                        mineral -rate, species j sigma_j rate (examples/15)
 *   DISSOL_MINERAL:     k, log10 Ksp, nu[S]  Omega of the water; below 1 the mineral dissolves at
 *                                        k (Omega - 1), releasing -nu_j times that */
struct DissolLaw {
    int law, S, sM;
    const double* p;
};

static void dissol_rate_p(const DissolLaw& L, const double* water, double mineral, double* subsR, double& mR) {
    const int S = L.S;
    for (int s = 0; s < S; ++s) subsR[s] = 0;
    mR = 0;
    const double* p = L.p;
    if (L.law == DISSOL_FIRST_ORDER) {
        const int h = (int)p[1];
        const double rate = p[0] * (h >= 0 ? std::max(water[h], 0.0) : 1.0) * std::max(mineral, 0.0);
        mR = -rate;
        for (int j = 0; j < S; ++j) subsR[j] = p[2 + j] * rate;
    } else if (L.law == DISSOL_MINERAL) {
        double la = 0;
        for (int j = 0; j < S; ++j)
            if (j != L.sM && p[2 + j] != 0.0) la += p[2 + j] * std::log10(std::max(water[j], 1e-30));
        const double om = std::pow(10.0, la - p[1]);
        if (om < 1.0) {
            mR = p[0] * (om - 1.0);
            for (int j = 0; j < S; ++j)
                if (j != L.sM) subsR[j] = -p[2 + j] * mR;
        }
    }
}

static const int DLOC[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// density of species s at voxel n as the processors see it between collide and stream
static double dens_post(const OrcAde* A, int s, size_t n) {
    if (!A->mobile[s]) return A->imm[s][n];
    double c = 0;
    for (int i = 0; i < Q7; ++i) c += A->gp[s][n * Q7 + i];
    return c + 1.0;
}

/* Dissolution of the stamped (precipitated) mineral voxels, added into dC[s][n]: pass 1 parks one
 * product share per open face in the mineral voxel's own increment slot and takes the mineral out
 * (surfaceDissolutionKinetics3D, dissolutionVOP.hh:379-605: water averaged over the open faces,
 * at most half the mineral per step, products scaled alike); pass 2 lets every open voxel collect
 * the shares of its mineral face neighbours, a negative share clamped to the headroom
 * (dissolutionGather3D, :608-742). dens(s, n) is the density the processors see, open(n) whether
 * the voxel is neither solid nor wall. */
extern "C++" {
template <typename Dens, typename Open>
static void dissolution_park_gather(int nx, int ny, int nz, int S, int sM, double dt, int surf, const uint8_t* stamp,
                                    const DissolLaw& L, Dens dens, Open open, std::vector<double>& dC) {
    const size_t N = (size_t)nx * ny * nz;
    auto id = [&](int x, int y, int z) { return ((size_t)x * ny + y) * nz + z; };
    // pass 1: park
    std::vector<double> water(S), subsR(S);
    for (int x = 1; x < nx - 1; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = id(x, y, z);
                if (!stamp[n]) continue;
                const double mineral = dens(sM, n);
                if (!(mineral > THRD)) continue;
                int opn[6], no = 0;
                for (int d = 0; d < 6; ++d) {
                    int X = x + DLOC[d][0], Y = y + DLOC[d][1], Z = z + DLOC[d][2];
                    if (X < 1 || X > nx - 2 || Y < 0 || Y > ny - 1 || Z < 0 || Z > nz - 1) continue;
                    if (!open(id(X, Y, Z))) continue;
                    opn[no++] = d;
                }
                if (no == 0 && surf) continue;
                for (int s2 = 0; s2 < S; ++s2) water[s2] = 0;
                if (no > 0) {
                    for (int k = 0; k < no; ++k) {
                        const int d = opn[k];
                        size_t m = id(x + DLOC[d][0], y + DLOC[d][1], z + DLOC[d][2]);
                        for (int s2 = 0; s2 < S; ++s2) water[s2] += dens(s2, m);
                    }
                    for (int s2 = 0; s2 < S; ++s2) water[s2] /= (double)no;
                }
                for (int s2 = 0; s2 < S; ++s2)
                    if (water[s2] < 0) water[s2] = 0;
                double mR;
                dissol_rate_p(L, water.data(), mineral, subsR.data(), mR);
                if (!(mR < 0)) continue;
                double dM = mR * dt;
                double scale = 1.0;
                const double maxRemove = 0.5 * mineral;
                if (-dM > maxRemove) scale = maxRemove / (-dM);
                dM *= scale;
                if (!(-dM > THRD)) continue;
                dC[(size_t)sM * N + n] += dM;
                if (no > 0)
                    for (int s2 = 0; s2 < S; ++s2) {
                        if (s2 == sM) continue;
                        const double rel = subsR[s2] * dt * scale;
                        if (std::fabs(rel) <= THRD) continue;
                        dC[(size_t)s2 * N + n] += rel / (double)no;
                    }
            }
    // pass 2: gather
    for (int x = 1; x < nx - 1; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = id(x, y, z);
                if (!open(n)) continue;
                for (int d = 0; d < 6; ++d) {
                    int X = x + DLOC[d][0], Y = y + DLOC[d][1], Z = z + DLOC[d][2];
                    if (X < 1 || X > nx - 2 || Y < 0 || Y > ny - 1 || Z < 0 || Z > nz - 1) continue;
                    size_t m = id(X, Y, Z);
                    if (!stamp[m]) continue;
                    for (int s2 = 0; s2 < S; ++s2) {
                        if (s2 == sM) continue;
                        const double share = dC[(size_t)s2 * N + m];
                        if (std::fabs(share) <= 1e-14) continue;
                        double give = share;
                        if (give < 0) {
                            const double have = dens(s2, n);
                            const double head = (have > 0 ? have : 0.0) + dC[(size_t)s2 * N + n];
                            if (give + head < 0) give = -head;
                            if (give > 0) give = 0;
                        }
                        if (!(std::fabs(give) > 1e-14)) continue;
                        dC[(size_t)s2 * N + n] += give;
                    }
                }
            }
}
}  // extern "C++"

/* One voxel of run_kinetics (complab3d_processors_part1.hh:85-187): concentrations and biomass
 * below the threshold read as zero, the rate law, increments R dt whose magnitude exceeds the
 * threshold, clamped so that no concentration or biomass goes below zero: dC = max(R dt, -C).
 * C and B are read and thresholded in place; dC / dB receive the increments (0 where none). */
/* The thermodynamic factor of Jin & Bethke (2003, 2005) on the concentrations the rate law saw,
 * used as activities (times the concentration scale, floored at cmin):
 *   ln Q = sum_i nu_i ln a_i,  dG = dG0 + R T ln Q + dGloss,  f = dG + m dG_ATP,
 *   F_T = max(0, 1 - exp(f / (chi R T)))   (0 at or past the threshold, 1 when exp underflows);
 * the steps and their order follow complab3d_thermo.hh:215-258. */
static double thermo_factor(const OrcAde* A, const double* C) {
    const double RT = A->gate_R * A->gate_T;
    double lq = 0.0;
    for (size_t i = 0; i < A->gate_nu.size(); ++i) {
        double a = C[A->gate_sp[i]] * A->gate_cscale;
        if (!(a > A->gate_cmin)) a = A->gate_cmin;
        lq += A->gate_nu[i] * std::log(a);
    }
    const double dG = A->gate_dG0 + RT * lq + A->gate_dGloss;
    const double f = dG + A->gate_atp * A->gate_dGatp;
    const double chi = A->gate_chi > 0.0 ? A->gate_chi : 1.0;
    const double x = f / (chi * RT);
    if (x >= 0.0) return 0.0;
    if (x < -700.0) return 1.0;
    const double F = 1.0 - std::exp(x);
    return F < 0.0 ? 0.0 : (F > 1.0 ? 1.0 : F);
}

// the organisms' .sym laws in one voxel (run_symbolic3D, complab3d_processors_symbolic.hh:100-200)
static void symbolic_voxel(const OrcAde* A, const double* C, const double* B, double* dC, double* dB) {
    const int S = A->S;
    std::vector<double> req(S, 0.0), x, y;
    for (int m = 0; m < A->M; ++m) {
        dB[m] = 0.0;
        const bool net = (A->gnn_mask >> m) & 1u;
        const bool srg = (A->srg_mask >> m) & 1u;
        if (!net && !srg && !((A->sym_mask >> m) & 1u)) continue;
        const double bm = B[m] > THRD ? B[m] : 0.0;
        if (!(bm > THRD)) continue;
        if (srg) {
            // run_surrogate3D (complab3d_processors_surrogate.hh:155-250) with the run-time network:
            // Michaelis-Menten uptake estimates (MetabolicConfig's unit chain,
            // complab3d_metabolic.hh:554-595) feed the network; its growth rate (or decay) moves the
            // biomass; the estimates are drawn from the substrates
            const SrgLaw& Q = A->srg[(size_t)m];
            std::vector<double> fin((size_t)S, 0.0);
            for (int s = 0; s < S; ++s) {
                const double av = C[s];
                const double mm = (Q.kc[(size_t)s] + av > 0.0) ? av / (Q.kc[(size_t)s] + av) : 0.0;
                double exh = 0.0;
                const double denom = bm * Q.mw * A->dt;
                if (denom > 1e-30) {
                    exh = -av * 3.6e6 / denom;
                    if (exh < -1e4) exh = -1e4;
                }
                double v = Q.vmax[(size_t)s] > THRD ? Q.vmax[(size_t)s] * mm : -exh * mm;
                const double cap = -exh;
                if (cap > 0.0 && v > cap) v = cap;
                fin[(size_t)s] = v;
            }
            std::vector<double> xs((size_t)Q.nIn), ys((size_t)Q.sizes.back());
            for (int i = 0; i < Q.nIn; ++i) xs[(size_t)i] = fin[(size_t)Q.subs[(size_t)i]];
            srg_outputs(Q, xs.data(), ys.data());
            double mu = ys[0];
            const double ft = (m == 0 && A->gate_on) ? thermo_factor(A, C) : 1.0;
            if (ft < 1.0) {
                for (auto& v : fin) v *= ft;
                mu *= ft;
            }
            double d = (std::fabs(mu) < THRD) ? -Q.kd * bm * A->dt : mu * bm * A->dt / 3600.0;
            if (d + bm < 0.0) d = -bm;
            if (d > THRD || d < -THRD) dB[m] = d;
            for (int s = 0; s < S; ++s) req[(size_t)s] += -(fin[(size_t)s] * (bm * Q.mw) * A->dt / 3.6e6);
            continue;
        }
        if (net) {
            // run_graphnet3D (complab3d_processors_graphnet.hh:120-200): the same budget
            const GnnLaw& G = A->gnn[(size_t)m];
            std::vector<double> xg((size_t)G.nS), yg((size_t)G.nS + 1);
            for (int i = 0; i < G.nS; ++i) xg[(size_t)i] = C[G.sp[(size_t)i]];
            gnn_rates(G, xg.data(), yg.data());
            const double ft = (m == 0 && A->gate_on) ? thermo_factor(A, C) : 1.0;
            for (int i = 0; i < G.nS; ++i) req[(size_t)G.sp[(size_t)i]] += yg[(size_t)i] * ft * A->dt;
            if (G.growth) {
                double d = yg[(size_t)G.nS] * ft * bm * A->dt;
                if (d > THRD || d < -THRD) {
                    if (d + bm < 0.0) d = -bm;
                    dB[m] = d;
                }
            }
            continue;
        }
        const SymLaw& L = A->sym[(size_t)m];
        x.resize(L.vars.size());
        y.resize(L.rates.size());
        for (size_t v = 0; v < L.vars.size(); ++v) x[v] = L.var_src[v] >= 0 ? C[L.var_src[v]] : bm;
        sym_rates(L, x.data(), y.data());
        const double ft = (m == 0 && A->gate_on) ? thermo_factor(A, C) : 1.0;
        double d = 0.0;
        for (size_t r = 0; r < y.size(); ++r) {
            if (L.rate_dst[r] >= 0) req[(size_t)L.rate_dst[r]] += y[r] * ft * A->dt;
            else d += y[r] * ft * bm * A->dt;
        }
        if (d > THRD || d < -THRD) {
            if (d + bm < 0.0) d = -bm;
            dB[m] = d;
        }
    }
    for (int s = 0; s < S; ++s) {
        dC[s] = 0.0;
        double draw = req[s];
        if (!(draw > THRD || draw < -THRD)) continue;
        if (draw + C[s] < 0.0) draw = -C[s];
        dC[s] = draw;
    }
}

static void biotic_voxel(const OrcAde* A, double* C, double* B, double* R, double* RB, double* dC, double* dB) {
    const int S = A->S;
    if (A->law == LAW_SYMBOLIC) {
        for (int s = 0; s < S; ++s) C[s] = C[s] > THRD ? C[s] : 0.0;
        symbolic_voxel(A, C, B, dC, dB);
        return;
    }
    for (int s = 0; s < S; ++s)
        if (C[s] < THRD) C[s] = 0;
    for (int m = 0; m < A->M; ++m)
        if (B[m] < THRD) B[m] = 0;
    rates(A, C, B, R, RB);
    // run_kinetics (complab3d_processors_part1.hh:134-141) scales the whole voxel's rates by the
    // factor of microbe 0's reaction block, so the gate acts only in a run with a microbe
    if (A->gate_on && A->M >= 1) {
        const double ft = thermo_factor(A, C);
        if (ft < 1.0) {
            for (int s = 0; s < S; ++s) R[s] *= ft;
            for (int m = 0; m < A->M; ++m) RB[m] *= ft;
        }
    }
    for (int s = 0; s < S; ++s) {
        double d = R[s] * A->dt;
        dC[s] = 0.0;
        if (!(d > THRD || d < -THRD)) continue;
        if (d + C[s] < 0.0) d = -C[s];
        if (!(d > THRD || d < -THRD)) continue;
        dC[s] = d;
    }
    for (int m = 0; m < A->M; ++m) {
        double d = RB[m] * A->dt;
        dB[m] = 0.0;
        if (!(d > THRD || d < -THRD)) continue;
        if (d + B[m] < 0.0) d = -B[m];
        dB[m] = d;
    }
}

/* The abiotic rate pass (run_abiotic_kinetics, complab3d_processors_part1.hh:199-297, or with the
 * surface-only rule surfaceAbioticKinetics3D, precipitationVOP.hh:53-153) over the interior
 * x-planes: increments R dt of magnitude above the threshold, clamped at -C, added into dC. */
extern "C++" {
template <class Dens>
static void abiotic_rate_pass(const OrcAde* A, Dens dens, double* dC) {
    const int nx = A->nx, ny = A->ny, nz = A->nz, S = A->S;
    const size_t N = A->N;
    auto inbox = [&](int x, int y, int z) { return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz; };
#pragma omp parallel for schedule(static)
    for (int x = 1; x < nx - 1; ++x) {
        std::vector<double> C(S), R(S);
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = A->id(x, y, z);
                if (!A->react[(uint8_t)A->mat[n]]) continue;
                if (A->surf) {
                    bool iface = false;
                    for (int d = 0; d < 6 && !iface; ++d) {
                        int X = x + DLOC[d][0], Y = y + DLOC[d][1], Z = z + DLOC[d][2];
                        if (!inbox(X, Y, Z)) continue;
                        if (!A->react[(uint8_t)A->mat[A->id(X, Y, Z)]]) iface = true;
                    }
                    if (!iface) continue;
                }
                for (int s2 = 0; s2 < S; ++s2) {
                    double c = dens(s2, n);
                    C[s2] = c < THRD ? 0.0 : c;
                }
                rates2(A, C.data(), R.data());
                for (int s2 = 0; s2 < S; ++s2) {
                    double d = R[s2] * A->dt;
                    if (!(d > THRD || d < -THRD)) continue;
                    if (d + C[s2] < 0.0) d = -C[s2];
                    if (!(d > THRD || d < -THRD)) continue;
                    dC[(size_t)s2 * N + n] += d;
                }
            }
    }
}
}  // extern "C++"

/* The abiotic block of complab.cpp:2460-2525 after the biotic increments are applied: abiotic
 * rates (with the clamp dC = max(R dt, -C)), dissolution of sealed mineral voxels parked per open
 * face (surfaceDissolutionKinetics3D, dissolutionVOP.hh:379-605), gathered by the open neighbours
 * with the headroom clamp (dissolutionGather3D, :608-742), all applied once
 * (update_abiotic_rxnLattices, complab3d_processors_part1.hh:299-404). */
static void abiotic_block(OrcAde* A) {
    const int nx = A->nx, ny = A->ny, nz = A->nz, S = A->S;
    const size_t N = A->N;
    std::vector<double> dC((size_t)S * N, 0.0);
    if (A->law2 != LAW_NONE)
        abiotic_rate_pass(A, [&](int s2, size_t n) { return dens_post(A, s2, n); }, dC.data());
    if (A->dis_on && A->sM >= 0) {
        const DissolLaw L{A->dis_law, S, A->sM, A->dprm.data()};
        dissolution_park_gather(
            nx, ny, nz, S, A->sM, A->dt, A->dis_surf, A->stamp.data(), L,
            [&](int s2, size_t n) { return dens_post(A, s2, n); },
            [&](size_t n) { return A->react[(uint8_t)A->mat[n]] != 0; }, dC);
    }
    // apply
#pragma omp parallel for schedule(static)
    for (int x = 1; x < nx - 1; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = A->id(x, y, z);
                const bool open = A->react[(uint8_t)A->mat[n]];
                for (int s2 = 0; s2 < S; ++s2) {
                    if (!open && A->mobile[s2]) continue;
                    const double d = dC[(size_t)s2 * N + n];
                    if (!(d > THRD || d < -THRD)) continue;
                    if (A->mobile[s2])
                        for (int i = 0; i < Q7; ++i) A->gp[s2][n * Q7 + i] += d * T7[i];
                    else
                        A->imm[s2][n] += d;
                }
            }
}

static void apply_speciation(OrcAde* A);

static void ade_step(OrcAde* A) {
    const int nx = A->nx, ny = A->ny, nz = A->nz, S = A->S;
    const size_t N = A->N, P = (size_t)ny * nz;
    // ---- 1. collide every mobile species
    for (int s = 0; s < S; ++s) {
        if (!A->mobile[s]) continue;
        std::vector<double>& G = A->g[s];
        std::vector<double>& GP = A->gp[s];
#pragma omp parallel for schedule(static)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    size_t n = A->id(x, y, z);
                    const double* c = &G[n * Q7];
                    double* o = &GP[n * Q7];
                    int d = A->node_dyn(s, x, n);
                    if (d == ADE_NONE) { for (int i = 0; i < Q7; ++i) o[i] = c[i]; continue; }
                    if (d == ADE_BB) { for (int i = 0; i < Q7; ++i) o[i] = c[opp7(i)]; continue; }
                    double w = (d == ADE_BIO) ? A->wbio[s] : A->wpore[s];
                    double gg[7];
                    for (int i = 0; i < Q7; ++i) gg[i] = c[i];
                    if (x == 0 || x == nx - 1) {
                        // AdvectionDiffusionBoundaryDynamics: complete the inward population
                        double rs = (x == 0 ? A->lstore[(size_t)s * P + (size_t)y * nz + z]
                                            : A->rstore[(size_t)s * P + (size_t)y * nz + z]) - 1.0;
                        int miss = (x == 0) ? 4 : 1;
                        double sum = 0;
                        for (int i = 0; i < Q7; ++i) if (i != miss) sum += gg[i];
                        gg[miss] = rs - sum;
                    }
                    double rb = 0;
                    for (int i = 0; i < Q7; ++i) rb += gg[i];
                    double rho = rb + 1.0;
                    double je[3] = {rho * A->u[n], rho * A->u[N + n], rho * A->u[2 * N + n]};
                    for (int i = 0; i < Q7; ++i) {
                        double cj = C7[i][0] * je[0] + C7[i][1] * je[1] + C7[i][2] * je[2];
                        o[i] = gg[i] * (1.0 - w) + w * (T7[i] * (rb + 4.0 * cj));
                    }
                }
    }
    // ---- 2. kinetics on post-collision densities, deposit t_i dC (update_rxnLattices)
    if (A->law != LAW_NONE) {
#pragma omp parallel for schedule(static)
        for (int x = 1; x < nx - 1; ++x) {
            std::vector<double> C(S), R(S), B(A->M + 1), RB(A->M + 1), dC(S), dB(A->M + 1);
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    size_t n = A->id(x, y, z);
                    if (!A->react[(uint8_t)A->mat[n]]) continue;
                    for (int s = 0; s < S; ++s) C[s] = dens_post(A, s, n);
                    for (int m = 0; m < A->M; ++m) B[m] = A->bio[(size_t)m * N + n];
                    biotic_voxel(A, C.data(), B.data(), R.data(), RB.data(), dC.data(), dB.data());
                    for (int s = 0; s < S; ++s) {
                        if (dC[s] == 0.0) continue;
                        if (A->mobile[s]) {
                            for (int i = 0; i < Q7; ++i) A->gp[s][n * Q7 + i] += dC[s] * T7[i];
                        } else {
                            A->imm[s][n] += dC[s];
                        }
                    }
                    for (int m = 0; m < A->M; ++m) A->bio[(size_t)m * N + n] += dB[m];
                }
        }
    }
    if (A->law2 != LAW_NONE || (A->dis_on && A->sM >= 0)) abiotic_block(A);
    // ---- speciation on the post-kinetics populations (complab.cpp:2564-2569)
    if (A->spec) apply_speciation(A);
    // ---- 3. stream, then the Neumann planes take the inner neighbour's density
    for (int s = 0; s < S; ++s) {
        if (!A->mobile[s]) continue;
        std::vector<double>& G = A->g[s];
        std::vector<double>& GP = A->gp[s];
#pragma omp parallel for schedule(static)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    size_t n = A->id(x, y, z);
                    G[n * Q7] = GP[n * Q7];
                    for (int i = 1; i < Q7; ++i) {
                        int sx = x - C7[i][0], sy = y - C7[i][1], sz = z - C7[i][2];
                        if (sx < 0 || sy < 0 || sz < 0 || sx >= nx || sy >= ny || sz >= nz)
                            G[n * Q7 + i] = GP[n * Q7 + opp7(i)];
                        else
                            G[n * Q7 + i] = GP[A->id(sx, sy, sz) * Q7 + i];
                    }
                }
        for (int side = 0; side < 2; ++side) {
            int bt = side == 0 ? A->ltype[s] : A->rtype[s];
            if (bt != BC_NEUMANN) continue;
            int xb = side == 0 ? 0 : nx - 1, xi = side == 0 ? 1 : nx - 2;
            std::vector<double>& st = side == 0 ? A->lstore : A->rstore;
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    size_t nb = A->id(xb, y, z), ni = A->id(xi, y, z);
                    int db = A->node_dyn(s, xb, nb), di = A->node_dyn(s, xi, ni);
                    if (db != ADE_PORE && db != ADE_BIO) continue;
                    if (di != ADE_PORE && di != ADE_BIO) continue;  // keep the previous value
                    double r = 1.0;
                    for (int i = 0; i < Q7; ++i) r += G[ni * Q7 + i];
                    st[(size_t)s * P + (size_t)y * nz + z] = r;
                }
        }
    }
    A->iters += 1;
}

void orc_ade_step(OrcAde* A, int n) {
    for (int k = 0; k < n; ++k) ade_step(A);
}

/* computeDensity of species s at every node: BGK nodes sum + 1; boundary nodes of a
 * Dirichlet / Neumann plane report their stored value; bounce-back nodes report the sum
 * of their populations + 1 (the "held" content the reference's diagnostics track). */
void orc_ade_density(OrcAde* A, int s, double* out) {
    const size_t N = A->N, P = (size_t)A->ny * A->nz;
    if (!A->mobile[s]) {
        for (size_t n = 0; n < N; ++n) out[n] = A->imm[s][n];
        return;
    }
    for (int x = 0; x < A->nx; ++x)
        for (int y = 0; y < A->ny; ++y)
            for (int z = 0; z < A->nz; ++z) {
                size_t n = A->id(x, y, z);
                int d = A->node_dyn(s, x, n);
                bool bgk = (d == ADE_PORE || d == ADE_BIO);
                if (bgk && x == 0) { out[n] = A->lstore[(size_t)s * P + (size_t)y * A->nz + z]; continue; }
                if (bgk && x == A->nx - 1) { out[n] = A->rstore[(size_t)s * P + (size_t)y * A->nz + z]; continue; }
                double r = 1.0;
                for (int i = 0; i < Q7; ++i) r += A->g[s][n * Q7 + i];
                out[n] = r;
            }
}

void orc_ade_populations(OrcAde* A, int s, double* out) {
    for (size_t n = 0; n < A->N; ++n)
        for (int i = 0; i < Q7; ++i) out[(size_t)i * A->N + n] = A->g[s][n * Q7 + i];
}

void orc_ade_biomass(OrcAde* A, double* out) {
    std::copy(A->bio.begin(), A->bio.end(), out);
}

void orc_ade_set_velocity(OrcAde* A, const double* u) { A->u.assign(u, u + 3 * A->N); }

void orc_ade_set_abiotic(OrcAde* A, int law, const double* prm, int nprm, int surface_only) {
    A->law2 = law;
    A->prm2.assign(prm, prm + nprm);
    A->surf = surface_only;
}

void orc_ade_set_precip(OrcAde* A, int mineral, double full, int precip_code, int dissolution, double reopen,
                        int pore_code, int dis_law, const double* dprm, int ndprm, int dis_surface_only) {
    A->pr_on = 1;
    A->sM = mineral;
    A->full = full;
    A->pcode = precip_code;
    A->dis_on = dissolution;
    A->reopen = reopen;
    A->porecode = pore_code;
    A->dis_law = dis_law;
    A->dprm.assign(dprm, dprm + ndprm);
    A->dis_surf = dis_surface_only;
    if (A->stamp.size() != A->N) A->stamp.assign(A->N, 0);
}

/* precipNodeConversion3D over Box3D(1, nx-2, ...) (precipitationVOP.hh:166-227, complab.cpp:3139-3146)
 * then, with dissolution, dissolNodeConversion3D (dissolutionVOP.hh:745-810). A voxel that changes
 * material changes dynamics on every species lattice (updateSoluteSolidDynamics3D) and keeps its
 * populations. Returns the number of voxels sealed and reopened. */
void orc_ade_geometry_update(OrcAde* A, int* sealed, int* reopened) {
    int ns = 0, nr = 0;
    const int nx = A->nx, ny = A->ny, nz = A->nz;
    for (int x = 1; x < nx - 1; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = A->id(x, y, z);
                if (!A->react[(uint8_t)A->mat[n]]) continue;
                if (A->imm[A->sM][n] >= A->full) {
                    A->mat[n] = (int8_t)A->pcode;
                    if (!A->dmat.empty()) A->dmat[n] = (int8_t)A->pcode;
                    A->stamp[n] = 1;
                    ++ns;
                }
            }
    if (A->dis_on)
        for (int x = 1; x < nx - 1; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    size_t n = A->id(x, y, z);
                    if (!A->stamp[n]) continue;
                    if (A->imm[A->sM][n] < A->reopen * A->full) {
                        A->mat[n] = (int8_t)A->porecode;
                        if (!A->dmat.empty()) A->dmat[n] = (int8_t)A->porecode;
                        A->stamp[n] = 0;
                        ++nr;
                    }
                }
    *sealed = ns;
    *reopened = nr;
}

/* One kinetics pass on given fields, without applying it (the increments run_kinetics and
 * run_abiotic_kinetics / surfaceAbioticKinetics3D leave in their dC / dB lattices, with the clamp):
 * C is [S][N] (post-collision densities), B is [M][N]; dC, dB receive [S][N], [M][N]. */
void orc_biotic_increments(OrcAde* A, const double* Cin, const double* Bin, double* dCout, double* dBout) {
    const int S = A->S, M = A->M;
    const size_t N = A->N;
    std::fill(dCout, dCout + (size_t)S * N, 0.0);
    std::fill(dBout, dBout + (size_t)M * N, 0.0);
    std::vector<double> C(S), R(S), B(M + 1), RB(M + 1), dC(S), dB(M + 1);
    for (int x = 1; x < A->nx - 1; ++x)
        for (int y = 0; y < A->ny; ++y)
            for (int z = 0; z < A->nz; ++z) {
                size_t n = A->id(x, y, z);
                if (!A->react[(uint8_t)A->mat[n]]) continue;
                for (int s = 0; s < S; ++s) C[s] = Cin[(size_t)s * N + n];
                for (int m = 0; m < M; ++m) B[m] = Bin[(size_t)m * N + n];
                biotic_voxel(A, C.data(), B.data(), R.data(), RB.data(), dC.data(), dB.data());
                for (int s = 0; s < S; ++s) dCout[(size_t)s * N + n] = dC[s];
                for (int m = 0; m < M; ++m) dBout[(size_t)m * N + n] = dB[m];
            }
}

void orc_abiotic_increments(OrcAde* A, const double* Cin, double* dCout) {
    const size_t N = A->N;
    std::fill(dCout, dCout + (size_t)A->S * N, 0.0);
    abiotic_rate_pass(A, [&](int s, size_t n) { return Cin[(size_t)s * N + n]; }, dCout);
}

// an immobile species' field and the precipitate stamps, as the conversions read them
void orc_ade_set_immobile(OrcAde* A, int s, const double* c) { A->imm[s].assign(c, c + A->N); }
void orc_ade_set_stamp(OrcAde* A, const uint8_t* st) { A->stamp.assign(st, st + A->N); }
void orc_ade_stamp(OrcAde* A, uint8_t* out) { std::copy(A->stamp.begin(), A->stamp.end(), out); }

void orc_ade_material(OrcAde* A, int8_t* out) { std::copy(A->mat.begin(), A->mat.end(), out); }

// ---------------------------------------------------------------- biofilm cellular automaton
/* The reference draws its random neighbour order from std::random_shuffle / std::rand, seeded by
 * the clock, so no two runs agree. The oracle (and the product) replace it with a counter-based
 * stream: voxel n in push sweep w draws from splitmix64 steps started at
 * seed ^ (w * 0x9E3779B97F4A7C15) ^ (n * 0xD1B54A32D192ED03); a shuffle of L entries is
 * Fisher-Yates from the top (j = draw % (i + 1)), a single pick is draw % L. */
static inline uint64_t sm64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static inline bool ca_open(const OrcAde* A, int m) { return m != A->bbc && m != A->solc; }
static inline bool ca_pore(const OrcAde* A, int m) {
    for (int c : A->pore_codes)
        if (m == c) return true;
    return false;
}

void orc_ca_setup(OrcAde* A, double Bmax, double frac, uint64_t seed, int n_pore, const int32_t* pore,
                  int bb, int solid, const int32_t* bio_codes) {
    const int nx = A->nx, ny = A->ny, nz = A->nz;
    const size_t N = A->N;
    A->ca_on = 1;
    A->half = 0;
    A->Bmax = Bmax;
    A->bfrac = frac;
    A->seed = seed;
    A->sweeps = 0;
    A->pore_codes.assign(pore, pore + n_pore);
    A->bio_code.assign(bio_codes, bio_codes + A->M);
    A->bbc = bb;
    A->solc = solid;
    if (A->dmat.empty()) A->dmat = A->mat;
    // initTotalbFilmLatticeDensity: the sum of the microbes' biomass
    A->total.assign(N, 0.0);
    for (size_t n = 0; n < N; ++n) {
        double t = 0;
        for (int m = 0; m < A->M; ++m) t += A->bio[(size_t)m * N + n];
        A->total[n] = t;
    }
    // createAgeDomain3D: solid / wall -1, pore 0, anything else (biofilm) 1
    A->age.assign(N, 0);
    A->distp.assign(N, 0);
    long long msum = 0;
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = A->id(x, y, z);
                const int m = A->mat[n];
                msum += m;
                A->age[n] = !ca_open(A, m) ? -1 : (ca_pore(A, m) ? 0 : 1);
                // calculateDistanceFromSolid (complab_functions.hh:220-291): positive exactly for
                // the voxels that are neither solid nor wall, off the last x, y and z planes
                A->distp[n] = (ca_open(A, m) && x < nx - 1 && y < ny - 1 && z < nz - 1) ? 1 : 0;
            }
    A->old_mask_sum = msum;
}

// updateLocalMaskNtotalLattices3D with a single pore code list (in place, lexicographic)
static void ca_mask_total(OrcAde* A) {
    const int nx = A->nx, ny = A->ny, nz = A->nz;
    const size_t N = A->N;
    const double thr = A->bfrac * A->Bmax;
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = A->id(x, y, z);
                const int m = A->mat[n];
                if (!ca_open(A, m)) continue;
                double bmass = 0;
                int newmask = 0;
                for (int mi = 0; mi < A->M; ++mi) {
                    const double bm = A->bio[(size_t)mi * N + n];
                    if (bm > 1e-14) {
                        bmass += bm;
                        newmask += A->bio_code[mi];
                    }
                }
                if (std::fabs(bmass - A->total[n]) > 1e-14) A->total[n] = bmass;
                const bool poreflag = ca_pore(A, m);
                if (!poreflag && bmass < thr) {
                    newmask = A->pore_codes[0];
                    if (A->pore_codes.size() > 1) {
                        const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
                        for (int d = 0; d < 6; ++d) {
                            int X = x + d6[d][0], Y = y + d6[d][1], Z = z + d6[d][2];
                            if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                            const int nm = A->mat[A->id(X, Y, Z)];
                            if (ca_open(A, nm) && ca_pore(A, nm)) { newmask = nm; break; }
                        }
                    }
                    A->mat[n] = (int8_t)newmask;
                } else if (poreflag && bmass >= thr) {
                    if (newmask > 0) A->mat[n] = (int8_t)newmask;
                }
            }
}

// pushExcessBiomass3D ('fraction', complab3d_processors_part1.hh:499-732) or
// halfPushExcessBiomass3D ('half', :735-970) of a single-block run, where every push lands inside
// the block. 'half' differs in four places: only biofilm voxels push (not pore), the excess is half
// the voxel's total (no threshold on it), the fallback target is a neighbour whose age is not above
// the voxel's (>= instead of >), and the fallback push always runs -- into the voxel itself
// (subtracted, then added back) when the first pass placed everything or no neighbour is open.
static void ca_push(OrcAde* A) {
    const int nx = A->nx, ny = A->ny, nz = A->nz;
    const size_t N = A->N;
    const double Bmax = A->Bmax;
    const uint64_t w = A->sweeps++;
    for (int x = 1; x <= nx - 2; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const size_t n = A->id(x, y, z);
                if (!ca_open(A, A->mat[n])) continue;
                if (A->half && ca_pore(A, A->mat[n])) continue;
                double bMt = A->total[n];
                if (!(bMt > Bmax)) continue;
                double bMd = A->half ? bMt * 0.5 : bMt - Bmax;
                if (!A->half && !(bMd > THRD)) continue;
                // neighbours in the reference's order, x limited to 1..nx-2
                size_t nb[6];
                int L = 0;
                const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
                for (int d = 0; d < 6; ++d) {
                    int X = x + d6[d][0], Y = y + d6[d][1], Z = z + d6[d][2];
                    if (X < 1 || X > nx - 2 || Y < 0 || Y >= ny || Z < 0 || Z >= nz) continue;
                    const size_t m = A->id(X, Y, Z);
                    if (!ca_open(A, A->mat[m])) continue;
                    nb[L++] = m;
                }
                uint64_t st = A->seed ^ (w * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)n * 0xD1B54A32D192ED03ULL);
                int perm[6] = {0, 1, 2, 3, 4, 5};
                if (L > 1)
                    for (int i = L - 1; i >= 1; --i) {
                        const int j = (int)(sm64(st) % (uint64_t)(i + 1));
                        std::swap(perm[i], perm[j]);
                    }
                bool chk = false;
                for (int t = 0; t < L; ++t) {
                    const size_t m = nb[L > 1 ? perm[t] : 0];
                    const double nbrbMt = ca_pore(A, A->mat[m]) ? 0.0 : A->total[m];
                    if (nbrbMt < Bmax) {
                        const double hold = Bmax - nbrbMt;
                        double partial = bMd;
                        if (bMd > hold) { partial = hold; bMd -= hold; }
                        else { bMd = 0; chk = true; }
                        for (int mi = 0; mi < A->M; ++mi) {
                            const double shove = A->bio[(size_t)mi * N + n] / bMt * partial;
                            if (shove > THRD) {
                                A->bio[(size_t)mi * N + n] -= shove;
                                A->bio[(size_t)mi * N + m] += shove;
                            }
                        }
                        bMt -= partial;
                    }
                    if (chk) break;
                }
                size_t m = n;  // 'half': with no fallback neighbour the push goes back into the voxel
                if (!chk && L > 0) {
                    const int id0 = A->age[n];
                    size_t cand[6];
                    int c = 0;
                    for (int t = 0; t < L; ++t)
                        if (A->half ? id0 >= A->age[nb[t]] : id0 > A->age[nb[t]]) cand[c++] = nb[t];
                    if (c > 1) m = cand[sm64(st) % (uint64_t)c];
                    else if (c == 1) m = cand[0];
                    else m = nb[L > 1 ? (int)(sm64(st) % (uint64_t)L) : 0];
                }
                if (A->half || (!chk && L > 0)) {
                    for (int mi = 0; mi < A->M; ++mi) {
                        const double shove = A->bio[(size_t)mi * N + n] / bMt * bMd;
                        A->bio[(size_t)mi * N + n] -= shove;
                        A->bio[(size_t)mi * N + m] += shove;
                    }
                }
            }
}

// updateAgeDistance3D: one in-place lexicographic sweep; returns the number of ages changed
static long ca_age_sweep(OrcAde* A) {
    const int nx = A->nx, ny = A->ny, nz = A->nz;
    const double Bmax = A->Bmax;
    long changed = 0;
    const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const size_t n = A->id(x, y, z);
                const double B = A->total[n];
                if (!(B > 1e-14)) continue;
                size_t D[6];
                int nd = 0;
                for (int d = 0; d < 6; ++d) {
                    int X = x + d6[d][0], Y = y + d6[d][1], Z = z + d6[d][2];
                    if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                    const size_t m = A->id(X, Y, Z);
                    if (A->distp[m]) D[nd++] = m;
                }
                const int a = A->age[n];
                int na = a;
                if (a == 0) na = 1;
                else if (a == 1 && (B - Bmax) > -1e-14) {
                    bool ok = true;
                    for (int t = 0; t < nd; ++t)
                        if (A->age[D[t]] == 0) { ok = false; break; }
                    if (ok) na = 2;
                } else {
                    int cnt = 0;
                    for (int t = 0; t < nd; ++t)
                        if (A->age[D[t]] >= a && (A->total[D[t]] - Bmax) > -1e-14) ++cnt;
                    if (cnt == nd) na = a + 1;
                }
                if (na != a) { A->age[n] = na; ++changed; }
            }
    return changed;
}

/* The CA block of one iteration (complab.cpp:2792-3055) followed by the age sweep the main loop
 * runs when the mask changed (:3074-3079). Returns 0, or -1 when the push stalls for 100 sweeps,
 * -2 when it does not settle in 1000 sweeps, -3 when the age relaxation does not settle in 1000. */
int orc_ca_step(OrcAde* A, int* sweeps_out, int* mask_changed) {
    const size_t N = A->N;
    ca_mask_total(A);
    auto gmax = [&]() { double g = -1e300; for (size_t n = 0; n < N; ++n) g = std::max(g, A->total[n]); return g; };
    double globalBmax = gmax();
    int whilecount = 0, rc = 0;
    if (globalBmax - A->Bmax > THRD) {
        double prev = globalBmax;
        int stall = 0;
        while (globalBmax - A->Bmax > THRD) {
            ca_push(A);
            ca_mask_total(A);
            globalBmax = gmax();
            if (globalBmax > prev - THRD) {
                if (++stall >= 100) { rc = -1; break; }
            } else {
                stall = 0;
            }
            prev = globalBmax;
            if (whilecount % 50 == 0) {
                int sub = 0;
                while (ca_age_sweep(A) != 0)
                    if (++sub > 1000) { rc = -3; break; }
                if (rc) break;
            }
            if (whilecount > 1000) { rc = -2; break; }
            ++whilecount;
        }
    }
    long long msum = 0;
    for (size_t n = 0; n < N; ++n) msum += A->mat[n];
    *mask_changed = msum != A->old_mask_sum;
    if (*mask_changed) {
        A->old_mask_sum = msum;
        ca_age_sweep(A);
    }
    *sweeps_out = whilecount;
    return rc;
}

/* updateSoluteDynamics3D (complab3d_processors_part2.hh:485-553): every open voxel's species
 * dynamics follow the mask, pore codes with the pore omega, any other open code with the
 * biofilm omega (the first microbe's code stands for it). */
void orc_ade_refresh_dynamics(OrcAde* A) {
    if (A->dmat.empty()) A->dmat = A->mat;
    const int bio0 = A->bio_code.empty() ? -1 : A->bio_code[0];
    for (size_t n = 0; n < A->N; ++n) {
        const int m = A->mat[n];
        if (!ca_open(A, m)) continue;
        A->dmat[n] = ca_pore(A, m) ? (int8_t)m : (int8_t)(bio0 >= 0 ? bio0 : m);
    }
}

void orc_ca_fields(OrcAde* A, double* total, int32_t* age) {
    std::copy(A->total.begin(), A->total.end(), total);
    std::copy(A->age.begin(), A->age.end(), age);
}

// single passes of the automaton on the current state (pinned to the reference's processors):
// the mask and total update once; the age relaxation until no age changes (at most max_sweeps),
// returning the number of sweeps that changed something
void orc_ca_mask_total_once(OrcAde* A) { ca_mask_total(A); }
void orc_ca_set_half(OrcAde* A, int half) { A->half = half ? 1 : 0; }
int orc_ca_age_relax(OrcAde* A, int max_sweeps) {
    int k = 0;
    while (k < max_sweeps && ca_age_sweep(A) != 0) ++k;
    return k;
}
// the age field and its open-region flags (age > -1 region of calculateDistanceFromSolid)
void orc_ca_age_flags(OrcAde* A, int32_t* distp) { std::copy(A->distp.begin(), A->distp.end(), distp); }

}  // extern "C"

// =====================================================================================
//                     EQUILIBRIUM SPECIATION (Newton-Raphson in log10)
// =====================================================================================
// Restates the reference's Newton-Raphson reserve solver
// (complab3d_processors_part4_eqsolver_NR_reserve.hh: calc_residual :309-328, calc_jacobian
// :356-375, partial-pivot Gaussian elimination :377-440 with singular threshold 1e-30,
// solve_equilibrium_NR :512-640 with Armijo backtracking of at most 40 halvings) on the species
// model of the active solver (complab3d_processors_part4_eqsolver.hh: calc_species :450-505 with
// log10 c clamped to [-30, 1] and c to [1e-30, 10], calc_component_totals :520-535,
// isEquilibriumSpecies :386-395), and the speciation step run_equilibrium_biotic (:1393-1545):
// x = 1..nx-2, mask neither solid nor wall, dC capped at max(1e-9, 0.1 |C|), the new
// concentration floored at 1e-20, deposited as t_i dC when |dC| > 1e-12.
namespace {
const double EQ_MIN_C = 1e-30, EQ_MAX_C = 10.0, EQ_MIN_LOG = -30.0, EQ_MAX_LOG = 1.0;
// Two departures from the reserve solver, both for robustness from a far initial guess: inside
// the Newton loop the species are taken without the [1e-30, 10] clamps (a species saturated at the
// clamp has a zero derivative the Jacobian does not see, and the iteration stalls); the clamps
// apply to the answer only. And no log10 component concentration moves by more than EQ_MAX_STEP
// in one step.
const double EQ_MAX_STEP = 2.0;

struct EqTableau {
    int ns = 0, nc = 0;
    std::vector<double> S, logK;  // S[i*nc + j]
    std::vector<int> comp;        // species index of component j or -1
    double tol = 1e-10;
    int max_it = 200;
    bool eq_species(int i) const {
        for (int j = 0; j < nc; ++j) if (std::fabs(S[i * nc + j]) > 1e-10) return true;
        return false;
    }
};

void eq_species_conc(const EqTableau& t, const double* x, const double* init, double* c) {
    for (int i = 0; i < t.ns; ++i) {
        if (!t.eq_species(i)) {
            c[i] = init[i] > EQ_MIN_C ? std::min(init[i], EQ_MAX_C) : EQ_MIN_C;
            continue;
        }
        double lc = t.logK[i];
        for (int j = 0; j < t.nc; ++j) lc += t.S[i * t.nc + j] * x[j];
        lc = std::max(std::min(lc, EQ_MAX_LOG), EQ_MIN_LOG);
        double v = std::pow(10.0, lc);
        if (std::isnan(v) || std::isinf(v)) v = init[i] > EQ_MIN_C ? init[i] : EQ_MIN_C;
        c[i] = std::max(std::min(v, EQ_MAX_C), EQ_MIN_C);
    }
}

// species inside the Newton loop: mass action without the concentration clamps
void eq_species_free(const EqTableau& t, const double* x, const double* init, double* c) {
    for (int i = 0; i < t.ns; ++i) {
        if (!t.eq_species(i)) {
            c[i] = init[i] > EQ_MIN_C ? std::min(init[i], EQ_MAX_C) : EQ_MIN_C;
            continue;
        }
        double lc = t.logK[i];
        for (int j = 0; j < t.nc; ++j) lc += t.S[i * t.nc + j] * x[j];
        c[i] = std::pow(10.0, std::max(std::min(lc, 300.0), -300.0));
    }
}

double eq_residual(const EqTableau& t, const double* x, const double* Ttot, const double* init, double* F) {
    double c[64];
    eq_species_free(t, x, init, c);
    double s = 0;
    for (int j = 0; j < t.nc; ++j) {
        double v = -Ttot[j];
        for (int i = 0; i < t.ns; ++i)
            if (t.eq_species(i)) v += t.S[i * t.nc + j] * c[i];
        F[j] = v;
        s += v * v;
    }
    return std::sqrt(s);
}

// returns iterations; *conv set
int eq_solve_nr(const EqTableau& t, const double* init, double* out, int* conv) {
    const int nc = t.nc, ns = t.ns;
    double Ttot[16], x[16], F[16], Fn[16], xn[16], d[16], A[16][17];
    *conv = 0;
    for (int j = 0; j < nc; ++j) {
        double v = 0;
        for (int i = 0; i < ns; ++i)
            if (t.eq_species(i)) v += t.S[i * nc + j] * std::max(std::min(init[i], EQ_MAX_C), EQ_MIN_C);
        Ttot[j] = std::max(v, EQ_MIN_C);
        double cc = t.comp[j] >= 0 ? init[t.comp[j]] : 1e-7;
        x[j] = std::log10(std::max(std::min(cc, EQ_MAX_C), EQ_MIN_C));
    }
    int it = 0;
    for (; it < t.max_it; ++it) {
        double fn = eq_residual(t, x, Ttot, init, F);
        if (fn < t.tol) { *conv = 1; ++it; break; }
        double c[64];
        eq_species_free(t, x, init, c);
        const double ln10 = std::log(10.0);
        for (int j = 0; j < nc; ++j) {
            for (int k = 0; k < nc; ++k) {
                double v = 0;
                for (int i = 0; i < ns; ++i)
                    if (t.eq_species(i)) v += ln10 * t.S[i * nc + j] * t.S[i * nc + k] * c[i];
                A[j][k] = v;
            }
            A[j][nc] = -F[j];
        }
        bool ok = true;
        for (int p = 0; p < nc && ok; ++p) {
            int r = p;
            double mv = std::fabs(A[p][p]);
            for (int q = p + 1; q < nc; ++q) if (std::fabs(A[q][p]) > mv) { mv = std::fabs(A[q][p]); r = q; }
            if (mv < 1e-30) { ok = false; break; }
            if (r != p) for (int q = 0; q <= nc; ++q) std::swap(A[p][q], A[r][q]);
            for (int q = p + 1; q < nc; ++q) {
                double fct = A[q][p] / A[p][p];
                for (int m = p; m <= nc; ++m) A[q][m] -= fct * A[p][m];
            }
        }
        if (!ok) { ++it; break; }
        for (int p = nc - 1; p >= 0; --p) {
            double v = A[p][nc];
            for (int q = p + 1; q < nc; ++q) v -= A[p][q] * d[q];
            d[p] = v / A[p][p];
        }
        // step limit: no log10 concentration moves by more than EQ_MAX_STEP in one iteration
        double dmax = 0;
        for (int j = 0; j < nc; ++j) dmax = std::max(dmax, std::fabs(d[j]));
        if (dmax > EQ_MAX_STEP)
            for (int j = 0; j < nc; ++j) d[j] *= EQ_MAX_STEP / dmax;
        double alpha = 1.0, fnew = 0;
        for (int ls = 0; ls < 40; ++ls) {
            for (int j = 0; j < nc; ++j) xn[j] = std::max(std::min(x[j] + alpha * d[j], EQ_MAX_LOG), EQ_MIN_LOG);
            fnew = eq_residual(t, xn, Ttot, init, Fn);
            if (fnew < fn * (1.0 - 0.0001 * alpha) || alpha < 1e-15) break;
            alpha *= 0.5;
        }
        for (int j = 0; j < nc; ++j) x[j] = xn[j];
        double dn = 0;
        for (int j = 0; j < nc; ++j) dn += d[j] * d[j];
        if (alpha * std::sqrt(dn) < t.tol * 1e-3 && fnew < t.tol * 100) { *conv = 1; ++it; break; }
    }
    eq_species_conc(t, x, init, out);
    for (int i = 0; i < ns; ++i) {
        if (std::isnan(out[i]) || std::isinf(out[i])) out[i] = init[i] > EQ_MIN_C ? std::min(init[i], EQ_MAX_C) : EQ_MIN_C;
        out[i] = std::max(std::min(out[i], EQ_MAX_C), EQ_MIN_C);
    }
    return it;
}
}  // namespace

extern "C" int orc_eq_nr(int ns, int nc, const double* stoich, const double* logK, const int* comp, double tol,
                         int max_it, const double* cin, double* cout, int* conv) {
    EqTableau t;
    t.ns = ns; t.nc = nc;
    t.S.assign(stoich, stoich + ns * nc);
    t.logK.assign(logK, logK + ns);
    t.comp.assign(comp, comp + nc);
    t.tol = tol;
    t.max_it = max_it;
    return eq_solve_nr(t, cin, cout, conv);
}

static void apply_speciation(OrcAde* A) {
    const EqTableau& t = *static_cast<const EqTableau*>(A->spec);
    const int nx = A->nx, ny = A->ny, nz = A->nz, ns = t.ns;
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 1; x < nx - 1; ++x) {
        double c[64], e[64];
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                size_t n = A->id(x, y, z);
                if (!A->react[(uint8_t)A->mat[n]]) continue;
                for (int s = 0; s < ns; ++s) {
                    double v;
                    if (A->mobile[s]) {
                        v = 1.0;
                        for (int i = 0; i < Q7; ++i) v += A->gp[s][n * Q7 + i];
                    } else {
                        v = A->imm[s][n];
                    }
                    c[s] = std::max(v, EQ_MIN_C);
                }
                int conv;
                eq_solve_nr(t, c, e, &conv);
                for (int s = 0; s < ns; ++s) {
                    double dC = e[s] - c[s];
                    const double cap = std::max(1e-9, 0.1 * std::fabs(c[s]));
                    if (std::fabs(dC) > cap) dC = dC > 0 ? cap : -cap;
                    if (c[s] + dC < 1e-20) dC = 1e-20 - c[s];
                    if (!(std::fabs(dC) > THRD)) continue;
                    if (A->mobile[s]) {
                        for (int i = 0; i < Q7; ++i) A->gp[s][n * Q7 + i] += dC * T7[i];
                    } else {
                        A->imm[s][n] += dC;
                    }
                }
            }
    }
}

extern "C" void orc_ade_set_speciation(OrcAde* A, int ns, int nc, const double* stoich, const double* logK,
                                       const int* comp, double tol, int max_it) {
    if (A->spec) delete static_cast<EqTableau*>(A->spec);
    EqTableau* t = new EqTableau();
    t->ns = ns; t->nc = nc;
    t->S.assign(stoich, stoich + ns * nc);
    t->logK.assign(logK, logK + ns);
    t->comp.assign(comp, comp + nc);
    t->tol = tol;
    t->max_it = max_it;
    A->spec = t;
}

/* The dissolution increments of one step for given fields, outside any lattice: densities C[s][N]
 * as the processors see them, material map, stamp (precipitated mineral voxels), the mineral
 * species sM and the dissolution law; dC[s][N] holds the increments already pending (abiotic
 * law) and receives the parked and gathered ones. Used to pin the restatement against the
 * reference's own surfaceDissolutionKinetics3D / dissolutionGather3D. */
extern "C" void orc_dissolution_increments(int nx, int ny, int nz, int S, int sM, double dt, int law,
                                           const double* prm, int surface_only, const int8_t* mat, int solid,
                                           int bb, const uint8_t* stamp, const double* C, double* dC) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<double> d(dC, dC + (size_t)S * N);
    const DissolLaw L{law, S, sM, prm};
    dissolution_park_gather(
        nx, ny, nz, S, sM, dt, surface_only, stamp, L, [&](int s, size_t n) { return C[(size_t)s * N + n]; },
        [&](size_t n) { return mat[n] != solid && mat[n] != bb; }, d);
    std::copy(d.begin(), d.end(), dC);
}

// =====================================================================================
//                 POROSITY-TARGETED SPHERE PACK (input maps of the CPU baseline)
// =====================================================================================
// The library's clb_geom_sphere_pack restated so the CPU baseline builds its input without the
// product library: walls on the listed axes, then spheres of radius U[rmin, rmax] at centres drawn
// from the reference's xorshift64* stream (complab3d_geometry.hh:77-83) carved as `grain` until
// the open fraction reaches `porosity`. Same voxels for the same arguments (tests/test_geometry.py).
namespace {
struct OrcXorShift {
    uint64_t s;
    explicit OrcXorShift(uint64_t seed) : s(seed ? seed : 1) {}
    uint64_t next() {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return s * 2685821657736338717ULL;
    }
    double uniform() { return (double)(next() >> 11) / 9007199254740992.0; }
    int below(int n) { return n > 0 ? (int)(uniform() * (double)n) : 0; }
};
}  // namespace

extern "C" int orc_sphere_pack(int nx, int ny, int nz, double porosity, double rmin, double rmax, uint64_t seed,
                               const char* walls, int grain, int wall, int pore, int8_t* out) {
    if (!out || nx < 1 || ny < 1 || nz < 1 || !(porosity > 0 && porosity < 1) || !(rmin > 0) || rmax < rmin) return 1;
    const size_t N = (size_t)nx * ny * nz;
    std::vector<int8_t> m(N, (int8_t)pore);
    const std::string w = walls ? walls : "";
    const bool all = w == "all";
    const bool wx = all || w.find('x') != std::string::npos, wy = all || w.find('y') != std::string::npos,
               wz = all || w.find('z') != std::string::npos;
    size_t open = N;
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const bool on = (wx && (x == 0 || x == nx - 1)) || (wy && (y == 0 || y == ny - 1)) ||
                                (wz && (z == 0 || z == nz - 1));
                if (on) { m[((size_t)x * ny + y) * nz + z] = (int8_t)wall; --open; }
            }
    OrcXorShift rng(seed);
    const size_t target = (size_t)(porosity * (double)N);
    for (int guard = 0; open > target && guard < 10000000; ++guard) {
        const int cx = rng.below(nx), cy = rng.below(ny), cz = rng.below(nz);
        const double r = rmin + (rmax - rmin) * rng.uniform();
        const int ri = (int)std::ceil(r);
        for (int x = std::max(0, cx - ri); x <= std::min(nx - 1, cx + ri); ++x)
            for (int y = std::max(0, cy - ri); y <= std::min(ny - 1, cy + ri); ++y)
                for (int z = std::max(0, cz - ri); z <= std::min(nz - 1, cz + ri); ++z) {
                    const double dx = x - cx, dy = y - cy, dz = z - cz;
                    if (dx * dx + dy * dy + dz * dz > r * r) continue;
                    int8_t& v = m[((size_t)x * ny + y) * nz + z];
                    if (v == (int8_t)pore) { v = (int8_t)grain; --open; }
                }
    }
    std::copy(m.begin(), m.end(), out);
    return 0;
}

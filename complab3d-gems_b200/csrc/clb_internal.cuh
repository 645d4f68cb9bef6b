// clb_internal.cuh -- shared declarations of the library's translation units.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/clb.h"
#include "symbolic.cuh"
#include "graphnet.cuh"
#include "srgnet.cuh"

namespace clb {

// ------------------------------------------------------------------ lattice constants
// D3Q19 in Palabos' order: 0 rest, 1..9 the "negative" half, i+9 the opposite of i.
__host__ __device__ constexpr int q19cx(int i) {
    return (i == 1 || i == 4 || i == 5 || i == 6 || i == 7) ? -1
         : (i == 10 || i == 13 || i == 14 || i == 15 || i == 16) ? 1 : 0;
}
__host__ __device__ constexpr int q19cy(int i) {
    return (i == 2 || i == 4 || i == 8 || i == 9 || i == 14) ? -1
         : (i == 5 || i == 11 || i == 13 || i == 17 || i == 18) ? 1 : 0;
}
__host__ __device__ constexpr int q19cz(int i) {
    return (i == 3 || i == 6 || i == 8 || i == 16 || i == 18) ? -1
         : (i == 7 || i == 9 || i == 12 || i == 15 || i == 17) ? 1 : 0;
}
__host__ __device__ constexpr double q19w(int i) {
    return i == 0 ? 1.0 / 3.0 : ((i == 1 || i == 2 || i == 3 || i == 10 || i == 11 || i == 12) ? 1.0 / 18.0 : 1.0 / 36.0);
}
__host__ __device__ constexpr int q19opp(int i) { return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9); }

// D3Q7 in Palabos' order: 0 rest, 1..3 = -x,-y,-z, 4..6 = +x,+y,+z.
__host__ __device__ constexpr int q7cx(int i) { return i == 1 ? -1 : (i == 4 ? 1 : 0); }
__host__ __device__ constexpr int q7cy(int i) { return i == 2 ? -1 : (i == 5 ? 1 : 0); }
__host__ __device__ constexpr int q7cz(int i) { return i == 3 ? -1 : (i == 6 ? 1 : 0); }
__host__ __device__ constexpr double q7w(int i) { return i == 0 ? 0.25 : 0.125; }
__host__ __device__ constexpr int q7opp(int i) { return i == 0 ? 0 : (i <= 3 ? i + 3 : i - 3); }

// Dynamics classes per material code.
enum : int8_t { DYN_BB = 0, DYN_NONE = 1, DYN_BGK = 2 };
enum : int8_t { ADE_BB = 0, ADE_NONE = 1, ADE_PORE = 2, ADE_BIO = 3 };

constexpr int MAX_CODES = 128;  // material codes 0..127 (int8, non-negative)
constexpr double THRD = 1e-12;  // complab3d_processors.hh:60

// ------------------------------------------------------------------ storage conversion
// FP16 storage holds the shifted populations f - t_i times 2^10: the small deviations of a flow
// lattice (1e-6 .. 1e-4) stay in half's normal range (subnormal below 6.1e-5 unscaled, below
// 6.0e-8 scaled), which keeps their 11 significant bits; the scaled range ends at |f - t_i| = 64.
// Scaling by a power of two is exact both ways, so only the rounding to 11 bits remains.
constexpr float HALF_SCALE = 1024.0f, HALF_INV = 1.0f / 1024.0f;
template <typename TS, typename TC>
__device__ __forceinline__ TC ld(const TS* p) { return (TC)(*p); }
template <>
__device__ __forceinline__ float ld<__half, float>(const __half* p) { return __half2float(*p) * HALF_INV; }
template <>
__device__ __forceinline__ double ld<__half, double>(const __half* p) { return (double)(__half2float(*p) * HALF_INV); }
template <typename TS>
__device__ __forceinline__ double ldd(const TS* p) { return (double)(*p); }
template <>
__device__ __forceinline__ double ldd<__half>(const __half* p) { return (double)(__half2float(*p) * HALF_INV); }
template <typename TS, typename TC>
__device__ __forceinline__ void st(TS* p, TC v) { *p = (TS)v; }
template <>
__device__ __forceinline__ void st<__half, float>(__half* p, float v) { *p = __float2half_rn(v * HALF_SCALE); }
// a double into FP16 storage (set-up and host writes)
__device__ __forceinline__ __half to_half(double v) { return __double2half(v * (double)HALF_SCALE); }

// Transport populations are stored as g_i - sigma t_i. Lattices computed in FP64 keep the
// reference's shifted form (sigma = 1: Palabos stores f_i - t_i and a density is 1 + the sum), so
// FP64 runs repeat the reference's rounding; lattices computed in FP32 (FP32 and FP16 storage) keep
// g_i itself (sigma = 0), so a concentration far below 1 keeps its relative precision instead of
// being the small difference of two numbers near t_i. The collision has the same form in both:
// with rb = the sum of the stored values, C = rb + sigma and g^eq_i - sigma t_i = t_i (rb + 4 c_i.j).
// The populations the C ABI exchanges are always the shifted ones, g_i - t_i.
template <typename T>
__host__ __device__ constexpr double ade_sigma() { return sizeof(T) == 8 ? 1.0 : 0.0; }

// ------------------------------------------------------------------ geometry of a domain
struct Geom {
    int nx, ny, nz;
    int64_t N;    // nx*ny*nz
    int plane;    // ny*nz
};

__device__ __forceinline__ void decode(const Geom& g, int64_t n, int& x, int& y, int& z) {
    x = (int)(n / g.plane);
    int r = (int)(n - (int64_t)x * g.plane);
    y = r / g.nz;
    z = r - y * g.nz;
}

// ------------------------------------------------------------------ convergence tracer
// util::ValueTracer<T>(1, 1000, eps) held on the device so a captured sequence of steps can
// stop itself: the last block of every step pushes the stored average energy and evaluates
// the criterion; later steps of the same batch see `converged` and do nothing.
constexpr int TRACER_WINDOW = 500;
struct Tracer {
    double ring[TRACER_WINDOW];
    double eps;
    double energy;          // last stored average energy
    int64_t iterations;     // collide-and-stream calls made
    int32_t count;          // values in the window
    int32_t head;           // next slot
    int32_t enabled;        // 1 while a solve runs
    int32_t converged;      // set once the criterion holds
    uint32_t done_blocks;   // completion counter of the running step
    int32_t pad;
};

// ------------------------------------------------------------------ flow parameters
struct FlowParams {
    Geom g;
    double omega[MAX_CODES];
    int8_t dyn[MAX_CODES];
    double rho_w, rho_e;    // pressure planes
    int64_t n_bgk;          // nodes that take statistics
};

// ------------------------------------------------------------------ ADE parameters
struct AdeParams {
    Geom g;
    int S;                  // species
    int M;                  // microbes with biomass fields
    int law;
    double dt;
    double prm[4 * CLB_MAX_SPECIES];
    int8_t dyn[MAX_CODES];
    int8_t react[MAX_CODES];
    int mobile[CLB_MAX_SPECIES];
    int slot[CLB_MAX_SPECIES];    // index of a mobile species among the mobile ones, -1 immobile
    int ltype[CLB_MAX_SPECIES], rtype[CLB_MAX_SPECIES];
    double lbc[CLB_MAX_SPECIES], rbc[CLB_MAX_SPECIES];
    double wpore[CLB_MAX_SPECIES], wbio[CLB_MAX_SPECIES];
    double c0[CLB_MAX_SPECIES];
    int donor;                          // internal index of the dual-Monod donor
    int acceptor[CLB_MAX_MICROBES];     // internal index of each microbe's acceptor, -1 none
    // abiotic law (internal species indices)
    int law2;                           // CLB_LAW_NONE, CLB_LAW_PRECIP, CLB_LAW_MINERAL
    int surf;                           // surface-only gate of the abiotic law
    double prm2[3 + CLB_MAX_SPECIES];
    // dissolution of sealed mineral voxels
    int dis_on, dis_law, dis_surf, sM;  // sM: internal index of the mineral
    double dprm[2 + CLB_MAX_SPECIES];
    // thermodynamic gate of the biotic rates (internal species indices; chi already >= 1 when unset)
    int gate_on, gate_n;
    int gate_sp[CLB_MAX_SPECIES];
    double gate_nu[CLB_MAX_SPECIES];
    double gate_dG0, gate_dGloss, gate_atp, gate_dGatp, gate_chi, gate_cmin, gate_RT, gate_cscale;
    double gate_x0, gate_inv_chi;   // (dG0 + dGloss + atp dGatp) / (chi RT) and 1 / chi
    int* nonfinite;                 // host-mapped flag a transport step sets on a NaN / Inf density
    // rate laws read from .sym files (law / law2 CLB_LAW_SYMBOLIC): programs [microbe], then the
    // abiotic one at [CLB_MAX_MICROBES]; sym_mask: the microbes that have one
    const SymProg* sym;
    uint32_t sym_mask;
    // graph networks read from .gnn files, in the same slots ([microbe], then the abiotic one);
    // gnn_mask: the microbes whose law is a network (law CLB_LAW_SYMBOLIC), gnn_abiotic: the abiotic
    // law (law2 CLB_LAW_SYMBOLIC) is a network
    const GnnNet* gnn;
    uint32_t gnn_mask;
    int gnn_abiotic;
    // surrogate organisms (.srg networks with their uptake parameters, [microbe]); srg_mask: the
    // microbes that are one (law CLB_LAW_SYMBOLIC)
    const SrgNet* srg;
    uint32_t srg_mask;
    // [K] per species-lattice node: 0 where no microbe's biomass reaches 1e-12 (so no organism
    // grows, decays or draws there), 1 where one may; kept by clb_set_biomass / clb_set_field and
    // by the automaton's mask passes, so the transport step reads biomass only where it can act
    const uint8_t* bflag;
};

// Per-node state of the precipitation / dissolution machinery (geometry_update.cu), passed to the
// fused transport step when an abiotic law or dissolution is active.
struct AdeExtra {
    const uint8_t* iface;   // [K] 1: a solid or wall face neighbour (surface-only abiotic gate)
    const int32_t* xidx;    // [K] row of the node in xdc, -1: none
    const double* xdc;      // [S][ng] abiotic increments of the nodes next to sealed voxels,
                            // gathered dissolution shares included
    int64_t ng;
};

}  // namespace clb

namespace clb {
// Host-owned device buffers of one compacted node layout (sparse.cuh).
struct SparseBuffers {
    int32_t* node = nullptr;
    int8_t* code = nullptr;
    uint32_t* wall = nullptr;
    int32_t* linkbase = nullptr;
    int32_t* rowstart = nullptr;
    uint32_t* rowmask = nullptr;
    int32_t* rowpre = nullptr;
    int32_t* idx_of = nullptr;
    // odd-step metadata (see sparse.cuh)
    uint32_t* meta = nullptr;   // [K][MW] packed wall / edge / row bits / link residual
    int16_t* dres = nullptr;    // [K][NR] neighbour-row rank residuals
    int32_t* tlb = nullptr;     // [T] link base of each 256-node tile
    int32_t* tdb = nullptr;     // [T][NR] neighbour-row rank bases of each tile
    int64_t K = 0, L = 0;
    int64_t KS = 0;             // population row stride: K rounded up to a multiple of 256
    int64_t SS = 0;             // species stride of a lattice whose link slots follow its q rows:
                                // q KS + L rounded up to a multiple of 256
    int W = 0, NR = 0;
};
}  // namespace clb

// ------------------------------------------------------------------ the handle
struct clb_handle_s {
    clb_domain_desc d;
    clb::Geom g;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int device = 0;
    int num_sms = 148;
    std::string err;
    int64_t launches = 0;             // kernels this handle enqueued on the coupled step's path
    void* d_sym = nullptr;            // SymProg[SYM_MAX_PROGS] on the device
    clb::SymProg sym_host[clb::SYM_MAX_PROGS];
    void* d_gnn = nullptr;            // GnnNet[SYM_MAX_PROGS] on the device
    clb::GnnNet* gnn_host = nullptr;  // host copies of the bound networks (SYM_MAX_PROGS, allocated on first use)
    void* d_srg = nullptr;            // SrgNet[CLB_MAX_MICROBES] on the device
    clb::SrgNet* srg_host = nullptr;  // host copies of the bound surrogates (CLB_MAX_MICROBES, on first use)
    std::vector<int8_t> h_mat;
    int8_t* d_mat = nullptr;

    // flow
    bool flow_ready = false;
    int flow_prec = CLB_F32;
    void* d_f = nullptr;              // [19][K] storage type, compacted stored nodes
    void* d_flink = nullptr;          // [L] wall link slots
    clb::SparseBuffers flow_sp;
    int64_t k_west_end = 0, k_east_begin = 0;  // compact index ranges of the planes x=0, x=nx-1
    clb::FlowParams fp;
    clb::Tracer* d_tracer = nullptr;
    double* d_partials = nullptr;     // per-block partial sums (scratch)
    int partial_cap = 0;
    int flow_grid = 0;
    int flow_even_tma = 1;            // even AA step through shared-memory tiles and bulk copies
    int flow_minb = 3;                // minimum resident CTAs per SM of the gather/scatter step (2 or 3)
    int flow_even_grid = 0;
    int flow_odd_pipe = 1;            // odd step pipelined through shared memory (4- and 8-byte storage)
    int flow_pipe_grid = 0;           // its resident-CTA grid; 0 where it is not available
    int* d_err = nullptr;             // device error flag (bounded waits that gave up)
    uint8_t* d_bflag = nullptr;       // [K] species-lattice nodes where biomass may act (AdeParams::bflag)
    int* h_flags = nullptr;           // host-mapped pinned flags: [0] a transport step met a non-finite
    int* d_flags = nullptr;           // density (its device alias)
    int64_t flow_iters = 0;           // host mirror of the device iteration count
    double delta_p = 0;

    // transport
    bool ade_ready = false;
    int ade_prec = CLB_F32;
    int S = 0, n_mobile = 0, M = 0;
    std::vector<clb_species_desc> species;  // user order
    int u2i[CLB_MAX_SPECIES];               // user species index -> internal (mobile first)
    int i2u[CLB_MAX_SPECIES];
    void* d_g = nullptr;              // [n_mobile][7][K] storage type, compacted stored nodes
    void* d_glink = nullptr;          // d_g + 7 KS: species m's wall link slots start at d_glink + m SS
                                      // (inside d_g, whose species m occupies [m SS, (m + 1) SS))
    clb::SparseBuffers ade_sp;
    int64_t ade_west_end = 0, ade_east_begin = 0;
    double* d_imm = nullptr;          // [S][N] immobile concentrations (unused rows stay empty)
    double* d_bio = nullptr;          // [M][N] biomass
    void* d_u = nullptr;              // [3][K] advection velocity (arithmetic type)
    double* d_neu = nullptr;          // [S][2][ny*nz] stored boundary densities
    double* d_red = nullptr;          // scratch of clb_reduce (partials, then the result)
    double* d_stage = nullptr;        // [N] staging of a field read back to the host
    clb::AdeParams ap;
    int64_t ade_iters = 0;
    int64_t neu_iter = -1;            // iteration whose stream the Neumann store reflects
    int ade_grid = 0;
    int ade_pipe = 0;                 // transport step with the next node's gathers in flight (where it fits)

    // speciation (SpecParams lives in speciation.cuh; kept as raw storage here)
    alignas(16) unsigned char sp_storage[2048];
    bool spec_ready = false;
    int spec_mode = 0;
    unsigned long long* d_spec_stats = nullptr;
    float* d_mlp = nullptr;             // params, Adam m, v, grad, scaling
    void* d_mlp_bf16 = nullptr;         // BF16 operand copies of W1, W2, W3
    bool mlp_ready = false;
    float mlp_margin = 0.02f, mlp_resid_tol = 1e-6f;
    int mlp_polish = 2;

    // precipitation / dissolution (geometry_update.cu)
    bool prc_ready = false;
    clb_precip_desc prc;
    uint8_t* d_stamp = nullptr;       // [N] 1 where precipitation sealed the voxel
    unsigned int* d_count = nullptr;  // conversion counters
    int8_t* d_mat_flow = nullptr;     // [N] the flow lattice's own material map once they differ
    std::vector<int8_t> h_mat_flow;
    uint8_t* d_iface = nullptr;       // [K_ade] surface gate of the abiotic law
    int32_t* d_seal = nullptr;        // sealed voxels: compact species-lattice index
    int64_t n_seal = 0, seal_cap = 0;
    int32_t* d_gath = nullptr;        // open voxels next to a sealed one: compact index
    int32_t* d_gath_nb = nullptr;     // [ng][6] row in the sealed list of each face neighbour, -1
    int64_t n_gath = 0, gath_cap = 0;
    int32_t* d_xidx = nullptr;        // [K_ade] row in the gather list, -1
    double* d_park = nullptr;         // [S][seal_cap] parked dissolution shares
    double* d_xdc = nullptr;          // [S][gath_cap] abiotic increments of the gather list

    // biofilm cellular automaton (biofilm_ca.cu)
    bool ca_ready = false;
    double ca_bmax = 0, ca_frac = 0;
    int ca_half = 0;                  // push mode: 0 'fraction', 1 'half' 
    uint64_t ca_seed = 0, ca_sweeps = 0;
    long long ca_mask_sum = 0;
    double* d_ca_total = nullptr;     // [N] total biomass as the automaton tracks it
    int* d_ca_age = nullptr;          // [N] age wavefront
    int32_t* d_ca_list[2] = {nullptr, nullptr};  // [N] each: voxels whose total biomass exceeds 1e-14
                                      // (the last mask pass's list and the one the next pass writes)
    int32_t* d_ca_ext = nullptr;      // [N] voxels a push sweep deposited into that are not active
    int32_t* d_ca_ext2 = nullptr;     // [N] of those, the ones off the biomass list
    int* d_ca_tmark = nullptr;        // [N] 1 while a voxel is on d_ca_ext
    bool ca_full = true;              // the next automaton step's first pass covers the whole box
    bool h_mat_stale = false;         // the automaton changed the device map since h_mat was copied
    void* h_ca_pin = nullptr;         // pinned host copies of the counters: [1] read back
    int8_t* d_ca_distp = nullptr;     // [N] 1 where the distance-from-wall field is positive
    int* d_ca_aidx = nullptr;         // [N] row of an active voxel in the sweep, -1
    int* d_ca_act = nullptr;          // [cap] active voxels of a sweep
    int* d_ca_done = nullptr;         // [cap] round in which each was processed
    int* d_ca_tgt = nullptr;          // [cap][7] push targets
    double* d_ca_amt = nullptr;       // [cap][7][M] pushed biomass
    double* d_ca_own = nullptr;       // [cap][M] biomass left in the voxel
    void* d_ca_sc = nullptr;          // device counters of the automaton
    int8_t* d_ca_mask0 = nullptr;     // mask before a pass (several pore codes)
    int ca_cap = 0;
    int ca_grid = 0;                  // blocks of the cooperative automaton step (all resident)
    // the window of the in-loop re-solves' tracer between re-solves (valid after the first)
    clb::Tracer resolve_tracer{};
    bool resolve_tracer_valid = false;
};

namespace clb {
// error helpers (api.cu)
clb_status fail(clb_handle* h, clb_status s, const std::string& msg);
// brings h_mat up to date with the device map after automaton passes changed it (api.cu)
clb_status host_mat_sync(clb_handle* h);
clb_status cuda_check(clb_handle* h, cudaError_t e, const char* what);

// flow.cu
clb_status flow_init(clb_handle* h, double delta_p);
clb_status flow_step(clb_handle* h, int n, bool trace, double eps);
// keep_window: the in-loop re-solves' ValueTracer (complab.cpp:2166, ns_convg2) is one object for
// the whole run, never reset, so each re-solve starts with the window the previous one left
clb_status flow_solve(clb_handle* h, int max_it, double eps, int* iterations, bool keep_window = false);
clb_status flow_autotune(clb_handle* h, int steps, char* report, int report_len);
clb_status flow_stats(clb_handle* h, double char_length, clb_flow_stats* out);
clb_status flow_velocity(clb_handle* h, void* dst, int dtype_device, bool to_host);
clb_status flow_velocity_at(clb_handle* h, const int32_t* nodes, int64_t count, void* u, int64_t stride, int dtype);
clb_status flow_populations(clb_handle* h, double* host);
clb_status flow_set_populations(clb_handle* h, const double* host);
void flow_free(clb_handle* h);

// ade.cu
clb_status ade_init(clb_handle* h, const clb_species_desc* sp, int S);
clb_status ade_step(clb_handle* h, int n);
clb_status ade_nonfinite_check(clb_handle* h);
clb_status ade_couple(clb_handle* h);
clb_status ade_set_kinetics(clb_handle* h, int law, const double* prm, int nprm, double dt);
clb_status ade_set_biomass(clb_handle* h, int M, const double* b);
clb_status ade_density(clb_handle* h, int s, double* host);
// shifted != 0: the C ABI's populations g_i - t_i; 0: the storage's own g_i - sigma t_i (exact round
// trips for restart files)
clb_status ade_populations(clb_handle* h, int s, double* host, int shifted = 1);
clb_status ade_set_populations(clb_handle* h, int s, const double* host, int shifted = 1);
clb_status ade_biomass(clb_handle* h, int m, double* host);
clb_status ade_velocity(clb_handle* h, double* host);
clb_status ade_set_velocity(clb_handle* h, const double* host);
clb_status ade_set_biomass_field(clb_handle* h, int m, const double* host);
clb_status ade_reduce(clb_handle* h, clb_stats* out);
clb_status ade_reduce_noalloc(clb_handle* h, clb_stats* out);
clb_status ade_set_abiotic(clb_handle* h, int law, const double* prm, int nprm, int surface_only);
clb_status ade_set_thermo(clb_handle* h, const clb_thermo_desc* d);
clb_status ade_set_immobile(clb_handle* h, int s, const double* host);
clb_status ade_set_concentration(clb_handle* h, int s, const double* host);
void ade_refresh_neumann(clb_handle* h);
void ade_free(clb_handle* h);

// geometry_update.cu
clb_status precip_setup(clb_handle* h, const clb_precip_desc* d);
clb_status geometry_update(clb_handle* h, int* sealed, int* reopened);
clb_status geometry_refresh(clb_handle* h);   // surface gate and dissolution lists from the map
clb_status dissolution_pre_step(clb_handle* h); // park + gather before a transport step
AdeExtra ade_extra(clb_handle* h);
void precip_free(clb_handle* h);
inline const int8_t* flow_mat(const clb_handle* h) { return h->d_mat_flow ? h->d_mat_flow : h->d_mat; }

// batch.cu
clb_status batch_create(clb_handle* const* hs, int n, clb_batch** out);
clb_status batch_step(clb_batch* b, int n, int flow, int ade);
clb_status batch_autotune(clb_batch* b, int steps, char* report, int report_len);
clb_status batch_destroy(clb_batch* b);
clb_status batch_counts(clb_batch* b, int64_t* flow_nodes, int64_t* ade_nodes);
clb_status batch_schedule(clb_batch* b, int persistent, int tile, int lag, int steps_per_launch, int ctas_per_sm);
clb_status batch_set_stream(clb_batch* b, void* stream);
clb_status batch_set_wait_limit(clb_batch* b, int64_t ns);
clb_status batch_get_schedule(clb_batch* b, int* persistent, int* tile, int* lag, int* steps_per_launch,
                              int* ctas_per_sm);

// biofilm_ca.cu
clb_status ca_setup(clb_handle* h, const clb_ca_desc* d);
clb_status ca_step(clb_handle* h, int* sweeps, int* mask_changed);
// the step enqueued only, and the results read back later (clb_run's loop)
clb_status ca_step_async(clb_handle* h, int64_t iter);
clb_status ca_read(clb_handle* h, int* step_sweeps, int* step_changed, int64_t* total_sweeps, int64_t* total_changes);
clb_status refresh_species_if_changed(clb_handle* h);
clb_status refresh_dynamics(clb_handle* h, int species, int flow);
clb_status ca_fields(clb_handle* h, int which, double* host);
void ca_free(clb_handle* h);

// driver.cu
clb_status run(clb_handle* h, const clb_run_desc* d, clb_run_report* r);

// symbolic.cu
clb_status symbolic_set(clb_handle* h, const char* path, const char* const* species_names, int microbe,
                        const char* microbe_name);
clb_status symbolic_eval(clb_handle* h, int which, const double* vars, int n, double* rates, int* n_rates);
void sym_eval_batch(clb_handle* h, int slot, const double* dvars, int n, double* drates);
clb_status graphnet_set(clb_handle* h, const char* path, const char* const* species_names, int microbe);
clb_status graphnet_eval(clb_handle* h, int which, const double* conc, int n, double* out, int* n_out,
                         long* n_clamped);
clb_status srg_set(clb_handle* h, const char* path, const char* const* species_names, int microbe,
                   const clb_surrogate_desc* d);
clb_status srg_eval_host(clb_handle* h, int microbe, const double* x, int n, double* out, int* n_out,
                         long* n_clamped);

// speciation.cu
clb_status speciation_setup(clb_handle* h, const clb_speciation_desc* d);
clb_status speciation_step(clb_handle* h);
clb_status speciation_solve(clb_handle* h, const double* cin, int n, double* cout, int* iters);
clb_status speciation_solve_device(clb_handle* h, const double* d_in, int n, double* d_out);
clb_status speciation_stats(clb_handle* h, clb_speciation_stats* out);
clb_status surrogate_train(clb_handle* h, const clb_surrogate_train_desc* d, clb_surrogate_report* rep);
clb_status surrogate_predict(clb_handle* h, const double* cin, int n, double* cout, int* accepted, int check);
clb_status surrogate_gradient(clb_handle* h, const float* X, const float* Y, int n, float* grad, float* loss);
clb_status surrogate_params(clb_handle* h, float* out, const float* in, float* scaling_out, const float* scaling_in);
int surrogate_param_count();

// list building (api.cu)
std::vector<int32_t> build_list(const clb_handle* h, const int8_t* cls_by_code);
}  // namespace clb

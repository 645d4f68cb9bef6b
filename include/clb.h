/* clb.h -- C ABI of the B200-native CompLaB3D reactive-transport step.
 *
 * One opaque handle owns every device buffer of one domain. Host buffers passed in are
 * copied; no pointer is retained across calls. Calls enqueue on the handle's CUDA stream
 * and return a clb_status; clb_last_error() gives the message of the last failure. No call
 * aborts the process or throws across the ABI.
 *
 * Layouts. Every per-voxel array is lexicographic with x slowest and z fastest:
 * index(x,y,z) = (x*ny + y)*nz + z -- the order of the reference's serial processor loops
 * (iX outer, iZ inner). nx counts the two ghost x-planes that the reference adds when it
 * reads a geometry (complab_functions.hh:999, readGeometry :178-207). Population arrays are
 * direction-major [q][N] in Palabos' velocity order, shifted by the lattice weights
 * (f_i - t_i), as Palabos stores them.
 *
 * Each entry point names the reference interface it replaces (paths inside the
 * CompLaB3D-GEMS project).
 */
#ifndef CLB_H
#define CLB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum clb_status {
    CLB_OK = 0,
    CLB_INVALID_ARG = 1,
    CLB_NOT_CONVERGED = 2,
    CLB_NONFINITE = 3,
    CLB_PERCOLATION_LOST = 4,
    CLB_CUDA_ERROR = 5,
    CLB_TIMEOUT = 6,
    CLB_NOT_INITIALIZED = 7,
    CLB_OUT_OF_MEMORY = 8
} clb_status;

/* Storage precision of lattice populations. Arithmetic is FP64 for CLB_F64 and FP32 for
 * the two others. CLB_F16S stores the Palabos shifted populations f - t_i in IEEE half. */
typedef enum clb_precision { CLB_F64 = 0, CLB_F32 = 1, CLB_F16S = 2 } clb_precision;

/* x-face boundary kinds of an advection-diffusion species (complab_functions.hh:404-438). */
typedef enum clb_face { CLB_DIRICHLET = 0, CLB_NEUMANN = 1, CLB_CLOSED = 2 } clb_face;

/* Rate laws compiled into the library (the reference compiles defineRxnKinetics /
 * defineAbioticRxnKinetics from config/kinetics/ into its binary). */
typedef enum clb_law {
    CLB_LAW_NONE = 0,
    CLB_LAW_DECAY = 1,      /* params k[S]:          R_s = -k_s C_s                        */
    CLB_LAW_MONOD = 2,      /* params k[S], Ks[S]:   R_s = -k_s C_s / (Ks_s + C_s)           */
    CLB_LAW_DUAL_MONOD = 3, /* params mu_max, Ks, Y, kd; microbe m grows on species 0 (donor)
                               and species 1+m (acceptor):
                               growth = mu_max C0/(Ks+C0) Ca/(Ks+Ca) B_m,
                               R_B = growth - kd B_m, R_0 -= growth/Y, R_a -= growth/Y     */
    /* abiotic laws (clb_set_abiotic_kinetics; defineAbioticRxnKinetics of the reference) */
    CLB_LAW_PRECIP = 4,     /* params kp, a, b, p: A + B -> P(s), R = kp max(C_a,0) max(C_b,0),
                               R_a = R_b = -R, R_p = +R (examples/13_precipitation)          */
    CLB_LAW_SYMBOLIC = 6,   /* a rate-law file read at run time (clb_set_symbolic_kinetics);
                               not selected through clb_set_kinetics / clb_set_abiotic_kinetics */
    CLB_LAW_MINERAL = 5     /* params k, log10 Ksp, p, nu[S]: saturation
                               Omega = 10^(sum_{j != p} nu_j log10 C_j - log10 Ksp),
                               R_p = k (Omega - 1), R_j = -nu_j R_p: the mineral p grows when the
                               water is supersaturated and dissolves (clamped at what there
                               is) when it is undersaturated                                 */
} clb_law;

#define CLB_MAX_MICROBES 8
#define CLB_MAX_PORE_CODES 8
#define CLB_MAX_SPECIES 16

/* The material-number surface of CompLaB.xml <material_numbers> plus the flow relaxation
 * (complab_functions.hh:1213-1285, NSdomainSetup :296-345). */
typedef struct clb_domain_desc {
    int32_t nx, ny, nz;           /* lattice size, ghost x-planes included                  */
    int32_t flow_precision;       /* clb_precision of the D3Q19 lattice                      */
    int32_t ade_precision;        /* clb_precision of the D3Q7 lattices                      */
    int32_t solid_code;           /* <solid>: NoDynamics on the flow lattice; -1 if none     */
    int32_t bounce_back_code;     /* <bounce_back>: inert wall; -1 if none                   */
    int32_t n_pore_codes;
    int32_t pore_codes[CLB_MAX_PORE_CODES];
    int32_t n_microbes;           /* biofilm material numbers, one per microbe               */
    int32_t bio_codes[CLB_MAX_MICROBES];
    double perm_ratio[CLB_MAX_MICROBES]; /* biofilm omega = 1/(r (1/omega - 1/2) + 1/2);
                                            r <= 1e-14 makes that biofilm bounce-back      */
    double tau;                   /* flow relaxation time                                    */
} clb_domain_desc;

/* One advection-diffusion species (soluteDomainSetup, complab_functions.hh:347-442;
 * relaxation rates as complab.cpp:1230-1253 derives them). */
typedef struct clb_species_desc {
    double omega_pore;
    double omega_biofilm;
    int32_t mobile;               /* 0: immobile -- never collides or streams               */
    int32_t left_type, right_type;/* clb_face                                                */
    double left_bc, right_bc;     /* Dirichlet values                                        */
    double c0;                    /* initial and background concentration                    */
} clb_species_desc;

typedef struct clb_flow_stats {
    double pore_mean_u;           /* mean |u| over x = 1..nx-2 (complab.cpp:1150)            */
    double pore_max_ux;           /* max u_x over x = 1..nx-2                                */
    double darcy_outlet_ux;       /* mean u_x over the plane x = nx-2                        */
    double permeability;          /* darcy_outlet_ux * nu * L / dP (complab.cpp:1160)        */
    double energy;                /* last stored average energy (half the mean |u|^2)       */
    int64_t iterations;           /* collide-and-stream calls made so far                    */
    int64_t bgk_nodes;            /* nodes that collide (pore + permeable biofilm)           */
    int64_t active_nodes;         /* nodes the step launches (BGK + no-dynamics)             */
} clb_flow_stats;

typedef struct clb_stats {
    double total[CLB_MAX_SPECIES];   /* sum of concentration over x=1..nx-2, open voxels     */
    double content[CLB_MAX_SPECIES]; /* sum over every node of (sum of populations + 1)      */
    double biomass[CLB_MAX_MICROBES];/* sum of biomass over x=1..nx-2                        */
    double min_c[CLB_MAX_SPECIES], max_c[CLB_MAX_SPECIES];
    int64_t open_voxels;             /* pore + biofilm voxels in x=1..nx-2                   */
    int64_t nonfinite;               /* non-finite concentrations found                      */
    int64_t ade_iterations;
} clb_stats;

/* Field identifiers for clb_get_field / clb_set_field. dtype: 0 = float64, 1 = float32,
 * 2 = int8. The material map is int8; clb_get_field reads the flow velocity as float64 or
 * float32 (half the copy to the host), every other field as float64. */
typedef enum clb_field {
    CLB_FIELD_MATERIAL = 0,       /* int8 [N]                                                */
    CLB_FIELD_FLOW_VELOCITY = 1,  /* [3][N]  computeVelocity of the flow lattice            */
    CLB_FIELD_FLOW_POPULATIONS = 2, /* [19][N] incoming (post-stream) populations            */
    CLB_FIELD_CONCENTRATION = 3,  /* [N] of species `index`: computeDensity. Written: an
                                     immobile species takes the field, a mobile one the
                                     equilibrium populations at rest with that density      */
    CLB_FIELD_ADE_POPULATIONS = 4,/* [7][N] of species `index`                               */
    CLB_FIELD_BIOMASS = 5,        /* [N] of microbe `index`                                  */
    CLB_FIELD_ADE_VELOCITY = 6,   /* [3][N] the advection velocity the species see          */
    CLB_FIELD_CA_TOTAL = 7,       /* [N] total biofilm biomass the automaton tracks          */
    CLB_FIELD_CA_AGE = 8          /* [N] age wavefront (integers)                            */
} clb_field;

typedef struct clb_handle_s clb_handle;

/* ---------------------------------------------------------------- lifetime */

/* Selects the CUDA device that later clb_create calls on this thread allocate on (the library
 * carries its own CUDA runtime, so a device chosen through another runtime is not seen). */
clb_status clb_set_device(int device);

/* Allocates the domain on the current CUDA device and uploads the material map.
 * Replaces: MultiScalarField3D<int> geometry + readGeometry (complab.cpp:1051-1052). */
clb_status clb_create(const clb_domain_desc* desc, const int8_t* material, clb_handle** out);
clb_status clb_destroy(clb_handle* h);
const char* clb_last_error(const clb_handle* h);
/* Message of the last failure of a call that had no handle to record it in. */
const char* clb_global_error(void);
clb_status clb_synchronize(clb_handle* h);

/* Every call of the handle enqueues on this stream (a cudaStream_t). By default the handle
 * owns a non-blocking stream; a caller that times or orders work with its own stream passes it
 * here (the handle then never destroys it). */
clb_status clb_set_stream(clb_handle* h, void* stream);
clb_status clb_get_stream(clb_handle* h, void** stream);

/* Launch-shape and kernel-variant knobs (used by the autotuner; defaults are tuned for B200):
 *   "flow_even_tma"  1: even AA step through shared-memory tiles and bulk copies (default),
 *                    0: the plain per-thread load/store step;
 *   "flow_min_blocks" 2 or 3: resident CTAs per SM the gather/scatter step is compiled for
 *                    (register budget 128 or 80 per thread); takes effect at clb_flow_init;
 *   "flow_odd_pipe"  1: odd AA step with the next node's gathers staged in shared memory by
 *                    asynchronous copies while a node is collided (default for FP64/FP32
 *                    storage; an error for FP16 storage, which always runs the plain step),
 *                    0: the plain step;
 *   "ade_pipe"       1: transport step with the next node's gathers staged in shared memory by
 *                    asynchronous copies while a node is finished (used for FP64/FP32 storage
 *                    where two slot sets per thread leave two resident CTAs per SM, i.e. up to
 *                    8 FP32 or 4 FP64 species), 0: the plain step (default: fewer resident
 *                    warps made the pipelined step slower on B200).
 * Unknown keys are an error. */
clb_status clb_tune(clb_handle* h, const char* key, int value);

/* Times every kernel variant of the flow step over `steps` steps on this domain and keeps the
 * fastest; the lattice state is saved and restored, so the simulation is unchanged. A one-line
 * report of the timings is written to `report` (may be NULL). */
clb_status clb_autotune(clb_handle* h, int steps, char* report, int report_len);

/* ---------------------------------------------------------------- flow (D3Q19) */

/* Dynamics from the material map, pressure planes at x=0 (rho=1) and x=nx-1
 * (rho=1-3 dP), PressureGradient equilibrium initial state.
 * Replaces: NSdomainSetup (complab_functions.hh:296-345). */
clb_status clb_flow_init(clb_handle* h, double delta_p);

/* n x nsLattice.collideAndStream() (complab.cpp:1120-1124 loop body). */
clb_status clb_flow_step(clb_handle* h, int n);

/* Runs collideAndStream until util::ValueTracer(1,1000,eps) on the stored average energy
 * converges or max_it calls are made (complab.cpp:1113-1124). *iterations receives the
 * number of collideAndStream calls made. Returns CLB_NOT_CONVERGED at the cap while the outlet
 * plane x = nx-2 still flows, CLB_PERCOLATION_LOST at the cap when its mean u_x is at most 1e-12
 * (the flow path is sealed; complab.cpp:3106-3113), and CLB_NONFINITE when the stored energy is
 * NaN or infinite (the solve diverged; complab.cpp:3116-3117). */
clb_status clb_flow_solve(clb_handle* h, int max_it, double eps, int* iterations);

/* Velocity statistics and permeability (complab.cpp:1136-1160). */
clb_status clb_flow_stats_get(clb_handle* h, double char_length, clb_flow_stats* out);

/* The Peclet rescale of complab.cpp:1156-1179: permeability from the solved field, the
 * pressure drop that gives u = Pe D / L with D = (tau_ade_fixed - 1/2)/4, and a re-solve
 * from a fresh initial state when that drop differs by more than 1 %. *delta_p_out
 * receives the drop in use afterwards. */
clb_status clb_flow_solve_peclet(clb_handle* h, double peclet, double char_length,
                                 double tau_ade_fixed, int max_it, double eps,
                                 double* delta_p_out, int* iterations);

/* ---------------------------------------------------------------- transport (D3Q7) */

/* Species lattices at equilibrium at c0, wall/solid nodes seeded at c0, x faces as
 * described. Replaces: soluteDomainSetup (complab_functions.hh:347-442) and the wall
 * seeding of complab.cpp:1506-1656. */
clb_status clb_ade_init(clb_handle* h, const clb_species_desc* species, int n_species);

/* Copies the flow velocity into the species' advection field.
 * Replaces: latticeToPassiveAdvDiff (complab.cpp:2014, 3119). */
clb_status clb_couple_velocity(clb_handle* h);

/* Selects the compiled rate law and the time step used for dC = R dt.
 * Replaces: run_kinetics + update_rxnLattices (complab3d_processors_part1.hh:85-187,
 * 406-497) with the clamp dC = max(R dt, -C). */
clb_status clb_set_kinetics(clb_handle* h, int law, const double* params, int n_params, double dt);

/* The abiotic rate law, evaluated after the biotic one on the concentrations it left
 * (run_abiotic_kinetics, complab3d_processors_part1.hh:199-297; complab.cpp:2460-2525), with the
 * same clamp dC = max(R dt, -C) and the time step of clb_set_kinetics. surface_only != 0 limits it
 * to voxels with a solid or wall face neighbour (surfaceAbioticKinetics3D,
 * precipitationVOP.hh:53-153). law: CLB_LAW_NONE, CLB_LAW_PRECIP or CLB_LAW_MINERAL; species
 * indices in params are user species indices. */
clb_status clb_set_abiotic_kinetics(clb_handle* h, int law, const double* params, int n_params, int surface_only);

/* One reaction block of the thermodynamic gate (a .thm file's `reaction`), energies in kJ/mol. */
typedef struct clb_thermo_desc {
    int32_t n_terms;                   /* terms of the stoich line; 0 turns the gate off          */
    int32_t species[CLB_MAX_SPECIES];  /* user species index of each term                         */
    double nu[CLB_MAX_SPECIES];        /* stoichiometric number: negative reactant, positive product */
    double dG0;                        /* standard free energy at `temperature`, kJ/mol           */
    double atp;                        /* mol ATP conserved per mol reaction (m)                  */
    double dGatp;                      /* free energy of ATP synthesis, kJ/mol ATP                */
    double chi;                        /* average stoichiometric number (<= 0 reads as 1)         */
    double cmin;                       /* activity floor, mol/L (> 0)                             */
    double dGloss;                     /* constant electron-transfer loss added to dG (>= 0)      */
    double temperature;                /* kelvin                                                  */
    double gas_constant;               /* kJ/mol/K (8.314462618e-3)                               */
    double conc_scale;                 /* solver concentration unit -> mol/L                      */
} clb_thermo_desc;

/* The thermodynamic gate of the biotic rates: per voxel, on the concentrations the rate law saw
 * (times conc_scale, floored at cmin), ln Q = sum nu_i ln a_i, dG = dG0 + R T ln Q + dGloss,
 * F_T = max(0, 1 - exp((dG + atp dGatp) / (chi R T))), and every substrate and biomass rate of the
 * voxel is multiplied by F_T before dC = max(R dt, -C). As in the reference, the block applies to
 * microbe 0, so the gate acts only in a run with biomass fields. desc NULL or n_terms 0: off.
 * F_T is evaluated in the lattice's arithmetic type (FP64 lattices: FP64; otherwise FP32).
 * The gate is compiled into the transport instantiations that also carry the abiotic block;
 * clb_batch_create refuses a gated domain.
 * Replaces: complab_thermo::gateFor (complab3d_thermo.hh:215-258, 669-692) in run_kinetics
 * (complab3d_processors_part1.hh:134-141) with one reaction block. */
clb_status clb_set_thermo_gate(clb_handle* h, const clb_thermo_desc* desc);

/* A rate law read at run time from a .sym file (the reference's complab3d_symbolic.hh format:
 * units / vars / range / rate / reaction / yield / biomass lines; expressions with + - * / ^,
 * exp log log10 sqrt abs tanh min max pow, pi, e; rate lines may use earlier ones; a 'reaction'
 * line derives the species lines), compiled on the host and evaluated per voxel in FP64 inside the
 * fused transport step. species_names[S] names the handle's species (user order) for the file's
 * variables and rate outputs.
 *   microbe >= 0: the law of the organism whose biomass field is `microbe` (a 'growth' line;
 *     microbe_name is its variable in the file): where its biomass exceeds 1e-12, the substrate
 *     rates are requested and the growth rate times the biomass grows it; the requests of all
 *     organisms of a voxel share each substrate's headroom (a draw never takes more than the
 *     voxel holds), as run_symbolic3D does (complab3d_processors_symbolic.hh:100-200).
 *   microbe = -1: an abiotic law (an 'extent' line), in place of clb_set_abiotic_kinetics, in every
 *     reacting voxel, each increment clamped at what the voxel holds.
 * Variables are clamped to the file's ranges; per_hour rates are divided by 3600; the time step is
 * clb_set_kinetics's dt. Replaces: complab_sym::load / evaluate (complab3d_symbolic.hh:420-1063)
 * and run_symbolic3D. */
clb_status clb_set_symbolic_kinetics(clb_handle* h, const char* sym_path, const char* const* species_names,
                                     int microbe, const char* microbe_name);

/* The bound law of `microbe` (-1: the abiotic one) on n rows of its variables in file order
 * (vars [n][n_vars], host) into rates [n][n_rates] (host; rate lines in file order, derived lines
 * last, units applied), evaluated by the device interpreter; *n_rates receives the rate count
 * (may be NULL). */
clb_status clb_symbolic_eval(clb_handle* h, int microbe, const double* vars, int n, double* rates, int* n_rates);

/* A rate law given as a graph network read at run time from a .gnn file (the reference's
 * complab3d_graphnet.hh format: a bipartite network over the species and reactions of the file's
 * stoichiometric matrix, `rounds` rounds of message passing of width `width` with tanh layers,
 * readout `species` or `extent`, an optional growth output, inputs clamped to trainmin..trainmax,
 * per_hour rates divided by 3600), evaluated per voxel in FP64 inside the fused transport step.
 * The file's species names are matched against species_names[S] (the handle's species, user
 * order).
 *   microbe >= 0: the law of the organism whose biomass field is `microbe`: where its biomass
 *     exceeds 1e-12 the network's species rates are requested and its growth rate times the
 *     biomass grows it; the requests of all organisms of a voxel (networks and .sym laws alike)
 *     share each substrate's headroom, a draw never taking more than the voxel holds, and
 *     production passing through (run_graphnet3D, complab3d_processors_graphnet.hh:70-200).
 *   microbe = -1: an abiotic network (no growth output) in every reacting voxel, each increment
 *     clamped at what the voxel holds (run_graphnet_abiotic3D,
 *     complab3d_processors_abiotic_learned.hh:163-250).
 * The time step is clb_set_kinetics's dt; a network replaces a .sym law bound to the same slot
 * and the other way round. Networks of up to 8 species, 8 reactions, width 16 and 4 rounds.
 * Replaces: complab_gnn::load / Network::eval / bindToSubstrates (complab3d_graphnet.hh:84-330,
 * 402-600). */
clb_status clb_set_graph_network(clb_handle* h, const char* gnn_path, const char* const* species_names,
                                 int microbe);

/* The bound network of `microbe` (-1: the abiotic one) on n rows of concentrations in the file's
 * species order (conc [n][nS], host) into out [n][n_out] (host; the species rates, then growth when
 * the file has it; units applied), evaluated on the device; *n_out receives the output count and
 * *n_clamped the rows the training-box clamp changed (either may be NULL). */
clb_status clb_graph_network_eval(clb_handle* h, int microbe, const double* conc, int n, double* out, int* n_out,
                                  long* n_clamped);

/* The uptake parameters of a surrogate organism, per species in user order: half-saturation
 * constants Kc (mol/L) and maximum uptake fluxes (mmol/gDW/h; 0: none, the flux that would exhaust
 * the voxel in one step stands in), the biomass molar mass (gDW/mol) and the decay coefficient
 * (1/s) that acts where the network predicts no growth. */
typedef struct {
    double half_saturation[CLB_MAX_SPECIES];
    double max_uptake_flux[CLB_MAX_SPECIES];
    double biomass_molar_mass;
    double decay;
} clb_surrogate_desc;

/* A surrogate organism: the growth rate of the organism whose biomass field is `microbe` from a
 * feed-forward network read at run time from a .srg file (the reference's complab3d_surrogate.hh
 * format: mapminmax scaling, tansig hidden layers, a linear output layer, output 0 the growth rate
 * in 1/h, optionally as log10; inputs clamped to trainmin..trainmax), fed, as the reference's
 * default surrogate model feeds it, with the organism's Michaelis-Menten uptake estimates of the
 * substrates the file names (inputnames matched against species_names[S], user order; a file
 * without names takes the substrates in order). Where its biomass B exceeds 1e-12: every
 * substrate's estimate v = vmax C/(Kc + C) (without vmax the one-step exhaustion flux
 * C 3.6e6/(B MW dt), capped at 1e4, times C/(Kc + C)), never above that exhaustion flux; growth
 * mu B dt/3600, or decay kd B dt where |mu| < 1e-12; the substrates drawn by v B MW dt/3.6e6 under
 * the shared headroom budget of the voxel's run-time organisms. The time step (seconds) is
 * clb_set_kinetics's dt. A surrogate replaces a .sym law or a network bound to the same organism.
 * Networks of up to 8 inputs, 4 layers and 32 units a layer.
 * Replaces: run_surrogate3D (complab3d_processors_surrogate.hh:96-293) with surrogateModel.hh's
 * run-time network (complab_srg::load / Network::eval / evalBound, complab3d_surrogate.hh:117-258,
 * 380-470, 1029-1049) and MetabolicConfig's unit chain (complab3d_metabolic.hh:554-595). */
clb_status clb_set_surrogate_organism(clb_handle* h, const char* srg_path, const char* const* species_names,
                                      int microbe, const clb_surrogate_desc* desc);

/* The bound surrogate network of `microbe` on n rows of its inputs (x [n][n_inputs], host) into
 * out [n][n_out] (host; every output, output 0 the growth rate with its log and floor), after the
 * training-box clamp, evaluated on the device; *n_out receives the output count and *n_clamped the
 * rows the clamp changed (either may be NULL). */
clb_status clb_surrogate_eval(clb_handle* h, int microbe, const double* x, int n, double* out, int* n_out,
                              long* n_clamped);

/* Biomass fields of the CA microbes, [n_microbes][N] float64. */
clb_status clb_set_biomass(clb_handle* h, int n_microbes, const double* biomass);

/* n transport iterations: collide every mobile species, kinetics, deposit, stream, Neumann
 * planes (complab.cpp:2307-2315, 2340-2452, 3251-3259), fused in one pass per step.
 * A step that meets a NaN or infinite concentration sets a flag the host reads without a copy;
 * the run then stops as the reference stops on non-finite values (complab.cpp:2796, 3116-3117):
 * the next clb_ade_step, and clb_synchronize once that step has completed, return
 * CLB_NONFINITE. clb_set_field of a species' populations clears the flag. */
clb_status clb_ade_step(clb_handle* h, int n);

/* FP64 reductions over the live fields (complab3d_processors_part3.hh:387-600). Warp shuffles and
 * a fixed order over warps and blocks, no atomics: the same fields give the same bits on every
 * call. Scratch is the handle's own (allocated by clb_ade_init); nothing is allocated per call. */
clb_status clb_reduce(clb_handle* h, clb_stats* out);

/* The same reductions as clb_reduce, computed without allocating: no counterpart in the
 * reference, whose reductions run inside Palabos data processors. For callers that must not
 * allocate while they monitor a run (an application that hands all device memory to its own
 * pool, or a loop that cannot absorb the device-wide synchronisation of a free). The partial
 * sums live in one fixed 65536-double buffer per device, built into the library; a handle whose
 * reduction needs more (2 x SMs x (5 x species + microbes + 1) + 4 x species + microbes + 2
 * doubles; 26,418 at 16 species and 8 microbes on 148 SMs) gets CLB_INVALID_ARG. Same
 * fixed-order tree as clb_reduce, so the two give the same bits. The buffer is shared by every handle on a device, so calls must not overlap
 * in time on one device (they would race on it). The first call on a device looks the buffer
 * up; make it before any stream capture begins. */
clb_status clb_reduce_noalloc(clb_handle* h, clb_stats* out);

/* ---------------------------------------------------------------- precipitation / dissolution */

/* Dissolution law of a sealed mineral voxel (defineDissolutionRate of the reference). */
typedef enum clb_dissolution_law {
    CLB_DISSOL_NONE = 0,
    CLB_DISSOL_FIRST_ORDER = 1, /* params kd, h, sigma[S]: rate = kd max(water_h,0) max(mineral,0)
                                   (h < 0: no water factor); the mineral loses rate, species j
                                   gains sigma_j rate (examples/15_precip_and_dissolution)    */
    CLB_DISSOL_MINERAL = 2      /* params k, log10 Ksp, nu[S]: Omega of the water; below 1 the
                                   mineral dissolves at k (1 - Omega), releasing nu_j times it */
} clb_dissolution_law;

/* <precipitation> and <dissolution> of CompLaB.xml with one precipitate phase. */
typedef struct clb_precip_desc {
    int32_t mineral_species;      /* immobile species holding the precipitate (user index)      */
    double full_density;          /* max_precipRho: a voxel seals at mineral >= this            */
    int32_t precip_code;          /* material code of sealed voxels; -1: the solid code         */
    int32_t seal_flow;            /* 0: the flow lattice keeps its dynamics at sealed voxels, as
                                     the reference's updateNsLatticesDynamics3D does (it skips
                                     solid voxels, complab3d_processors_part2.hh:785-806);
                                     1: sealed voxels become bounce-back on the flow lattice
                                     (permeable IncBGK if seal_perm_ratio > 0) and the flow is
                                     re-solved after every change                             */
    double seal_perm_ratio;       /* <precipitation><perm_ratio>                               */
    int32_t flow_max_iterations;  /* re-solve cap (ns_max_iT2)                                 */
    double flow_eps;              /* re-solve convergence (ns_convergence_iT2)                 */
    int32_t dissolution;          /* 1: sealed voxels dissolve and may reopen                   */
    double reopen_fraction;       /* reopen below this fraction of full_density (0.9)           */
    int32_t pore_code;            /* material of a reopened voxel; -1: the first pore code      */
    int32_t dissolution_law;      /* clb_dissolution_law                                        */
    double dissolution_params[CLB_MAX_SPECIES + 2];
    int32_t dissolution_surface_only; /* 1: a voxel with no open face neighbour does not dissolve */
} clb_precip_desc;

/* Replaces: the <precipitation>/<dissolution> set-up of complab.cpp (phase lattice, precipitate
 * phase). Dissolution, when on, runs inside every later clb_ade_step as the reference runs it in
 * the abiotic block: surfaceDissolutionKinetics3D (dissolutionVOP.hh:379-605) parks the products
 * per open face, dissolutionGather3D (:608-742) lets the open neighbours collect them. */
clb_status clb_precip_setup(clb_handle* h, const clb_precip_desc* desc);

/* The node conversions of one update interval: precipNodeConversion3D (precipitationVOP.hh:166-227)
 * seals open voxels of x = 1..nx-2 whose mineral reached full_density, dissolNodeConversion3D
 * (dissolutionVOP.hh:745-810) reopens sealed voxels below reopen_fraction x full_density. The
 * species lattices switch dynamics there and keep their populations
 * (updateSoluteSolidDynamics3D, complab3d_processors_part2.hh:585-647); with seal_flow the flow
 * lattice does too and is re-solved, then its velocity is coupled again (complab.cpp:3139-3247).
 * sealed / reopened (may be NULL) receive the voxel counts. */
clb_status clb_geometry_update(clb_handle* h, int* sealed, int* reopened);

/* ---------------------------------------------------------------- biofilm cellular automaton */

/* The <microbiology> settings of the CA microbes (solver type CA; the biomass fields are those of
 * clb_set_biomass, microbe m living in material bio_codes[m]). */
/* Push modes of the automaton (<microbiology><CA_method> of CompLaB.xml, halfflag):
 * CLB_PUSH_FRACTION  pushExcessBiomass3D (complab3d_processors_part1.hh:499-732): every open voxel
 *                    above max_biomass pushes the excess over it;
 * CLB_PUSH_HALF      halfPushExcessBiomass3D (:735-970): every biofilm voxel above max_biomass
 *                    pushes half its biomass, the fallback neighbour may have an equal age, and the
 *                    fallback push always runs (into the voxel itself when nothing is left or no
 *                    neighbour is open). */
#define CLB_PUSH_FRACTION 0
#define CLB_PUSH_HALF 1

typedef struct clb_ca_desc {
    double max_biomass;           /* max_bMassRho: excess above it is pushed to neighbours      */
    double biofilm_fraction;      /* thrd_bFilmFrac: pore <-> biofilm at this fraction of max   */
    uint64_t seed;                /* seed of the random neighbour choices (the reference seeds
                                     std::rand from the clock); a voxel's draws in a sweep are
                                     splitmix64 steps from seed ^ sweep*0x9E3779B97F4A7C15
                                     ^ voxel*0xD1B54A32D192ED03                               */
    int32_t push_mode;            /* CLB_PUSH_FRACTION or CLB_PUSH_HALF                          */
} clb_ca_desc;

/* Age and distance fields from the current mask (createAgeDomain3D, calculateDistanceFromSolid;
 * complab.cpp:1078-1090) and the total biomass (initTotalbFilmLatticeDensity). */
clb_status clb_ca_setup(clb_handle* h, const clb_ca_desc* desc);

/* The CA block of one iteration (complab.cpp:2792-3055): mask and total update
 * (updateLocalMaskNtotalLattices3D), then, while the largest total exceeds max_biomass, push
 * sweeps (pushExcessBiomass3D or halfPushExcessBiomass3D, by push_mode) each followed by the mask
 * update, with the age
 * relaxation (updateAgeDistance3D) every 50 sweeps; then one age sweep when the mask changed
 * (:3074-3079). Results equal the sequential lexicographic sweeps bit for bit. *sweeps receives
 * the push sweeps made, *mask_changed whether the mask changed. Returns CLB_NOT_CONVERGED where
 * the reference stops the run (no progress in 100 sweeps, more than 1000 sweeps, or an age
 * relaxation that does not settle). Voxels of the ghost planes x = 0 and x = nx-1 never push. */
clb_status clb_ca_step(clb_handle* h, int* sweeps, int* mask_changed);
/* (clb_ca_step returns CLB_NONFINITE when a biomass value is NaN or infinite, complab.cpp:2796.) */

/* Dynamics follow the mask: species != 0 runs updateSoluteDynamics3D (pore / biofilm relaxation,
 * complab3d_processors_part2.hh:485-553), flow != 0 updateNsLatticesDynamics3D (:748-818). The
 * reference runs them every ade_update_interval / ns_update_interval iterations after a mask
 * change; re-solve the flow and couple its velocity afterwards as it does. */
clb_status clb_refresh_dynamics(clb_handle* h, int species, int flow);

/* ---------------------------------------------------------------- the coupled step, driven */

/* The schedule of the reference's main loop (complab.cpp:2178-3262) for clb_run. */
typedef struct clb_run_desc {
    int32_t iterations;           /* transport iterations this call advances                      */
    int32_t ca;                   /* 1: the biofilm automaton every iteration (clb_ca_setup first) */
    int32_t ade_update_interval;  /* species dynamics follow a changed mask at iterations that are
                                     multiples of it (<ade_update_interval>; 0: never)            */
    int32_t ns_update_interval;   /* flow dynamics follow a changed mask and the flow is re-solved
                                     at iterations that are multiples of it (the reference's
                                     schedule: the mask changed at that very iteration; 0: never) */
    int32_t resolve_every;        /* re-solve the flow every this many iterations whatever the mask
                                     did (the flow dynamics follow the mask first if it changed since
                                     the previous re-solve); 0: off                               */
    int32_t geometry_interval;    /* precipitation / dissolution node conversion every this many
                                     iterations (clb_geometry_update; clb_precip_setup first); 0: off */
    int32_t flow_max_iterations;  /* cap of each re-solve (ns_max_iT2)                              */
    double flow_eps;              /* ValueTracer criterion of each re-solve (ns_converge_iT2)        */
} clb_run_desc;

typedef struct clb_run_report {
    int64_t iterations;           /* transport iterations made                                      */
    int64_t ca_sweeps;            /* push sweeps of the automaton                                   */
    int64_t mask_changes;         /* iterations whose automaton changed the mask                    */
    int64_t flow_resolves;        /* flow re-solves made (not counting clb_geometry_update's own)   */
    int64_t flow_iterations;      /* collide-and-stream calls of those re-solves                    */
    int64_t flow_unconverged;     /* re-solves that reached their cap with the outlet still flowing */
    int64_t sealed, reopened;     /* voxels converted by the geometry updates                       */
    double ms_transport;          /* device time of the fused transport steps (CUDA events)         */
    double ms_ca;                 /* device time of the automaton and the species' dynamics refresh */
    double ms_flow;               /* device time of the re-solves and velocity couplings            */
    double ms_geometry;           /* device time of the geometry updates (their re-solves included) */
    double seconds;               /* wall clock of the call                                         */
    int64_t launches;             /* kernels the call launched                                      */
} clb_run_report;

/* Advances d->iterations coupled iterations in the reference's order: the fused transport step
 * (collide, kinetics, speciation, stream), the biofilm automaton, the dynamics refresh and flow
 * re-solve after a mask change, the precipitation / dissolution conversions. Stops where the
 * reference stops: CLB_NONFINITE (non-finite concentrations, biomass or flow energy),
 * CLB_PERCOLATION_LOST (a re-solve found no flow through the outlet), CLB_NOT_CONVERGED (the
 * automaton could not settle); a re-solve that reaches its cap while the outlet still flows is
 * counted in report->flow_unconverged and the run goes on. report may be NULL.
 * Replaces: the body of the main loop, complab.cpp:2178-3262. */
clb_status clb_run(clb_handle* h, const clb_run_desc* d, clb_run_report* report);

/* ---------------------------------------------------------------- ensembles of domains */

/* A parameter sweep: many independent domains (each its own handle, with its own size, geometry,
 * relaxation times and species) advanced together, so many small uneven domains are not bound by
 * launch overhead. Two schedules:
 *   persistent (the default): one launch runs several steps of every lattice of every domain,
 *     walking a table of (step, domain, lattice, tile) items in which an item waits only for the
 *     same lattice of the same domain at the previous step; launches are replayed from a captured
 *     CUDA graph;
 *   per lattice: one launch per lattice and step covering the nodes of all domains, pairs of
 *     steps replayed from a captured CUDA graph.
 * Results are those of stepping each domain on its own, bit for bit, on either schedule. No
 * counterpart in the reference (one domain per run there). The handles must share a device and
 * storage precisions, be at the same step parity, and have no abiotic law, dissolution or
 * speciation; they must stay unchanged (no re-initialisation) while the batch exists. */
typedef struct clb_batch_s clb_batch;
clb_status clb_batch_create(clb_handle* const* handles, int n, clb_batch** out);

/* n steps of the flow lattices (flow != 0) and/or the species lattices (transport != 0) of every
 * domain; returns once they are done. Each handle's iteration counters advance by n. CLB_TIMEOUT:
 * a dependency wait of the persistent schedule gave up (bounded at two seconds; the domains'
 * state is then undefined). */
clb_status clb_batch_step(clb_batch* batch, int n, int flow, int transport);

/* Times the schedules and launch shapes of the batched steps over `steps` steps each (rounded up
 * to a multiple of 8) and keeps the fastest; the timed steps are real steps (the handles'
 * counters show them). */
clb_status clb_batch_autotune(clb_batch* batch, int steps, char* report, int report_len);

/* Sets the schedule: persistent == 1 with `tile` nodes per item (a multiple of 256), a lag of
 * `lag` >= 1 domains between a domain's successive steps in the item table, an even 2..8 steps
 * per launch, and registers budgeted for `ctas_per_sm` resident CTAs per SM (4 always; 6 and 8
 * for FP32 / FP16 storage with up to 4 mobile species); persistent == 0: one launch per lattice
 * and step (the other arguments are ignored); persistent == 2: the same with the flow step
 * through the staged kernels (bulk-copied tiles on even steps, the next node's gathers in flight
 * on odd steps; FP32 / FP64 flow storage). The persistent schedule needs one storage type for
 * flow and transport. clb_batch_get_schedule reports the same three values. */
clb_status clb_batch_schedule(clb_batch* batch, int persistent, int tile, int lag, int steps_per_launch,
                              int ctas_per_sm);
clb_status clb_batch_get_schedule(clb_batch* batch, int* persistent, int* tile, int* lag, int* steps_per_launch,
                                  int* ctas_per_sm);

/* Enqueue the batch's work on `stream` (a cudaStream_t; NULL: the batch's own stream). */
clb_status clb_batch_set_stream(clb_batch* batch, void* stream);

/* The limit of one dependency wait of the persistent schedule, in nanoseconds (default 2 s). A
 * wait that reaches it gives up: the launch skips its remaining items, the step returns
 * CLB_TIMEOUT and the domains' state is undefined; the device stays usable. */
clb_status clb_batch_set_wait_limit(clb_batch* batch, int64_t ns);

/* Open (collide / stream) nodes of the flow and species lattices over all domains. */
clb_status clb_batch_counts(clb_batch* batch, int64_t* flow_nodes, int64_t* transport_nodes);
clb_status clb_batch_destroy(clb_batch* batch);

/* ---------------------------------------------------------------- equilibrium speciation */

#define CLB_MAX_EQ_SPECIES 16
#define CLB_MAX_COMPONENTS 8

/* The <equilibrium> block of CompLaB.xml: tableau rows are the handle's species 0..n_species-1
 * (user order), columns the components (complab.cpp:614-723). */
typedef struct clb_speciation_desc {
    int32_t n_species, n_components;
    double stoich[CLB_MAX_EQ_SPECIES][CLB_MAX_COMPONENTS];
    double logK[CLB_MAX_EQ_SPECIES];
    int32_t component_species[CLB_MAX_COMPONENTS]; /* species that is each component, -1 none */
    double tolerance;             /* Newton-Raphson: |S^T c - T|_2 below this (absolute)      */
    int32_t max_iterations;
} clb_speciation_desc;

typedef enum clb_speciation_mode {
    CLB_SPEC_OFF = 0,
    CLB_SPEC_NR = 1,              /* FP64 Newton-Raphson in log10 concentration              */
    CLB_SPEC_MLP = 2,             /* trained surrogate only                                   */
    CLB_SPEC_MLP_NR = 3           /* surrogate, Newton-Raphson where the input is outside the
                                     trained range or the surrogate's residual check fails    */
} clb_speciation_mode;

typedef struct clb_speciation_stats {
    int64_t solves, converged, surrogate_used, fallbacks, iterations;
} clb_speciation_stats;

/* Replaces: EquilibriumChemistry configuration (complab.cpp:614-723). */
clb_status clb_speciation_setup(clb_handle* h, const clb_speciation_desc* desc);

/* Runs the speciation step inside every later clb_ade_step, after the kinetics and before the
 * stream, as run_equilibrium_biotic does (complab3d_processors_part4_eqsolver.hh:1393-1545:
 * x = 1..nx-2, mask neither solid nor wall, dC capped at max(1e-9, 0.1 |C|), floored at 1e-20). */
clb_status clb_set_speciation_mode(clb_handle* h, int mode);
clb_status clb_speciation_stats_get(clb_handle* h, clb_speciation_stats* out);

/* Solves n independent tableau problems: conc_in [n][n_species] (host), conc_out likewise,
 * iterations [n] (may be NULL). Replaces: EquilibriumChemistry::calculate_species_concentrations
 * (complab3d_processors_part4_eqsolver.hh:1195-1215), here by Newton-Raphson on the GPU. */
clb_status clb_speciation_solve(clb_handle* h, const double* conc_in, int n, double* conc_out, int* iterations);

/* ---------------------------------------------------------------- speciation surrogate */

/* The surrogate replaces the per-voxel Newton-Raphson solve: n_components log10 totals in, two
 * hidden layers of 64 tanh units, n_species log10 concentrations out, mapminmax scaling of
 * inputs and outputs (the recipe of the reference's FBA surrogate, complab3d_surrogate.hh:117-258
 * evalAll and :660-806 fitNetwork: Adam, held-out early stopping). Training data are Newton-
 * Raphson solves made on the GPU from species states with log10 c uniform in
 * [log_c_lo, log_c_hi]. Forward passes run on the tensor cores (BF16 operands, FP32 accumulate);
 * the backward pass and the Adam update are FP32. */
typedef struct clb_surrogate_train_desc {
    int32_t n_samples, epochs, batch, patience;
    double learning_rate, val_fraction;
    uint64_t seed;
    double log_c_lo[CLB_MAX_EQ_SPECIES], log_c_hi[CLB_MAX_EQ_SPECIES];
    int32_t source;               /* 0: states with log10 c uniform in [log_c_lo, log_c_hi];
                                     1: the species states of the domain's open voxels as they
                                     stand (the states the run itself generates), each species
                                     scaled by 10^u with u uniform in [-jitter, jitter]        */
    double jitter;
} clb_surrogate_train_desc;

typedef struct clb_surrogate_report {
    double train_mse, val_mse, seconds;  /* mean squared error on the scaled outputs            */
    int32_t epochs, steps, n_train, n_val;
} clb_surrogate_report;

clb_status clb_surrogate_train(clb_handle* h, const clb_surrogate_train_desc* desc, clb_surrogate_report* out);

/* How the speciation step uses the surrogate: its answer is used only when every scaled input
 * lies within 1 + range_margin of the trained range; it then starts newton_polish FP64
 * Newton-Raphson iterations (the surrogate's component concentrations are the initial point).
 * Mode CLB_SPEC_MLP keeps the polished answer; mode CLB_SPEC_MLP_NR keeps it only if its relative
 * mass-balance residual max_j |S^T c - T|_j / T_j is at most residual_tol and otherwise continues
 * Newton-Raphson from there (outside the trained range it starts Newton-Raphson afresh).
 * Defaults 0.02, 2 and 1e-6. */
clb_status clb_surrogate_set_check(clb_handle* h, double range_margin, int newton_polish, double residual_tol);

/* Surrogate speciation of n states ([n][n_species] host arrays), polished as above; accepted[n]
 * (may be NULL) reports the acceptance test (the convergence check when residual_check != 0). */
clb_status clb_surrogate_predict(clb_handle* h, const double* conc_in, int n, double* conc_out, int* accepted,
                                 int residual_check);

/* Parameter blob (clb_surrogate_param_count() floats: W1[64][16], b1[64], W2[64][64], b2[64],
 * W3[16][64], b3[16]) and the 64-float scaling block (input lo[16], hi[16], output lo[16],
 * hi[16]); either pointer pair may be NULL. Setting parameters makes the surrogate usable. */
clb_status clb_surrogate_params(clb_handle* h, float* params_out, const float* params_in, float* scaling_out,
                                const float* scaling_in);
int clb_surrogate_param_count(void);

/* Loss (sum of squared errors over the n x n_species scaled outputs) and its gradient with
 * respect to the parameter blob, for scaled inputs X[n][16] and targets Y[n][16], computed by
 * the training kernels themselves (gradient of the mean: the blob is scaled by 1/(n n_species)). */
clb_status clb_surrogate_gradient(clb_handle* h, const float* X, const float* Y, int n, float* grad, float* loss);

/* ---------------------------------------------------------------- fields */

clb_status clb_get_field(clb_handle* h, int field, int index, void* host, int dtype);
clb_status clb_set_field(clb_handle* h, int field, int index, const void* host, int dtype);

/* ---------------------------------------------------------------- checkpoints */

#define CLB_CKPT_FLOW 1        /* the flow lattice's incoming populations                        */
#define CLB_CKPT_TRANSPORT 2   /* every species (mobile: populations, immobile: concentration),
                                  the biomass fields and the advection velocity                  */

/* A restart file of the handle's lattices (`what`: CLB_CKPT_FLOW | CLB_CKPT_TRANSPORT) in FP64,
 * exact for every storage precision, with the step counters and the material map. Loading it
 * into a handle created on the same material map and set up the same way (clb_flow_init,
 * clb_ade_init, kinetics, biomass fields) continues the run exactly as the saved handle would.
 * Not for runs with the automaton or precipitation set up (their state is not in the file).
 * Replaces: saveBinaryBlock / loadBinaryBlock of the flow, substrate and biomass lattices
 * (complab.cpp:2004, 2292-2302; 1106-1108, 2044-2055). */
clb_status clb_checkpoint_save(clb_handle* h, const char* path, int what);
clb_status clb_checkpoint_load(clb_handle* h, const char* path);

/* ---------------------------------------------------------------- output */

/* One VTK ImageData file (.vti, XML, inline base64 binary, UInt64 headers) of a domain field over
 * the interior x-planes 1..nx-2, x fastest, spacing 1, as the reference's writers produce it:
 *   CLB_FIELD_FLOW_VELOCITY   "velocityNorm" + "velocity" (float32)  writeNsVTI
 *   CLB_FIELD_MATERIAL        "tag" (float32)                        writePorousMediumVTI
 *   CLB_FIELD_CONCENTRATION   "Density" of species `index` (float64) writeAdvVTI
 *   CLB_FIELD_BIOMASS         "Density" of microbe `index` (float64) writeAdvVTI
 * Replaces: complab_functions.hh:96-176 (the caller names the file, e.g. nameid + 7-digit
 * iteration + ".vti" as createFileName does). */
clb_status clb_write_vti(clb_handle* h, int field, int index, const char* path);

/* The writer itself, for host arrays: n_arrays point-data arrays, array a [components[a]][N] in
 * this library's layout (x slowest, N = nx ny nz), dtypes[a] 0 float64 or 1 float32 (written as
 * stored), cropped to x = 1..nx-2. */
clb_status clb_vti_write(const char* path, int nx, int ny, int nz, int n_arrays, const char* const* names,
                         const int32_t* components, const int32_t* dtypes, const void* const* data);

/* ---------------------------------------------------------------- run descriptions (CompLaB.xml) */

/* A parsed CompLaB.xml. Replaces: initialize_complab (complab_functions.hh:825-1602) for the
 * parameters of the reactive-transport path -- <path>, <LB_numerics> (domain, material numbers,
 * delta_P, Peclet, tau, iteration), <chemistry> (substrates, <immobile>), <microbiology>
 * (cellular-automaton microbes, maximum_biomass_density, thrd_biofilm_fraction, CA_method),
 * <equilibrium>, <precipitation> -- with the reference's element names, defaults and checks.
 * Errors (a missing required element, a malformed number, an unknown boundary type, ...) return
 * CLB_INVALID_ARG with the message in clb_case_error(). Rate laws are compiled code in the
 * reference (defineRxnKinetics); after clb_case_setup they are selected with clb_set_kinetics. */
typedef struct clb_case_s clb_case;
clb_status clb_case_load(const char* xml_path, clb_case** out);
clb_status clb_case_free(clb_case* c);
const char* clb_case_error(void);

/* A number of the run description by name: "nx" (ghost planes included), "ny", "nz", "dx" (m),
 * "char_length" (lattice units), "tau", "delta_P", "Peclet", "ns_max_iT1", "ns_max_iT2",
 * "ns_converge_iT1", "ns_converge_iT2", "ns_update_interval", "ade_update_interval", "ade_max_iT",
 * "n_substrates", "n_microbes", "substrate.<i>.{c0,d_pore,d_biofilm,left_type,right_type,left_bc,
 * right_bc,mobile}", "microbe.<m>.{code,perm_ratio}"; after clb_case_setup also the unit chain
 * "refNu", "refTau", "ade_dt" (s per iteration), "substrate.<i>.omega_pore" / "omega_biofilm", and
 * with flow "pore_mean_u", "delta_P_used", "flow_iterations", "flow_converged". */
clb_status clb_case_get(const clb_case* c, const char* key, double* value);

/* The set-up phases of the reference's main program (complab.cpp:1036-1290) on the current
 * device: the geometry file (<input_path>/<filename> beside the XML) with its ghost planes, the
 * handle, at Pe > 0 the flow solved to ns_converge_iT1 with the Peclet rescale and PoreMeanU
 * (complab.cpp:1093-1183), the unit chain refNu / refTau / ade_dt and every species' relaxation
 * rates (complab.cpp:1213-1253), the species lattices with the velocity coupled, the biomass fields
 * from initial_densities and the automaton, the equilibrium tableau (Newton-Raphson speciation in
 * every step), the precipitation phase. *out receives the handle (the caller destroys it). */
clb_status clb_case_setup(clb_case* c, int flow_precision, int ade_precision, clb_handle** out);

/* iterations (< 0: the description's ade_max_iT) coupled iterations through clb_run with the
 * description's schedule (ade/ns update intervals, ns_max_iT2 / ns_converge_iT2 re-solves, the
 * precipitation interval); with output_dir and save_VTK_interval > 0, one .vti file per substrate
 * every interval (<name>_<7-digit iteration>.vti, as writeAdvVTI names them). */
clb_status clb_case_run(clb_case* c, clb_handle* h, int iterations, const char* output_dir, clb_run_report* report);

/* ---------------------------------------------------------------- geometry (host) */

/* complab_geom::GenOptions (complab3d_geometry.hh:111-120). */
typedef struct clb_geom_options {
    const char* kind;             /* channel, spheres, cylinders, random, fracture, layered  */
    double porosity, radius, aperture, roughness;
    int32_t count, layers;
    uint64_t seed;
    const char* walls;            /* "y", "yz", "none", ...                                  */
} clb_geom_options;

/* complab_geom::generate (complab3d_geometry.hh:138-200): the same voxels for the same
 * options. Output in this library's layout (x slowest) of an nx*ny*nz grid. */
clb_status clb_geom_generate(const clb_geom_options* opt, int nx, int ny, int nz, int8_t* out);

/* Porosity-targeted sphere pack: spheres with radius uniform in [rmin, rmax] and centres
 * uniform in the box, drawn from the reference's xorshift64* stream, are carved as `grain`
 * until the open fraction reaches `porosity`; then walls (code `wall`) on the listed axes. */
clb_status clb_geom_sphere_pack(int nx, int ny, int nz, double porosity, double rmin, double rmax,
                                uint64_t seed, const char* walls, int grain, int wall, int pore,
                                int8_t* out);

/* readGeometry (complab_functions.hh:178-207): a .dat file of nx_inner slices (x slowest,
 * z fastest) into an (nx_inner+2)*ny*nz map whose ghost planes duplicate slices 1 and
 * nx_inner. */
clb_status clb_geom_read_dat(const char* path, int nx_inner, int ny, int nz, int8_t* out);

typedef struct clb_inspection {
    double porosity;
    int64_t open_voxels, isolated_voxels;
    int32_t clusters, spanning_clusters, percolates, quasi_2d;
} clb_inspection;

/* complab_geom::inspect (complab3d_geometry.hh:287-355) on a map in this library's layout:
 * open = code >= 2, 6-connected clusters, spanning = touches x=0 and x=nx-1. */
clb_status clb_geom_inspect(const int8_t* map, int nx, int ny, int nz, clb_inspection* out);

#ifdef __cplusplus
}
#endif

#endif /* CLB_H */

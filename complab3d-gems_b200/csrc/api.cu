// api.cu -- the extern "C" surface: handle lifetime, status reporting, field transfer.
#include "clb_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

// Every entry point that uses a handle runs on the handle's device, whatever the calling
// thread has current.
#define CLB_ON_DEVICE(h) cudaSetDevice((h)->device)

namespace clb {

static thread_local std::string g_global_err;

clb_status fail(clb_handle* h, clb_status s, const std::string& msg) {
    if (h) h->err = msg;
    else g_global_err = msg;
    return s;
}

clb_status cuda_check(clb_handle* h, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CLB_OK;
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(h, e == cudaErrorMemoryAllocation ? CLB_OUT_OF_MEMORY : CLB_CUDA_ERROR, m);
}

// The host copy of the material map follows the device's lazily: a mask pass of the automaton that
// changes voxels marks it stale, and the readers of h_mat refresh it here first, so the automaton
// moves no map to the host in iterations where nobody reads it.
clb_status host_mat_sync(clb_handle* h) {
    if (!h->h_mat_stale) return CLB_OK;
    cudaError_t e = cudaMemcpy(h->h_mat.data(), h->d_mat, (size_t)h->g.N, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_check(h, e, "material copy");
    h->h_mat_stale = false;
    return CLB_OK;
}

// Compacted list of nodes whose class (by material code) is nonzero, in lexicographic order.
std::vector<int32_t> build_list(const clb_handle* h, const int8_t* cls_by_code) {
    std::vector<int32_t> list;
    list.reserve((size_t)h->g.N / 2);
    for (int64_t n = 0; n < h->g.N; ++n)
        if (cls_by_code[(uint8_t)h->h_mat[n] & 127]) list.push_back((int32_t)n);
    return list;
}

}  // namespace clb

using namespace clb;

extern "C" {

const char* clb_last_error(const clb_handle* h) { return h ? h->err.c_str() : g_global_err.c_str(); }
const char* clb_global_error(void) { return g_global_err.c_str(); }

clb_status clb_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, CLB_CUDA_ERROR, std::string("set device: ") + cudaGetErrorString(e));
    return CLB_OK;
}

clb_status clb_create(const clb_domain_desc* desc, const int8_t* material, clb_handle** out) {
    if (!desc || !material || !out) return fail(nullptr, CLB_INVALID_ARG, "null argument");
    *out = nullptr;
    if (desc->nx < 3 || desc->ny < 1 || desc->nz < 1) return fail(nullptr, CLB_INVALID_ARG, "domain too small");
    const int64_t N = (int64_t)desc->nx * desc->ny * desc->nz;
    if (N > (int64_t)INT32_MAX / 2) return fail(nullptr, CLB_INVALID_ARG, "domain exceeds 2^30 voxels");
    if (!(desc->tau > 0.5)) return fail(nullptr, CLB_INVALID_ARG, "tau must exceed 1/2");
    if (desc->n_microbes < 0 || desc->n_microbes > CLB_MAX_MICROBES)
        return fail(nullptr, CLB_INVALID_ARG, "microbe count out of range");
    {
        // any negative code sets the sign bit of the OR (a branch-free pass the compiler vectorises)
        uint8_t acc = 0;
        const uint8_t* m = reinterpret_cast<const uint8_t*>(material);
        for (int64_t n = 0; n < N; ++n) acc |= m[n];
        if (acc & 0x80u) return fail(nullptr, CLB_INVALID_ARG, "negative material code");
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(nullptr, CLB_CUDA_ERROR, "no CUDA device");
    clb_handle* h = new (std::nothrow) clb_handle_s();
    if (!h) return fail(nullptr, CLB_OUT_OF_MEMORY, "host allocation");
    h->d = *desc;
    h->device = dev;
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev);
    h->g.nx = desc->nx;
    h->g.ny = desc->ny;
    h->g.nz = desc->nz;
    h->g.N = N;
    h->g.plane = desc->ny * desc->nz;
    h->h_mat.assign(material, material + N);
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_mat, N);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_mat, material, N, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        std::string m = std::string("create: ") + cudaGetErrorString(e);
        if (h->d_mat) cudaFree(h->d_mat);
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return fail(nullptr, CLB_CUDA_ERROR, m);
    }
    *out = h;
    return CLB_OK;
}

clb_status clb_destroy(clb_handle* h) {
    if (!h) return CLB_OK;
    cudaStreamSynchronize(h->stream);
    flow_free(h);
    ade_free(h);
    cudaFree(h->d_mat);
    cudaFree(h->d_mat_flow);
    cudaFree(h->d_err);
    cudaFree(h->d_spec_stats);
    cudaFree(h->d_mlp);
    cudaFree(h->d_mlp_bf16);
    cudaFree(h->d_sym);
    cudaFree(h->d_gnn);
    delete[] h->gnn_host;
    cudaFree(h->d_srg);
    delete[] h->srg_host;
    if (h->h_flags) cudaFreeHost(h->h_flags);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return CLB_OK;
}

clb_status clb_synchronize(clb_handle* h) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    clb_status s = cuda_check(h, cudaStreamSynchronize(h->stream), "synchronize");
    if (s != CLB_OK) return s;
    if (!h->d_err) return ade_nonfinite_check(h);
    int flag = 0;
    cudaMemcpy(&flag, h->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (flag) return fail(h, CLB_TIMEOUT, "a bounded device wait gave up (bulk copy did not complete)");
    return ade_nonfinite_check(h);
}

clb_status clb_set_stream(clb_handle* h, void* stream) {
    if (!h || !stream) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_check(h, e, "set stream");
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return CLB_OK;
}

clb_status clb_get_stream(clb_handle* h, void** stream) {
    if (!h || !stream) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    *stream = (void*)h->stream;
    return CLB_OK;
}

clb_status clb_tune(clb_handle* h, const char* key, int value) {
    if (!h || !key) return fail(h, CLB_INVALID_ARG, "null argument");
    const std::string k = key;
    if (k == "flow_even_tma") { h->flow_even_tma = value ? 1 : 0; return CLB_OK; }
    if (k == "ade_pipe") { h->ade_pipe = value ? 1 : 0; return CLB_OK; }
    if (k == "flow_odd_pipe") {
        if (value && h->flow_ready && !h->flow_pipe_grid)
            return fail(h, CLB_INVALID_ARG, "flow_odd_pipe needs 4- or 8-byte flow storage");
        h->flow_odd_pipe = value ? 1 : 0;
        return CLB_OK;
    }
    if (k == "flow_min_blocks") {
        if (value != 2 && value != 3) return fail(h, CLB_INVALID_ARG, "flow_min_blocks is 2 or 3");
        h->flow_minb = value;
        return CLB_OK;
    }
    return fail(h, CLB_INVALID_ARG, "unknown tuning key '" + k + "'");
}

clb_status clb_autotune(clb_handle* h, int steps, char* report, int report_len) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    return flow_autotune(h, steps, report, report_len);
}

clb_status clb_flow_init(clb_handle* h, double delta_p) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (!std::isfinite(delta_p)) return fail(h, CLB_INVALID_ARG, "delta_p not finite");
    return flow_init(h, delta_p);
}

clb_status clb_flow_step(clb_handle* h, int n) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    if (n < 0) return fail(h, CLB_INVALID_ARG, "negative step count");
    return flow_step(h, n, false, 0.0);
}

clb_status clb_flow_solve(clb_handle* h, int max_it, double eps, int* iterations) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    if (max_it < 0 || !(eps > 0)) return fail(h, CLB_INVALID_ARG, "bad solve arguments");
    clb_status s = flow_solve(h, max_it, eps, iterations);
    if (s == CLB_NOT_CONVERGED) h->err = "flow did not converge within the iteration cap";
    return s;  // CLB_NONFINITE: diverged; CLB_PERCOLATION_LOST: no outlet flow at the cap
}

clb_status clb_flow_stats_get(clb_handle* h, double char_length, clb_flow_stats* out) {
    if (!h || !out) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    return flow_stats(h, char_length, out);
}

clb_status clb_flow_solve_peclet(clb_handle* h, double peclet, double char_length, double tau_ade_fixed, int max_it,
                                 double eps, double* delta_p_out, int* iterations) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    int it1 = 0, it2 = 0;
    clb_status s = flow_solve(h, max_it, eps, &it1);
    if (s != CLB_OK && s != CLB_NOT_CONVERGED) return s;
    clb_flow_stats st;
    clb_status s2 = flow_stats(h, char_length, &st);
    if (s2 != CLB_OK) return s2;
    const double nu = (h->d.tau - 0.5) / 3.0;
    const double d_fixed = 0.25 * (tau_ade_fixed - 0.5);
    const double u_target = peclet * d_fixed / char_length;
    if (!(st.permeability > 0)) return fail(h, CLB_PERCOLATION_LOST, "zero permeability: no flow path");
    const double dp_new = u_target * nu * char_length / st.permeability;
    if (std::fabs(dp_new - h->delta_p) / h->delta_p > 0.01) {
        s2 = flow_init(h, dp_new);
        if (s2 != CLB_OK) return s2;
        s = flow_solve(h, max_it, eps, &it2);
        if (s != CLB_OK && s != CLB_NOT_CONVERGED) return s;
    }
    if (delta_p_out) *delta_p_out = h->delta_p;
    if (iterations) *iterations = it1 + it2;
    if (s == CLB_NOT_CONVERGED) h->err = "flow did not converge within the iteration cap";
    return s;
}

clb_status clb_ade_init(clb_handle* h, const clb_species_desc* species, int n_species) {
    if (!h || !species) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    for (int s = 0; s < n_species; ++s) {
        const clb_species_desc& sp = species[s];
        if (sp.mobile && (!(sp.omega_pore > 0 && sp.omega_pore < 2) || !(sp.omega_biofilm > 0 && sp.omega_biofilm < 2)))
            return fail(h, CLB_INVALID_ARG, "species omega outside (0, 2)");
        if (sp.left_type < 0 || sp.left_type > 2 || sp.right_type < 0 || sp.right_type > 2)
            return fail(h, CLB_INVALID_ARG, "unknown face type");
    }
    return ade_init(h, species, n_species);
}

clb_status clb_couple_velocity(clb_handle* h) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return ade_couple(h);
}

clb_status clb_set_kinetics(clb_handle* h, int law, const double* params, int n_params, double dt) {
    if (!h || (n_params > 0 && !params)) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return ade_set_kinetics(h, law, params, n_params, dt);
}

clb_status clb_set_thermo_gate(clb_handle* h, const clb_thermo_desc* desc) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return ade_set_thermo(h, desc);
}

clb_status clb_set_biomass(clb_handle* h, int n_microbes, const double* biomass) {
    if (!h || (n_microbes > 0 && !biomass)) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return ade_set_biomass(h, n_microbes, biomass);
}

clb_status clb_set_symbolic_kinetics(clb_handle* h, const char* sym_path, const char* const* species_names,
                                     int microbe, const char* microbe_name) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return symbolic_set(h, sym_path, species_names, microbe, microbe_name);
}

clb_status clb_symbolic_eval(clb_handle* h, int microbe, const double* vars, int n, double* rates, int* n_rates) {
    if (!h || (n > 0 && (!vars || !rates))) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return symbolic_eval(h, microbe, vars, n, rates, n_rates);
}

clb_status clb_set_graph_network(clb_handle* h, const char* gnn_path, const char* const* species_names,
                                 int microbe) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return graphnet_set(h, gnn_path, species_names, microbe);
}

clb_status clb_graph_network_eval(clb_handle* h, int microbe, const double* conc, int n, double* out, int* n_out,
                                  long* n_clamped) {
    if (!h || (n > 0 && (!conc || !out))) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return graphnet_eval(h, microbe, conc, n, out, n_out, n_clamped);
}

clb_status clb_set_surrogate_organism(clb_handle* h, const char* srg_path, const char* const* species_names,
                                      int microbe, const clb_surrogate_desc* desc) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return srg_set(h, srg_path, species_names, microbe, desc);
}

clb_status clb_surrogate_eval(clb_handle* h, int microbe, const double* x, int n, double* out, int* n_out,
                              long* n_clamped) {
    if (!h || (n > 0 && (!x || !out))) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return srg_eval_host(h, microbe, x, n, out, n_out, n_clamped);
}

clb_status clb_ade_step(clb_handle* h, int n) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (n < 0) return fail(h, CLB_INVALID_ARG, "negative step count");
    return ade_step(h, n);
}

clb_status clb_reduce(clb_handle* h, clb_stats* out) {
    if (!h || !out) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return ade_reduce(h, out);
}

clb_status clb_set_abiotic_kinetics(clb_handle* h, int law, const double* params, int n_params, int surface_only) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    if (n_params > 0 && !params) return fail(h, CLB_INVALID_ARG, "null parameters");
    CLB_ON_DEVICE(h);
    return ade_set_abiotic(h, law, params, n_params, surface_only);
}

clb_status clb_precip_setup(clb_handle* h, const clb_precip_desc* desc) {
    if (!h || !desc) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return precip_setup(h, desc);
}

clb_status clb_geometry_update(clb_handle* h, int* sealed, int* reopened) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return geometry_update(h, sealed, reopened);
}

clb_status clb_ca_setup(clb_handle* h, const clb_ca_desc* desc) {
    if (!h || !desc) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return ca_setup(h, desc);
}

clb_status clb_ca_step(clb_handle* h, int* sweeps, int* mask_changed) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return ca_step(h, sweeps, mask_changed);
}

clb_status clb_refresh_dynamics(clb_handle* h, int species, int flow) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    return refresh_dynamics(h, species, flow);
}

clb_status clb_run(clb_handle* h, const clb_run_desc* d, clb_run_report* report) {
    if (!h || !d) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    clb_run_report local;
    return run(h, d, report ? report : &local);
}

clb_status clb_batch_create(clb_handle* const* handles, int n, clb_batch** out) {
    if (!handles || !out) return fail(nullptr, CLB_INVALID_ARG, "null argument");
    *out = nullptr;
    return batch_create(handles, n, out);
}

clb_status clb_batch_step(clb_batch* batch, int n, int flow, int transport) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_step(batch, n, flow, transport);
}

clb_status clb_batch_autotune(clb_batch* batch, int steps, char* report, int report_len) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_autotune(batch, steps, report, report_len);
}

clb_status clb_batch_counts(clb_batch* batch, int64_t* flow_nodes, int64_t* transport_nodes) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_counts(batch, flow_nodes, transport_nodes);
}

clb_status clb_batch_schedule(clb_batch* batch, int persistent, int tile, int lag, int steps_per_launch,
                              int ctas_per_sm) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_schedule(batch, persistent, tile, lag, steps_per_launch, ctas_per_sm);
}

clb_status clb_batch_get_schedule(clb_batch* batch, int* persistent, int* tile, int* lag, int* steps_per_launch,
                                  int* ctas_per_sm) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_get_schedule(batch, persistent, tile, lag, steps_per_launch, ctas_per_sm);
}

clb_status clb_batch_set_wait_limit(clb_batch* batch, int64_t ns) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_set_wait_limit(batch, ns);
}

clb_status clb_batch_set_stream(clb_batch* batch, void* stream) {
    if (!batch) return fail(nullptr, CLB_INVALID_ARG, "null batch");
    return batch_set_stream(batch, stream);
}

clb_status clb_batch_destroy(clb_batch* batch) { return batch_destroy(batch); }

clb_status clb_reduce_noalloc(clb_handle* h, clb_stats* out) {
    if (!h || !out) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return ade_reduce_noalloc(h, out);
}

clb_status clb_speciation_setup(clb_handle* h, const clb_speciation_desc* desc) {
    if (!h || !desc) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return speciation_setup(h, desc);
}

clb_status clb_set_speciation_mode(clb_handle* h, int mode) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    if (mode < CLB_SPEC_OFF || mode > CLB_SPEC_MLP_NR) return fail(h, CLB_INVALID_ARG, "unknown speciation mode");
    if (mode != CLB_SPEC_OFF && !h->spec_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_speciation_setup first");
    if ((mode == CLB_SPEC_MLP || mode == CLB_SPEC_MLP_NR) && !h->mlp_ready)
        return fail(h, CLB_NOT_INITIALIZED, "train or load the surrogate first");
    h->spec_mode = mode;
    return CLB_OK;
}

clb_status clb_speciation_stats_get(clb_handle* h, clb_speciation_stats* out) {
    if (!h || !out) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return speciation_stats(h, out);
}

clb_status clb_speciation_solve(clb_handle* h, const double* conc_in, int n, double* conc_out, int* iterations) {
    if (!h || (n > 0 && (!conc_in || !conc_out))) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return speciation_solve(h, conc_in, n, conc_out, iterations);
}

clb_status clb_surrogate_train(clb_handle* h, const clb_surrogate_train_desc* desc, clb_surrogate_report* out) {
    if (!h || !desc) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return surrogate_train(h, desc, out);
}

clb_status clb_surrogate_set_check(clb_handle* h, double range_margin, int newton_polish, double residual_tol) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    if (!(range_margin >= 0) || newton_polish < 0 || newton_polish > 50 || !(residual_tol > 0))
        return fail(h, CLB_INVALID_ARG, "bad acceptance settings");
    h->mlp_margin = (float)range_margin;
    h->mlp_polish = newton_polish;
    h->mlp_resid_tol = (float)residual_tol;
    return CLB_OK;
}

clb_status clb_surrogate_predict(clb_handle* h, const double* conc_in, int n, double* conc_out, int* accepted,
                                 int residual_check) {
    if (!h || (n > 0 && (!conc_in || !conc_out))) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    return surrogate_predict(h, conc_in, n, conc_out, accepted, residual_check);
}

clb_status clb_surrogate_params(clb_handle* h, float* params_out, const float* params_in, float* scaling_out,
                                const float* scaling_in) {
    if (!h) return fail(nullptr, CLB_INVALID_ARG, "null handle");
    CLB_ON_DEVICE(h);
    if (!h->spec_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_speciation_setup first");
    return surrogate_params(h, params_out, params_in, scaling_out, scaling_in);
}

int clb_surrogate_param_count(void) { return surrogate_param_count(); }

clb_status clb_surrogate_gradient(clb_handle* h, const float* X, const float* Y, int n, float* grad, float* loss) {
    if (!h || !X || !Y || !grad || !loss || n < 1) return fail(h, CLB_INVALID_ARG, "bad arguments");
    CLB_ON_DEVICE(h);
    return surrogate_gradient(h, X, Y, n, grad, loss);
}

clb_status clb_get_field(clb_handle* h, int field, int index, void* host, int dtype) {
    if (!h || !host) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    const size_t N = (size_t)h->g.N;
    if (field == CLB_FIELD_MATERIAL) {
        if (dtype != 2) return fail(h, CLB_INVALID_ARG, "material is int8");
        clb_status st = host_mat_sync(h);
        if (st != CLB_OK) return st;
        std::memcpy(host, h->h_mat.data(), N);
        return CLB_OK;
    }
    if (field == CLB_FIELD_FLOW_VELOCITY) {
        if (dtype != 0 && dtype != 1) return fail(h, CLB_INVALID_ARG, "the flow velocity is read as float64 or float32");
        if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
        return flow_velocity(h, host, dtype, true);
    }
    if (dtype != 0) return fail(h, CLB_INVALID_ARG, "fields are read as float64");
    switch (field) {
        case CLB_FIELD_FLOW_POPULATIONS:
            if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
            return flow_populations(h, (double*)host);
        case CLB_FIELD_CONCENTRATION: return ade_density(h, index, (double*)host);
        case CLB_FIELD_ADE_POPULATIONS: return ade_populations(h, index, (double*)host);
        case CLB_FIELD_BIOMASS: return ade_biomass(h, index, (double*)host);
        case CLB_FIELD_ADE_VELOCITY: return ade_velocity(h, (double*)host);
        case CLB_FIELD_CA_TOTAL: return ca_fields(h, 0, (double*)host);
        case CLB_FIELD_CA_AGE: return ca_fields(h, 1, (double*)host);
        default: return fail(h, CLB_INVALID_ARG, "unknown field");
    }
}

clb_status clb_set_field(clb_handle* h, int field, int index, const void* host, int dtype) {
    if (!h || !host) return fail(h, CLB_INVALID_ARG, "null argument");
    CLB_ON_DEVICE(h);
    if (dtype != 0) return fail(h, CLB_INVALID_ARG, "fields are written as float64");
    switch (field) {
        case CLB_FIELD_FLOW_POPULATIONS:
            if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
            return flow_set_populations(h, (const double*)host);
        case CLB_FIELD_ADE_POPULATIONS: return ade_set_populations(h, index, (const double*)host);
        case CLB_FIELD_CONCENTRATION: return ade_set_concentration(h, index, (const double*)host);
        case CLB_FIELD_ADE_VELOCITY: return ade_set_velocity(h, (const double*)host);
        case CLB_FIELD_BIOMASS: return ade_set_biomass_field(h, index, (const double*)host);
        default: return fail(h, CLB_INVALID_ARG, "field is read-only");
    }
}

}  // extern "C"

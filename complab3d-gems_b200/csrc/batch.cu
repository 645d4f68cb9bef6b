// batch.cu -- an ensemble of independent domains (a parameter sweep) advanced together: one
// launch per lattice and step covers the nodes of every domain, and pairs of steps are replayed
// from a captured CUDA graph, so a sweep of many small uneven domains is not bound by launch
// overhead. Each domain keeps its own handle, layout and parameters; the batched kernels run the
// very same per-node code as the single-domain steps, so a batched run matches stepping each
// domain on its own bit for bit.
#include "batch.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>

struct clb_batch_s {
    std::vector<clb_handle*> hs;
    int device = 0, num_sms = 148;
    cudaStream_t stream = nullptr;
    int flow_prec = 0, ade_prec = 0, nm = 1;
    bool has_flow = false, has_ade = false;
    clb::BatchDomain* d_dom = nullptr;
    int64_t *d_foff = nullptr, *d_aoff = nullptr, *d_joff = nullptr;
    clb::NeumannJob* d_jobs = nullptr;
    clb::BatchView view{};
    int64_t flow_nodes = 0, ade_nodes = 0;
    int flow_threads = 256, flow_mult = 4, ade_mult = 1, neu_grid = 148;
    std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;  // (flow parity, ade parity, flow, ade)
    std::string err;
};

namespace clb {

static clb_status bfail(clb_batch* b, clb_status s, const std::string& msg) {
    if (b) b->err = msg;
    return fail(nullptr, s, msg);
}

static void drop_graphs(clb_batch* b) {
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

static void batch_free(clb_batch* b) {
    drop_graphs(b);
    cudaFree(b->d_dom);
    cudaFree(b->d_foff);
    cudaFree(b->d_aoff);
    cudaFree(b->d_jobs);
    cudaFree(b->d_joff);
    if (b->stream) cudaStreamDestroy(b->stream);
}

clb_status batch_create(clb_handle* const* hs, int n, clb_batch** out) {
    if (n < 1 || n > BATCH_MAX_DOMAINS) return fail(nullptr, CLB_INVALID_ARG, "batch size out of range");
    clb_batch* b = new clb_batch_s();
    b->hs.assign(hs, hs + n);
    clb_handle* h0 = hs[0];
    b->device = h0->device;
    b->num_sms = h0->num_sms;
    b->has_flow = h0->flow_ready;
    b->has_ade = h0->ade_ready;
    b->flow_prec = h0->flow_prec;
    b->ade_prec = h0->ade_prec;
    for (int i = 0; i < n; ++i) {
        clb_handle* h = hs[i];
        if (!h) { delete b; return fail(nullptr, CLB_INVALID_ARG, "null handle in batch"); }
        if (h->device != b->device) { delete b; return fail(nullptr, CLB_INVALID_ARG, "batch handles must share a device"); }
        if (h->flow_ready != b->has_flow || h->ade_ready != b->has_ade) {
            delete b;
            return fail(nullptr, CLB_INVALID_ARG, "batch handles must all have (or all lack) flow and transport");
        }
        if ((b->has_flow && h->flow_prec != b->flow_prec) || (b->has_ade && h->ade_prec != b->ade_prec)) {
            delete b;
            return fail(nullptr, CLB_INVALID_ARG, "batch handles must share their storage precisions");
        }
        if (b->has_ade && (h->ap.law2 != CLB_LAW_NONE || h->ap.dis_on || h->ap.gate_on || h->ap.law == CLB_LAW_SYMBOLIC ||
                           h->spec_mode != CLB_SPEC_OFF)) {
            delete b;
            return fail(nullptr, CLB_INVALID_ARG,
                        "batched transport has no abiotic law, dissolution, thermodynamic gate or speciation");
        }
        if (b->has_ade && h->M > 0 && !h->d_bio) { delete b; return fail(nullptr, CLB_INVALID_ARG, "biomass missing"); }
        if (b->has_ade) b->nm = std::max(b->nm, h->S);
    }
    if (!b->has_flow && !b->has_ade) { delete b; return fail(nullptr, CLB_INVALID_ARG, "nothing to step in the batch"); }
    cudaSetDevice(b->device);
    std::vector<BatchDomain> dom((size_t)n);
    std::vector<int64_t> foff((size_t)n + 1, 0), aoff((size_t)n + 1, 0), joff(1, 0);
    std::vector<NeumannJob> jobs;
    for (int i = 0; i < n; ++i) {
        clb_handle* h = hs[i];
        BatchDomain& d = dom[(size_t)i];
        std::memset(&d, 0, sizeof d);
        if (b->has_flow) {
            d.f = h->d_f;
            d.flink = h->d_flink;
            d.fs = view_of(h->flow_sp);
            d.fkw = h->k_west_end;
            d.fke = h->k_east_begin;
            d.fp = h->fp;
            foff[(size_t)i + 1] = foff[(size_t)i] + h->flow_sp.K;
        }
        if (b->has_ade) {
            d.g = h->d_g;
            d.glink = h->d_glink;
            d.as = view_of(h->ade_sp);
            d.akw = h->ade_west_end;
            d.ake = h->ade_east_begin;
            d.ap = h->ap;
            d.imm = h->d_imm;
            d.bio = h->d_bio;
            d.u = h->d_u;
            d.neu = h->d_neu;
            d.mob = (const int*)(h->d_neu + (size_t)h->S * 2 * h->g.plane);  // the mobile-species table
            d.mat = h->d_mat;
            d.n_mobile = h->n_mobile;
            aoff[(size_t)i + 1] = aoff[(size_t)i] + h->ade_sp.K;
            for (int s = 0; s < h->S; ++s) {
                const int m = h->ap.slot[s];
                if (m < 0) continue;
                for (int side = 0; side < 2; ++side) {
                    if ((side == 0 ? h->ap.ltype[s] : h->ap.rtype[s]) != CLB_NEUMANN) continue;
                    jobs.push_back({i, s, m, side});
                    joff.push_back(joff.back() + h->g.plane);
                }
            }
        }
    }
    b->flow_nodes = foff.back();
    b->ade_nodes = aoff.back();
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_dom, sizeof(BatchDomain) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_foff, sizeof(int64_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_aoff, sizeof(int64_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs, sizeof(NeumannJob) * std::max<size_t>(1, jobs.size()));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_joff, sizeof(int64_t) * joff.size());
    if (e == cudaSuccess) e = cudaMemcpy(b->d_dom, dom.data(), sizeof(BatchDomain) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_foff, foff.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_aoff, aoff.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !jobs.empty())
        e = cudaMemcpy(b->d_jobs, jobs.data(), sizeof(NeumannJob) * jobs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_joff, joff.data(), sizeof(int64_t) * joff.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        batch_free(b);
        delete b;
        return fail(nullptr, CLB_CUDA_ERROR, std::string("batch set-up: ") + cudaGetErrorString(e));
    }
    b->view.dom = b->d_dom;
    b->view.foff = b->d_foff;
    b->view.aoff = b->d_aoff;
    b->view.ndom = n;
    b->view.jobs = b->d_jobs;
    b->view.joff = b->d_joff;
    b->view.njobs = (int)jobs.size();
    b->neu_grid = std::max<int64_t>(1, std::min<int64_t>((joff.back() + 255) / 256, b->num_sms * 4));
    *out = b;
    return CLB_OK;
}

// one step of the requested lattices at the given parities, on the batch stream
static void batch_launch_step(clb_batch* b, int fodd, int aodd, bool flow, bool ade) {
    if (flow) {
        const int grid = b->num_sms * b->flow_mult;
        launch_flow_batch(b->view, b->flow_prec, fodd != 0, grid, b->flow_threads, b->stream);
    }
    if (ade) {
        launch_neumann_batch(b->view, b->ade_prec, aodd != 0, b->neu_grid, b->stream);
        launch_ade_batch(b->view, b->ade_prec, aodd != 0, b->nm, b->ade_mult, b->num_sms, b->stream);
    }
}

// bring each handle's counters (and the flow tracer's) up to date after n batched steps
static clb_status batch_commit(clb_batch* b, int n, bool flow, bool ade) {
    for (clb_handle* h : b->hs) {
        if (flow) {
            h->flow_iters += n;
            if (h->d_tracer)
                cudaMemcpyAsync(&h->d_tracer->iterations, &h->flow_iters, sizeof(int64_t), cudaMemcpyHostToDevice, b->stream);
        }
        if (ade) {
            h->ade_iters += n;
            h->neu_iter = -1;
        }
    }
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch step: ") + cudaGetErrorString(e));
    return CLB_OK;
}

clb_status batch_step(clb_batch* b, int n, int flow_on, int ade_on) {
    if (n < 0) return bfail(b, CLB_INVALID_ARG, "negative step count");
    const bool flow = flow_on && b->has_flow, ade = ade_on && b->has_ade;
    if (!flow && !ade) return bfail(b, CLB_INVALID_ARG, "nothing to step");
    cudaSetDevice(b->device);
    const int fodd = (int)(b->hs[0]->flow_iters & 1), aodd = (int)(b->hs[0]->ade_iters & 1);
    for (clb_handle* h : b->hs) {
        if ((flow && (int)(h->flow_iters & 1) != fodd) || (ade && (int)(h->ade_iters & 1) != aodd))
            return bfail(b, CLB_INVALID_ARG, "batched domains must be at the same step parity");
        cudaError_t e = cudaStreamSynchronize(h->stream);  // their own pending work first
        if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch step: ") + cudaGetErrorString(e));
    }
    int done = 0;
    if (n >= 4) {
        const auto key = std::make_tuple(fodd, aodd, (int)flow, (int)ade);
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            // two direct steps first: every kernel variant is set up before the capture
            batch_launch_step(b, fodd, aodd, flow, ade);
            batch_launch_step(b, fodd ^ 1, aodd ^ 1, flow, ade);
            done = 2;
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                batch_launch_step(b, fodd, aodd, flow, ade);
                batch_launch_step(b, fodd ^ 1, aodd ^ 1, flow, ade);
                e = cudaStreamEndCapture(b->stream, &graph);
            }
            cudaGraphExec_t exec = nullptr;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch graph: ") + cudaGetErrorString(e));
            it = b->graphs.emplace(key, exec).first;
        }
        for (; done + 2 <= n; done += 2) {
            cudaError_t e = cudaGraphLaunch(it->second, b->stream);
            if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch graph: ") + cudaGetErrorString(e));
        }
    }
    for (; done < n; ++done) batch_launch_step(b, fodd ^ (done & 1), aodd ^ (done & 1), flow, ade);
    return batch_commit(b, n, flow, ade);
}

// Times the launch shapes of the batched steps and keeps the fastest: flow with 128 or 256
// threads per block and 2, 4 or 8 blocks per SM, transport with 1 or 2 times the resident grid.
// Every timed step is a real step of the domains: their iteration counters show the advance.
clb_status batch_autotune(clb_batch* b, int steps, char* report, int report_len) {
    cudaSetDevice(b->device);
    steps = std::max(2, steps + (steps & 1));
    int taken = 0;
    std::string rep;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto time_steps = [&](bool flow, bool ade) {
        const int fodd = (int)((b->hs[0]->flow_iters + taken) & 1), aodd = (int)((b->hs[0]->ade_iters + taken) & 1);
        batch_launch_step(b, fodd, aodd, flow, ade);  // set-up outside the timing
        batch_launch_step(b, fodd ^ 1, aodd ^ 1, flow, ade);
        cudaEventRecord(e0, b->stream);
        for (int s = 0; s < steps; ++s) batch_launch_step(b, fodd ^ (s & 1), aodd ^ (s & 1), flow, ade);
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        taken += steps + 2;
        return ms / steps;
    };
    for (clb_handle* h : b->hs) cudaStreamSynchronize(h->stream);
    if (b->has_flow) {
        float best = 1e30f;
        int bt = 256, bm = 4;
        for (int threads : {128, 256})
            for (int mult : {2, 4, 8}) {
                b->flow_threads = threads;
                b->flow_mult = mult * (256 / threads);
                const float ms = time_steps(true, false);
                char buf[96];
                std::snprintf(buf, sizeof buf, "flow %dx%d:%.1fus ", threads, b->flow_mult, ms * 1e3f);
                rep += buf;
                if (ms < best) { best = ms; bt = threads; bm = b->flow_mult; }
            }
        b->flow_threads = bt;
        b->flow_mult = bm;
        // the flow counters advanced by the timed steps
        for (clb_handle* h : b->hs) h->flow_iters += taken;
        taken = 0;
    }
    if (b->has_ade) {
        float best = 1e30f;
        int bm = 1;
        for (int mult : {1, 2}) {
            b->ade_mult = mult;
            const float ms = time_steps(false, true);
            char buf[96];
            std::snprintf(buf, sizeof buf, "transport x%d:%.1fus ", mult, ms * 1e3f);
            rep += buf;
            if (ms < best) { best = ms; bm = mult; }
        }
        b->ade_mult = bm;
        for (clb_handle* h : b->hs) { h->ade_iters += taken; h->neu_iter = -1; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs(b);
    for (clb_handle* h : b->hs)
        if (b->has_flow && h->d_tracer)
            cudaMemcpyAsync(&h->d_tracer->iterations, &h->flow_iters, sizeof(int64_t), cudaMemcpyHostToDevice, b->stream);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (report && report_len > 0) {
        std::strncpy(report, rep.c_str(), (size_t)report_len - 1);
        report[report_len - 1] = 0;
    }
    if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch autotune: ") + cudaGetErrorString(e));
    return CLB_OK;
}

clb_status batch_destroy(clb_batch* b) {
    if (!b) return CLB_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    batch_free(b);
    delete b;
    return CLB_OK;
}

clb_status batch_counts(clb_batch* b, int64_t* flow_nodes, int64_t* ade_nodes) {
    if (flow_nodes) *flow_nodes = b->flow_nodes;
    if (ade_nodes) *ade_nodes = b->ade_nodes;
    return CLB_OK;
}

}  // namespace clb

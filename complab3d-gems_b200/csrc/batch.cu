// batch.cu -- an ensemble of independent domains (a parameter sweep) advanced together, on one
// of two schedules:
//   persistent: one launch runs several steps of every lattice of every domain, walking a table
//     of (step, domain, lattice, tile) items with per-domain dependencies (ade.cu,
//     k_batch_persistent); the launches are replayed from a captured CUDA graph;
//   per lattice: one launch per lattice and step covers the nodes of every domain, pairs of steps
//     replayed from a captured CUDA graph.
// The autotuner times both (tile size, lag and steps per launch of the persistent schedule, block
// shapes of the other) and keeps the fastest. Each domain keeps its own handle, layout and
// parameters; the batched kernels run the very same per-node code as the single-domain steps, so
// a batched run matches stepping each domain on its own bit for bit, whatever the schedule.
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
    int64_t *d_foff = nullptr, *d_aoff = nullptr, *d_joff = nullptr, *d_face_off = nullptr;
    clb::NeumannJob* d_jobs = nullptr;
    clb::BatchTile *d_ftiles = nullptr, *d_atiles = nullptr;
    clb::NeumannFace* d_faces = nullptr;
    clb::BatchView view{};
    int64_t flow_nodes = 0, ade_nodes = 0;
    int flow_threads = 256, flow_mult = 4, ade_mult = 1, ade_resident = 4, neu_grid = 148;
    bool flow_staged = false;  // the flow step through the staged kernels (4- and 8-byte storage)
    // graphs by (flow parity, ade parity, flow, ade, steps per launch (0: per lattice), tile, lag)
    std::map<std::tuple<int, int, int, int, int, int, int>, cudaGraphExec_t> graphs;
    // persistent schedule
    bool persistent = true;
    int tile = 2048, lag = 8, per_launch = 2, minb = 4, resident = 0;
    int64_t wait_ns = 2000000000;
    std::vector<int64_t> kf, ka;  // flow and transport nodes of each domain
    std::vector<int> jbeg;        // Neumann jobs of domain d: [jbeg[d], jbeg[d + 1])
    int* d_sync = nullptr;        // [0] status, [1] ticket, [2 ..] finished items per (step, lattice, domain)
    struct Table {
        clb::BatchItem* items = nullptr;
        int* need = nullptr;
        int n = 0;
    };
    std::map<std::tuple<int, int, int, int, int>, Table> tables;  // (steps, flow, ade, tile, lag)
    int* d_jbeg = nullptr;
    cudaStream_t user_stream = nullptr;
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

static void drop_tables(clb_batch* b) {
    for (auto& kv : b->tables) {
        cudaFree(kv.second.items);
        cudaFree(kv.second.need);
    }
    b->tables.clear();
}

static void batch_free(clb_batch* b) {
    drop_graphs(b);
    drop_tables(b);
    cudaFree(b->d_sync);
    cudaFree(b->d_jbeg);
    cudaFree(b->d_dom);
    cudaFree(b->d_foff);
    cudaFree(b->d_aoff);
    cudaFree(b->d_jobs);
    cudaFree(b->d_joff);
    cudaFree(b->d_ftiles);
    cudaFree(b->d_atiles);
    cudaFree(b->d_faces);
    cudaFree(b->d_face_off);
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
    std::vector<BatchTile> ftiles, atiles;
    std::vector<NeumannFace> faces;
    std::vector<int64_t> face_off(1, 0);
    b->kf.assign((size_t)n, 0);
    b->ka.assign((size_t)n, 0);
    b->jbeg.assign((size_t)n + 1, 0);
    for (int i = 0; i < n; ++i) {
        clb_handle* h = hs[i];
        BatchDomain& d = dom[(size_t)i];
        b->jbeg[(size_t)i] = (int)jobs.size();
        std::memset(&d, 0, sizeof d);
        if (b->has_flow) {
            d.f = h->d_f;
            d.flink = h->d_flink;
            d.fs = view_of(h->flow_sp);
            d.fkw = h->k_west_end;
            d.fke = h->k_east_begin;
            d.fp = h->fp;
            foff[(size_t)i + 1] = foff[(size_t)i] + h->flow_sp.K;
            b->kf[(size_t)i] = h->flow_sp.K;
            for (int64_t k = 0; k < h->flow_sp.K; k += BATCH_FLOW_TILE)
                ftiles.push_back({i, (int)std::min<int64_t>(BATCH_FLOW_TILE, h->flow_sp.K - k), k});
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
            b->ka[(size_t)i] = h->ade_sp.K;
            for (int64_t k = 0; k < h->ade_sp.K; k += BATCH_ADE_TILE)
                atiles.push_back({i, (int)std::min<int64_t>(BATCH_ADE_TILE, h->ade_sp.K - k), k});
            for (int side = 0; side < 2; ++side) {
                bool any = false;
                for (int s = 0; s < h->S; ++s)
                    any = any || (h->ap.slot[s] >= 0 && (side == 0 ? h->ap.ltype[s] : h->ap.rtype[s]) == CLB_NEUMANN);
                if (!any) continue;
                faces.push_back({i, side});
                face_off.push_back(face_off.back() + h->g.plane);
            }
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
    b->jbeg[(size_t)n] = (int)jobs.size();
    b->flow_nodes = foff.back();
    b->ade_nodes = aoff.back();
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_dom, sizeof(BatchDomain) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_foff, sizeof(int64_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_aoff, sizeof(int64_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs, sizeof(NeumannJob) * std::max<size_t>(1, jobs.size()));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_joff, sizeof(int64_t) * joff.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_jbeg, sizeof(int) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ftiles, sizeof(BatchTile) * std::max<size_t>(1, ftiles.size()));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_atiles, sizeof(BatchTile) * std::max<size_t>(1, atiles.size()));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_faces, sizeof(NeumannFace) * std::max<size_t>(1, faces.size()));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_face_off, sizeof(int64_t) * face_off.size());
    if (e == cudaSuccess && !ftiles.empty())
        e = cudaMemcpy(b->d_ftiles, ftiles.data(), sizeof(BatchTile) * ftiles.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !atiles.empty())
        e = cudaMemcpy(b->d_atiles, atiles.data(), sizeof(BatchTile) * atiles.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !faces.empty())
        e = cudaMemcpy(b->d_faces, faces.data(), sizeof(NeumannFace) * faces.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_face_off, face_off.data(), sizeof(int64_t) * face_off.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_sync, sizeof(int) * (2 + (size_t)PERSIST_MAX_STEPS * 3 * n));
    if (e == cudaSuccess) e = cudaMemset(b->d_sync, 0, sizeof(int) * (2 + (size_t)PERSIST_MAX_STEPS * 3 * n));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_jbeg, b->jbeg.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
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
    b->view.ftiles = b->d_ftiles;
    b->view.nft = (int)ftiles.size();
    b->view.atiles = b->d_atiles;
    b->view.nat = (int)atiles.size();
    b->view.faces = b->d_faces;
    b->view.foff_faces = b->d_face_off;
    b->view.nfaces = (int)faces.size();
    b->view.status = b->d_sync;
    b->neu_grid = std::max<int64_t>(1, std::min<int64_t>((face_off.back() + 255) / 256, b->num_sms * 4));
    b->resident = batch_persistent_resident(b->has_ade ? b->ade_prec : b->flow_prec, b->nm, b->minb);
    if (b->has_flow && b->has_ade && b->flow_prec != b->ade_prec) b->persistent = false;  // one storage type per launch
    *out = b;
    return CLB_OK;
}

static cudaStream_t bstream(const clb_batch* b) { return b->user_stream ? b->user_stream : b->stream; }

// The item table of a launch of `steps` steps: step s of domain d is placed by the key d + lag s
// (later steps first among equal keys); within it the flow tiles, then the Neumann planes, then
// the transport tiles. An item depends only on items of a smaller key.
static clb_status persist_table(clb_batch* b, int steps, bool flow, bool ade, clb_batch_s::Table** out) {
    const auto key = std::make_tuple(steps, (int)flow, (int)ade, b->tile, b->lag);
    auto it = b->tables.find(key);
    if (it != b->tables.end()) { *out = &it->second; return CLB_OK; }
    const int nd = (int)b->hs.size(), T = b->tile, W = b->lag;
    std::vector<int> need((size_t)3 * nd, 0);
    for (int d = 0; d < nd; ++d) {
        if (flow) need[(size_t)BI_FLOW * nd + d] = (int)((b->kf[(size_t)d] + T - 1) / T);
        if (ade) {
            need[(size_t)BI_NEUMANN * nd + d] = b->jbeg[(size_t)d + 1] > b->jbeg[(size_t)d] ? 1 : 0;
            need[(size_t)BI_TRANSPORT * nd + d] = (int)((b->ka[(size_t)d] + T - 1) / T);
        }
    }
    std::vector<BatchItem> items;
    const int keys = nd + W * (steps - 1);
    for (int k = 0; k < keys; ++k)
        for (int s = steps - 1; s >= 0; --s) {
            const int d = k - W * s;
            if (d < 0 || d >= nd) continue;
            auto tiles = [&](int kind, int64_t K) {
                for (int64_t f0 = 0; f0 < K; f0 += T)
                    items.push_back({d, (int16_t)kind, (int16_t)s, f0, (int)std::min<int64_t>(T, K - f0), 0});
            };
            if (flow) tiles(BI_FLOW, b->kf[(size_t)d]);
            if (ade) {
                if (need[(size_t)BI_NEUMANN * nd + d]) items.push_back({d, (int16_t)BI_NEUMANN, (int16_t)s, 0, 0, 0});
                tiles(BI_TRANSPORT, b->ka[(size_t)d]);
            }
        }
    clb_batch_s::Table t;
    t.n = (int)items.size();
    cudaError_t e = cudaMalloc(&t.items, sizeof(BatchItem) * std::max<size_t>(1, items.size()));
    if (e == cudaSuccess) e = cudaMalloc(&t.need, sizeof(int) * need.size());
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(t.items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t.need, need.data(), sizeof(int) * need.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(t.items);
        cudaFree(t.need);
        return bfail(b, CLB_CUDA_ERROR, std::string("batch schedule: ") + cudaGetErrorString(e));
    }
    *out = &b->tables.emplace(key, t).first->second;
    return CLB_OK;
}

// one persistent launch of `steps` steps from the given parities (counters cleared first)
static clb_status persist_launch(clb_batch* b, int steps, int fodd, int aodd, bool flow, bool ade) {
    clb_batch_s::Table* t = nullptr;
    clb_status st = persist_table(b, steps, flow, ade, &t);
    if (st != CLB_OK) return st;
    const int nd = (int)b->hs.size();
    PersistView V;
    V.B = b->view;
    V.items = t->items;
    V.n_items = t->n;
    V.need = t->need;
    V.jbeg = b->d_jbeg;
    V.status = b->d_sync;
    V.ticket = b->d_sync + 1;
    V.done = b->d_sync + 2;
    V.fodd = fodd;
    V.aodd = aodd;
    V.wait_ns = b->wait_ns;
    cudaMemsetAsync(b->d_sync + 1, 0, sizeof(int) * (1 + (size_t)steps * 3 * nd), bstream(b));
    launch_batch_persistent(V, ade ? b->ade_prec : b->flow_prec, b->nm, b->minb, b->resident, b->num_sms, bstream(b));
    return CLB_OK;
}

// one step of the requested lattices at the given parities, on the batch stream
static void batch_launch_step(clb_batch* b, int fodd, int aodd, bool flow, bool ade) {
    if (flow) {
        if (b->flow_staged) {
            launch_flow_batch_staged(b->view, b->flow_prec, fodd != 0, b->num_sms, bstream(b));
        } else {
            const int grid = b->num_sms * b->flow_mult;
            launch_flow_batch(b->view, b->flow_prec, fodd != 0, grid, b->flow_threads, bstream(b));
        }
    }
    if (ade) {
        launch_neumann_batch(b->view, b->ade_prec, aodd != 0, b->neu_grid, bstream(b));
        launch_ade_batch(b->view, b->ade_prec, aodd != 0, b->nm, b->ade_mult, b->ade_resident, b->num_sms, bstream(b));
    }
}

// bring each handle's counters (and the flow tracer's) up to date after n batched steps
static clb_status batch_commit(clb_batch* b, int n, bool flow, bool ade) {
    for (clb_handle* h : b->hs) {
        if (flow) {
            h->flow_iters += n;
            if (h->d_tracer)
                cudaMemcpyAsync(&h->d_tracer->iterations, &h->flow_iters, sizeof(int64_t), cudaMemcpyHostToDevice, bstream(b));
        }
        if (ade) {
            h->ade_iters += n;
            h->neu_iter = -1;
        }
    }
    int status = 0;
    cudaMemcpyAsync(&status, b->d_sync, sizeof(int), cudaMemcpyDeviceToHost, bstream(b));
    cudaError_t e = cudaStreamSynchronize(bstream(b));
    if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch step: ") + cudaGetErrorString(e));
    if (status) {
        cudaMemset(b->d_sync, 0, sizeof(int));
        return bfail(b, CLB_TIMEOUT, "batch step: a dependency wait of the persistent schedule gave up; the domains' "
                                     "state is undefined");
    }
    return CLB_OK;
}

// n steps on the persistent schedule: launches of per_launch steps (replayed from a graph when
// there are at least two of them), then one launch for the remainder
static clb_status persist_steps(clb_batch* b, int n, int fodd, int aodd, bool flow, bool ade) {
    const int S = b->per_launch;
    int done = 0;
    if (n / S >= 2) {
        const auto key = std::make_tuple(fodd, aodd, (int)flow, (int)ade, S, b->tile, b->lag);
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            // one direct launch first: the table and the kernel are set up before the capture
            clb_status st = persist_launch(b, S, fodd, aodd, flow, ade);
            if (st != CLB_OK) return st;
            done = S;
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(bstream(b), cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                st = persist_launch(b, S, fodd ^ (S & 1), aodd ^ (S & 1), flow, ade);
                e = cudaStreamEndCapture(bstream(b), &graph);
                if (st != CLB_OK) {
                    if (graph) cudaGraphDestroy(graph);
                    return st;
                }
            }
            cudaGraphExec_t exec = nullptr;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch graph: ") + cudaGetErrorString(e));
            it = b->graphs.emplace(key, exec).first;
        }
        // S is even, so every replay starts at the same parities
        for (; done + S <= n; done += S) {
            cudaError_t e = cudaGraphLaunch(it->second, bstream(b));
            if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch graph: ") + cudaGetErrorString(e));
        }
    }
    while (done < n) {
        const int k = std::min(S, n - done);
        clb_status st = persist_launch(b, k, fodd ^ (done & 1), aodd ^ (done & 1), flow, ade);
        if (st != CLB_OK) return st;
        done += k;
    }
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
    if (b->persistent) {
        clb_status st = persist_steps(b, n, fodd, aodd, flow, ade);
        if (st != CLB_OK) return st;
        return batch_commit(b, n, flow, ade);
    }
    int done = 0;
    if (n >= 4) {
        const auto key = std::make_tuple(fodd, aodd, (int)flow, (int)ade, 0, 0, 0);
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            // two direct steps first: every kernel variant is set up before the capture
            batch_launch_step(b, fodd, aodd, flow, ade);
            batch_launch_step(b, fodd ^ 1, aodd ^ 1, flow, ade);
            done = 2;
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(bstream(b), cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                batch_launch_step(b, fodd, aodd, flow, ade);
                batch_launch_step(b, fodd ^ 1, aodd ^ 1, flow, ade);
                e = cudaStreamEndCapture(bstream(b), &graph);
            }
            cudaGraphExec_t exec = nullptr;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch graph: ") + cudaGetErrorString(e));
            it = b->graphs.emplace(key, exec).first;
        }
        for (; done + 2 <= n; done += 2) {
            cudaError_t e = cudaGraphLaunch(it->second, bstream(b));
            if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch graph: ") + cudaGetErrorString(e));
        }
    }
    for (; done < n; ++done) batch_launch_step(b, fodd ^ (done & 1), aodd ^ (done & 1), flow, ade);
    return batch_commit(b, n, flow, ade);
}

// Times the schedules of the batched steps and keeps the fastest. Per-lattice launches: flow with
// 128 or 256 threads per block and 2, 4 or 8 blocks per SM, or the staged flow kernels; transport
// with shared memory for 4 or 6 resident blocks per SM and 1 or 2 times the resident grid. Persistent launches (when the lattices share one storage type): tiles of 1024,
// 2048 or 4096 nodes, lags of 2, 8 or 32 domains, 2 or 8 steps per launch, registers budgeted for
// 4, 6 or 8 resident CTAs per SM where those kernels are built. Every timed step is a
// real step of the domains: their iteration counters show the advance.
clb_status batch_autotune(clb_batch* b, int steps, char* report, int report_len) {
    cudaSetDevice(b->device);
    steps = std::max(8, (steps + 7) / 8 * 8);
    std::string rep;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int64_t ftaken = 0, ataken = 0;
    auto parities = [&](int& fodd, int& aodd) {
        fodd = (int)((b->hs[0]->flow_iters + ftaken) & 1);
        aodd = (int)((b->hs[0]->ade_iters + ataken) & 1);
    };
    auto elapsed = [&]() {
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / steps;
    };
    auto time_steps = [&](bool flow, bool ade) {
        int fodd, aodd;
        parities(fodd, aodd);
        batch_launch_step(b, fodd, aodd, flow, ade);  // set-up outside the timing
        batch_launch_step(b, fodd ^ 1, aodd ^ 1, flow, ade);
        cudaEventRecord(e0, bstream(b));
        for (int s = 0; s < steps; ++s) batch_launch_step(b, fodd ^ (s & 1), aodd ^ (s & 1), flow, ade);
        cudaEventRecord(e1, bstream(b));
        if (flow) ftaken += steps + 2;
        if (ade) ataken += steps + 2;
        return elapsed();
    };
    auto time_persist = [&]() {
        int fodd, aodd;
        parities(fodd, aodd);
        const int S = b->per_launch;
        clb_status st = persist_launch(b, S, fodd, aodd, b->has_flow, b->has_ade);  // table and kernel set-up
        if (st != CLB_OK) return 1e30f;
        cudaEventRecord(e0, bstream(b));
        for (int s = 0; s < steps; s += S) persist_launch(b, S, fodd, aodd, b->has_flow, b->has_ade);
        cudaEventRecord(e1, bstream(b));
        if (b->has_flow) ftaken += steps + S;
        if (b->has_ade) ataken += steps + S;
        return elapsed();
    };
    for (clb_handle* h : b->hs) cudaStreamSynchronize(h->stream);
    float legacy = 0.f;
    if (b->has_flow) {
        float best = 1e30f;
        int bt = 256, bm = 4;
        b->flow_staged = false;
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
        bool staged = false;
        if (flow_batch_staged_available(b->flow_prec)) {
            b->flow_staged = true;
            const float ms = time_steps(true, false);
            char buf[96];
            std::snprintf(buf, sizeof buf, "flow staged:%.1fus ", ms * 1e3f);
            rep += buf;
            if (ms < best) { best = ms; staged = true; }
        }
        b->flow_staged = staged;
        b->flow_threads = bt;
        b->flow_mult = bm;
        legacy += best;
    }
    if (b->has_ade) {
        float best = 1e30f;
        int bm = 1, br = 4;
        for (int resident : {4, 6})
            for (int mult : {1, 2}) {
                b->ade_mult = mult;
                b->ade_resident = resident;
                const float ms = time_steps(false, true);
                char buf[96];
                std::snprintf(buf, sizeof buf, "transport %dx%d:%.1fus ", resident, mult, ms * 1e3f);
                rep += buf;
                if (ms < best) { best = ms; bm = mult; br = resident; }
            }
        b->ade_mult = bm;
        b->ade_resident = br;
        legacy += best;
    }
    // the flow and transport steps of the per-lattice schedule run one after the other
    b->persistent = false;
    float best = legacy;
    const bool can_persist = !(b->has_flow && b->has_ade && b->flow_prec != b->ade_prec);
    if (can_persist) {
        const int prec = b->has_ade ? b->ade_prec : b->flow_prec;
        int bt = b->tile, bw = b->lag, bs = b->per_launch, bb = b->minb;
        for (int mb : {4, 6, 8}) {
            if (persist_minb(prec, b->nm, mb) != mb) continue;
            b->minb = mb;
            b->resident = batch_persistent_resident(prec, b->nm, mb);
            for (int tile : {1024, 2048, 4096})
                for (int lag : {2, 8, 32})
                    for (int S : {2, 8}) {
                        b->tile = tile;
                        b->lag = lag;
                        b->per_launch = S;
                        const float ms = time_persist();
                        char buf[96];
                        std::snprintf(buf, sizeof buf, "persistent %d/%d/%d/%dx%d:%.1fus ", tile, lag, S, mb, b->resident,
                                      ms * 1e3f);
                        rep += buf;
                        if (ms < best) { best = ms; bt = tile; bw = lag; bs = S; bb = mb; b->persistent = true; }
                    }
        }
        b->tile = bt;
        b->lag = bw;
        b->per_launch = bs;
        b->minb = bb;
        b->resident = batch_persistent_resident(prec, b->nm, bb);
    }
    {
        char buf[128];
        if (b->persistent)
            std::snprintf(buf, sizeof buf, "-> persistent tile %d lag %d steps/launch %d ctas/SM %d", b->tile, b->lag,
                          b->per_launch, b->minb);
        else
            std::snprintf(buf, sizeof buf, "-> per-lattice launches");
        rep += buf;
    }
    for (clb_handle* h : b->hs) {
        h->flow_iters += ftaken;
        if (ataken) { h->ade_iters += ataken; h->neu_iter = -1; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs(b);
    for (clb_handle* h : b->hs)
        if (b->has_flow && h->d_tracer)
            cudaMemcpyAsync(&h->d_tracer->iterations, &h->flow_iters, sizeof(int64_t), cudaMemcpyHostToDevice, bstream(b));
    int status = 0;
    cudaMemcpyAsync(&status, b->d_sync, sizeof(int), cudaMemcpyDeviceToHost, bstream(b));
    cudaError_t e = cudaStreamSynchronize(bstream(b));
    if (report && report_len > 0) {
        std::strncpy(report, rep.c_str(), (size_t)report_len - 1);
        report[report_len - 1] = 0;
    }
    if (e != cudaSuccess) return bfail(b, CLB_CUDA_ERROR, std::string("batch autotune: ") + cudaGetErrorString(e));
    if (status) {
        cudaMemset(b->d_sync, 0, sizeof(int));
        return bfail(b, CLB_TIMEOUT, "batch autotune: a dependency wait of the persistent schedule gave up");
    }
    return CLB_OK;
}

// Sets the schedule: persistent (tile nodes per item, lag in domains, steps per launch: even, at
// most PERSIST_MAX_STEPS, the register budget in resident CTAs per SM) or, persistent == 0, one
// launch per lattice and step.
clb_status batch_schedule(clb_batch* b, int persistent, int tile, int lag, int steps_per_launch, int ctas_per_sm) {
    if (persistent < 0 || persistent > 2) return bfail(b, CLB_INVALID_ARG, "schedule: persistent is 0, 1 or 2");
    if (persistent == 1) {
        if (b->has_flow && b->has_ade && b->flow_prec != b->ade_prec)
            return bfail(b, CLB_INVALID_ARG, "the persistent schedule needs one storage type for flow and transport");
        if (tile < 256 || tile % 256 || tile > (1 << 20) || lag < 1 || steps_per_launch < 2 ||
            steps_per_launch > PERSIST_MAX_STEPS || steps_per_launch % 2)
            return bfail(b, CLB_INVALID_ARG, "schedule: tile a multiple of 256, lag >= 1, an even 2..8 steps per launch");
        const int prec = b->has_ade ? b->ade_prec : b->flow_prec;
        if (ctas_per_sm != 4 && persist_minb(prec, b->nm, ctas_per_sm) != ctas_per_sm)
            return bfail(b, CLB_INVALID_ARG, "schedule: no persistent kernel built for that number of CTAs per SM");
        b->tile = tile;
        b->lag = lag;
        b->per_launch = steps_per_launch;
        b->minb = ctas_per_sm;
        b->resident = batch_persistent_resident(prec, b->nm, ctas_per_sm);
    }
    if (persistent == 2 && b->has_flow && !flow_batch_staged_available(b->flow_prec))
        return bfail(b, CLB_INVALID_ARG, "schedule: the staged flow step needs 4- or 8-byte flow storage");
    b->persistent = persistent == 1;
    b->flow_staged = persistent == 2;
    drop_graphs(b);
    return CLB_OK;
}

// The limit of one dependency wait of the persistent schedule (nanoseconds); a wait that reaches
// it gives up, the launch skips its remaining items and the step returns CLB_TIMEOUT.
clb_status batch_set_wait_limit(clb_batch* b, int64_t ns) {
    if (ns < 0) return bfail(b, CLB_INVALID_ARG, "wait limit must not be negative");
    cudaStreamSynchronize(bstream(b));
    b->wait_ns = ns;
    drop_graphs(b);  // the limit is a parameter of the captured launches
    return CLB_OK;
}

// The stream the batch's work is enqueued on (nullptr: the batch's own); the steps still return
// once their work is done.
clb_status batch_set_stream(clb_batch* b, void* stream) {
    cudaStreamSynchronize(bstream(b));
    b->user_stream = static_cast<cudaStream_t>(stream);
    drop_graphs(b);
    return CLB_OK;
}

// The schedule in force (for reports).
clb_status batch_get_schedule(clb_batch* b, int* persistent, int* tile, int* lag, int* steps_per_launch,
                              int* ctas_per_sm) {
    if (persistent) *persistent = b->persistent ? 1 : (b->flow_staged ? 2 : 0);
    if (ctas_per_sm) *ctas_per_sm = b->minb;
    if (tile) *tile = b->tile;
    if (lag) *lag = b->lag;
    if (steps_per_launch) *steps_per_launch = b->per_launch;
    return CLB_OK;
}

clb_status batch_destroy(clb_batch* b) {
    if (!b) return CLB_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(bstream(b));
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

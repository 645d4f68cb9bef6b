// checkpoint.cu -- restart files of a domain's lattices (the reference's .chk checkpoints:
// saveBinaryBlock of the flow lattice, complab.cpp:2004, and of every substrate and biomass
// lattice, :2292-2302; loadBinaryBlock at :1106-1108 and :2044-2055). One file per call holds the
// flow lattice's incoming populations, and/or every species (mobile: incoming populations in the
// storage's own convention, g_i - t_i for FP64 lattices and g_i for FP32 / FP16 ones; immobile:
// concentration), the biomass fields and the advection velocity, in FP64 (exact for every storage
// precision), with the step counters; loading it into a handle set up on the same material map and
// precisions continues the run exactly as the saved handle would.
//
// The header records which species are mobile and the biofilm material codes, because a species'
// block size follows from its mobility: a handle whose mobile set differs would otherwise read
// misaligned blocks. A save writes `path`.tmp and renames it over `path` once the file is complete,
// so a crash or a full disk during a save leaves the previous restart point intact. A load reads
// and checks the whole file into host memory before it changes the handle, so a truncated or
// mismatched file leaves the handle exactly as it was.
#include "clb_internal.cuh"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace clb;

namespace {

const char MAGIC[8] = {'C', 'L', 'B', 'C', 'K', 'P', 'T', '1'};
constexpr int32_t VERSION = 3;

struct Header {
    char magic[8];
    int32_t version, nx, ny, nz, flow_prec, ade_prec, S, M, what, pad;
    int64_t flow_iters, ade_iters;
    uint32_t mobile_mask;                   // bit s: user species s is mobile
    int32_t n_microbes;                     // the domain's biofilm materials
    int32_t bio_codes[CLB_MAX_MICROBES];
    int32_t pad2;
};

bool put(std::FILE* f, const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }
bool get(std::FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

bool mobile(const clb_handle* h, int s) { return h->ap.slot[h->u2i[s]] >= 0; }

uint32_t mobile_mask(const clb_handle* h) {
    uint32_t m = 0;
    for (int s = 0; s < h->S; ++s)
        if (mobile(h, s)) m |= 1u << s;
    return m;
}

}  // namespace

extern "C" {

clb_status clb_checkpoint_save(clb_handle* h, const char* path, int what) {
    if (!h || !path) return fail(h, CLB_INVALID_ARG, "null argument");
    if (what <= 0 || (what & ~(CLB_CKPT_FLOW | CLB_CKPT_TRANSPORT)))
        return fail(h, CLB_INVALID_ARG, "checkpoint contents: CLB_CKPT_FLOW and/or CLB_CKPT_TRANSPORT");
    if ((what & CLB_CKPT_FLOW) && !h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    if ((what & CLB_CKPT_TRANSPORT) && !h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (h->ca_ready || h->prc_ready)
        return fail(h, CLB_INVALID_ARG, "checkpoints hold no automaton or precipitation state; save before clb_ca_setup / clb_precip_setup");
    const size_t N = (size_t)h->g.N;
    Header hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, MAGIC, 8);
    hd.version = VERSION;
    hd.nx = h->g.nx; hd.ny = h->g.ny; hd.nz = h->g.nz;
    hd.flow_prec = h->flow_prec;
    hd.ade_prec = h->ade_prec;
    hd.S = (what & CLB_CKPT_TRANSPORT) ? h->S : 0;
    hd.M = (what & CLB_CKPT_TRANSPORT) ? h->M : 0;
    hd.what = what;
    hd.flow_iters = h->flow_iters;
    hd.ade_iters = h->ade_iters;
    hd.mobile_mask = (what & CLB_CKPT_TRANSPORT) ? mobile_mask(h) : 0;
    hd.n_microbes = h->d.n_microbes;
    for (int m = 0; m < h->d.n_microbes && m < CLB_MAX_MICROBES; ++m) hd.bio_codes[m] = h->d.bio_codes[m];
    {
        clb_status hs = host_mat_sync(h);
        if (hs != CLB_OK) return hs;
    }
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return fail(h, CLB_INVALID_ARG, "cannot open " + tmp);
    bool ok = put(f, &hd, sizeof(hd)) && put(f, h->h_mat.data(), N);
    clb_status st = CLB_OK;
    std::vector<double> buf;
    if (ok && (what & CLB_CKPT_FLOW)) {
        buf.resize(19 * N);
        st = clb_get_field(h, CLB_FIELD_FLOW_POPULATIONS, 0, buf.data(), 0);
        ok = st == CLB_OK && put(f, buf.data(), sizeof(double) * buf.size());
    }
    if (ok && (what & CLB_CKPT_TRANSPORT)) {
        for (int s = 0; ok && s < h->S; ++s) {
            const bool mob = mobile(h, s);
            buf.resize((mob ? 7 : 1) * N);
            st = mob ? ade_populations(h, s, buf.data(), 0) : clb_get_field(h, CLB_FIELD_CONCENTRATION, s, buf.data(), 0);
            ok = st == CLB_OK && put(f, buf.data(), sizeof(double) * buf.size());
        }
        for (int m = 0; ok && m < h->M; ++m) {
            buf.resize(N);
            st = clb_get_field(h, CLB_FIELD_BIOMASS, m, buf.data(), 0);
            ok = st == CLB_OK && put(f, buf.data(), sizeof(double) * N);
        }
        if (ok) {
            buf.resize(3 * N);
            st = clb_get_field(h, CLB_FIELD_ADE_VELOCITY, 0, buf.data(), 0);
            ok = st == CLB_OK && put(f, buf.data(), sizeof(double) * buf.size());
        }
    }
    if (ok && std::fflush(f) != 0) ok = false;
    if (std::fclose(f) != 0) ok = false;
    if (!ok || st != CLB_OK) {
        std::remove(tmp.c_str());
        if (st != CLB_OK) return st;
        return fail(h, CLB_INVALID_ARG, "cannot write " + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return fail(h, CLB_INVALID_ARG, std::string("cannot replace ") + path);
    }
    return CLB_OK;
}

clb_status clb_checkpoint_load(clb_handle* h, const char* path) {
    if (!h || !path) return fail(h, CLB_INVALID_ARG, "null argument");
    cudaSetDevice(h->device);
    const size_t N = (size_t)h->g.N;
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return fail(h, CLB_INVALID_ARG, std::string("cannot open ") + path);
    Header hd;
    std::vector<int8_t> mat(N);
    auto bad = [&](const std::string& why) {
        std::fclose(f);
        return fail(h, CLB_INVALID_ARG, "checkpoint " + std::string(path) + ": " + why);
    };
    if (!get(f, &hd, sizeof(hd)) || std::memcmp(hd.magic, MAGIC, 8) != 0 || hd.version != VERSION)
        return bad("not a checkpoint of this library version");
    if (hd.nx != h->g.nx || hd.ny != h->g.ny || hd.nz != h->g.nz) return bad("lattice size differs");
    if (!get(f, mat.data(), N)) return bad("truncated");
    if (host_mat_sync(h) != CLB_OK) return bad("cannot read the handle's material map");
    if (std::memcmp(mat.data(), h->h_mat.data(), N) != 0) return bad("saved on a different material map");
    if (hd.n_microbes != h->d.n_microbes) return bad("biofilm materials differ");
    for (int m = 0; m < hd.n_microbes && m < CLB_MAX_MICROBES; ++m)
        if (hd.bio_codes[m] != h->d.bio_codes[m]) return bad("biofilm materials differ");
    if (hd.what & CLB_CKPT_FLOW) {
        if (!h->flow_ready) return bad("holds the flow lattice; clb_flow_init first");
        if (hd.flow_prec != h->flow_prec) return bad("flow storage precision differs");
    }
    if (hd.what & CLB_CKPT_TRANSPORT) {
        if (!h->ade_ready) return bad("holds the species lattices; clb_ade_init first");
        if (hd.ade_prec != h->ade_prec) return bad("transport storage precision differs");
        if (hd.S != h->S || hd.M != h->M) return bad("species or microbe count differs");
        if (hd.mobile_mask != mobile_mask(h)) return bad("mobile species differ");
    }
    // the whole payload into host memory first: nothing of the handle changes unless all of it is there
    std::vector<double> flow, vel;
    std::vector<std::vector<double>> spec, bio;
    if (hd.what & CLB_CKPT_FLOW) {
        flow.resize(19 * N);
        if (!get(f, flow.data(), sizeof(double) * flow.size())) return bad("truncated");
    }
    if (hd.what & CLB_CKPT_TRANSPORT) {
        spec.resize(h->S);
        for (int s = 0; s < h->S; ++s) {
            spec[s].resize((mobile(h, s) ? 7 : 1) * N);
            if (!get(f, spec[s].data(), sizeof(double) * spec[s].size())) return bad("truncated");
        }
        bio.resize(h->M);
        for (int m = 0; m < h->M; ++m) {
            bio[m].resize(N);
            if (!get(f, bio[m].data(), sizeof(double) * N)) return bad("truncated");
        }
        vel.resize(3 * N);
        if (!get(f, vel.data(), sizeof(double) * vel.size())) return bad("truncated");
    }
    if (std::fgetc(f) != EOF) return bad("trailing data after the last field");
    std::fclose(f);

    const int64_t save_flow = h->flow_iters, save_ade = h->ade_iters;
    clb_status st = CLB_OK;
    if (hd.what & CLB_CKPT_FLOW) {
        // the counter first: the populations go into the slots of the step parity it gives
        h->flow_iters = hd.flow_iters;
        Tracer tz;
        std::memset(&tz, 0, sizeof(tz));
        tz.iterations = hd.flow_iters;
        cudaError_t e = cudaMemcpy(h->d_tracer, &tz, sizeof(tz), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { h->flow_iters = save_flow; return cuda_check(h, e, "tracer"); }
        if ((st = clb_set_field(h, CLB_FIELD_FLOW_POPULATIONS, 0, flow.data(), 0)) != CLB_OK) return st;
    }
    if (hd.what & CLB_CKPT_TRANSPORT) {
        h->ade_iters = hd.ade_iters;
        for (int s = 0; s < h->S; ++s) {
            st = mobile(h, s) ? ade_set_populations(h, s, spec[s].data(), 0) : ade_set_immobile(h, s, spec[s].data());
            if (st != CLB_OK) { h->ade_iters = save_ade; return st; }
        }
        for (int m = 0; m < h->M; ++m)
            if ((st = clb_set_field(h, CLB_FIELD_BIOMASS, m, bio[m].data(), 0)) != CLB_OK) return st;
        if ((st = clb_set_field(h, CLB_FIELD_ADE_VELOCITY, 0, vel.data(), 0)) != CLB_OK) return st;
    }
    return CLB_OK;
}

}  // extern "C"

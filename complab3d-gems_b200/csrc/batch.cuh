// batch.cuh -- many independent domains advanced by one launch per lattice and step.
#pragma once

#include "sparse.cuh"

namespace clb {

// Everything the batched kernels need of one domain (device copy, one per domain).
struct BatchDomain {
    // flow lattice
    void* f;
    void* flink;
    SparseView fs;
    int64_t fkw, fke;  // compact index ranges of the planes x = 0, x = nx-1
    FlowParams fp;
    // species lattices
    void* g;
    void* glink;
    SparseView as;
    int64_t akw, ake;
    AdeParams ap;
    double* imm;
    double* bio;
    const void* u;
    double* neu;
    const int* mob;
    const int8_t* mat;
    int n_mobile;
};

// one Neumann plane of one mobile species of one domain
struct NeumannJob {
    int d, s, m, side;
};

// A run of consecutive compact nodes of one domain's lattice: the unit the per-lattice batched
// launches hand to a CTA, which holds the domain's description in shared memory while it works.
struct BatchTile {
    int d;
    int count;
    int64_t first;
};
constexpr int BATCH_FLOW_TILE = 1024;  // flow nodes per tile
constexpr int BATCH_ADE_TILE = 512;    // transport nodes per tile
// the staged flow kernels step whole 256-node tiles of the layout: a run of the tile table must not
// split one
static_assert(BATCH_FLOW_TILE % TILE == 0, "flow tiles are whole layout tiles");

// One x-face of one domain that at least one mobile species treats as Neumann
struct NeumannFace {
    int d, side;
};

struct BatchView {
    const BatchDomain* dom;
    const int64_t* foff;  // [ndom + 1] prefix sums of the flow node counts
    const int64_t* aoff;  // [ndom + 1] prefix sums of the species node counts
    int ndom;
    const NeumannJob* jobs;
    const int64_t* joff;  // [njobs + 1] prefix sums of the plane sizes
    int njobs;
    const BatchTile* ftiles;  // flow tiles, domain by domain
    int nft;
    const BatchTile* atiles;  // transport tiles, domain by domain
    int nat;
    const NeumannFace* faces;
    const int64_t* foff_faces;  // [nfaces + 1] prefix sums of the face sizes
    int nfaces;
    int* status;  // nonzero: a bounded wait of a staged step gave up
};

constexpr int BATCH_MAX_DOMAINS = 2048;

// One entry of the persistent schedule: a tile of one lattice of one domain at one step of the
// launch (or the Neumann planes of the domain's species at that step).
constexpr int BI_FLOW = 0, BI_NEUMANN = 1, BI_TRANSPORT = 2;
struct BatchItem {
    int d;
    int16_t kind;   // BI_FLOW, BI_NEUMANN or BI_TRANSPORT
    int16_t step;   // step within the launch
    int64_t first;  // first compact node of the tile
    int count;      // nodes in the tile
    int pad;
};
constexpr int PERSIST_MAX_STEPS = 8;

struct PersistView {
    BatchView B;
    const BatchItem* items;
    int n_items;
    const int* need;  // [3][ndom]: items of each kind per domain and step
    const int* jbeg;  // [ndom + 1]: the Neumann jobs of domain d are jobs[jbeg[d] .. jbeg[d + 1])
    int* done;        // [steps][3][ndom]: items finished, zero when the launch starts
    int* ticket;      // next item to take, zero when the launch starts
    int* status;      // nonzero: a wait gave up (the launch's remaining items were skipped)
    int fodd, aodd;   // parities of the launch's first step
    int64_t wait_ns;  // limit of one wait
};

// flow.cu (staged: the even step through bulk-copied tiles, the odd step with the next node's
// gathers in flight, 4- and 8-byte storage; else the plain per-node step)
void launch_flow_batch(const BatchView& B, int prec, bool odd, int grid, int threads, cudaStream_t st);
bool flow_batch_staged_available(int prec);
void launch_flow_batch_staged(const BatchView& B, int prec, bool odd, int num_sms, cudaStream_t st);
// ade.cu (nm: species register bucket 1, 2, 4, 8 or 16)
void launch_ade_batch(const BatchView& B, int prec, bool odd, int nm, int grid_mult, int resident, int num_sms,
                      cudaStream_t st);
void launch_neumann_batch(const BatchView& B, int prec, bool odd, int grid, cudaStream_t st);
// the persistent schedule: one launch runs the whole item table
void launch_batch_persistent(const PersistView& V, int prec, int nm, int minb, int blocks_per_sm, int num_sms,
                             cudaStream_t st);
int batch_persistent_resident(int prec, int nm, int minb);  // resident CTAs per SM of that launch
int persist_minb(int prec, int nm, int minb);                // the register budget built for that request

}  // namespace clb

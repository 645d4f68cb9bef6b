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

struct BatchView {
    const BatchDomain* dom;
    const int64_t* foff;  // [ndom + 1] prefix sums of the flow node counts
    const int64_t* aoff;  // [ndom + 1] prefix sums of the species node counts
    int ndom;
    const NeumannJob* jobs;
    const int64_t* joff;  // [njobs + 1] prefix sums of the plane sizes
    int njobs;
};

constexpr int BATCH_MAX_DOMAINS = 2048;

// flow.cu
void launch_flow_batch(const BatchView& B, int prec, bool odd, int grid, int threads, cudaStream_t st);
// ade.cu (nm: species register bucket 1, 2, 4, 8 or 16)
void launch_ade_batch(const BatchView& B, int prec, bool odd, int nm, int grid_mult, int num_sms, cudaStream_t st);
void launch_neumann_batch(const BatchView& B, int prec, bool odd, int grid, cudaStream_t st);

}  // namespace clb

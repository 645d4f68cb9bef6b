// biofilm_ca.cu -- the biofilm cellular automaton: excess biomass pushed to face neighbours
// ('fraction' and 'half' modes), the mask / total-biomass update and the age wavefront, on the
// GPU with the same results as the sequential lexicographic algorithm.
//
// Reference behaviour (complab.cpp:2792-3055 and :3074-3079):
//   updateLocalMaskNtotalLattices3D (complab3d_processors_part2.hh:71-259): the total biomass of
//     every open voxel (species above 1e-14), pore -> biofilm at thrd_bFilmFrac x Bmax (the mask
//     becomes the sum of the present microbes' codes), biofilm -> pore below it;
//   while max(total) exceeds Bmax: pushExcessBiomass3D (complab3d_processors_part1.hh:499-732)
//     over the voxels in lexicographic order: the excess goes to the face neighbours in a random
//     order, each taking up to its room (Bmax - its total, a pore neighbour counting as empty),
//     split over the microbes in proportion; what is left goes to one neighbour chosen among
//     those with a lower age (else any); then the mask / total update; every 50 sweeps the age
//     relaxation (updateAgeDistance3D, part2.hh:840-965) until no age changes; a sweep that does
//     not lower the maximum for 100 sweeps in a row, or more than 1000 sweeps, is a failure;
//   after the block, if the mask changed, one age sweep.
// A single-block run never takes the push's block-boundary path, so the copy lattices and
// pullExcessBiomass3D (part1.hh:973-1150) have no effect there and are not built.
//
// Random choices: the reference draws from std::random_shuffle / std::rand seeded by the clock.
// Here voxel n of push sweep w draws from splitmix64 steps started at
// seed ^ (w * 0x9E3779B97F4A7C15) ^ (n * 0xD1B54A32D192ED03) (shuffle: Fisher-Yates from the top,
// draw % (i + 1); pick: draw % L), so a run is reproducible and the draws do not depend on the
// order in which voxels are processed.
//
// Parallel schedule with sequential results. In a sweep the only state a voxel's push reads that
// another voxel's push writes is its own per-microbe biomass, which its lexicographically earlier
// face neighbours (x-1, y-1, z-1) may have pushed into. Every other input (totals, masks, ages)
// is fixed during the sweep. So the active voxels are processed in rounds: a voxel runs once its
// earlier active neighbours have run, starting from its biomass plus their pushes into it (added
// in their lexicographic order), and records its pushes instead of writing them; a final pass
// adds to every voxel the pushes it received, in the order the sequential sweep adds them. The
// results are bit-identical to the sequential sweep.
//
// The age sweep after a mask change is one in-place lexicographic sweep: it runs as wavefronts
// over x + y + z, each voxel seeing its earlier neighbours updated and its later ones not. The
// relaxation to convergence runs as unordered in-place sweeps over the voxels that hold biomass
// (the only ones the rule changes; the mask pass lists them): the update is monotone and only ever
// raises an age, so any order of updates reaches the same least fixed point as the reference's
// lexicographic in-place sweeps. Counters cross to the host through pinned memory.
//
// Passes over the biomass list, not the box. A mask pass lists the voxels whose total exceeds
// 1e-14 afterwards. A voxel off that list holds every microbe below 1e-12 (a microbe at or above
// it makes the sum differ from a stored total at or below 1e-14 by more than 1e-14, so the pass
// stores the new total and lists the voxel) and a pore or closed code (a biofilm code below the
// biofilm threshold reverts). The rate laws leave biomass below 1e-12 as it is, and such a voxel
// is a fixed point of the mask rule, so the next pass needs only the listed voxels plus those a
// push sweep deposited into. The mask sum is carried along by the changes each pass makes. The
// pushes of a sweep likewise change only the active voxels and the voxels their records name, so
// the apply pass walks those two lists. A pass over the whole box runs after set-up and after
// the host or a geometry update wrote biomass or the material map (`full`).
#include "sparse.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>

namespace clb {

constexpr int CA_THREADS = 256;
constexpr int CA_REC = 7;  // push records per voxel: up to six neighbours plus the remainder

struct CaView {
    Geom g;
    double bmax, thr;        // Bmax, thrd_bFilmFrac x Bmax
    int M;
    int half;                // push mode: 0 'fraction' (pushExcessBiomass3D), 1 'half' (halfPushExcessBiomass3D)
    int bb, solid;
    int n_pore;
    int pore[CLB_MAX_PORE_CODES];
    int bio_code[CLB_MAX_MICROBES];
};

__device__ __forceinline__ bool ca_open(const CaView& C, int m) { return m != C.bb && m != C.solid; }
__device__ __forceinline__ bool ca_pore(const CaView& C, int m) {
    for (int i = 0; i < C.n_pore; ++i)
        if (m == C.pore[i]) return true;
    return false;
}
__device__ __forceinline__ uint64_t sm64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
// doubles ordered as signed 64-bit integers (for atomicMax)
__device__ __forceinline__ long long ordered(double v) {
    long long i = __double_as_longlong(v);
    return i < 0 ? i ^ 0x7FFFFFFFFFFFFFFFLL : i;
}

// Counters and control state of the automaton in device memory. The pass and sweep counters are
// cleared and read inside one step (the first pass's by the step before, or at set-up); the step
// results and the totals are what the host reads back.
struct CaScalars {
    long long gmax;         // ordered bits of max(total) over the voxels the pass visits, at least 0
    long long msum;         // whole-box pass: the mask sum; list pass: the change it made to it
    unsigned int nonfinite; // biomass values that are NaN or infinite (mask pass)
    unsigned int nout;      // voxels the mask pass lists
    unsigned int moved;     // voxels whose material the passes of the step changed
    unsigned int active;    // voxels collected for the sweep
    unsigned int remaining;
    unsigned int changed;   // ages changed by a sweep
    unsigned int overflow;  // active voxels beyond the capacity
    unsigned int next;      // voxels the sweep pushed into that are not active themselves
    unsigned int next2;     // of those, the ones not on the biomass list
    unsigned int nlist;     // voxels on the current biomass list
    int list;               // which of the two list buffers holds it
    long long mask_run;     // the mask sum as it stands
    int status;             // CA_OK, or why a step stopped (kept until the host reads it)
    int fail_iter;          // the iteration whose step set `status`
    int step_sweeps;        // push sweeps of the last step
    int step_changed;       // 1: the last step changed the mask sum
    unsigned int moved_any; // a step changed voxels since the host last looked
    long long ca_mask_sum;  // the mask sum after the last step
    unsigned long long sweep_counter;  // push sweeps since set-up: the random streams' sweep number
    long long total_sweeps, total_changes;  // over all steps since set-up
};

enum : int { CA_OK = 0, CA_NONFINITE = 1, CA_STALL = 2, CA_AGE = 3, CA_SWEEPS = 4, CA_CAPACITY = 5, CA_ROUNDS = 6 };

// the device buffers one step of the automaton works on
struct CaBufs {
    int8_t* mat;
    int8_t* mask0;  // the mask before a pass (several pore codes), else null
    double* bio;
    double* total;
    int* age;
    const int8_t* distp;
    int* aidx;
    int* act;
    int* done;
    int* tgt;
    double* amt;
    double* own;
    int32_t* list[2];  // the biomass list and the one the next mask pass writes
    int32_t* ext;      // voxels a sweep pushed into that are not active
    int32_t* ext2;     // of those, the ones off the biomass list
    int* tmark;        // 1 while a voxel is on ext (cleared after the sweep)
    uint8_t* bflag;    // the transport step's biomass flags per species node (see below), or null
    const int32_t* sidx;  // species-lattice node of each voxel, -1
    int cap;
    uint64_t seed;
};

// ------------------------------------------------------------------ set-up and mask update

__global__ void k_ca_init(const CaView C, const int8_t* __restrict__ mat, const double* __restrict__ bio,
                          double* __restrict__ total, int* __restrict__ age, int8_t* __restrict__ distp,
                          int* __restrict__ aidx, CaScalars* sc) {
    const Geom G = C.g;
    long long msum = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(G, n, x, y, z);
        double t = 0.0;
        for (int m = 0; m < C.M; ++m) t += bio[(int64_t)m * G.N + n];
        total[n] = t;
        const int mk = mat[n];
        msum += mk;
        age[n] = !ca_open(C, mk) ? -1 : (ca_pore(C, mk) ? 0 : 1);
        distp[n] = (ca_open(C, mk) && x < G.nx - 1 && y < G.ny - 1 && z < G.nz - 1) ? 1 : 0;
        aidx[n] = -1;
    }
    atomicAdd((unsigned long long*)&sc->mask_run, (unsigned long long)msum);
}

// updateLocalMaskNtotalLattices3D; with several pore codes a reopened voxel copies the first
// pore neighbour found in `mask0` (the mask as it stood before the pass).
// One voxel of the pass, from its loaded material, previous total and biomass; returns whether it
// goes on the biomass list. `msum` takes the voxel's code (DELTA false: a whole-box pass sums the
// mask) or the change the pass made to it (DELTA true: a list pass carries the sum along).
template <bool DELTA>
__device__ __forceinline__ bool ca_mask_voxel(const CaView& C, const CaBufs& B, CaScalars* sc, int64_t n, int mk,
                                              double told, const double* bm, long long& best, long long& msum) {
    const Geom G = C.g;
    double tn = told;
    if (ca_open(C, mk)) {
        double bmass = 0.0;
        int newmask = 0;
        for (int m = 0; m < C.M; ++m) {
            if (!isfinite(bm[m])) atomicAdd(&sc->nonfinite, 1u);  // the run stops (complab.cpp:2796)
            if (bm[m] > 1e-14) {
                bmass += bm[m];
                newmask += C.bio_code[m];
            }
        }
        if (fabs(bmass - told) > 1e-14) {
            B.total[n] = bmass;
            tn = bmass;
        }
        const bool poreflag = ca_pore(C, mk);
        int out = mk;
        if (!poreflag && bmass < C.thr) {
            out = C.pore[0];
            if (C.n_pore > 1) {
                int x, y, z;
                decode(G, n, x, y, z);
                const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
                for (int d = 0; d < 6; ++d) {
                    const int X = x + d6[d][0], Y = y + d6[d][1], Z = z + d6[d][2];
                    if (X < 0 || Y < 0 || Z < 0 || X >= G.nx || Y >= G.ny || Z >= G.nz) continue;
                    const int nm = B.mask0[(int64_t)X * G.plane + (int64_t)Y * G.nz + Z];
                    if (ca_open(C, nm) && ca_pore(C, nm)) { out = nm; break; }
                }
            }
        } else if (poreflag && bmass >= C.thr && newmask > 0) {
            out = newmask;
        }
        if (out != mk) {
            B.mat[n] = (int8_t)out;
            atomicAdd(&sc->moved, 1u);
        }
        msum += DELTA ? out - mk : out;
    } else if (!DELTA) {
        msum += mk;
    }
    best = max(best, ordered(tn));
    // the transport step reads this voxel's biomass only when it is listed (a voxel off the list
    // holds every microbe below 1e-12, where no rate law acts); a NaN total stays flagged
    if (B.bflag) {
        const int32_t k = B.sidx[n];
        if (k >= 0) B.bflag[k] = !(tn <= 1e-14);
    }
    return tn > 1e-14;
}

// appends n (where `listed`) to `out` (count in *nout), one atomic per warp; the whole warp calls it
__device__ __forceinline__ void ca_list_append(int32_t* __restrict__ out, unsigned int* nout, int64_t n, bool listed) {
    const int lane = threadIdx.x & 31;
    const unsigned int bal = __ballot_sync(0xffffffffu, listed);
    if (!bal) return;
    unsigned int base = 0;
    if (lane == 0) base = atomicAdd(nout, (unsigned int)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (listed) out[base + __popc(bal & ((1u << lane) - 1u))] = (int32_t)n;
}

// appends n (where `listed`) to `out` (count in *nout) with one atomic per block: a pass over a
// list runs with whole blocks in step, and one counter taken by every warp of the grid would
// serialise thousands of atomics on one address. Every thread of the block calls it; s_cnt holds
// blockDim.x / 32 + 1 counts.
__device__ __forceinline__ void ca_list_append_block(int32_t* __restrict__ out, unsigned int* nout, int64_t n,
                                                     bool listed, unsigned int* s_cnt) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned int bal = __ballot_sync(0xffffffffu, listed);
    if (lane == 0) s_cnt[w] = (unsigned int)__popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int tot = 0;
        for (int i = 0; i < nw; ++i) {
            const unsigned int c = s_cnt[i];
            s_cnt[i] = tot;
            tot += c;
        }
        s_cnt[nw] = tot ? atomicAdd(nout, tot) : 0u;
    }
    __syncthreads();
    if (listed) out[s_cnt[nw] + s_cnt[w] + (unsigned int)__popc(bal & ((1u << lane) - 1u))] = (int32_t)n;
    __syncthreads();  // the counts are reused by the next call
}

// updateLocalMaskNtotalLattices3D. FULL: over every voxel; each thread takes UNR voxels a grid
// stride apart per round and issues their loads together, so the pass is not bound by one voxel's
// latency. Otherwise over the voxels of in[0, n_in) and in2[0, n_in2) (disjoint lists), every other
// voxel being a fixed point of the rule. The voxels whose total exceeds 1e-14 afterwards go to
// `out` (count in sc->nout); max(total), the mask sum (FULL) or its change, and the counts go to
// the pass counters.
template <bool FULL>
__device__ void ca_mask_pass(const CaView& C, const CaBufs& B, CaScalars* sc, const int32_t* __restrict__ in,
                             int n_in, const int32_t* __restrict__ in2, int n_in2, int32_t* __restrict__ out) {
    const Geom G = C.g;
    long long best = 0, msum = 0;  // ordered(+0.0) == 0: totals are never below zero
    const int64_t S = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (FULL) {
        constexpr int UNR = 4;
        // whole warps run the loop together, so the list append is warp-wide
        const int64_t span = (G.N + 31) / 32 * 32;
        if (C.M <= 2) {
            for (int64_t n0 = t0; n0 < span; n0 += UNR * S) {
                int mk[UNR];
                double told[UNR], b0[UNR], b1[UNR];
#pragma unroll
                for (int j = 0; j < UNR; ++j) {
                    const int64_t n = n0 + j * S;
                    const bool inb = n < G.N;
                    mk[j] = inb ? (int)B.mat[n] : C.bb;
                    told[j] = inb ? B.total[n] : 0.0;
                }
                // biomass only where the voxel is open (most voxels of a pack are not)
#pragma unroll
                for (int j = 0; j < UNR; ++j) {
                    const int64_t n = n0 + j * S;
                    const bool op = n < G.N && ca_open(C, mk[j]);
                    b0[j] = op ? B.bio[n] : 0.0;
                    b1[j] = (op && C.M > 1) ? B.bio[G.N + n] : 0.0;
                }
#pragma unroll
                for (int j = 0; j < UNR; ++j) {
                    const int64_t n = n0 + j * S;
                    if (n >= span) break;  // uniform per warp: span and S are multiples of 32
                    bool listed = false;
                    if (n < G.N) {
                        const double bm[2] = {b0[j], b1[j]};
                        listed = ca_mask_voxel<false>(C, B, sc, n, mk[j], told[j], bm, best, msum);
                    }
                    ca_list_append(out, &sc->nout, n, listed);
                }
            }
        } else {
            for (int64_t n = t0; n < span; n += S) {
                bool listed = false;
                if (n < G.N) {
                    double bm[CLB_MAX_MICROBES];
                    for (int m = 0; m < C.M; ++m) bm[m] = B.bio[(int64_t)m * G.N + n];
                    listed = ca_mask_voxel<false>(C, B, sc, n, B.mat[n], B.total[n], bm, best, msum);
                }
                ca_list_append(out, &sc->nout, n, listed);
            }
        }
    } else {
        const int64_t n_all = (int64_t)n_in + n_in2;
        __shared__ unsigned int s_cnt[CA_THREADS / 32 + 1];
        // whole blocks run the loop together (the list append is block-wide)
        for (int64_t jb = (int64_t)blockIdx.x * blockDim.x; jb < n_all; jb += S) {
            const int64_t j = jb + threadIdx.x;
            bool listed = false;
            int64_t n = 0;
            if (j < n_all) {
                n = j < n_in ? in[j] : in2[j - n_in];
                const int mk = B.mat[n];
                double bm[CLB_MAX_MICROBES];
                const bool op = ca_open(C, mk);
                for (int m = 0; m < C.M; ++m) bm[m] = op ? B.bio[(int64_t)m * G.N + n] : 0.0;
                listed = ca_mask_voxel<true>(C, B, sc, n, mk, B.total[n], bm, best, msum);
            }
            ca_list_append_block(out, &sc->nout, n, listed, s_cnt);
        }
    }
    // warp, then block reduction; one atomic per block, and none where the value is the identity
    for (int o = 16; o > 0; o >>= 1) {
        best = max(best, __shfl_down_sync(0xffffffffu, best, o));
        msum += __shfl_down_sync(0xffffffffu, msum, o);
    }
    __shared__ long long s_best[CA_THREADS / 32], s_msum[CA_THREADS / 32];
    if ((threadIdx.x & 31) == 0) {
        s_best[threadIdx.x >> 5] = best;
        s_msum[threadIdx.x >> 5] = msum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long b = 0, m = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            b = max(b, s_best[i]);
            m += s_msum[i];
        }
        if (b > 0) atomicMax(&sc->gmax, b);
        if (m != 0) atomicAdd((unsigned long long*)&sc->msum, (unsigned long long)m);
    }
    __syncthreads();  // the block's partials are reused by the next pass of a cooperative step
}

// ------------------------------------------------------------------ push sweep

// the voxels of x = 1..nx-2 that push, from the biomass list (any voxel above the maximum is on it)
__device__ void ca_collect(const CaView& C, const CaBufs& B, CaScalars* sc, const int32_t* __restrict__ blist,
                           int nb) {
    const Geom G = C.g;
    const int8_t* __restrict__ mat = B.mat;
    const double* __restrict__ total = B.total;
    int* __restrict__ aidx = B.aidx;
    int* __restrict__ act = B.act;
    int* __restrict__ done = B.done;
    const int cap = B.cap;
    const int64_t lo = G.plane, hi = G.N - G.plane;  // x = 1..nx-2
    // whole warps run the loop together: one atomic per warp takes the rows of its active voxels
    const int span = (nb + 31) / 32 * 32;
    const int lane = threadIdx.x & 31;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < span; j += gridDim.x * blockDim.x) {
        bool take = false;
        int64_t n = 0;
        if (j < nb) {
            n = blist[j];
            if (n >= lo && n < hi && ca_open(C, mat[n])) {
                const double t = total[n];
                if (C.half) take = !ca_pore(C, mat[n]) && t > C.bmax;  // 'half': biofilm voxels, any excess
                else take = t > C.bmax && t - C.bmax > THRD;
            }
        }
        const unsigned int bal = __ballot_sync(0xffffffffu, take);
        if (!bal) continue;
        unsigned int base = 0;
        if (lane == 0) base = atomicAdd(&sc->active, (unsigned int)__popc(bal));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (!take) continue;
        const unsigned int i = base + __popc(bal & ((1u << lane) - 1u));
        if ((int)i >= cap) { atomicAdd(&sc->overflow, 1u); continue; }
        act[i] = (int)n;
        aidx[n] = (int)i;
        done[i] = 0;
    }
}

// the pushes source j recorded into voxel n, added in record order
__device__ __forceinline__ void add_records(const CaView& C, int j, int64_t n, const int* __restrict__ tgt,
                                            const double* __restrict__ amt, double* b) {
    for (int t = 0; t < CA_REC; ++t) {
        if (tgt[j * CA_REC + t] != (int)n) continue;
        for (int m = 0; m < C.M; ++m) b[m] += amt[((int64_t)j * CA_REC + t) * C.M + m];
    }
}

__device__ void ca_round(const CaView& C, const CaBufs& B, int count, int round, uint64_t sweep, CaScalars* sc) {
    const Geom G = C.g;
    const int8_t* __restrict__ mat = B.mat;
    const double* __restrict__ total = B.total;
    const int* __restrict__ age = B.age;
    const double* __restrict__ bio = B.bio;
    const int* __restrict__ aidx = B.aidx;
    const int* __restrict__ act = B.act;
    int* __restrict__ done = B.done;
    int* __restrict__ tgt = B.tgt;
    double* __restrict__ amt = B.amt;
    double* __restrict__ own = B.own;
    const uint64_t seed = B.seed;
    unsigned int fin = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        if (done[i]) continue;
        const int64_t n = act[i];
        int x, y, z;
        decode(G, n, x, y, z);
        // sources that push before this voxel in lexicographic order: x-1, y-1, z-1
        int pre[3] = {-1, -1, -1};
        if (x > 1) pre[0] = aidx[n - G.plane];
        if (y > 0) pre[1] = aidx[n - G.nz];
        if (z > 0) pre[2] = aidx[n - 1];
        bool ready = true;
        for (int q = 0; q < 3; ++q)
            if (pre[q] >= 0) {
                const int dq = done[pre[q]];
                if (dq == 0 || dq == round) ready = false;
            }
        if (!ready) continue;
        double b[CLB_MAX_MICROBES];
        for (int m = 0; m < C.M; ++m) b[m] = bio[(int64_t)m * G.N + n];
        for (int q = 0; q < 3; ++q)
            if (pre[q] >= 0) add_records(C, pre[q], n, tgt, amt, b);
        for (int t = 0; t < CA_REC; ++t) tgt[i * CA_REC + t] = -1;
        double bMt = total[n];
        double bMd = C.half ? bMt * 0.5 : bMt - C.bmax;  // 'half' pushes half the voxel's biomass
        int64_t nb[6];
        int L = 0;
        const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        for (int d = 0; d < 6; ++d) {
            const int X = x + d6[d][0], Y = y + d6[d][1], Z = z + d6[d][2];
            if (X < 1 || X > G.nx - 2 || Y < 0 || Y >= G.ny || Z < 0 || Z >= G.nz) continue;
            const int64_t m = (int64_t)X * G.plane + (int64_t)Y * G.nz + Z;
            if (!ca_open(C, mat[m])) continue;
            nb[L++] = m;
        }
        uint64_t st = seed ^ (sweep * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)n * 0xD1B54A32D192ED03ULL);
        int perm[6] = {0, 1, 2, 3, 4, 5};
        if (L > 1)
            for (int a = L - 1; a >= 1; --a) {
                const int j = (int)(sm64(st) % (uint64_t)(a + 1));
                const int tmp = perm[a];
                perm[a] = perm[j];
                perm[j] = tmp;
            }
        int rec = 0;
        bool chk = false;
        for (int t = 0; t < L; ++t) {
            const int64_t m = nb[L > 1 ? perm[t] : 0];
            const double nbrbMt = ca_pore(C, mat[m]) ? 0.0 : total[m];
            if (nbrbMt < C.bmax) {
                const double hold = C.bmax - nbrbMt;
                double partial = bMd;
                if (bMd > hold) { partial = hold; bMd -= hold; }
                else { bMd = 0.0; chk = true; }
                tgt[i * CA_REC + rec] = (int)m;
                for (int mi = 0; mi < C.M; ++mi) {
                    const double shove = b[mi] / bMt * partial;
                    double give = 0.0;
                    if (shove > THRD) {
                        b[mi] -= shove;
                        give = shove;
                    }
                    amt[((int64_t)i * CA_REC + rec) * C.M + mi] = give;
                }
                ++rec;
                bMt -= partial;
            }
            if (chk) break;
        }
        if (!chk && L > 0) {
            const int id0 = age[n];
            int64_t cand[6];
            int c = 0;
            for (int t = 0; t < L; ++t)
                if (C.half ? id0 >= age[nb[t]] : id0 > age[nb[t]]) cand[c++] = nb[t];
            int64_t m;
            if (c > 1) m = cand[sm64(st) % (uint64_t)c];
            else if (c == 1) m = cand[0];
            else m = nb[L > 1 ? (int)(sm64(st) % (uint64_t)L) : 0];
            tgt[i * CA_REC + rec] = (int)m;
            for (int mi = 0; mi < C.M; ++mi) {
                const double shove = b[mi] / bMt * bMd;
                b[mi] -= shove;
                amt[((int64_t)i * CA_REC + rec) * C.M + mi] = shove;
            }
        } else if (C.half) {
            // 'half' always makes the last push; with everything placed (bMd = 0) or no open
            // neighbour its target is the voxel itself: subtracted, then added back
            for (int mi = 0; mi < C.M; ++mi) {
                const double shove = b[mi] / bMt * bMd;
                b[mi] -= shove;
                b[mi] += shove;
            }
        }
        for (int m = 0; m < C.M; ++m) own[(int64_t)i * C.M + m] = b[m];
        done[i] = round;
        ++fin;
    }
    // the voxels this round finished, one atomic per warp (every lane reaches this point)
    for (int o = 16; o > 0; o >>= 1) fin += __shfl_down_sync(0xffffffffu, fin, o);
    if ((threadIdx.x & 31) == 0 && fin) atomicSub(&sc->remaining, fin);
}

// The voxels a sweep pushed into that are not active themselves, each once (ext), and of those the
// ones off the biomass list (ext2: their total is at most 1e-14, which is the list's criterion;
// the total changes only in mask passes). Every voxel whose biomass the sweep changes is active
// or on ext.
__device__ void ca_targets(const CaBufs& B, CaScalars* sc, int count) {
    const int* __restrict__ tgt = B.tgt;
    const int* __restrict__ aidx = B.aidx;
    const double* __restrict__ total = B.total;
    // whole warps run the loop together, so the appends take one atomic per warp
    const int span = (count + 31) / 32 * 32;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < span; i += gridDim.x * blockDim.x) {
        for (int t = 0; t < CA_REC; ++t) {
            bool take = false, off_list = false;
            int m = 0;
            if (i < count) {
                m = tgt[i * CA_REC + t];
                if (m >= 0 && aidx[m] < 0 && atomicExch(&B.tmark[m], 1) == 0) {
                    take = true;
                    off_list = !(total[m] > 1e-14);
                }
            }
            ca_list_append(B.ext, &sc->next, m, take);
            ca_list_append(B.ext2, &sc->next2, m, off_list);
        }
    }
}

// every voxel takes the pushes it received, in the order the sequential sweep adds them: the
// active voxels (act[0, count)) and the voxels they pushed into (ext[0, next)); no other voxel's
// biomass changes
__device__ void ca_apply(const CaView& C, const CaBufs& B, int count, int next) {
    const Geom G = C.g;
    double* __restrict__ bio = B.bio;
    const int* __restrict__ aidx = B.aidx;
    const int* __restrict__ tgt = B.tgt;
    const double* __restrict__ amt = B.amt;
    const double* __restrict__ own = B.own;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count + next; j += gridDim.x * blockDim.x) {
        const int64_t n = j < count ? B.act[j] : B.ext[j - count];
        int x, y, z;
        decode(G, n, x, y, z);
        const int a = aidx[n];
        int pre[3] = {-1, -1, -1}, post[3] = {-1, -1, -1};
        if (x > 1) pre[0] = aidx[n - G.plane];
        if (y > 0) pre[1] = aidx[n - G.nz];
        if (z > 0) pre[2] = aidx[n - 1];
        if (z < G.nz - 1) post[0] = aidx[n + 1];
        if (y < G.ny - 1) post[1] = aidx[n + G.nz];
        if (x < G.nx - 2) post[2] = aidx[n + G.plane];
        if (a < 0 && pre[0] < 0 && pre[1] < 0 && pre[2] < 0 && post[0] < 0 && post[1] < 0 && post[2] < 0) continue;
        double b[CLB_MAX_MICROBES];
        if (a >= 0) {
            for (int m = 0; m < C.M; ++m) b[m] = own[(int64_t)a * C.M + m];
        } else {
            for (int m = 0; m < C.M; ++m) b[m] = bio[(int64_t)m * G.N + n];
            for (int q = 0; q < 3; ++q)
                if (pre[q] >= 0) add_records(C, pre[q], n, tgt, amt, b);
        }
        for (int q = 0; q < 3; ++q)
            if (post[q] >= 0) add_records(C, post[q], n, tgt, amt, b);
        for (int m = 0; m < C.M; ++m) bio[(int64_t)m * G.N + n] = b[m];
    }
}

__device__ void ca_clear(const CaBufs& B, int count, int next) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count + next; i += gridDim.x * blockDim.x) {
        if (i < count) B.aidx[B.act[i]] = -1;
        else B.tmark[B.ext[i - count]] = 0;
    }
}

// ------------------------------------------------------------------ age wavefront

// new age of voxel n from the ages it sees (updateAgeDistance3D); returns the old age when unchanged
__device__ __forceinline__ int age_rule(const CaView& C, int64_t n, const int* age,
                                        const int8_t* __restrict__ distp, const double* __restrict__ total) {
    const Geom G = C.g;
    const int a = age[n];
    const double B = total[n];
    if (!(B > 1e-14)) return a;
    int x, y, z;
    decode(G, n, x, y, z);
    int64_t D[6];
    int nd = 0;
    const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int d = 0; d < 6; ++d) {
        const int X = x + d6[d][0], Y = y + d6[d][1], Z = z + d6[d][2];
        if (X < 0 || Y < 0 || Z < 0 || X >= G.nx || Y >= G.ny || Z >= G.nz) continue;
        const int64_t m = (int64_t)X * G.plane + (int64_t)Y * G.nz + Z;
        if (distp[m]) D[nd++] = m;
    }
    if (a == 0) return 1;
    if (a == 1 && (B - C.bmax) > -1e-14) {
        for (int t = 0; t < nd; ++t)
            if (age[D[t]] == 0) return a;
        return 2;
    }
    int cnt = 0;
    for (int t = 0; t < nd; ++t)
        if (age[D[t]] >= a && (total[D[t]] - C.bmax) > -1e-14) ++cnt;
    return cnt == nd ? a + 1 : a;
}

// One relaxation sweep over the biomass list, in place (the rule leaves every other voxel as it
// is). A voxel may read a neighbour's age before or after that neighbour's update in the same
// sweep: both are iterates of the same monotone, inflationary rule, so the sweeps still reach the
// least fixed point above the start, the one the reference's in-place sweeps reach, and a sweep
// that changes nothing has read only final values.
__device__ void ca_age_relax(const CaView& C, const CaBufs& B, CaScalars* sc, const int32_t* __restrict__ blist,
                             int nb) {
    int* age = B.age;
    const int8_t* __restrict__ distp = B.distp;
    const double* __restrict__ total = B.total;
    unsigned int ch = 0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nb; j += gridDim.x * blockDim.x) {
        const int64_t n = blist[j];
        const int old = age[n];
        const int v = age_rule(C, n, age, distp, total);
        if (v != old) {
            age[n] = v;
            ++ch;
        }
    }
    for (int o = 16; o > 0; o >>= 1) ch += __shfl_down_sync(0xffffffffu, ch, o);
    if ((threadIdx.x & 31) == 0 && ch) atomicAdd(&sc->changed, ch);
}

// voxels with x + y + z = level, in place
__device__ void ca_age_level(const CaView& C, const CaBufs& B, int level) {
    const Geom G = C.g;
    int* age = B.age;
    const int8_t* __restrict__ distp = B.distp;
    const double* __restrict__ total = B.total;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)G.nx * G.ny;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t / G.ny), y = (int)(t - (int64_t)x * G.ny);
        const int z = level - x - y;
        if (z < 0 || z >= G.nz) continue;
        const int64_t n = (int64_t)x * G.plane + (int64_t)y * G.nz + z;
        age[n] = age_rule(C, n, age, distp, total);
    }
}

// ------------------------------------------------------------------ one step, on the device

// The step's first mask pass as an ordinary launch over every resident thread the pass can use
// (many more than the cooperative step keeps resident): over the whole box when `full`, else over
// the biomass list; it writes the other list buffer. The step before cleared its counters.
__global__ void __launch_bounds__(CA_THREADS) k_ca_mask_first(const CaView C, const CaBufs B, CaScalars* sc, int full) {
    if (sc->status != CA_OK) return;
    if (B.mask0) return;  // several pore codes: the cooperative step snapshots the mask and runs this pass
    const int cur = sc->list;
    if (full) ca_mask_pass<true>(C, B, sc, nullptr, 0, nullptr, 0, B.list[cur ^ 1]);
    else ca_mask_pass<false>(C, B, sc, B.list[cur], (int)sc->nlist, nullptr, 0, B.list[cur ^ 1]);
}

// the mask as it stands before a pass, for the reopening rule with several pore codes
__device__ __forceinline__ void ca_snapshot_mask(const CaView& C, const CaBufs& B) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < C.g.N; n += (int64_t)gridDim.x * blockDim.x)
        B.mask0[n] = B.mat[n];
}

__device__ __forceinline__ double unordered_dev(long long i) {
    if (i < 0) i ^= 0x7FFFFFFFFFFFFFFFLL;
    return __longlong_as_double(i);
}

// the counters of a mask pass, cleared by one thread ahead of a barrier
__device__ __forceinline__ void ca_pass_reset(CaScalars* sc) {
    sc->gmax = 0;  // ordered(+0.0)
    sc->msum = 0;
    sc->nonfinite = 0;
    sc->nout = 0;
}

// One step of the automaton (ca_step's sequence: mask pass; while max(total) exceeds Bmax, push
// sweeps with their mask passes, the stall and sweep limits and, every 50 sweeps, the age
// relaxation; the in-place age sweep after a mask change) in one cooperative launch, with grid-wide
// barriers between the phases, so no phase waits for the host. Every block makes the same decisions
// from values it reads after a barrier; a value is changed again only after a further barrier, so no
// block can read a later value than another. Every loop is bounded: rounds by the active count
// (each round finishes at least the lexicographically first unfinished voxel), sweeps by 1001, age
// sweeps by 1001 per relaxation. A failure is recorded in `status` with the iteration and later
// steps do nothing until the host has read it. The biomass list alternates between two buffers:
// every block tracks which one is current and its length, and the step leaves both for the next.
__global__ void __launch_bounds__(CA_THREADS, 4) k_ca_step(const CaView C, const CaBufs B, CaScalars* sc, int iter,
                                                            int full) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    // `status`, `list`, `nlist` and `mask_run` are written only after the last barrier of a step, so
    // every block reads the same values
    if (sc->status != CA_OK) return;
    int cur = sc->list;
    int nlist = (int)sc->nlist;
    if (B.mask0) {
        // the first pass, which k_ca_mask_first leaves to this launch with several pore codes
        ca_snapshot_mask(C, B);
        grid.sync();
        if (full) ca_mask_pass<true>(C, B, sc, nullptr, 0, nullptr, 0, B.list[cur ^ 1]);
        else ca_mask_pass<false>(C, B, sc, B.list[cur], nlist, nullptr, 0, B.list[cur ^ 1]);
    }
    grid.sync();
    double gmax = unordered_dev(sc->gmax);
    long long msum = full ? sc->msum : sc->mask_run + sc->msum;  // the mask sum now
    int status = (sc->nonfinite || !isfinite(gmax)) ? CA_NONFINITE : CA_OK;
    cur ^= 1;
    nlist = (int)sc->nout;
    uint64_t sweep = sc->sweep_counter;
    const long long mask_sum0 = sc->ca_mask_sum;
    grid.sync();
    int whilecount = 0, stall = 0, count = 0, next = 0;
    double prev = gmax;
    if (status == CA_OK && gmax - C.bmax > THRD) {
        while (gmax - C.bmax > THRD) {
            // ---- push sweep: the voxels above the maximum, their rounds, the pushes applied
            if (lead) {
                sc->active = 0;
                sc->overflow = 0;
                sc->next = 0;
                sc->next2 = 0;
            }
            grid.sync();
            ca_collect(C, B, sc, B.list[cur], nlist);
            grid.sync();
            count = (int)sc->active;
            const bool over = sc->overflow != 0;
            grid.sync();
            if (over) {
                count = count < B.cap ? count : B.cap;  // the rows written; cleared below
                status = CA_CAPACITY;
                break;
            }
            int next2 = 0;
            next = 0;
            if (count > 0) {
                if (lead) sc->remaining = (unsigned int)count;
                grid.sync();
                for (int round = 1;; ++round) {
                    ca_round(C, B, count, round, sweep, sc);
                    grid.sync();
                    const unsigned int rem = sc->remaining;
                    grid.sync();
                    if (rem == 0) break;
                    if (round >= count) { status = CA_ROUNDS; break; }
                }
                if (status != CA_OK) break;
                ca_targets(B, sc, count);
                grid.sync();
                next = (int)sc->next;
                next2 = (int)sc->next2;
                ca_apply(C, B, count, next);
                grid.sync();
                ca_clear(B, count, next);
                count = next = 0;
            }
            ++sweep;
            // ---- mask pass after the sweep: the list and the voxels pushed into off it
            if (lead) ca_pass_reset(sc);
            if (B.mask0) ca_snapshot_mask(C, B);
            grid.sync();
            ca_mask_pass<false>(C, B, sc, B.list[cur], nlist, B.ext2, next2, B.list[cur ^ 1]);
            grid.sync();
            gmax = unordered_dev(sc->gmax);
            msum += sc->msum;
            cur ^= 1;
            nlist = (int)sc->nout;
            const bool nonf = sc->nonfinite != 0;
            grid.sync();
            if (nonf || !isfinite(gmax)) { status = CA_NONFINITE; break; }
            if (gmax > prev - THRD) {
                if (++stall >= 100) { status = CA_STALL; break; }
            } else {
                stall = 0;
            }
            prev = gmax;
            if (whilecount % 50 == 0) {
                bool settled = false;
                for (int k = 0; k < 1001 && !settled; ++k) {
                    if (lead) sc->changed = 0;
                    grid.sync();
                    ca_age_relax(C, B, sc, B.list[cur], nlist);
                    grid.sync();
                    settled = sc->changed == 0;
                    grid.sync();
                }
                if (!settled) { status = CA_AGE; break; }
            }
            if (whilecount > 1000) { status = CA_SWEEPS; break; }
            ++whilecount;
        }
    }
    // a sweep that stopped before its pushes were applied leaves its active voxels marked: unmark
    // them (after the barrier the break followed), so the handle can step again once the host has
    // read the failure
    if (count > 0) ca_clear(B, count, 0);
    bool changed = false;
    if (status != CA_NONFINITE) {
        // after the block, a changed mask takes one in-place age sweep (wavefronts over x + y + z)
        changed = msum != mask_sum0;
        if (changed) {
            const int levels = C.g.nx + C.g.ny + C.g.nz - 2;
            for (int l = 0; l < levels; ++l) {
                ca_age_level(C, B, l);
                grid.sync();
            }
        }
    }
    // every block read the counters before a barrier it has passed, so the lead may reset them
    if (lead) {
        sc->step_sweeps = whilecount;
        sc->step_changed = changed ? 1 : 0;
        if (changed) sc->ca_mask_sum = msum;
        sc->mask_run = msum;
        sc->list = cur;
        sc->nlist = (unsigned int)nlist;
        sc->sweep_counter = sweep;
        sc->total_sweeps += whilecount;
        sc->total_changes += changed ? 1 : 0;
        if (sc->moved) sc->moved_any = 1;
        sc->moved = 0;
        ca_pass_reset(sc);  // for the next step's first pass
        if (status != CA_OK) {
            sc->status = status;
            sc->fail_iter = iter;
        }
    }
}

// ------------------------------------------------------------------ dynamics refresh

// updateSoluteDynamics3D: open voxels take the pore or the biofilm dynamics from the mask
// guard: when given, the pass acts only if the automaton's last step changed the mask
__global__ void k_refresh_species(int8_t* __restrict__ code, const int32_t* __restrict__ node, int64_t K,
                                  const int8_t* __restrict__ mat, const CaView C, int bio0, const int* guard) {
    if (guard && *guard == 0) return;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int m = mat[node[k]];
        if (!ca_open(C, m)) continue;
        code[k] = (int8_t)(ca_pore(C, m) ? m : bio0);
    }
}

// updateNsLatticesDynamics3D (complab3d_processors_part2.hh:785-806): a biofilm voxel with the
// pore dynamics takes the biofilm dynamics of the first microbe, a pore voxel with any other
// dynamics the pore dynamics; solid and wall voxels keep theirs.
__global__ void k_refresh_flow_map(int8_t* __restrict__ fmat, const int8_t* __restrict__ mat, const CaView C,
                                   const FlowParams F, double pore_omega, int bio0) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < C.g.N; n += (int64_t)gridDim.x * blockDim.x) {
        const int m = mat[n];
        if (!ca_open(C, m)) continue;
        const int prev = fmat[n];
        const bool pore_dyn = F.dyn[prev & 127] == DYN_BGK && fabs(F.omega[prev & 127] - pore_omega) < 1e-14;
        if (ca_pore(C, m)) {
            if (!pore_dyn) fmat[n] = (int8_t)m;
        } else if (pore_dyn && bio0 >= 0) {
            fmat[n] = (int8_t)bio0;
        }
    }
}

__global__ void k_codes_from_map(int8_t* __restrict__ code, const int32_t* __restrict__ node, int64_t K,
                                 const int8_t* __restrict__ map) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x)
        code[k] = map[node[k]];
}

// ------------------------------------------------------------------ host side

static CaScalars* SC(clb_handle* h) { return static_cast<CaScalars*>(h->d_ca_sc); }

static CaView ca_view(const clb_handle* h) {
    CaView C;
    std::memset(&C, 0, sizeof C);
    C.g = h->g;
    C.bmax = h->ca_bmax;
    C.thr = h->ca_frac * h->ca_bmax;
    C.M = h->M;
    C.half = h->ca_half;
    C.bb = h->d.bounce_back_code;
    C.solid = h->d.solid_code;
    C.n_pore = h->d.n_pore_codes > 0 ? h->d.n_pore_codes : 1;
    if (h->d.n_pore_codes > 0)
        for (int i = 0; i < h->d.n_pore_codes; ++i) C.pore[i] = h->d.pore_codes[i];
    else
        C.pore[0] = 2;
    for (int m = 0; m < CLB_MAX_MICROBES; ++m) C.bio_code[m] = m < h->d.n_microbes ? h->d.bio_codes[m] : 0;
    return C;
}

void ca_free(clb_handle* h) {
    cudaFree(h->d_ca_total); h->d_ca_total = nullptr;
    cudaFree(h->d_ca_age); h->d_ca_age = nullptr;
    for (int i = 0; i < 2; ++i) {
        cudaFree(h->d_ca_list[i]);
        h->d_ca_list[i] = nullptr;
    }
    cudaFree(h->d_ca_ext); h->d_ca_ext = nullptr;
    cudaFree(h->d_ca_ext2); h->d_ca_ext2 = nullptr;
    cudaFree(h->d_ca_tmark); h->d_ca_tmark = nullptr;
    if (h->h_ca_pin) cudaFreeHost(h->h_ca_pin);
    h->h_ca_pin = nullptr;
    cudaFree(h->d_ca_distp); h->d_ca_distp = nullptr;
    cudaFree(h->d_ca_aidx); h->d_ca_aidx = nullptr;
    cudaFree(h->d_ca_act); h->d_ca_act = nullptr;
    cudaFree(h->d_ca_done); h->d_ca_done = nullptr;
    cudaFree(h->d_ca_tgt); h->d_ca_tgt = nullptr;
    cudaFree(h->d_ca_amt); h->d_ca_amt = nullptr;
    cudaFree(h->d_ca_own); h->d_ca_own = nullptr;
    cudaFree(h->d_ca_sc); h->d_ca_sc = nullptr;
    cudaFree(h->d_ca_mask0); h->d_ca_mask0 = nullptr;
    h->ca_cap = 0;
    h->ca_ready = false;
}

static clb_status ca_reserve(clb_handle* h, int cap) {
    cudaFree(h->d_ca_act); cudaFree(h->d_ca_done); cudaFree(h->d_ca_tgt); cudaFree(h->d_ca_amt); cudaFree(h->d_ca_own);
    h->d_ca_act = h->d_ca_done = h->d_ca_tgt = nullptr;
    h->d_ca_amt = h->d_ca_own = nullptr;
    const int M = std::max(1, h->M);
    cudaError_t e = cudaMalloc(&h->d_ca_act, sizeof(int) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_done, sizeof(int) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_tgt, sizeof(int) * cap * CA_REC);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_amt, sizeof(double) * (size_t)cap * CA_REC * M);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_own, sizeof(double) * (size_t)cap * M);
    if (e != cudaSuccess) return cuda_check(h, e, "cellular automaton buffers");
    h->ca_cap = cap;
    return CLB_OK;
}

clb_status ca_setup(clb_handle* h, const clb_ca_desc* d) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (h->M < 1 || !h->d_bio) return fail(h, CLB_INVALID_ARG, "the automaton needs biomass fields (clb_set_biomass)");
    if (h->M > h->d.n_microbes) return fail(h, CLB_INVALID_ARG, "every biomass field needs a biofilm material code");
    if (!(d->max_biomass > 0)) return fail(h, CLB_INVALID_ARG, "max_biomass must be positive");
    if (d->push_mode != CLB_PUSH_FRACTION && d->push_mode != CLB_PUSH_HALF)
        return fail(h, CLB_INVALID_ARG, "push_mode is CLB_PUSH_FRACTION or CLB_PUSH_HALF");
    int codesum = 0;
    for (int m = 0; m < h->M; ++m) codesum += h->d.bio_codes[m];
    if (codesum > 127) return fail(h, CLB_INVALID_ARG, "the sum of the biofilm codes must fit a material code");
    ca_free(h);
    const size_t N = (size_t)h->g.N;
    cudaError_t e = cudaMalloc(&h->d_ca_total, sizeof(double) * N);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_age, sizeof(int) * N);
    for (int i = 0; i < 2; ++i)
        if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_list[i], sizeof(int32_t) * N);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_ext, sizeof(int32_t) * N);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_ext2, sizeof(int32_t) * N);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_tmark, sizeof(int) * N);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_ca_tmark, 0, sizeof(int) * N, h->stream);
    if (e == cudaSuccess) e = cudaHostAlloc(&h->h_ca_pin, 3 * sizeof(CaScalars), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_distp, N);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_aidx, sizeof(int) * N);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ca_sc, sizeof(CaScalars));
    if (e == cudaSuccess && h->d.n_pore_codes > 1) e = cudaMalloc(&h->d_ca_mask0, N);
    if (e != cudaSuccess) return cuda_check(h, e, "cellular automaton fields");
    // room for every voxel that can push (open voxels of x = 1..nx-2), so a sweep never overflows
    int open_inner = 0;
    {
        clb_status hs = host_mat_sync(h);
        if (hs != CLB_OK) return hs;
        const CaView C0 = ca_view(h);
        auto open_code = [&](int m) { return m != C0.bb && m != C0.solid; };  // ca_open
        for (int64_t n = h->g.plane; n < h->g.N - h->g.plane; ++n) open_inner += open_code(h->h_mat[n]) ? 1 : 0;
    }
    clb_status st = ca_reserve(h, std::max(1024, open_inner));
    if (st != CLB_OK) return st;
    if (!h->d_mat_flow) {
        // from now on the mask moves with the automaton; the flow keeps its own map until a refresh
        h->h_mat_flow = h->h_mat;
        e = cudaMalloc(&h->d_mat_flow, N);
        if (e == cudaSuccess) e = cudaMemcpy(h->d_mat_flow, h->h_mat_flow.data(), N, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_check(h, e, "flow material map");
    }
    h->ca_bmax = d->max_biomass;
    h->ca_frac = d->biofilm_fraction;
    h->ca_half = d->push_mode;
    h->ca_seed = d->seed;
    h->ca_sweeps = 0;
    // pinned copies: [1] read back ([0] and [2] unused)
    CaScalars* pin = static_cast<CaScalars*>(h->h_ca_pin);
    std::memset(pin, 0, 3 * sizeof(CaScalars));
    // all counters zero: the first pass's are cleared (gmax 0 is ordered(+0.0)), the list is empty,
    // and the first step's pass runs over the whole box
    cudaMemsetAsync(SC(h), 0, sizeof(CaScalars), h->stream);
    h->ca_full = true;
    const CaView C = ca_view(h);
    k_ca_init<<<h->num_sms * 8, CA_THREADS, 0, h->stream>>>(C, h->d_mat, h->d_bio, h->d_ca_total, h->d_ca_age,
                                                             h->d_ca_distp, h->d_ca_aidx, SC(h));
    // the mask sum the steps compare against
    cudaMemcpyAsync(&SC(h)->ca_mask_sum, &SC(h)->mask_run, sizeof(long long), cudaMemcpyDeviceToDevice, h->stream);
    CaScalars s;
    e = cudaMemcpyAsync(&s, SC(h), sizeof s, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_check(h, e, "cellular automaton set-up");
    h->ca_mask_sum = s.mask_run;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_ca_step, CA_THREADS, 0);
    if (e != cudaSuccess || per_sm < 1) return cuda_check(h, e == cudaSuccess ? cudaErrorLaunchOutOfResources : e, "automaton step");
    h->ca_grid = h->num_sms * per_sm;  // every resident block: the full-box passes are latency-bound
    h->ca_ready = true;
    return CLB_OK;
}

static clb_status ca_scalars(clb_handle* h, CaScalars& s) {
    CaScalars* pin = static_cast<CaScalars*>(h->h_ca_pin);
    cudaError_t e = cudaMemcpyAsync(&pin[1], SC(h), sizeof s, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    s = pin[1];
    return e == cudaSuccess ? CLB_OK : cuda_check(h, e, "cellular automaton counters");
}

// mask / total pass; returns max(total) and the mask sum
static CaBufs ca_bufs(clb_handle* h) {
    CaBufs B;
    B.mat = h->d_mat;
    B.mask0 = h->d_ca_mask0;
    B.bio = h->d_bio;
    B.total = h->d_ca_total;
    B.age = h->d_ca_age;
    B.distp = h->d_ca_distp;
    B.aidx = h->d_ca_aidx;
    B.act = h->d_ca_act;
    B.done = h->d_ca_done;
    B.tgt = h->d_ca_tgt;
    B.amt = h->d_ca_amt;
    B.own = h->d_ca_own;
    B.list[0] = h->d_ca_list[0];
    B.list[1] = h->d_ca_list[1];
    B.ext = h->d_ca_ext;
    B.ext2 = h->d_ca_ext2;
    B.tmark = h->d_ca_tmark;
    B.bflag = h->d_bflag;
    B.sidx = h->ade_sp.idx_of;
    B.cap = h->ca_cap;
    B.seed = h->ca_seed;
    return B;
}

// Enqueues one step of the automaton (k_ca_step); `iter` is the iteration a failure is recorded with.
clb_status ca_step_async(clb_handle* h, int64_t iter) {
    if (!h->ca_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ca_setup first");
    CaView C = ca_view(h);
    CaBufs B = ca_bufs(h);
    CaScalars* sc = SC(h);
    int it = (int)std::min<int64_t>(iter, INT32_MAX);
    int full = h->ca_full ? 1 : 0;  // biomass or the map written outside the automaton: whole box
    void* args[] = {&C, &B, &sc, &it, &full};
    // the first pass (its counters were cleared by the step before), then the rest of the step
    h->launches += 2;
    k_ca_mask_first<<<h->num_sms * 8, CA_THREADS, 0, h->stream>>>(C, B, sc, full);
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_ca_step, dim3(h->ca_grid), dim3(CA_THREADS), args, 0,
                                                h->stream);
    if (e == cudaSuccess) h->ca_full = false;
    return cuda_check(h, e, "automaton step");
}

// Reads the automaton's results back (synchronises): the last step's sweeps and mask change, the
// totals, and a failure a step recorded (cleared once read, so the handle can step again).
clb_status ca_read(clb_handle* h, int* step_sweeps, int* step_changed, int64_t* total_sweeps, int64_t* total_changes) {
    CaScalars s;
    clb_status st = ca_scalars(h, s);
    if (st != CLB_OK) return st;
    if (step_sweeps) *step_sweeps = s.step_sweeps;
    if (step_changed) *step_changed = s.step_changed;
    if (total_sweeps) *total_sweeps = s.total_sweeps;
    if (total_changes) *total_changes = s.total_changes;
    h->ca_sweeps = s.sweep_counter;
    if (s.moved_any) {
        cudaMemsetAsync(&SC(h)->moved_any, 0, sizeof(unsigned int), h->stream);
        h->h_mat_stale = true;
        if ((st = geometry_refresh(h)) != CLB_OK) return st;
    }
    if (s.status == CA_OK) return CLB_OK;
    cudaMemsetAsync(&SC(h)->status, 0, sizeof(int), h->stream);
    const std::string at = " (iteration " + std::to_string(s.fail_iter) + ")";
    switch (s.status) {
        case CA_NONFINITE: return fail(h, CLB_NONFINITE, "non-finite biomass (NaN or Inf) in the biofilm fields" + at);
        case CA_STALL: return fail(h, CLB_NOT_CONVERGED, "biofilm push stalled: excess biomass cannot spread" + at);
        case CA_AGE: return fail(h, CLB_NOT_CONVERGED, "age relaxation did not settle in 1000 sweeps" + at);
        case CA_SWEEPS: return fail(h, CLB_NOT_CONVERGED, "biofilm push did not settle in 1000 sweeps" + at);
        default: return fail(h, CLB_CUDA_ERROR, "automaton step: active voxels beyond the sweep's bounds" + at);
    }
}

// One step of the automaton, synchronously (clb_ca_step): the results are read back at once.
clb_status ca_step(clb_handle* h, int* sweeps_out, int* mask_changed) {
    if (!h->ca_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ca_setup first");
    clb_status st = ca_step_async(h, h->ade_iters);
    if (st == CLB_OK) st = ca_read(h, sweeps_out, mask_changed, nullptr, nullptr);
    return st;
}

clb_status refresh_dynamics(clb_handle* h, int species, int flow) {
    const CaView C = ca_view(h);
    const int bio0 = h->d.n_microbes > 0 ? h->d.bio_codes[0] : -1;
    const int grid = h->num_sms * 8;
    if (species && h->ade_ready) ++h->launches;
    if (species && h->ade_ready)
        k_refresh_species<<<grid, CA_THREADS, 0, h->stream>>>(h->ade_sp.code, h->ade_sp.node, h->ade_sp.K, h->d_mat, C,
                                                              bio0, nullptr);
    if (flow && h->flow_ready) {
        const int64_t N = h->g.N;
        cudaError_t e = cudaSuccess;
        if (!h->d_mat_flow) {
            h->h_mat_flow = h->h_mat;
            e = cudaMalloc(&h->d_mat_flow, (size_t)N);
            if (e == cudaSuccess)
                e = cudaMemcpy(h->d_mat_flow, h->h_mat_flow.data(), (size_t)N, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return cuda_check(h, e, "flow material map");
        }
        h->launches += 2;
        k_refresh_flow_map<<<grid, CA_THREADS, 0, h->stream>>>(h->d_mat_flow, h->d_mat, C, h->fp, 1.0 / h->d.tau, bio0);
        k_codes_from_map<<<grid, CA_THREADS, 0, h->stream>>>(h->flow_sp.code, h->flow_sp.node, h->flow_sp.K, h->d_mat_flow);
        h->h_mat_flow.resize((size_t)N);
        e = cudaMemcpyAsync(h->h_mat_flow.data(), h->d_mat_flow, (size_t)N, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_check(h, e, "flow material map");
        int64_t nbgk = 0;
        for (int64_t n = 0; n < N; ++n) nbgk += h->fp.dyn[(uint8_t)h->h_mat_flow[n] & 127] == DYN_BGK;
        h->fp.n_bgk = nbgk;
    }
    return cuda_check(h, cudaGetLastError(), "dynamics refresh");
}

// updateSoluteDynamics3D enqueued after an automaton step, acting only if that step changed the mask
clb_status refresh_species_if_changed(clb_handle* h) {
    const CaView C = ca_view(h);
    const int bio0 = h->d.n_microbes > 0 ? h->d.bio_codes[0] : -1;
    ++h->launches;
    k_refresh_species<<<h->num_sms * 8, CA_THREADS, 0, h->stream>>>(h->ade_sp.code, h->ade_sp.node, h->ade_sp.K,
                                                                     h->d_mat, C, bio0, &SC(h)->step_changed);
    return cuda_check(h, cudaGetLastError(), "dynamics refresh");
}

clb_status ca_fields(clb_handle* h, int which, double* host) {
    if (!h->ca_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ca_setup first");
    const size_t N = (size_t)h->g.N;
    cudaError_t e;
    if (which == 0) {
        e = cudaMemcpy(host, h->d_ca_total, sizeof(double) * N, cudaMemcpyDeviceToHost);
    } else {
        std::vector<int> a(N);
        e = cudaMemcpy(a.data(), h->d_ca_age, sizeof(int) * N, cudaMemcpyDeviceToHost);
        for (size_t n = 0; n < N; ++n) host[n] = a[n];
    }
    return cuda_check(h, e, "automaton field");
}

}  // namespace clb

// flow.cu -- D3Q19 incompressible BGK flow lattice on the AA in-place pattern.
//
// Reference behaviour (Palabos dynamics installed by NSdomainSetup,
// complab_functions.hh:296-345, driven by complab.cpp:1095-1206):
//   IncBGK collision with per-material omega (pore, biofilm: omega_bio =
//   1/(permRatio (1/omega - 1/2) + 1/2), :323), BounceBack walls (full-way: populations are
//   held one step in the wall node), NoDynamics solids (no collision, populations stream
//   through), Palabos' local regularized density boundary on the planes x = 0 (rho = 1) and
//   x = nx-1 (rho = 1 - 3 dP), reflection of populations whose source lies outside the box.
//
// Layout: only collide-or-stream nodes are stored (sparse.cuh): f[19][K] of the storage type
// in lexicographic node order, plus one link slot per (node, direction into a wall). One array,
// updated in place with the AA pattern:
//   even step: node a reads f[i][a], collides, writes outgoing i to f[opp(i)][a];
//   odd step:  node a reads incoming i from f[opp(i)][a - c_i], collides, writes outgoing
//              i to f[i][a + c_i].
// Each slot is read and written by exactly one node per step, so a step needs no second array
// and no synchronisation. A full-way bounce-back node is the identity on its AA slots, so it is
// never launched; each link from a stored node into a wall is a two-step delay line held in the
// node's own opposite slot on odd steps and in a link slot on even steps (sparse.cuh). A source
// or destination outside the box maps to the node's own opposite slot: Palabos' reflection at the
// block edge. The even step touches only the node's own slots and its link slots; the odd step
// gathers and scatters through the precomputed neighbour-row offsets and writes every stored slot
// exactly once.
//
// Algorithmic bytes per node update: 2 * 19 * sizeof(storage). Metadata read per node: 1 byte
// material code and 4 bytes wall mask + link offset (even step); 1 byte code, 8 bytes masks and
// 16 bytes neighbour-row offsets (odd step).
#include "batch.cuh"
#include "flow_node.cuh"
#include "tma.cuh"

#include <algorithm>
#include <mutex>
#include <vector>
#include <cmath>
#include <cstring>

namespace clb {

constexpr int FLOW_THREADS = 256;
constexpr int PIPE_THREADS = 256;  // CTA of the pipelined odd step (shared memory per thread: 2 nodes)


// Block-wide FP64 sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
    __syncthreads();
    return r;
}

// The last block of a step turns the partial sums into the stored average energy and runs
// the tracer. Deterministic: fixed grid, fixed reduction order.
__device__ void finish_step(Tracer* tr, double* partials, double block_total, int64_t n_bgk, int trace) {
    __shared__ bool s_last;
    __shared__ double sh[32];
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = block_total;
        __threadfence();
        unsigned t = atomicAdd(&tr->done_blocks, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double v = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) v += ((volatile double*)partials)[k];
    double tot = block_sum(v, sh);
    __shared__ double s_mean;
    __shared__ int s_count;
    if (threadIdx.x == 0) {
        double e = n_bgk > 0 ? 0.5 * tot / (double)n_bgk : 0.0;
        tr->energy = e;
        tr->iterations += 1;
        tr->done_blocks = 0;
        s_count = 0;
        if (trace) {
            tr->ring[tr->head] = e;
            tr->head = (tr->head + 1) % TRACER_WINDOW;
            if (tr->count < TRACER_WINDOW) tr->count += 1;
            s_count = tr->count;
        }
    }
    __syncthreads();
    if (!trace || s_count < TRACER_WINDOW) return;
    v = 0;
    for (int k = threadIdx.x; k < TRACER_WINDOW; k += blockDim.x) v += tr->ring[k];
    double sum = block_sum(v, sh);
    if (threadIdx.x == 0) s_mean = sum / (double)TRACER_WINDOW;
    __syncthreads();
    v = 0;
    for (int k = threadIdx.x; k < TRACER_WINDOW; k += blockDim.x) {
        double d = tr->ring[k] - s_mean;
        v += d * d;
    }
    double sq = block_sum(v, sh);
    if (threadIdx.x == 0) {
        double sd = sqrt(sq / (double)(TRACER_WINDOW - 1));
        double r = sd / s_mean;
        if (isnan(r) || fabs(r) < tr->eps) tr->converged = 1;
    }
}



// Odd AA step with the gathers of the next node in flight while a node is collided: each thread
// stages a node's 19 incoming populations in its own two shared-memory slots with asynchronous
// copies (4- and 8-byte storage), one node ahead, and the node after that has its metadata
// loading. The odd step is an in-place permutation: outgoing population j of node k goes to the
// slot incoming opp(j) came from, so the 19 slot offsets computed for the gathers are kept in
// registers (two sets, the loop unrolled by two nodes) and reused by the stores. Same arithmetic
// as the plain step.
template <typename TS, typename TC, int MINB>
__global__ void __launch_bounds__(PIPE_THREADS, MINB)
    k_flow_odd_pipe(TS* __restrict__ f, TS* __restrict__ link, const SparseView S, const FlowParams P,
                    Tracer* __restrict__ tr, double* __restrict__ partials, int trace, int64_t k_west_end,
                    int64_t k_east_begin) {
    if (trace && tr->converged) return;
    extern __shared__ __align__(16) unsigned char flow_smem[];
    const int tid = threadIdx.x, nt = blockDim.x;
    TS* buf = reinterpret_cast<TS*>(flow_smem);  // [2][19][nt]
    const int64_t K = S.K;
    const uint32_t K32 = (uint32_t)S.KS;
    const int64_t stride = (int64_t)gridDim.x * nt;
    double esum = 0;
    uint32_t A[19], B[19];
    auto issue = [&](int64_t kk, const FlowMeta& M, int q, uint32_t (&ad)[19]) {
        const OddRows R = odd_rows(S, kk, M);
        TS* dst = buf + (q * 19) * nt + tid;
#pragma unroll
        for (int i = 0; i < 19; ++i) {
            ad[i] = odd_src(i, kk, R, K32);
            cp_async<sizeof(TS)>(dst + i * nt, f + ad[i]);
        }
    };
    int64_t k = (int64_t)blockIdx.x * nt + tid;
    FlowMeta cur, nxt;
    if (k < K) {
        cur = flow_meta<true>(S, k);
        issue(k, cur, 0, A);
    }
    cp_async_commit();
    int64_t kn = k + stride;
    if (kn < K) nxt = flow_meta<true>(S, kn);
    // one node: gathers of the next node issued into the other slot, then this node collided
    auto node = [&](int q, uint32_t (&ac)[19], uint32_t (&an)[19]) {
        if (kn < K) issue(kn, nxt, q ^ 1, an);
        cp_async_commit();
        const int64_t knn = kn + stride;
        FlowMeta nn;
        if (knn < K) nn = flow_meta<true>(S, knn);
        cp_async_wait_group<1>();  // this node's populations have landed
        const int code = cur.code;
        if (P.dyn[code] != DYN_BB) {  // a stored bounce-back node: identity on AA slots
            TC g[19];
            const TS* src = buf + (q * 19) * nt + tid;
#pragma unroll
            for (int i = 0; i < 19; ++i) g[i] = ld<TS, TC>(src + i * nt);
            if (P.dyn[code] == DYN_BGK) {
                if (k < k_west_end) regularize19<TC>(g, -1, (TC)(P.rho_w - 1.0));
                else if (k >= k_east_begin) regularize19<TC>(g, 1, (TC)(P.rho_e - 1.0));
                esum += (double)bgk19<TC>(g, (TC)P.omega[code]);
            }
#pragma unroll
            for (int i = 0; i < 19; ++i) st<TS, TC>(f + ac[q19opp(i)], g[i]);
        }
        k = kn;
        kn = knn;
        cur = nxt;
        nxt = nn;
    };
    while (k < K) {
        node(0, A, B);
        if (k >= K) break;
        node(1, B, A);
    }
    cp_async_wait_group<0>();
    __shared__ double sh[32];
    double bt = block_sum(esum, sh);
    finish_step(tr, partials, bt, P.n_bgk, trace);
}

template <typename TS, typename TC, bool ODD, int MINB>
__global__ void __launch_bounds__(FLOW_THREADS, MINB)
    k_flow_aa(TS* __restrict__ f, TS* __restrict__ link, const SparseView S, const FlowParams P,
              Tracer* __restrict__ tr, double* __restrict__ partials, int trace, int64_t k_west_end,
              int64_t k_east_begin) {
    if (trace && tr->converged) return;  // a batch continues past convergence as no-ops
    const int64_t K = S.K;
    double esum = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    FlowMeta cur;
    if (k < K) cur = flow_meta<ODD>(S, k);
    while (k < K) {
        const int64_t kn = k + stride;
        FlowMeta nxt;
        if (kn < K) nxt = flow_meta<ODD>(S, kn);  // the next node's metadata in flight meanwhile
        esum += flow_node_m<TS, TC, ODD>(f, link, S, P, k, k_west_end, k_east_begin, cur);
        cur = nxt;
        k = kn;
    }
    __shared__ double sh[32];
    double bt = block_sum(esum, sh);
    finish_step(tr, partials, bt, P.n_bgk, trace);
}


// Even AA step through shared memory: a persistent CTA walks 256-node tiles; one thread moves the
// tile's 19 population rows (contiguous, 16-byte aligned thanks to the padded row stride) into
// shared memory with bulk copies completing on an mbarrier, keeping NSTAGE-1 tiles in flight
// ahead of the one being collided. Each thread collides its node in place in shared memory; the
// rows go back with bulk stores. A wall link (a, i) takes its incoming opp(i) from its even-step
// slot X (a global load issued alongside the tile's), writes outgoing i to X, and leaves its
// odd-step slot Y = f[opp(i)][a] untouched in the tile, so the bulk store rewrites it unchanged.
constexpr int NSTAGE = 2;  // 2 stages x 4 resident CTAs (4-byte storage) beat 3 x 3 on B200

template <typename TS, typename TC>
__global__ void __launch_bounds__(TILE, sizeof(TS) == 8 ? 2 : 4)
    k_flow_even_tma(TS* __restrict__ f, TS* __restrict__ link, const SparseView S, const FlowParams P,
                    Tracer* __restrict__ tr, double* __restrict__ partials, int trace, int64_t k_west_end,
                    int64_t k_east_begin, int* __restrict__ err) {
    if (trace && tr->converged) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TS* stages = reinterpret_cast<TS*>(smem_raw);
    __shared__ __align__(8) uint64_t full[NSTAGE];
    __shared__ int s_abort;
    const int tid = threadIdx.x;
    const int64_t K = S.K, KS = S.KS;
    const int ntiles = (int)((K + TILE - 1) / TILE);
    const uint32_t row_bytes = TILE * sizeof(TS);
    if (tid == 0) {
        for (int q = 0; q < NSTAGE; ++q) mbar_init(&full[q], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    auto issue_load = [&](int t, int q) {
        TS* dst = stages + (size_t)q * 19 * TILE;
        mbar_expect_tx(&full[q], 19 * row_bytes);
        for (int i = 0; i < 19; ++i) bulk_g2s(dst + i * TILE, f + (int64_t)i * KS + (int64_t)t * TILE, row_bytes, &full[q]);
    };
    double esum = 0;
    if (tid == 0)
        for (int q = 0; q < NSTAGE - 1; ++q) {
            const int t = blockIdx.x + q * gridDim.x;
            if (t < ntiles) issue_load(t, q);
        }
    int j = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++j) {
        const int q = j % NSTAGE;
        TS* buf = stages + (size_t)q * 19 * TILE;
        // keep NSTAGE-1 tiles in flight: refill the stage of the previous tile once its bulk store
        // has read it
        const int tn = t + (NSTAGE - 1) * gridDim.x;
        if (tid == 0 && tn < ntiles) {
            bulk_wait_read_all();
            issue_load(tn, (j + NSTAGE - 1) % NSTAGE);
        }
        const int64_t k = (int64_t)t * TILE + tid;
        int code = 0;
        if (k < K) code = S.code[k];
        // a stored bounce-back node leaves its tile slots and links as they are (identity)
        const bool live = k < K && P.dyn[code] != DYN_BB;
        uint32_t wm = 0;
        int lb = 0;
        TC xv[19];
        if (live) {
            const uint32_t m0 = S.meta[2 * k];
            wm = m0 & 0x7FFFFu;
            lb = S.tlb[t] + (int)(m0 >> 19);
            int r = 0;
#pragma unroll
            for (int i = 1; i < 19; ++i) {
                const bool wl = (wm >> i) & 1u;
                xv[q19opp(i)] = wl ? ld<TS, TC>(link + lb + r) : (TC)0;
                r += wl;
            }
        }
        if (!mbar_wait(&full[q], (uint32_t)((j / NSTAGE) & 1))) {
            if (tid == 0) { atomicExch(err, 1); s_abort = 1; }
        }
        __syncthreads();
        if (s_abort) break;
        if (live) {
            TC g[19];
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                const bool wsrc = i != 0 && ((wm >> q19opp(i)) & 1u);
                g[i] = wsrc ? xv[i] : ld<TS, TC>(buf + i * TILE + tid);
            }
            if (P.dyn[code] == DYN_BGK) {
                if (k < k_west_end) regularize19<TC>(g, -1, (TC)(P.rho_w - 1.0));
                else if (k >= k_east_begin) regularize19<TC>(g, 1, (TC)(P.rho_e - 1.0));
                esum += (double)bgk19<TC>(g, (TC)P.omega[code]);
            }
            int r = 0;
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                const bool wl = (wm >> i) & 1u;
                if (wl) st<TS, TC>(link + lb + r, g[i]);
                else st<TS, TC>(buf + q19opp(i) * TILE + tid, g[i]);
                r += wl;
            }
        }
        fence_async_smem();  // this thread's writes to the tile, ordered before the bulk stores read it
        __syncthreads();
        if (tid == 0) {
            for (int i = 0; i < 19; ++i) bulk_s2g(f + (int64_t)i * KS + (int64_t)t * TILE, buf + i * TILE, row_bytes);
            bulk_commit();
        }
    }
    if (tid == 0) bulk_wait_all();
    __shared__ double sh[32];
    double bt = block_sum(esum, sh);
    finish_step(tr, partials, bt, P.n_bgk, trace);
}

// ------------------------------------------------------------------ batched step of many domains

// One AA step of every domain's flow lattice. Each CTA takes a contiguous run of the tile table
// (tiles are in domain order) and copies a tile's domain description into shared memory when it
// differs from the previous tile's, so the node loop reads the layout and the parameters from
// shared memory with the very same per-node code as the single-domain step.
template <typename TS, typename TC, bool ODD>
__global__ void __launch_bounds__(256) k_flow_batch(const BatchView B) {
    __shared__ __align__(16) BatchDomain sd;
    const int tid = threadIdx.x;
    const int per = (B.nft + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * per, t1 = min(B.nft, t0 + per);
    int cur = -1;
    for (int t = t0; t < t1; ++t) {
        const BatchTile T = B.ftiles[t];
        if (T.d != cur) {
            __syncthreads();  // every thread is done with the previous domain
            const uint64_t* src = reinterpret_cast<const uint64_t*>(B.dom + T.d);
            uint64_t* dst = reinterpret_cast<uint64_t*>(&sd);
            for (int q = tid; q < (int)(sizeof(BatchDomain) / 8); q += blockDim.x) dst[q] = src[q];
            __syncthreads();
            cur = T.d;
        }
        TS* f = (TS*)sd.f;
        TS* fl = (TS*)sd.flink;
        for (int64_t k = T.first + tid; k < T.first + T.count; k += blockDim.x)
            flow_node<TS, TC, ODD>(f, fl, sd.fs, sd.fp, k, sd.fkw, sd.fke);
    }
}

void launch_flow_batch(const BatchView& B, int prec, bool odd, int grid, int threads, cudaStream_t st) {
    grid = std::max(1, std::min(grid, B.nft));
#define CLB_FB(TS, TC)                                                                      \
    if (odd) k_flow_batch<TS, TC, true><<<grid, threads, 0, st>>>(B);                      \
    else k_flow_batch<TS, TC, false><<<grid, threads, 0, st>>>(B);
    switch (prec) {
        case CLB_F64: CLB_FB(double, double); break;
        case CLB_F32: CLB_FB(float, float); break;
        default: CLB_FB(__half, float); break;
    }
#undef CLB_FB
}

// The staged batched steps: a CTA's run of the tile table is cut into segments of consecutive
// tiles of one domain; for each segment the domain's description goes to shared memory and the
// segment's nodes are stepped as the single-domain staged kernels step a lattice (the even step
// through bulk-copied 256-node tiles, the odd step with each thread's next node's gathers in
// flight). Tile-table runs start on 1024-node boundaries, so no two CTAs share a 256-node tile.

// the segment of a CTA's run that starts at tile t (t < t1): tiles [t, returned) of one domain,
// compact nodes [kb, ke)
__device__ __forceinline__ int batch_segment(const BatchTile* __restrict__ tiles, int t, int t1, int64_t& kb,
                                             int64_t& ke) {
    const int d = tiles[t].d;
    kb = tiles[t].first;
    ke = kb;
    int te = t;
    while (te < t1 && tiles[te].d == d) {
        ke = tiles[te].first + tiles[te].count;
        ++te;
    }
    return te;
}

__device__ __forceinline__ void batch_load_domain(BatchDomain& sd, const BatchDomain* src, int tid, int nt) {
    const uint64_t* a = reinterpret_cast<const uint64_t*>(src);
    uint64_t* b = reinterpret_cast<uint64_t*>(&sd);
    for (int q = tid; q < (int)(sizeof(BatchDomain) / 8); q += nt) b[q] = a[q];
}

template <typename TS, typename TC>
__global__ void __launch_bounds__(PIPE_THREADS, 2) k_flow_batch_odd(const BatchView B) {
    extern __shared__ __align__(16) unsigned char flow_smem[];
    __shared__ __align__(16) BatchDomain sd;
    const int tid = threadIdx.x, nt = blockDim.x;
    TS* buf = reinterpret_cast<TS*>(flow_smem);  // [2][19][nt]
    const int per = (B.nft + gridDim.x - 1) / gridDim.x;
    int t = blockIdx.x * per;
    const int t1 = min(B.nft, t + per);
    while (t < t1) {
        int64_t kb, ke;
        const int d = B.ftiles[t].d;
        t = batch_segment(B.ftiles, t, t1, kb, ke);
        __syncthreads();  // every thread is done with the previous domain
        batch_load_domain(sd, B.dom + d, tid, nt);
        __syncthreads();
        TS* f = (TS*)sd.f;
        const SparseView& S = sd.fs;
        const FlowParams& P = sd.fp;
        const uint32_t K32 = (uint32_t)S.KS;
        const int64_t kw = sd.fkw, kE = sd.fke;
        uint32_t A[19], C[19];
        auto issue = [&](int64_t kk, const FlowMeta& M, int q, uint32_t (&ad)[19]) {
            const OddRows R = odd_rows(S, kk, M);
            TS* dst = buf + (q * 19) * nt + tid;
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                ad[i] = odd_src(i, kk, R, K32);
                cp_async<sizeof(TS)>(dst + i * nt, f + ad[i]);
            }
        };
        int64_t k = kb + tid;
        FlowMeta cur, nxt;
        if (k < ke) {
            cur = flow_meta<true>(S, k);
            issue(k, cur, 0, A);
        }
        cp_async_commit();
        int64_t kn = k + nt;
        if (kn < ke) nxt = flow_meta<true>(S, kn);
        auto node = [&](int q, uint32_t (&ac)[19], uint32_t (&an)[19]) {
            if (kn < ke) issue(kn, nxt, q ^ 1, an);
            cp_async_commit();
            const int64_t knn = kn + nt;
            FlowMeta nn;
            if (knn < ke) nn = flow_meta<true>(S, knn);
            cp_async_wait_group<1>();  // this node's populations have landed
            const int code = cur.code;
            if (P.dyn[code] != DYN_BB) {
                TC g[19];
                const TS* src = buf + (q * 19) * nt + tid;
#pragma unroll
                for (int i = 0; i < 19; ++i) g[i] = ld<TS, TC>(src + i * nt);
                if (P.dyn[code] == DYN_BGK) {
                    if (k < kw) regularize19<TC>(g, -1, (TC)(P.rho_w - 1.0));
                    else if (k >= kE) regularize19<TC>(g, 1, (TC)(P.rho_e - 1.0));
                    bgk19<TC>(g, (TC)P.omega[code]);
                }
#pragma unroll
                for (int i = 0; i < 19; ++i) st<TS, TC>(f + ac[q19opp(i)], g[i]);
            }
            k = kn;
            kn = knn;
            cur = nxt;
            nxt = nn;
        };
        while (k < ke) {
            node(0, A, C);
            if (k >= ke) break;
            node(1, C, A);
        }
        cp_async_wait_group<0>();
    }
}

template <typename TS, typename TC>
__global__ void __launch_bounds__(TILE, sizeof(TS) == 8 ? 2 : 4) k_flow_batch_even(const BatchView B) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TS* stages = reinterpret_cast<TS*>(smem_raw);
    __shared__ __align__(8) uint64_t full[NSTAGE];
    __shared__ __align__(16) BatchDomain sd;
    __shared__ int s_abort;
    const int tid = threadIdx.x;
    const uint32_t row_bytes = TILE * sizeof(TS);
    if (tid == 0) {
        for (int q = 0; q < NSTAGE; ++q) mbar_init(&full[q], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    const int per = (B.nft + gridDim.x - 1) / gridDim.x;
    int t = blockIdx.x * per;
    const int t1 = min(B.nft, t + per);
    int j = 0;  // tiles stepped by this CTA: stage j % NSTAGE, its phase (j / NSTAGE) & 1
    while (t < t1) {
        int64_t kb, ke;
        const int d = B.ftiles[t].d;
        t = batch_segment(B.ftiles, t, t1, kb, ke);
        __syncthreads();  // every thread is done with the previous domain
        batch_load_domain(sd, B.dom + d, tid, TILE);
        __syncthreads();
        TS* f = (TS*)sd.f;
        TS* link = (TS*)sd.flink;
        const SparseView& S = sd.fs;
        const FlowParams& P = sd.fp;
        const int64_t K = S.K, KS = S.KS;
        const int tb = (int)(kb / TILE), te = (int)((ke + TILE - 1) / TILE);
        auto issue_load = [&](int tt, int q) {
            TS* dst = stages + (size_t)q * 19 * TILE;
            mbar_expect_tx(&full[q], 19 * row_bytes);
            for (int i = 0; i < 19; ++i)
                bulk_g2s(dst + i * TILE, f + (int64_t)i * KS + (int64_t)tt * TILE, row_bytes, &full[q]);
        };
        if (tid == 0) {
            bulk_wait_read_all();  // the stages' earlier bulk stores have read them
            for (int q = 0; q < NSTAGE - 1; ++q)
                if (tb + q < te) issue_load(tb + q, (j + q) % NSTAGE);
        }
        for (int tt = tb; tt < te; ++tt, ++j) {
            const int q = j % NSTAGE;
            TS* buf = stages + (size_t)q * 19 * TILE;
            const int tn = tt + NSTAGE - 1;
            if (tid == 0 && tn < te) {
                bulk_wait_read_all();
                issue_load(tn, (j + NSTAGE - 1) % NSTAGE);
            }
            const int64_t k = (int64_t)tt * TILE + tid;
            int code = 0;
            if (k < K) code = S.code[k];
            const bool live = k < K && P.dyn[code] != DYN_BB;
            uint32_t wm = 0;
            int lb = 0;
            TC xv[19];
            if (live) {
                const uint32_t m0 = S.meta[2 * k];
                wm = m0 & 0x7FFFFu;
                lb = S.tlb[tt] + (int)(m0 >> 19);
                int r = 0;
#pragma unroll
                for (int i = 1; i < 19; ++i) {
                    const bool wl = (wm >> i) & 1u;
                    xv[q19opp(i)] = wl ? ld<TS, TC>(link + lb + r) : (TC)0;
                    r += wl;
                }
            }
            if (!mbar_wait(&full[q], (uint32_t)((j / NSTAGE) & 1))) {
                if (tid == 0) {
                    atomicExch(B.status, 1);
                    s_abort = 1;
                }
            }
            __syncthreads();
            if (s_abort) break;
            if (live) {
                TC g[19];
#pragma unroll
                for (int i = 0; i < 19; ++i) {
                    const bool wsrc = i != 0 && ((wm >> q19opp(i)) & 1u);
                    g[i] = wsrc ? xv[i] : ld<TS, TC>(buf + i * TILE + tid);
                }
                if (P.dyn[code] == DYN_BGK) {
                    if (k < sd.fkw) regularize19<TC>(g, -1, (TC)(P.rho_w - 1.0));
                    else if (k >= sd.fke) regularize19<TC>(g, 1, (TC)(P.rho_e - 1.0));
                    bgk19<TC>(g, (TC)P.omega[code]);
                }
                int r = 0;
#pragma unroll
                for (int i = 0; i < 19; ++i) {
                    const bool wl = (wm >> i) & 1u;
                    if (wl) st<TS, TC>(link + lb + r, g[i]);
                    else st<TS, TC>(buf + q19opp(i) * TILE + tid, g[i]);
                    r += wl;
                }
            }
            fence_async_smem();  // this thread's writes to the tile, ordered before the bulk stores read it
            __syncthreads();
            if (tid == 0) {
                for (int i = 0; i < 19; ++i)
                    bulk_s2g(f + (int64_t)i * KS + (int64_t)tt * TILE, buf + i * TILE, row_bytes);
                bulk_commit();
            }
        }
        if (s_abort) break;
    }
    if (tid == 0) bulk_wait_all();
}

// PressureGradient equilibrium (complab_functions.hh:82-94): BGK nodes t_i (rho(x) - 1),
// no-dynamics nodes zero (BounceBack / NoDynamics equilibria are zero). For a wall link (a, i)
// the even-step slot X holds a's equilibrium incoming opp(i) and the odd-step slot
// Y = f[opp(i)][a] the wall's initial (zero) population.
template <typename TS>
__global__ void k_flow_init(TS* __restrict__ f, TS* __restrict__ link, const SparseView S, const FlowParams P,
                            double delta_p) {
    const Geom G = P.g;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < S.K; k += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(S.node[k] / G.plane);
        const double rho = 1.0 - delta_p * 3.0 / (double)(G.nx - 1) * (double)x;
        const bool bgk = P.dyn[S.code[k]] == DYN_BGK;
        const uint32_t wm = S.wall[k];
#pragma unroll
        for (int i = 0; i < 19; ++i) {
            const double eq = bgk ? q19w(i) * (rho - 1.0) : 0.0;
            const bool wall_src = i != 0 && ((wm >> q19opp(i)) & 1u);
            const double v = wall_src ? 0.0 : eq;
            if constexpr (std::is_same<TS, __half>::value) f[(int64_t)i * S.KS + k] = to_half(v);
            else f[(int64_t)i * S.KS + k] = (TS)v;
            if (wall_src) {
                TS* x_ = link_slot(S, link, (int)k, q19opp(i));
                if constexpr (std::is_same<TS, __half>::value) *x_ = to_half(eq);
                else *x_ = (TS)eq;
            }
        }
    }
}

// computeVelocity at the dense nodes `nodes[0..count)` (all nodes when nodes == nullptr):
// BGK u = j; pressure-plane BGK nodes (j_x from the known populations, 0, 0); others 0.
// Output u[3][stride] at position t (the node's rank in `nodes`).
template <typename TS, typename TC, typename TO>
__global__ void k_flow_velocity(const TS* __restrict__ f, const TS* __restrict__ link, const SparseView S,
                                const int8_t* __restrict__ mat, const FlowParams P, int odd,
                                const int32_t* __restrict__ nodes, int64_t count, TO* __restrict__ u, int64_t stride) {
    const Geom G = P.g;
    const TC zero[19] = {};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = nodes ? nodes[t] : t;
        TC jx = 0, jy = 0, jz = 0;
        if (P.dyn[mat[n]] == DYN_BGK) {
            TC g[19];
            natural<TS, TC, 19>(S, G, f, link, n, odd, zero, g);
            const int x = (int)(n / G.plane);
            if (x == 0 || x == G.nx - 1) {
                const int o = (x == 0) ? -1 : 1;
                const TC rb = (TC)((x == 0 ? P.rho_w : P.rho_e) - 1.0);
                TC r0 = 0, rn = 0;
                for (int i = 0; i < 19; ++i) {
                    if (q19cx(i) == 0) r0 += g[i];
                    else if (q19cx(i) == o) rn += g[i];
                }
                jx = (TC)o * (r0 + (TC)2 * rn - rb);
            } else {
                for (int i = 0; i < 19; ++i) {
                    jx += (TC)q19cx(i) * g[i];
                    jy += (TC)q19cy(i) * g[i];
                    jz += (TC)q19cz(i) * g[i];
                }
            }
        }
        u[t] = (TO)jx;
        u[stride + t] = (TO)jy;
        u[2 * stride + t] = (TO)jz;
    }
}

template <typename TS>
__global__ void k_flow_get_pops(const TS* __restrict__ f, const TS* __restrict__ link, const SparseView S,
                                const Geom G, int odd, double* __restrict__ out) {
    const double zero[19] = {};
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        double g[19];
        natural<TS, double, 19>(S, G, f, link, n, odd, zero, g);
        for (int i = 0; i < 19; ++i) out[(int64_t)i * G.N + n] = g[i];
    }
}

template <typename TS>
__global__ void k_flow_set_pops(TS* __restrict__ f, TS* __restrict__ link, const SparseView S, const Geom G, int odd,
                                const double* __restrict__ in) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        double g[19];
        for (int i = 0; i < 19; ++i) g[i] = in[(int64_t)i * G.N + n];
        put_natural<TS, 19>(S, G, f, link, n, odd, g);
    }
}

__global__ void k_flow_vstats(const double* __restrict__ u, const Geom G, double* __restrict__ acc) {
    // acc[0] sum |u| over x=1..nx-2, acc[1] max u_x (as ordered bits), acc[2] sum u_x on x=nx-2
    __shared__ double sh[32];
    double s_norm = 0, s_out = 0, m = -1e300;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(n / G.plane);
        if (x < 1 || x > G.nx - 2) continue;
        const double ux = u[n], uy = u[G.N + n], uz = u[2 * G.N + n];
        s_norm += sqrt(ux * ux + uy * uy + uz * uz);
        m = fmax(m, ux);
        if (x == G.nx - 2) s_out += ux;
    }
    double a = block_sum(s_norm, sh);
    double b = block_sum(s_out, sh);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double smax[32];
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = -1e300;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mm = fmax(mm, smax[k]);
        atomicAdd(&acc[0], a);
        atomicAdd(&acc[2], b);
        // max of doubles via the ordered-integer trick
        long long bits = __double_as_longlong(mm);
        long long key = bits >= 0 ? bits : (bits ^ 0x7fffffffffffffffLL);
        atomicMax((long long*)&acc[1], key);
    }
}

// ------------------------------------------------------------------ host side


// ------------------------------------------------------------------ host side

static size_t storage_size(int prec) { return prec == CLB_F64 ? 8 : (prec == CLB_F32 ? 4 : 2); }

template <typename TS>
static size_t even_smem() {
    return (size_t)NSTAGE * 19 * TILE * sizeof(TS);
}

// two slots of 19 populations per thread for the pipelined odd step
template <typename TS>
static size_t pipe_smem() {
    return (size_t)2 * 19 * PIPE_THREADS * sizeof(TS);
}

// resident-CTA grid of the pipelined odd step (0: not available for 2-byte storage, whose
// populations are below the 4-byte granule of the asynchronous copy)
template <typename TS, typename TC>
static int pipe_grid_of(clb_handle* h) {
    if (sizeof(TS) < 4) return 0;
    int per_sm = 0;
    const size_t sm = pipe_smem<TS>();
    cudaFuncSetAttribute(k_flow_odd_pipe<TS, TC, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow_odd_pipe<TS, TC, 2>, PIPE_THREADS, sm);
    return h->num_sms * std::min(16, std::max(1, per_sm));
}


template <typename F>
static int grid_for(clb_handle* h, F kernel, int threads) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    if (per_sm < 1) per_sm = 1;
    return h->num_sms * per_sm;
}

void flow_free(clb_handle* h) {
    cudaFree(h->d_f); h->d_f = nullptr;
    cudaFree(h->d_flink); h->d_flink = nullptr;
    sparse_free(h->flow_sp);
    cudaFree(h->d_tracer); h->d_tracer = nullptr;
    cudaFree(h->d_partials); h->d_partials = nullptr;
    h->flow_ready = false;
}

static int flow_gather_grid(clb_handle* h) {
    switch (h->flow_prec) {
        case CLB_F64: return h->flow_minb == 2 ? grid_for(h, k_flow_aa<double, double, true, 2>, FLOW_THREADS) : grid_for(h, k_flow_aa<double, double, true, 3>, FLOW_THREADS);
        case CLB_F32: return h->flow_minb == 2 ? grid_for(h, k_flow_aa<float, float, true, 2>, FLOW_THREADS) : grid_for(h, k_flow_aa<float, float, true, 3>, FLOW_THREADS);
        default: return h->flow_minb == 2 ? grid_for(h, k_flow_aa<__half, float, true, 2>, FLOW_THREADS) : grid_for(h, k_flow_aa<__half, float, true, 3>, FLOW_THREADS);
    }
}

clb_status flow_init(clb_handle* h, double delta_p) {
    h->resolve_tracer_valid = false;  // a new flow: the in-loop tracer starts empty again
    const clb_domain_desc& d = h->d;
    FlowParams& P = h->fp;
    std::memset(&P, 0, sizeof(P));
    P.g = h->g;
    const double omega = 1.0 / d.tau;
    // NSdomainSetup: IncBGK(omega) everywhere, pore codes IncBGK, bounce-back, no-dynamics,
    // biofilm IncBGK(omega_bio) or BounceBack when impermeable.
    for (int c = 0; c < MAX_CODES; ++c) { P.dyn[c] = DYN_BGK; P.omega[c] = omega; }
    if (d.bounce_back_code >= 0 && d.bounce_back_code < MAX_CODES) P.dyn[d.bounce_back_code] = DYN_BB;
    if (d.solid_code >= 0 && d.solid_code < MAX_CODES) P.dyn[d.solid_code] = DYN_NONE;
    for (int m = 0; m < d.n_microbes; ++m) {
        int c = d.bio_codes[m];
        if (c < 0 || c >= MAX_CODES) continue;
        if (d.perm_ratio[m] > 1e-14) {
            P.dyn[c] = DYN_BGK;
            P.omega[c] = 1.0 / (d.perm_ratio[m] * (1.0 / omega - 0.5) + 0.5);
        } else {
            P.dyn[c] = DYN_BB;
        }
    }
    P.rho_w = 1.0;
    P.rho_e = 1.0 - delta_p * 3.0;
    h->delta_p = delta_p;
    // the flow lattice's own map once precipitation has changed the species' one
    const std::vector<int8_t>& fmat = h->h_mat_flow.empty() ? h->h_mat : h->h_mat_flow;
    // biofilm voxels are nodes even when impermeable (bounce-back nodes are skipped by the step),
    // so that the automaton can turn them back into pore without a new layout
    int8_t cls[MAX_CODES];
    for (int c = 0; c < MAX_CODES; ++c) cls[c] = (P.dyn[c] != DYN_BB);
    for (int m = 0; m < d.n_microbes; ++m)
        if (d.bio_codes[m] >= 0 && d.bio_codes[m] < MAX_CODES) cls[d.bio_codes[m]] = 1;
    // BGK node count from a histogram of the codes (four interleaved counters, no data-dependent
    // branch), the node counts of the first and last x-planes from those planes alone
    int64_t nbgk = 0, kw = 0, ke = 0;
    {
        std::vector<int64_t> hist(4 * 128, 0);
        const uint8_t* m = reinterpret_cast<const uint8_t*>(fmat.data());
        const int64_t N = h->g.N, plane = h->g.plane;
        int64_t n = 0;
        for (; n + 4 <= N; n += 4) {
            ++hist[m[n] & 127];
            ++hist[128 + (m[n + 1] & 127)];
            ++hist[256 + (m[n + 2] & 127)];
            ++hist[384 + (m[n + 3] & 127)];
        }
        for (; n < N; ++n) ++hist[m[n] & 127];
        for (int c = 0; c < 128; ++c)
            if (P.dyn[c] == DYN_BGK) nbgk += hist[c] + hist[128 + c] + hist[256 + c] + hist[384 + c];
        for (int64_t i = 0; i < plane; ++i) {
            kw += cls[m[i] & 127];
            ke += cls[m[N - plane + i] & 127];
        }
    }
    P.n_bgk = nbgk;

    flow_free(h);
    clb_status s = sparse_build(h, cls, 19, h->flow_sp, &fmat);
    if (s != CLB_OK) return s;
    const int64_t K = h->flow_sp.K;
    h->k_west_end = kw;
    h->k_east_begin = K - ke;
    h->flow_prec = d.flow_precision;
    const size_t es = storage_size(h->flow_prec);
    cudaError_t e;
    if ((e = cudaMalloc(&h->d_f, es * 19 * (size_t)h->flow_sp.KS)) != cudaSuccess)
        return cuda_check(h, e, "flow populations");
    // +16 bytes: the FP16 even step copies whole aligned 4-byte words around each link slot
    if ((e = cudaMalloc(&h->d_flink, es * (size_t)std::max<int64_t>(1, h->flow_sp.L) + 16)) != cudaSuccess)
        return cuda_check(h, e, "flow links");
    if ((e = cudaMalloc(&h->d_tracer, sizeof(Tracer))) != cudaSuccess) return cuda_check(h, e, "tracer");
    cudaMemsetAsync(h->d_tracer, 0, sizeof(Tracer), h->stream);
    cudaMemsetAsync(h->d_flink, 0, es * (size_t)std::max<int64_t>(1, h->flow_sp.L), h->stream);

    int grid = flow_gather_grid(h);
    h->flow_grid = grid;
    // the even step's tiled kernel: persistent CTAs, shared-memory stages sized by precision
    {
        int per_sm = 0;
        size_t sm = 0;
        switch (h->flow_prec) {
            case CLB_F64:
                sm = even_smem<double>();
                cudaFuncSetAttribute(k_flow_even_tma<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow_even_tma<double, double>, TILE, sm);
                break;
            case CLB_F32:
                sm = even_smem<float>();
                cudaFuncSetAttribute(k_flow_even_tma<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow_even_tma<float, float>, TILE, sm);
                break;
            default:
                sm = even_smem<__half>();
                cudaFuncSetAttribute(k_flow_even_tma<__half, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow_even_tma<__half, float>, TILE, sm);
                break;
        }
        h->flow_even_grid = h->num_sms * std::max(1, per_sm);
    }
    switch (h->flow_prec) {
        case CLB_F64: h->flow_pipe_grid = pipe_grid_of<double, double>(h); break;
        case CLB_F32: h->flow_pipe_grid = pipe_grid_of<float, float>(h); break;
        default: h->flow_pipe_grid = 0; break;
    }
    if (!h->flow_pipe_grid) h->flow_odd_pipe = 0;
    // partials sized for the largest grid any variant uses
    const int pcap = h->num_sms * 16;
    if ((e = cudaMalloc(&h->d_partials, sizeof(double) * pcap)) != cudaSuccess) return cuda_check(h, e, "partials");
    h->partial_cap = pcap;
    if (!h->d_err) {
        if ((e = cudaMalloc(&h->d_err, sizeof(int))) != cudaSuccess) return cuda_check(h, e, "error flag");
    }
    cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);

    const int ig = h->num_sms * 8;
    const SparseView S = view_of(h->flow_sp);
    switch (h->flow_prec) {
        case CLB_F64: k_flow_init<double><<<ig, 256, 0, h->stream>>>((double*)h->d_f, (double*)h->d_flink, S, P, delta_p); break;
        case CLB_F32: k_flow_init<float><<<ig, 256, 0, h->stream>>>((float*)h->d_f, (float*)h->d_flink, S, P, delta_p); break;
        default: k_flow_init<__half><<<ig, 256, 0, h->stream>>>((__half*)h->d_f, (__half*)h->d_flink, S, P, delta_p); break;
    }
    h->flow_iters = 0;
    h->flow_ready = true;
    return cuda_check(h, cudaGetLastError(), "flow init");
}

static void launch_flow(clb_handle* h, bool odd, int trace) {
    ++h->launches;  // one step launch per call
    const FlowParams& P = h->fp;
    const SparseView S = view_of(h->flow_sp);
    const int grid = h->flow_grid;
    if (!odd && h->flow_even_tma) {
        const int eg = h->flow_even_grid;
#define CLB_EVEN(TS, TC)                                                                                       \
        k_flow_even_tma<TS, TC><<<eg, TILE, even_smem<TS>(), h->stream>>>((TS*)h->d_f, (TS*)h->d_flink, S, P,  \
                                                                       h->d_tracer, h->d_partials, trace,     \
                                                                       h->k_west_end, h->k_east_begin, h->d_err);
        switch (h->flow_prec) {
            case CLB_F64: CLB_EVEN(double, double); break;
            case CLB_F32: CLB_EVEN(float, float); break;
            default: CLB_EVEN(__half, float); break;
        }
#undef CLB_EVEN
        return;
    }
    if (odd && h->flow_odd_pipe && h->flow_pipe_grid) {
        const int pg = h->flow_pipe_grid;
#define CLB_PIPE(TS, TC)                                                                                       \
        k_flow_odd_pipe<TS, TC, 2><<<pg, PIPE_THREADS, pipe_smem<TS>(), h->stream>>>(                          \
            (TS*)h->d_f, (TS*)h->d_flink, S, P, h->d_tracer, h->d_partials, trace, h->k_west_end, h->k_east_begin);
        switch (h->flow_prec) {
            case CLB_F64: CLB_PIPE(double, double); return;
            case CLB_F32: CLB_PIPE(float, float); return;
            default: break;
        }
#undef CLB_PIPE
    }
#define CLB_LAUNCH_B(TS, TC, B)                                                                                \
    if (odd)                                                                                                   \
        k_flow_aa<TS, TC, true, B><<<grid, FLOW_THREADS, 0, h->stream>>>((TS*)h->d_f, (TS*)h->d_flink, S, P,    \
                                                                          h->d_tracer, h->d_partials, trace,   \
                                                                          h->k_west_end, h->k_east_begin);     \
    else                                                                                                       \
        k_flow_aa<TS, TC, false, B><<<grid, FLOW_THREADS, 0, h->stream>>>((TS*)h->d_f, (TS*)h->d_flink, S, P,   \
                                                                           h->d_tracer, h->d_partials, trace,  \
                                                                           h->k_west_end, h->k_east_begin);
#define CLB_LAUNCH(TS, TC) if (h->flow_minb == 2) { CLB_LAUNCH_B(TS, TC, 2) } else { CLB_LAUNCH_B(TS, TC, 3) }
    switch (h->flow_prec) {
        case CLB_F64: CLB_LAUNCH(double, double); break;
        case CLB_F32: CLB_LAUNCH(float, float); break;
        default: CLB_LAUNCH(__half, float); break;
    }
#undef CLB_LAUNCH
#undef CLB_LAUNCH_B
}

clb_status flow_step(clb_handle* h, int n, bool trace, double eps) {
    (void)eps;
    for (int k = 0; k < n; ++k) {
        launch_flow(h, (h->flow_iters & 1) != 0, trace ? 1 : 0);
        h->flow_iters += 1;
    }
    return cuda_check(h, cudaGetLastError(), "flow step");
}

clb_status flow_solve(clb_handle* h, int max_it, double eps, int* iterations, bool keep_window) {
    // a fresh util::ValueTracer (empty window, new epsilon), or the in-loop one as the previous
    // re-solve left it
    Tracer t0;
    std::memset(&t0, 0, sizeof(t0));
    if (keep_window && h->resolve_tracer_valid) {
        std::memcpy(t0.ring, h->resolve_tracer.ring, sizeof(t0.ring));
        t0.count = h->resolve_tracer.count;
        t0.head = h->resolve_tracer.head;
    }
    Tracer cur;
    cudaError_t e = cudaMemcpyAsync(&cur, h->d_tracer, sizeof(Tracer), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_check(h, e, "tracer read");
    t0.eps = eps;
    t0.iterations = cur.iterations;
    t0.energy = cur.energy;
    cudaMemcpyAsync(h->d_tracer, &t0, sizeof(Tracer), cudaMemcpyHostToDevice, h->stream);
    const int64_t start = cur.iterations;
    int done = 0;
    int chunk = 64;
    bool conv = false;
    while (done < max_it) {
        int k = std::min(chunk, max_it - done);
        clb_status s = flow_step(h, k, true, eps);
        if (s != CLB_OK) return s;
        done += k;
        e = cudaMemcpyAsync(&cur, h->d_tracer, sizeof(Tracer), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_check(h, e, "tracer read");
        if (cur.converged) { conv = true; break; }
        if (chunk < 1024) chunk *= 2;
    }
    h->flow_iters = cur.iterations;  // steps after convergence were no-ops
    if (iterations) *iterations = (int)(cur.iterations - start);
    if (keep_window) {
        h->resolve_tracer = cur;
        h->resolve_tracer_valid = true;
    }
    // leave the tracer disabled for plain steps
    int zero = 0;
    cudaMemcpyAsync(&h->d_tracer->converged, &zero, sizeof(int), cudaMemcpyHostToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
    // a diverged solve (NaN or Inf stored energy; the tracer reads a NaN window as settled) stops
    // the run cleanly, as complab.cpp:3116-3117 does
    if (!std::isfinite(cur.energy))
        return fail(h, CLB_NONFINITE, "flow solve diverged: the stored average energy is not finite");
    if (!conv) {
        // at the cap with nothing leaving through the outlet plane the flow path is sealed: the
        // reference's percolation limit (complab.cpp:3106-3113, outlet u_x <= 1e-12)
        clb_flow_stats st;
        clb_status s = flow_stats(h, 1.0, &st);
        if (s != CLB_OK) return s;
        if (!(st.darcy_outlet_ux > THRD))
            return fail(h, CLB_PERCOLATION_LOST, "percolation lost: no flow through the outlet plane at the iteration cap");
        return CLB_NOT_CONVERGED;
    }
    return CLB_OK;
}

// Velocity at `count` dense nodes (all nodes when nodes == nullptr) into a device buffer
// u[3][stride] of float64 (dtype 0) or float32 (dtype 1).
clb_status flow_velocity_at(clb_handle* h, const int32_t* nodes, int64_t count, void* u, int64_t stride, int dtype) {
    const FlowParams& P = h->fp;
    const SparseView S = view_of(h->flow_sp);
    const int odd = (int)(h->flow_iters & 1);
    const int grid = h->num_sms * 8;
    ++h->launches;
#define CLB_VEL(TS, TC)                                                                                         \
    if (dtype == 0)                                                                                             \
        k_flow_velocity<TS, TC, double><<<grid, 256, 0, h->stream>>>((const TS*)h->d_f, (const TS*)h->d_flink, S, \
                                                                     flow_mat(h), P, odd, nodes, count, (double*)u, stride); \
    else                                                                                                        \
        k_flow_velocity<TS, TC, float><<<grid, 256, 0, h->stream>>>((const TS*)h->d_f, (const TS*)h->d_flink, S,  \
                                                                    flow_mat(h), P, odd, nodes, count, (float*)u, stride);
    switch (h->flow_prec) {
        case CLB_F64: CLB_VEL(double, double); break;
        case CLB_F32: CLB_VEL(float, float); break;
        default: CLB_VEL(__half, float); break;
    }
#undef CLB_VEL
    return cuda_check(h, cudaGetLastError(), "flow velocity");
}

clb_status flow_velocity(clb_handle* h, void* dst, int dtype_device, bool to_host) {
    void* out = dst;
    const size_t es = dtype_device == 0 ? 8 : 4;
    if (to_host) {
        cudaError_t e = cudaMalloc(&out, es * 3 * (size_t)h->g.N);
        if (e != cudaSuccess) return cuda_check(h, e, "velocity buffer");
    }
    clb_status s = flow_velocity_at(h, nullptr, h->g.N, out, h->g.N, dtype_device);
    if (to_host) {
        cudaError_t e = cudaMemcpyAsync(dst, out, es * 3 * (size_t)h->g.N, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(out);
        if (e != cudaSuccess) return cuda_check(h, e, "velocity copy");
    }
    return s;
}

clb_status flow_populations(clb_handle* h, double* host) {
    double* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, sizeof(double) * 19 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "population buffer");
    const int odd = (int)(h->flow_iters & 1);
    const int grid = h->num_sms * 8;
    const SparseView S = view_of(h->flow_sp);
    switch (h->flow_prec) {
        case CLB_F64: k_flow_get_pops<double><<<grid, 256, 0, h->stream>>>((const double*)h->d_f, (const double*)h->d_flink, S, h->g, odd, buf); break;
        case CLB_F32: k_flow_get_pops<float><<<grid, 256, 0, h->stream>>>((const float*)h->d_f, (const float*)h->d_flink, S, h->g, odd, buf); break;
        default: k_flow_get_pops<__half><<<grid, 256, 0, h->stream>>>((const __half*)h->d_f, (const __half*)h->d_flink, S, h->g, odd, buf); break;
    }
    e = cudaMemcpyAsync(host, buf, sizeof(double) * 19 * (size_t)h->g.N, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    return cuda_check(h, e, "population copy");
}

clb_status flow_set_populations(clb_handle* h, const double* host) {
    double* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, sizeof(double) * 19 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "population buffer");
    e = cudaMemcpyAsync(buf, host, sizeof(double) * 19 * (size_t)h->g.N, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) { cudaFree(buf); return cuda_check(h, e, "population copy"); }
    const int odd = (int)(h->flow_iters & 1);
    const int grid = h->num_sms * 8;
    const SparseView S = view_of(h->flow_sp);
    switch (h->flow_prec) {
        case CLB_F64: k_flow_set_pops<double><<<grid, 256, 0, h->stream>>>((double*)h->d_f, (double*)h->d_flink, S, h->g, odd, buf); break;
        case CLB_F32: k_flow_set_pops<float><<<grid, 256, 0, h->stream>>>((float*)h->d_f, (float*)h->d_flink, S, h->g, odd, buf); break;
        default: k_flow_set_pops<__half><<<grid, 256, 0, h->stream>>>((__half*)h->d_f, (__half*)h->d_flink, S, h->g, odd, buf); break;
    }
    e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    return cuda_check(h, e, "set populations");
}

clb_status flow_stats(clb_handle* h, double char_length, clb_flow_stats* out) {
    double* u = nullptr;
    double* acc = nullptr;
    cudaError_t e = cudaMalloc(&u, sizeof(double) * 3 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "stats buffer");
    e = cudaMalloc(&acc, sizeof(double) * 3);
    if (e != cudaSuccess) { cudaFree(u); return cuda_check(h, e, "stats buffer"); }
    clb_status s = flow_velocity(h, u, 0, false);
    if (s != CLB_OK) { cudaFree(u); cudaFree(acc); return s; }
    double init[3] = {0.0, 0.0, 0.0};
    long long neg = (long long)0x8000000000000000ULL;  // below every ordered key
    std::memcpy(&init[1], &neg, sizeof(double));
    cudaMemcpyAsync(acc, init, sizeof(init), cudaMemcpyHostToDevice, h->stream);
    k_flow_vstats<<<h->num_sms * 4, 256, 0, h->stream>>>(u, h->g, acc);
    double r[3];
    Tracer t;
    cudaMemcpyAsync(r, acc, sizeof(r), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(&t, h->d_tracer, sizeof(Tracer), cudaMemcpyDeviceToHost, h->stream);
    e = cudaStreamSynchronize(h->stream);
    cudaFree(u);
    cudaFree(acc);
    if (e != cudaSuccess) return cuda_check(h, e, "stats");
    long long key;
    std::memcpy(&key, &r[1], sizeof(key));
    long long bits = key >= 0 ? key : (key ^ 0x7fffffffffffffffLL);
    double mx;
    std::memcpy(&mx, &bits, sizeof(mx));
    const int64_t inner = (int64_t)(h->g.nx - 2) * h->g.plane;
    out->pore_mean_u = r[0] / (double)inner;
    out->pore_max_ux = mx;
    out->darcy_outlet_ux = r[2] / (double)h->g.plane;
    const double nu = (h->d.tau - 0.5) / 3.0;
    out->permeability = h->delta_p != 0 ? out->darcy_outlet_ux * nu * char_length / h->delta_p : 0.0;
    out->energy = t.energy;
    out->iterations = t.iterations;
    out->bgk_nodes = h->fp.n_bgk;
    out->active_nodes = h->flow_sp.K;
    return CLB_OK;
}

// Times every kernel variant (even step through TMA tiles or not; odd step compiled for 2 or 3
// resident CTAs, or pipelined through shared memory) over `steps` steps and keeps the fastest. The lattice state is saved before
// and restored after, so the run is unchanged. Writes a one-line report into `report`.
clb_status flow_autotune(clb_handle* h, int steps, char* report, int report_len) {
    if (steps < 2) steps = 2;
    steps += steps & 1;
    const size_t es = storage_size(h->flow_prec);
    const size_t fb = es * 19 * (size_t)h->flow_sp.KS, lb = es * (size_t)std::max<int64_t>(1, h->flow_sp.L) + 16;
    void* sf = nullptr;
    void* sl = nullptr;
    cudaError_t e = cudaMalloc(&sf, fb);
    if (e == cudaSuccess) e = cudaMalloc(&sl, lb);
    if (e != cudaSuccess) { cudaFree(sf); return cuda_check(h, e, "autotune buffers"); }
    Tracer tsave;
    cudaMemcpyAsync(sf, h->d_f, fb, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(sl, h->d_flink, lb, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(&tsave, h->d_tracer, sizeof(Tracer), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    const int64_t iters0 = h->flow_iters;
    const int save_tma = h->flow_even_tma, save_minb = h->flow_minb, save_pipe = h->flow_odd_pipe;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    int best_tma = save_tma, best_minb = save_minb, best_pipe = save_pipe;
    std::string rep;
    for (int tma = 1; tma >= 0; --tma)
        for (int v = 0; v < 3; ++v) {  // odd step: 3 or 2 resident CTAs, or pipelined
            const int minb = v == 1 ? 2 : 3, pipe = v == 2 ? 1 : 0;
            if (pipe && !h->flow_pipe_grid) continue;
            h->flow_even_tma = tma;
            h->flow_minb = minb;
            h->flow_odd_pipe = pipe;
            h->flow_grid = flow_gather_grid(h);
            flow_step(h, 2, false, 0.0);  // warm
            cudaEventRecord(a, h->stream);
            flow_step(h, steps, false, 0.0);
            cudaEventRecord(b, h->stream);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            char buf[96];
            if (pipe) snprintf(buf, sizeof(buf), "%stma=%d,pipe:%.1fus", rep.empty() ? "" : " ", tma, 1e3f * ms / steps);
            else snprintf(buf, sizeof(buf), "%stma=%d,minb=%d:%.1fus", rep.empty() ? "" : " ", tma, minb, 1e3f * ms / steps);
            rep += buf;
            if (ms < best) { best = ms; best_tma = tma; best_minb = minb; best_pipe = pipe; }
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->flow_even_tma = best_tma;
    h->flow_minb = best_minb;
    h->flow_odd_pipe = best_pipe;
    h->flow_grid = flow_gather_grid(h);
    cudaMemcpyAsync(h->d_f, sf, fb, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->d_flink, sl, lb, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->d_tracer, &tsave, sizeof(Tracer), cudaMemcpyHostToDevice, h->stream);
    e = cudaStreamSynchronize(h->stream);
    cudaFree(sf);
    cudaFree(sl);
    h->flow_iters = iters0;
    char buf[64];
    if (best_pipe) snprintf(buf, sizeof(buf), " -> tma=%d,pipe", best_tma);
    else snprintf(buf, sizeof(buf), " -> tma=%d,minb=%d", best_tma, best_minb);
    rep += buf;
    if (report && report_len > 0) {
        std::strncpy(report, rep.c_str(), (size_t)report_len - 1);
        report[report_len - 1] = 0;
    }
    return cuda_check(h, e, "autotune");
}

bool flow_batch_staged_available(int prec) { return prec == CLB_F64 || prec == CLB_F32; }

// resident CTAs of a staged batched kernel times the SM count (set up once per kernel)
static int batch_staged_grid(const void* kern, int threads, size_t smem, int num_sms) {
    struct Known { const void* kern; int blocks; };
    static std::mutex mu;
    static std::vector<Known> known;
    std::lock_guard<std::mutex> lock(mu);
    for (auto& kv : known)
        if (kv.kern == kern) return kv.blocks * num_sms;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem) != cudaSuccess || nb < 1) nb = 1;
    known.push_back({kern, nb});
    return nb * num_sms;
}

template <typename TS, typename TC>
static void launch_flow_batch_staged_t(const BatchView& B, bool odd, int num_sms, cudaStream_t st) {
    if (odd) {
        auto kern = k_flow_batch_odd<TS, TC>;
        const size_t sm = pipe_smem<TS>();
        const int grid = std::max(1, std::min(batch_staged_grid((const void*)kern, PIPE_THREADS, sm, num_sms), B.nft));
        kern<<<grid, PIPE_THREADS, sm, st>>>(B);
    } else {
        auto kern = k_flow_batch_even<TS, TC>;
        const size_t sm = even_smem<TS>();
        const int grid = std::max(1, std::min(batch_staged_grid((const void*)kern, TILE, sm, num_sms), B.nft));
        kern<<<grid, TILE, sm, st>>>(B);
    }
}

void launch_flow_batch_staged(const BatchView& B, int prec, bool odd, int num_sms, cudaStream_t st) {
    if (prec == CLB_F64) launch_flow_batch_staged_t<double, double>(B, odd, num_sms, st);
    else launch_flow_batch_staged_t<float, float>(B, odd, num_sms, st);
}

}  // namespace clb

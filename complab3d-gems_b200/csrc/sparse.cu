// sparse.cu -- construction of the compacted node layout (see sparse.cuh) on the device.
#include "sparse.cuh"

#include <algorithm>
#include <cstring>

namespace clb {

void sparse_free(SparseBuffers& b) {
    cudaFree(b.node); cudaFree(b.code); cudaFree(b.wall); cudaFree(b.linkbase);
    cudaFree(b.rowstart); cudaFree(b.rowmask); cudaFree(b.rowpre); cudaFree(b.idx_of);
    cudaFree(b.meta); cudaFree(b.dres); cudaFree(b.tlb); cudaFree(b.tdb);
    b = SparseBuffers();
}

// ------------------------------------------------------------------ device construction
//
// The layout is built on the device from the material map in a handful of passes: row-word
// masks and counts, an exclusive scan (rank bases), the node list and inverse index, the wall /
// edge masks with per-node link counts, a second scan (link bases), and one block per 256-node
// tile for the odd-step metadata (row bases as the midpoint of the tile's range, 16-bit
// residuals). Only K, L and an error flag come back to the host.

constexpr int SB_THREADS = 256;
constexpr int SCAN_ITEMS = 4;                        // elements per thread of a scan block
constexpr int SCAN_BLOCK = SB_THREADS * SCAN_ITEMS;  // elements per scan block

struct StoredTable {
    int8_t s[128];
};

// exclusive scan of one SCAN_BLOCK chunk of 32-bit counts; the chunk's total goes to bsum
__global__ void k_scan_chunks(const int32_t* __restrict__ in, int32_t* __restrict__ out, int64_t n,
                              int32_t* __restrict__ bsum) {
    __shared__ int32_t warp_tot[SB_THREADS / 32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + (int64_t)threadIdx.x * SCAN_ITEMS;
    int32_t v[SCAN_ITEMS], run = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        const int32_t t = base + j < n ? in[base + j] : 0;
        v[j] = run;  // exclusive within the thread
        run += t;
    }
    // exclusive scan of the thread totals over the block
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int32_t w = lane < SB_THREADS / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SB_THREADS / 32) warp_tot[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const int32_t off = (x - run) + (wid > 0 ? warp_tot[wid - 1] : 0);
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j)
        if (base + j < n) out[base + j] = v[j] + off;
    if (threadIdx.x == SB_THREADS - 1) bsum[blockIdx.x] = off + run;
}

__global__ void k_scan_add(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ boff) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += boff[i / SCAN_BLOCK];
}

// out = exclusive prefix sums of in[0..n) (in and out may alias: a block reads its whole chunk
// before it writes); *total (device) = the sum. Totals stay below 2^31 (the layout checks K and L).
static cudaError_t scan_exclusive(const int32_t* in, int32_t* out, int64_t n, int32_t* total, cudaStream_t st) {
    const int64_t nb = std::max<int64_t>(1, (n + SCAN_BLOCK - 1) / SCAN_BLOCK);
    int32_t* bsum = nullptr;
    cudaError_t e = cudaMalloc(&bsum, sizeof(int32_t) * (nb + 1));
    if (e != cudaSuccess) return e;
    k_scan_chunks<<<(unsigned)nb, SB_THREADS, 0, st>>>(in, out, n, bsum);
    if (nb > 1) {
        e = scan_exclusive(bsum, bsum, nb, total, st);
        if (e == cudaSuccess)
            k_scan_add<<<(unsigned)((n + SB_THREADS - 1) / SB_THREADS), SB_THREADS, 0, st>>>(out, n, bsum);
    } else {
        e = cudaMemcpyAsync(total, bsum, sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    cudaFree(bsum);
    return e;
}

// stored bits of every 32-voxel word of every row, and their counts
__global__ void k_sb_words(const int8_t* __restrict__ mat, const StoredTable T, int R, int nz, int W,
                           uint32_t* __restrict__ rowmask, int32_t* __restrict__ wcount) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)R * W) return;
    const int r = (int)(i / W), w = (int)(i - (int64_t)r * W);
    uint32_t m = 0;
    for (int b = 0; b < 32; ++b) {
        const int z = w * 32 + b;
        if (z >= nz) break;
        if (T.s[(uint8_t)mat[(int64_t)r * nz + z] & 127]) m |= 1u << b;
    }
    rowmask[i] = m;
    wcount[i] = __popc(m);
}

// row bases from the scanned word prefixes
__global__ void k_sb_rows(const int32_t* __restrict__ wpre, int R, int W, int32_t* __restrict__ rowstart,
                          int32_t* __restrict__ rowpre) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)R * W) return;
    const int r = (int)(i / W);
    const int32_t s0 = wpre[(int64_t)r * W];
    rowpre[i] = wpre[i] - s0;
    if (i == (int64_t)r * W) rowstart[r] = s0;
}

// node list, codes and inverse index (lexicographic order: x slowest, z fastest)
__global__ void k_sb_nodes(const int8_t* __restrict__ mat, int64_t N, int nz, int W, const uint32_t* __restrict__ rowmask,
                           const int32_t* __restrict__ wpre, int32_t* __restrict__ idx, int32_t* __restrict__ node,
                           int8_t* __restrict__ code) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int64_t r = n / nz;
    const int z = (int)(n - r * nz), w = z >> 5;
    const uint32_t m = rowmask[r * W + w];
    if (!((m >> (z & 31)) & 1u)) {
        idx[n] = -1;
        return;
    }
    const int32_t k = wpre[r * W + w] + __popc(m & ((1u << (z & 31)) - 1u));
    idx[n] = k;
    node[k] = (int32_t)n;
    code[k] = mat[n];
}

// wall mask (neighbour in the box and not stored), edge mask (neighbour outside the box), links
template <int Q>
__global__ void k_sb_wall(const int32_t* __restrict__ node, const int32_t* __restrict__ idx, int64_t K, Geom G,
                          uint32_t* __restrict__ wall, uint32_t* __restrict__ edge, int32_t* __restrict__ lcount) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    int x, y, z;
    decode(G, node[k], x, y, z);
    uint32_t wm = 0, em = 0;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        int cx, cy, cz, oi;
        qdir<Q>(i, cx, cy, cz, oi);
        const int X = x + cx, Y = y + cy, Z = z + cz;
        if ((unsigned)X >= (unsigned)G.nx || (unsigned)Y >= (unsigned)G.ny || (unsigned)Z >= (unsigned)G.nz) {
            em |= 1u << i;
            continue;
        }
        if (idx[(int64_t)X * G.plane + (int64_t)Y * G.nz + Z] < 0) wm |= 1u << i;
    }
    wall[k] = wm;
    edge[k] = em;
    lcount[k] = __popc(wm);
}

__device__ __forceinline__ int32_t sb_rank(const int32_t* rowstart, const int32_t* rowpre, const uint32_t* rowmask,
                                           int W, int r, int z) {
    const int w = z >> 5;
    return rowstart[r] + rowpre[(int64_t)r * W + w] + __popc(rowmask[(int64_t)r * W + w] & ((1u << (z & 31)) - 1u));
}

// odd-step metadata of one 256-node tile per block (TILE threads)
template <int Q>
__global__ void __launch_bounds__(TILE) k_sb_tiles(const int32_t* __restrict__ node, int64_t K, Geom G, int W,
                                                   const int32_t* __restrict__ rowstart, const int32_t* __restrict__ rowpre,
                                                   const uint32_t* __restrict__ rowmask, const uint32_t* __restrict__ wall,
                                                   const uint32_t* __restrict__ edge, const int32_t* __restrict__ linkbase,
                                                   uint32_t* __restrict__ meta, int16_t* __restrict__ dres,
                                                   int32_t* __restrict__ tlb, int32_t* __restrict__ tdb, int* __restrict__ err) {
    constexpr int NR = Q == 19 ? 8 : 4;
    __shared__ int32_t lo[NR], hi[NR], base[NR];
    const int t = blockIdx.x;
    const int64_t k0 = (int64_t)t * TILE, k = k0 + threadIdx.x;
    if (threadIdx.x < NR) {
        lo[threadIdx.x] = INT32_MAX;
        hi[threadIdx.x] = INT32_MIN;
    }
    __syncthreads();
    int32_t d[NR];
    uint32_t rbits = 0;
    const bool live = k < K;
    if (live) {
        int x, y, z;
        decode(G, node[k], x, y, z);
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                if (dx == 0 && dy == 0) continue;
                if (Q == 7 && dx != 0 && dy != 0) continue;
                const int s_ = Q == 19 ? row8(dx, dy) : row4(dx, dy);
                int32_t v = 0;
                if (x + dx >= 0 && x + dx < G.nx && y + dy >= 0 && y + dy < G.ny) {
                    const int r2 = (x + dx) * G.ny + (y + dy);
                    v = sb_rank(rowstart, rowpre, rowmask, W, r2, z) - (int32_t)k;
                    if (Q == 19 && ((rowmask[(int64_t)r2 * W + (z >> 5)] >> (z & 31)) & 1u)) rbits |= 1u << s_;
                }
                d[s_] = v;
                atomicMin(&lo[s_], v);
                atomicMax(&hi[s_], v);
            }
    }
    __syncthreads();
    if (threadIdx.x < NR) {
        const int s_ = threadIdx.x;
        const int32_t b = lo[s_] == INT32_MAX ? 0 : (int32_t)(((int64_t)lo[s_] + hi[s_]) / 2);
        if (lo[s_] != INT32_MAX && ((int64_t)hi[s_] - b > 32767 || (int64_t)b - lo[s_] > 32767)) atomicExch(err, 1);
        base[s_] = b;
        tdb[(int64_t)t * NR + s_] = b;
    }
    if (threadIdx.x == 0) tlb[t] = linkbase[k0];
    __syncthreads();
    if (!live) return;
#pragma unroll
    for (int s_ = 0; s_ < NR; ++s_) dres[k * NR + s_] = (int16_t)(d[s_] - base[s_]);
    const uint32_t lres = (uint32_t)(linkbase[k] - linkbase[k0]);
    if (Q == 19) {
        meta[2 * k] = (wall[k] & 0x7FFFFu) | (lres << 19);
        meta[2 * k + 1] = (edge[k] & 0x7FFFFu) | (rbits << 19);
    } else {
        meta[k] = (wall[k] & 0x7Fu) | ((edge[k] & 0x7Fu) << 7) | (lres << 14);
    }
}

static unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + SB_THREADS - 1) / SB_THREADS); }

clb_status sparse_build(clb_handle* h, const int8_t* stored_by_code, int q, SparseBuffers& out,
                        const std::vector<int8_t>* map) {
    sparse_free(out);
    if (!map) {
        clb_status st = host_mat_sync(h);
        if (st != CLB_OK) return st;
    }
    const std::vector<int8_t>& mat = map ? *map : h->h_mat;
    const Geom& G = h->g;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int64_t N = G.N;
    const int R = nx * ny, W = (nz + 31) / 32;
    const int64_t RW = (int64_t)R * W;
    const int NR = q == 19 ? 8 : 4;
    // node ranks and link counts are scanned in 32 bits: at most N nodes, (q - 1) links each
    if (N * (int64_t)(q - 1) > INT32_MAX) return fail(h, CLB_INVALID_ARG, "lattice too large for 32-bit node indices");
    cudaStream_t st = h->stream;
    StoredTable T;
    for (int c = 0; c < 128; ++c) T.s[c] = stored_by_code[c] ? 1 : 0;

    int8_t* dmat = nullptr;
    int32_t *wcount = nullptr, *scal = nullptr, *lcount = nullptr;
    uint32_t* edge = nullptr;
    int* err = nullptr;
    int32_t hs[2] = {0, 0};
    int herr = 0;
    cudaError_t e = cudaMalloc(&dmat, (size_t)N);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmat, mat.data(), (size_t)N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMalloc(&scal, sizeof(int32_t) * 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(scal, 0, sizeof(int32_t) * 2, st);
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMalloc(&out.rowmask, sizeof(uint32_t) * RW);
    if (e == cudaSuccess) e = cudaMalloc(&wcount, sizeof(int32_t) * RW);
    if (e == cudaSuccess) {
        k_sb_words<<<blocks_for(RW), SB_THREADS, 0, st>>>(dmat, T, R, nz, W, out.rowmask, wcount);
        e = scan_exclusive(wcount, wcount, RW, scal, st);  // wcount now holds the word prefixes
    }
    if (e == cudaSuccess) e = cudaMemcpy(&hs[0], scal, sizeof(int32_t), cudaMemcpyDeviceToHost);
    const int64_t K = hs[0];
    if (e == cudaSuccess) e = cudaMalloc(&out.rowstart, sizeof(int32_t) * std::max(1, R));
    if (e == cudaSuccess) e = cudaMalloc(&out.rowpre, sizeof(int32_t) * RW);
    if (e == cudaSuccess) e = cudaMalloc(&out.idx_of, sizeof(int32_t) * N);
    if (e == cudaSuccess) e = cudaMalloc(&out.node, sizeof(int32_t) * std::max<int64_t>(1, K));
    if (e == cudaSuccess) e = cudaMalloc(&out.code, std::max<int64_t>(1, K));
    if (e == cudaSuccess) {
        k_sb_rows<<<blocks_for(RW), SB_THREADS, 0, st>>>(wcount, R, W, out.rowstart, out.rowpre);
        k_sb_nodes<<<blocks_for(N), SB_THREADS, 0, st>>>(dmat, N, nz, W, out.rowmask, wcount, out.idx_of, out.node,
                                                          out.code);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMalloc(&out.wall, sizeof(uint32_t) * std::max<int64_t>(1, K));
    if (e == cudaSuccess) e = cudaMalloc(&edge, sizeof(uint32_t) * std::max<int64_t>(1, K));
    if (e == cudaSuccess) e = cudaMalloc(&lcount, sizeof(int32_t) * std::max<int64_t>(1, K));
    if (e == cudaSuccess) e = cudaMalloc(&out.linkbase, sizeof(int32_t) * std::max<int64_t>(1, K));
    if (e == cudaSuccess && K > 0) {
        if (q == 19) k_sb_wall<19><<<blocks_for(K), SB_THREADS, 0, st>>>(out.node, out.idx_of, K, G, out.wall, edge, lcount);
        else k_sb_wall<7><<<blocks_for(K), SB_THREADS, 0, st>>>(out.node, out.idx_of, K, G, out.wall, edge, lcount);
        e = scan_exclusive(lcount, out.linkbase, K, scal + 1, st);
        if (e == cudaSuccess) e = cudaMemcpy(&hs[1], scal + 1, sizeof(int32_t), cudaMemcpyDeviceToHost);
    }
    const int64_t L = hs[1];
    const int64_t T_ = std::max<int64_t>(1, (K + TILE - 1) / TILE);
    if (e == cudaSuccess) e = cudaMalloc(&out.meta, sizeof(uint32_t) * std::max<int64_t>(1, K) * (q == 19 ? 2 : 1));
    if (e == cudaSuccess) e = cudaMalloc(&out.dres, sizeof(int16_t) * std::max<int64_t>(1, K) * NR);
    if (e == cudaSuccess) e = cudaMalloc(&out.tlb, sizeof(int32_t) * T_);
    if (e == cudaSuccess) e = cudaMalloc(&out.tdb, sizeof(int32_t) * T_ * NR);
    if (e == cudaSuccess && K > 0) {
        const unsigned nt = (unsigned)((K + TILE - 1) / TILE);
        if (q == 19)
            k_sb_tiles<19><<<nt, TILE, 0, st>>>(out.node, K, G, W, out.rowstart, out.rowpre, out.rowmask, out.wall, edge,
                                                 out.linkbase, out.meta, out.dres, out.tlb, out.tdb, err);
        else
            k_sb_tiles<7><<<nt, TILE, 0, st>>>(out.node, K, G, W, out.rowstart, out.rowpre, out.rowmask, out.wall, edge,
                                                out.linkbase, out.meta, out.dres, out.tlb, out.tdb, err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dmat);
    cudaFree(wcount);
    cudaFree(scal);
    cudaFree(lcount);
    cudaFree(edge);
    cudaFree(err);
    if (e != cudaSuccess) return cuda_check(h, e, "sparse layout");
    if (herr) return fail(h, CLB_INVALID_ARG, "neighbour-row offsets within a 256-node tile exceed 16 bits");
    const int64_t KS = ((int64_t)K + TILE - 1) / TILE * TILE;
    if (KS * q > INT32_MAX) return fail(h, CLB_INVALID_ARG, "lattice exceeds 2^31 populations per species");
    out.K = K;
    out.L = L;
    out.W = W;
    out.NR = NR;
    out.KS = std::max<int64_t>(KS, TILE);
    out.SS = q * out.KS + std::max<int64_t>(TILE, (L + TILE - 1) / TILE * TILE);
    if (out.SS > INT32_MAX) return fail(h, CLB_INVALID_ARG, "lattice exceeds 2^31 slots per species");
    return CLB_OK;
}

}  // namespace clb

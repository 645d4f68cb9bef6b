// sparse.cuh -- the compacted node layout shared by the flow and transport lattices.
//
// Only the nodes a step launches (collide or stream nodes) are stored: node k = 0..K-1 in
// lexicographic order, populations f[q][K]. A full-way bounce-back node is a no-op on the AA
// pattern; the only part of its state that matters is, for every link (a, i) from a stored node
// a into it, the one population a sent into it on the last odd step. That population is kept in
// a link slot: link[linkbase[k] + rank of i among k's wall links] (node-major). Every other slot
// of a wall node is never read by a stored node and is not kept.
//
// Neighbour indices come from per-row bitmasks (a row = one (x, y) column along z): the compact
// index of (x', y', z) is rowstart[r'] + rowpre[r'*W + z/32] + popc(rowmask[r'*W + z/32] below z),
// about 0.3 bytes of metadata per voxel instead of 4 bytes per neighbour.
#pragma once

#include "clb_internal.cuh"

namespace clb {

struct SparseView {
    const int32_t* node;      // [K] dense index of compact node k
    const int8_t* code;       // [K] material code
    const uint32_t* wall;     // [K] bit i: x + c_i lies in the box and is not stored
    const int32_t* linkbase;  // [K] first link slot of node k
    const int32_t* rowstart;  // [R] compact index of the first stored node of row r
    const uint32_t* rowmask;  // [R*W] stored bits of row r
    const int32_t* rowpre;    // [R*W] stored nodes of row r in words < w
    const int32_t* idx_of;    // [N] compact index or -1 (non-hot kernels)
    const uint32_t* meta;     // odd-step metadata, see below
    const int16_t* dres;
    const int32_t* tlb;
    const int32_t* tdb;
    int64_t K, L;
    int64_t KS;               // population row stride (K rounded up to a multiple of TILE)
    int64_t SS;               // species stride (transport lattices): 7 rows, then the link slots
    int W, NR;
};

inline SparseView view_of(const SparseBuffers& b) {
    return SparseView{b.node, b.code, b.wall, b.linkbase, b.rowstart, b.rowmask, b.rowpre, b.idx_of,
                      b.meta, b.dres, b.tlb, b.tdb, b.K, b.L, b.KS, b.SS, b.W, b.NR};
}

// Odd-step metadata, built once per geometry so the gather step needs no coordinate decode and
// no row lookups. Nodes are grouped in tiles of 256 (tile t = k >> 8).
//   D3Q19, two words per node:
//     meta[2k]   bits 0..18 wall mask, bits 19..31 link slot of the node minus tlb[t]
//     meta[2k+1] bits 0..18 edge mask (a + c_i outside the box), bits 19..26 row bits: whether
//                (x+dx, y+dy, z) is stored, for the 8 neighbour rows
//   D3Q7, one word per node: bits 0..6 wall mask, 7..13 edge mask, 14..31 link residual.
//   dres[k*NR + s] + tdb[t*NR + s] = rank of (x+dx, y+dy, z) in its row (compact index of the
//   first stored node of that row at or above z) minus k, for the NR neighbour rows
//   (D3Q19: the 8 rows (dx, dy) != (0, 0) in row-slot order; D3Q7: (+1,0), (-1,0), (0,+1), (0,-1)).
constexpr int TILE = 256;
__host__ __device__ constexpr int row8(int dx, int dy) {
    return (dx + 1) * 3 + (dy + 1) < 4 ? (dx + 1) * 3 + (dy + 1) : (dx + 1) * 3 + (dy + 1) - 1;
}
__host__ __device__ constexpr int row4(int dx, int dy) {
    return dx == 1 ? 0 : (dx == -1 ? 1 : (dy == 1 ? 2 : 3));
}

// Build on the host from the material map: a node is stored when stored_by_code[code] != 0.
// q = 19 or 7 selects the velocity set of the wall masks.
// `map` (default: the handle's material map) gives the material of every voxel.
clb_status sparse_build(clb_handle* h, const int8_t* stored_by_code, int q, SparseBuffers& out,
                        const std::vector<int8_t>* map = nullptr);
void sparse_free(SparseBuffers& b);

// rank of z in row r: stored nodes of the row below z, plus the row's start
__device__ __forceinline__ int row_rank(const SparseView& S, int r, int z) {
    const int w = z >> 5;
    const int o = r * S.W + w;
    return S.rowstart[r] + S.rowpre[o] + __popc(S.rowmask[o] & ((1u << (z & 31)) - 1u));
}
__device__ __forceinline__ bool row_bit(const SparseView& S, int r, int z) {
    return (S.rowmask[r * S.W + (z >> 5)] >> (z & 31)) & 1u;
}

// Wall links and the AA parity. A full-way bounce-back link (a, i) (a stored, b = a + c_i a
// wall) is a two-step delay line: what a sends into b comes back as a's incoming opp(i) two
// steps later. It needs two slots, one per step parity:
//   odd steps  use Y = f[opp(i)][a] (a's own slot): read as incoming opp(i), then overwritten
//              with outgoing i -- exactly the edge-reflection rule, so an odd step touches no
//              link and writes every stored slot once (no partially written sectors);
//   even steps use X = link slot (a, i): read as incoming opp(i), overwritten with outgoing i;
//              Y keeps its value (the even step writes it back unchanged so its sector is whole).
// Natural (post-stream, incoming) populations of dense node n in terms of this storage:
//   n stored (k), source s = n - c_i:
//     out of box -> f[i][k];  wall -> even state X(k, opp(i)), odd state f[i][k];
//     stored (ks) -> even state f[i][k], odd state f[opp(i)][ks]
//   n a wall node, a = n - c_i stored (ka) -> even state f[opp(i)][ka], odd state X(ka, i);
//   anything else is never touched and keeps its initial value.
// "even state" = the next step is even (after an odd step, or at initialisation).
template <typename TS>
__device__ __forceinline__ TS* link_slot(const SparseView& S, TS* link, int k, int j) {
    return link + S.linkbase[k] + __popc(S.wall[k] & ((1u << j) - 1u));
}

template <int Q>
__device__ __forceinline__ void qdir(int i, int& cx, int& cy, int& cz, int& oi) {
    cx = (Q == 19) ? q19cx(i) : q7cx(i);
    cy = (Q == 19) ? q19cy(i) : q7cy(i);
    cz = (Q == 19) ? q19cz(i) : q7cz(i);
    oi = (Q == 19) ? q19opp(i) : q7opp(i);
}

// Storage location of natural population i of dense node n (nullptr: untouched, initial value).
template <typename TS, int Q>
__device__ __forceinline__ TS* natural_slot(const SparseView& S, const Geom& G, TS* f, TS* link, int64_t n, int x,
                                            int y, int z, int i, int odd) {
    const int k = S.idx_of[n];
    int cx, cy, cz, oi;
    qdir<Q>(i, cx, cy, cz, oi);
    if (k >= 0) {
        if (i == 0) return f + k;
        const int sx = x - cx, sy = y - cy, sz = z - cz;
        if ((unsigned)sx >= (unsigned)G.nx || (unsigned)sy >= (unsigned)G.ny || (unsigned)sz >= (unsigned)G.nz)
            return f + (int64_t)i * S.KS + k;
        const int ks = S.idx_of[(int64_t)sx * G.plane + sy * G.nz + sz];
        if (ks < 0) return odd ? f + (int64_t)i * S.KS + k : link_slot(S, link, k, oi);
        return odd ? f + (int64_t)oi * S.KS + ks : f + (int64_t)i * S.KS + k;
    }
    if (i == 0) return nullptr;
    const int ax = x - cx, ay = y - cy, az = z - cz;
    if ((unsigned)ax >= (unsigned)G.nx || (unsigned)ay >= (unsigned)G.ny || (unsigned)az >= (unsigned)G.nz)
        return nullptr;
    const int ka = S.idx_of[(int64_t)ax * G.plane + ay * G.nz + az];
    if (ka < 0) return nullptr;
    return odd ? link_slot(S, link, ka, i) : f + (int64_t)oi * S.KS + ka;
}

template <typename TS, typename TC, int Q>
__device__ __forceinline__ void natural(const SparseView& S, const Geom& G, const TS* __restrict__ f,
                                        const TS* __restrict__ link, int64_t n, int odd, const TC* init,
                                        TC* out) {
    int x, y, z;
    decode(G, n, x, y, z);
    for (int i = 0; i < Q; ++i) {
        const TS* p = natural_slot<const TS, Q>(S, G, f, link, n, x, y, z, i, odd);
        out[i] = p ? ld<TS, TC>(p) : init[i];
    }
}

// Inverse of natural(): write the natural populations of node n into the storage; populations
// that no stored node ever reads are dropped.
template <typename TS, int Q>
__device__ __forceinline__ void put_natural(const SparseView& S, const Geom& G, TS* __restrict__ f,
                                            TS* __restrict__ link, int64_t n, int odd, const double* in) {
    int x, y, z;
    decode(G, n, x, y, z);
    for (int i = 0; i < Q; ++i) {
        TS* p = natural_slot<TS, Q>(S, G, f, link, n, x, y, z, i, odd);
        if (!p) continue;
        if constexpr (std::is_same<TS, __half>::value) *p = to_half(in[i]);
        else *p = (TS)in[i];
    }
}

}  // namespace clb

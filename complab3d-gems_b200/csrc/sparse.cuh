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
    int64_t K, L;
    int W;
};

inline SparseView view_of(const SparseBuffers& b) {
    return SparseView{b.node, b.code, b.wall, b.linkbase, b.rowstart, b.rowmask, b.rowpre, b.idx_of, b.K, b.L, b.W};
}

// Build on the host from the material map: a node is stored when stored_by_code[code] != 0.
// q = 19 or 7 selects the velocity set of the wall masks.
clb_status sparse_build(clb_handle* h, const int8_t* stored_by_code, int q, SparseBuffers& out);
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

// Value of the dense AA slot (j, m) (population j stored at node m) in the sparse layout:
// stored node -> f; wall node reached by a link from m - c_j -> that link slot; otherwise the
// slot is never touched and holds its initial value `init`.
template <typename TS, typename TC, int Q>
__device__ __forceinline__ TC dense_slot(const SparseView& S, const Geom& G, const TS* __restrict__ f,
                                         const TS* __restrict__ link, int j, int64_t m, int mx, int my, int mz,
                                         TC init) {
    const int k = S.idx_of[m];
    if (k >= 0) return ld<TS, TC>(f + (int64_t)j * S.K + k);
    const int cx = (Q == 19) ? q19cx(j) : q7cx(j);
    const int cy = (Q == 19) ? q19cy(j) : q7cy(j);
    const int cz = (Q == 19) ? q19cz(j) : q7cz(j);
    const int px = mx - cx, py = my - cy, pz = mz - cz;
    if (j == 0 || (unsigned)px >= (unsigned)G.nx || (unsigned)py >= (unsigned)G.ny || (unsigned)pz >= (unsigned)G.nz)
        return init;
    const int p = S.idx_of[(int64_t)px * G.plane + py * G.nz + pz];
    if (p < 0) return init;
    const uint32_t wm = S.wall[p];
    return ld<TS, TC>(link + S.linkbase[p] + __popc(wm & ((1u << j) - 1u)));
}

// Natural (incoming, post-stream) populations of dense node n under the AA parity rule.
template <typename TS, typename TC, int Q>
__device__ __forceinline__ void natural(const SparseView& S, const Geom& G, const TS* __restrict__ f,
                                        const TS* __restrict__ link, int64_t n, int odd, const TC* init,
                                        TC* out) {
    int x, y, z;
    decode(G, n, x, y, z);
    for (int i = 0; i < Q; ++i) {
        const int cx = (Q == 19) ? q19cx(i) : q7cx(i);
        const int cy = (Q == 19) ? q19cy(i) : q7cy(i);
        const int cz = (Q == 19) ? q19cz(i) : q7cz(i);
        const int oi = (Q == 19) ? q19opp(i) : q7opp(i);
        if (!odd || i == 0) {
            out[i] = dense_slot<TS, TC, Q>(S, G, f, link, i, n, x, y, z, init[i]);
        } else {
            const int sx = x - cx, sy = y - cy, sz = z - cz;
            if ((unsigned)sx < (unsigned)G.nx && (unsigned)sy < (unsigned)G.ny && (unsigned)sz < (unsigned)G.nz)
                out[i] = dense_slot<TS, TC, Q>(S, G, f, link, oi, (int64_t)sx * G.plane + sy * G.nz + sz, sx, sy,
                                               sz, init[oi]);
            else
                out[i] = dense_slot<TS, TC, Q>(S, G, f, link, i, n, x, y, z, init[i]);
        }
    }
}

// Inverse of natural(): write the natural populations of node n into the sparse layout; slots
// that are never touched by a stored node are dropped.
template <typename TS, int Q>
__device__ __forceinline__ void put_dense_slot(const SparseView& S, const Geom& G, TS* __restrict__ f,
                                               TS* __restrict__ link, int j, int64_t m, int mx, int my, int mz,
                                               double v) {
    const int k = S.idx_of[m];
    TS* dst = nullptr;
    if (k >= 0) {
        dst = f + (int64_t)j * S.K + k;
    } else if (j != 0) {
        const int cx = (Q == 19) ? q19cx(j) : q7cx(j);
        const int cy = (Q == 19) ? q19cy(j) : q7cy(j);
        const int cz = (Q == 19) ? q19cz(j) : q7cz(j);
        const int px = mx - cx, py = my - cy, pz = mz - cz;
        if ((unsigned)px < (unsigned)G.nx && (unsigned)py < (unsigned)G.ny && (unsigned)pz < (unsigned)G.nz) {
            const int p = S.idx_of[(int64_t)px * G.plane + py * G.nz + pz];
            if (p >= 0) dst = link + S.linkbase[p] + __popc(S.wall[p] & ((1u << j) - 1u));
        }
    }
    if (!dst) return;
    if constexpr (std::is_same<TS, __half>::value) *dst = __double2half(v);
    else *dst = (TS)v;
}

template <typename TS, int Q>
__device__ __forceinline__ void put_natural(const SparseView& S, const Geom& G, TS* __restrict__ f,
                                            TS* __restrict__ link, int64_t n, int odd, const double* in) {
    int x, y, z;
    decode(G, n, x, y, z);
    for (int i = 0; i < Q; ++i) {
        const int cx = (Q == 19) ? q19cx(i) : q7cx(i);
        const int cy = (Q == 19) ? q19cy(i) : q7cy(i);
        const int cz = (Q == 19) ? q19cz(i) : q7cz(i);
        const int oi = (Q == 19) ? q19opp(i) : q7opp(i);
        const int sx = x - cx, sy = y - cy, sz = z - cz;
        if (odd && i != 0 && (unsigned)sx < (unsigned)G.nx && (unsigned)sy < (unsigned)G.ny &&
            (unsigned)sz < (unsigned)G.nz)
            put_dense_slot<TS, Q>(S, G, f, link, oi, (int64_t)sx * G.plane + sy * G.nz + sz, sx, sy, sz, in[i]);
        else
            put_dense_slot<TS, Q>(S, G, f, link, i, n, x, y, z, in[i]);
    }
}

}  // namespace clb

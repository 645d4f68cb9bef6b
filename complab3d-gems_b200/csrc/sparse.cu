// sparse.cu -- host construction of the compacted node layout (see sparse.cuh).
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

template <typename T>
static cudaError_t upload(T*& dst, const std::vector<T>& src, cudaStream_t s) {
    cudaError_t e = cudaMalloc(&dst, sizeof(T) * std::max<size_t>(1, src.size()));
    if (e != cudaSuccess || src.empty()) return e;
    return cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, s);
}

clb_status sparse_build(clb_handle* h, const int8_t* stored_by_code, int q, SparseBuffers& out,
                        const std::vector<int8_t>* map) {
    sparse_free(out);
    const std::vector<int8_t>& mat = map ? *map : h->h_mat;
    const Geom& G = h->g;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int64_t N = G.N;
    const int R = nx * ny, W = (nz + 31) / 32;
    std::vector<int32_t> idx(N, -1), node, rowstart(R), rowpre((size_t)R * W);
    std::vector<int8_t> code;
    std::vector<uint32_t> rowmask((size_t)R * W, 0u);
    node.reserve(N / 2);
    code.reserve(N / 2);
    int32_t K = 0;
    for (int r = 0; r < R; ++r) {
        rowstart[r] = K;
        int32_t pre = 0;
        for (int w = 0; w < W; ++w) {
            rowpre[(size_t)r * W + w] = pre;
            uint32_t m = 0;
            for (int b = 0; b < 32; ++b) {
                const int z = w * 32 + b;
                if (z >= nz) break;
                const int64_t n = (int64_t)r * nz + z;
                const int8_t c = mat[n];
                if (stored_by_code[(uint8_t)c & 127]) {
                    m |= 1u << b;
                    idx[n] = K++;
                    node.push_back((int32_t)n);
                    code.push_back(c);
                }
            }
            rowmask[(size_t)r * W + w] = m;
            pre += __builtin_popcount(m);
        }
    }
    std::vector<uint32_t> wall(K, 0u);
    std::vector<int32_t> linkbase(K, 0);
    int64_t L = 0;
    for (int32_t k = 0; k < K; ++k) {
        const int64_t n = node[k];
        const int x = (int)(n / G.plane), rr = (int)(n - (int64_t)x * G.plane), y = rr / nz, z = rr - y * nz;
        uint32_t wm = 0;
        for (int i = 1; i < q; ++i) {
            const int cx = q == 19 ? q19cx(i) : q7cx(i), cy = q == 19 ? q19cy(i) : q7cy(i),
                      cz = q == 19 ? q19cz(i) : q7cz(i);
            const int X = x + cx, Y = y + cy, Z = z + cz;
            if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
            if (idx[(int64_t)X * G.plane + (int64_t)Y * nz + Z] < 0) wm |= 1u << i;
        }
        wall[k] = wm;
        linkbase[k] = (int32_t)L;
        L += __builtin_popcount(wm);
    }
    if (L > INT32_MAX) return fail(h, CLB_INVALID_ARG, "too many wall links");
    const int64_t KS = ((int64_t)K + TILE - 1) / TILE * TILE;
    if (KS * q > INT32_MAX) return fail(h, CLB_INVALID_ARG, "lattice exceeds 2^31 populations per species");

    // ---- odd-step metadata
    const int NR = q == 19 ? 8 : 4;
    const int64_t T = ((int64_t)K + TILE - 1) / TILE;
    std::vector<uint32_t> meta((size_t)K * (q == 19 ? 2 : 1));
    std::vector<int16_t> dres((size_t)K * NR);
    std::vector<int32_t> tlb(std::max<int64_t>(1, T)), tdb((size_t)std::max<int64_t>(1, T) * NR);
    std::vector<int64_t> dkf((size_t)TILE * NR);
    auto rank = [&](int r, int z) -> int64_t {
        const int w = z >> 5;
        const uint32_t m = rowmask[(size_t)r * W + w] & ((1u << (z & 31)) - 1u);
        return (int64_t)rowstart[r] + rowpre[(size_t)r * W + w] + __builtin_popcount(m);
    };
    for (int64_t t = 0; t < T; ++t) {
        const int64_t k0 = t * TILE, k1 = std::min<int64_t>(K, k0 + TILE);
        tlb[t] = linkbase[k0];
        std::vector<int64_t> lo(NR, INT64_MAX), hi(NR, INT64_MIN);
        std::fill(dkf.begin(), dkf.end(), 0);
        for (int64_t k = k0; k < k1; ++k) {
            const int64_t n = node[k];
            const int x = (int)(n / G.plane), rr = (int)(n - (int64_t)x * G.plane), y = rr / nz, z = rr - y * nz;
            uint32_t edge = 0, rbits = 0;
            for (int i = 1; i < q; ++i) {
                const int cx = q == 19 ? q19cx(i) : q7cx(i), cy = q == 19 ? q19cy(i) : q7cy(i),
                          cz = q == 19 ? q19cz(i) : q7cz(i);
                const int X = x + cx, Y = y + cy, Z = z + cz;
                if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) edge |= 1u << i;
            }
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy) {
                    if (dx == 0 && dy == 0) continue;
                    if (q == 7 && dx != 0 && dy != 0) continue;
                    const int s_ = q == 19 ? row8(dx, dy) : row4(dx, dy);
                    int64_t d = 0;
                    if (x + dx >= 0 && x + dx < nx && y + dy >= 0 && y + dy < ny) {
                        const int r2 = (x + dx) * ny + (y + dy);
                        d = rank(r2, z) - k;
                        if (q == 19 && ((rowmask[(size_t)r2 * W + (z >> 5)] >> (z & 31)) & 1u)) rbits |= 1u << s_;
                    }
                    dkf[(size_t)(k - k0) * NR + s_] = d;
                    lo[(size_t)s_] = std::min(lo[(size_t)s_], d);
                    hi[(size_t)s_] = std::max(hi[(size_t)s_], d);
                }
            const uint32_t lres = (uint32_t)(linkbase[k] - tlb[t]);
            if (q == 19) {
                meta[(size_t)2 * k] = (wall[k] & 0x7FFFFu) | (lres << 19);
                meta[(size_t)2 * k + 1] = (edge & 0x7FFFFu) | (rbits << 19);
            } else {
                meta[(size_t)k] = (wall[k] & 0x7Fu) | ((edge & 0x7Fu) << 7) | (lres << 14);
            }
        }
        for (int s_ = 0; s_ < NR; ++s_) {
            const int64_t base = lo[(size_t)s_] == INT64_MAX ? 0 : (lo[(size_t)s_] + hi[(size_t)s_]) / 2;
            if (lo[(size_t)s_] != INT64_MAX && (hi[(size_t)s_] - base > 32767 || base - lo[(size_t)s_] > 32767))
                return fail(h, CLB_INVALID_ARG, "neighbour-row offsets within a 256-node tile exceed 16 bits");
            tdb[(size_t)t * NR + s_] = (int32_t)base;
            for (int64_t k = k0; k < k1; ++k)
                dres[(size_t)k * NR + s_] = (int16_t)(dkf[(size_t)(k - k0) * NR + s_] - base);
        }
    }
    cudaError_t e = cudaSuccess;
    cudaStream_t s = h->stream;
    if (e == cudaSuccess) e = upload(out.node, node, s);
    if (e == cudaSuccess) e = upload(out.code, code, s);
    if (e == cudaSuccess) e = upload(out.wall, wall, s);
    if (e == cudaSuccess) e = upload(out.linkbase, linkbase, s);
    if (e == cudaSuccess) e = upload(out.rowstart, rowstart, s);
    if (e == cudaSuccess) e = upload(out.rowmask, rowmask, s);
    if (e == cudaSuccess) e = upload(out.rowpre, rowpre, s);
    if (e == cudaSuccess) e = upload(out.idx_of, idx, s);
    if (e == cudaSuccess) e = upload(out.meta, meta, s);
    if (e == cudaSuccess) e = upload(out.dres, dres, s);
    if (e == cudaSuccess) e = upload(out.tlb, tlb, s);
    if (e == cudaSuccess) e = upload(out.tdb, tdb, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host vectors die here
    out.K = K;
    out.L = L;
    out.W = W;
    out.NR = NR;
    out.KS = std::max<int64_t>(KS, TILE);
    out.SS = q * out.KS + std::max<int64_t>(TILE, (L + TILE - 1) / TILE * TILE);
    if (out.SS > INT32_MAX) return fail(h, CLB_INVALID_ARG, "lattice exceeds 2^31 slots per species");
    return cuda_check(h, e, "sparse layout");
}

}  // namespace clb
